"""The library's per-device memory pool: how much it holds, and handing its unused part back.

Scratch buffers, point tables and mesh outputs are stream-ordered allocations from a pool that
keeps up to 16 GB of freed memory mapped for the next call.  The reference's WebGPU buffers
return their memory when destroyed (fusion/tsdf-volume.ts:279-290,
mvs/dense-stereo.ts:357-370); `trim_memory` does that on request for the current device.
"""
from __future__ import annotations

import ctypes as C

from . import _lib


def trim_memory(keep_bytes: int = 0) -> None:
    """Waits for the current device's queued work, then releases the pool's unused memory
    until at most `keep_bytes` stay reserved.  Memory held by live handles stays."""
    _lib.check(_lib.load().l3d_memory_trim(int(keep_bytes)))


def memory_reserved() -> tuple[int, int]:
    """(reserved, used) bytes of the current device's pool; (0, 0) before its first use."""
    r, u = C.c_int64(0), C.c_int64(0)
    _lib.check(_lib.load().l3d_memory_reserved(C.byref(r), C.byref(u)))
    return r.value, u.value
