"""TSDF fusion: the host-side mirror of BrickGrid and TsdfVolume
(frontend/src/app/vision/fusion/tsdf-volume.ts) over libluvas3d.so.

Two layouts: the reference's brick pool (8^3 bricks, voxel (b, x, y, z) at b*512 + x + 8y + 64z,
chosen by BrickGrid around the surface) and a dense grid (x fastest).  Two weight storages: f32
(the reference's) and uint16 Q8.8 fixed point.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass
from typing import Sequence

import numpy as np

from . import _lib
from .camera import Intrinsics, Pose

BRICK = 8                 # tsdf-volume.ts:5
MAX_WEIGHT = 96.0         # tsdf-volume.ts:7
PRIOR_WEIGHT = 0.12       # tsdf-volume.ts:8


class BrickGrid:
    """Sparse set of 8^3 voxel bricks on a bounded grid (BrickGrid, tsdf-volume.ts:13-65)."""

    def __init__(self, origin, voxel: float, extent):
        self.origin = tuple(float(o) for o in origin)
        self.voxel = float(voxel)
        side = self.voxel * BRICK
        self.dims = tuple(max(1, math.ceil(float(e) / side)) for e in extent)
        self.marks = np.zeros(self.dims[0] * self.dims[1] * self.dims[2], dtype=np.uint8)

    @property
    def cells(self) -> int:
        return self.marks.size

    def mark(self, x: float, y: float, z: float, radius: float) -> None:
        """Marks every brick touched by the cube of half-size radius around a point."""
        side = self.voxel * BRICK
        ox, oy, oz = self.origin
        dx, dy, dz = self.dims
        x0 = max(0, math.floor((x - radius - ox) / side))
        x1 = min(dx - 1, math.floor((x + radius - ox) / side))
        y0 = max(0, math.floor((y - radius - oy) / side))
        y1 = min(dy - 1, math.floor((y + radius - oy) / side))
        z0 = max(0, math.floor((z - radius - oz) / side))
        z1 = min(dz - 1, math.floor((z + radius - oz) / side))
        if x1 < x0 or y1 < y0 or z1 < z0:
            return
        m = self.marks.reshape(dz, dy, dx)
        m[z0:z1 + 1, y0:y1 + 1, x0:x1 + 1] = 1

    def build(self) -> tuple[np.ndarray, np.ndarray, int]:
        """Pool layout: brick coords (count, 4) int32 (x, y, z, 0) and the grid -> pool lookup."""
        dx, dy, _ = self.dims
        idx = np.flatnonzero(self.marks)
        lookup = np.full(self.marks.size, -1, dtype=np.int32)
        lookup[idx] = np.arange(idx.size, dtype=np.int32)
        coords = np.zeros((idx.size, 4), dtype=np.int32)
        coords[:, 0] = idx % dx
        coords[:, 1] = (idx // dx) % dy
        coords[:, 2] = idx // (dx * dy)
        return coords, lookup, int(idx.size)


@dataclass
class IntegrationView:
    """IntegrationView (tsdf-volume.ts:67-79)."""

    intrinsics: Intrinsics
    pose: Pose
    max_depth: float
    prior: np.ndarray | None = None
    confidence: float = 0.0


def _host_ptr(a, count: int, itemsize: int):
    """Address of a host buffer of at least `count` elements of `itemsize` bytes: a C-contiguous
    numpy array or a contiguous CPU tensor.  None stays None."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        ok = a.flags.c_contiguous and a.size >= count and a.itemsize == itemsize
        addr = a.ctypes.data
    else:
        if getattr(a, "is_cuda", False):
            raise ValueError("integrate_many_read writes host buffers, not device tensors")
        ok = a.is_contiguous() and a.numel() >= count and a.element_size() == itemsize
        addr = a.data_ptr()
    if not ok:
        raise ValueError(f"host buffer must be contiguous with >= {count} elements of {itemsize} bytes")
    return C.c_void_p(addr)


def _c_view(v: IntegrationView, keep: list):
    cv = _lib.IntegrationView()
    k = v.intrinsics
    cv.intrinsics = _lib.Intrinsics(k.fx, k.fy, k.cx, k.cy)
    cv.pose.R[:] = list(np.asarray(v.pose.R, dtype=np.float64).reshape(9))
    cv.pose.t[:] = list(np.asarray(v.pose.t, dtype=np.float64).reshape(3))
    cv.max_depth = float(v.max_depth)
    cv.confidence = float(v.confidence)
    if v.prior is not None:
        p = np.ascontiguousarray(v.prior, dtype=np.float32).reshape(-1)
        keep.append(p)
        cv.prior = p.ctypes.data_as(C.POINTER(C.c_float))
    return cv


class TsdfVolume:
    """Truncated signed distance volume on the GPU (TsdfVolume, tsdf-volume.ts:157-291).

    dense=(X, Y, Z) builds a dense grid; otherwise `grid` and `layout` (BrickGrid.build()) give the
    reference's brick pool.  truncation defaults to 4 voxels (tsdf-volume.ts:179).
    """

    def __init__(self, width: int, height: int, voxel: float, origin, *, dense=None,
                 grid: BrickGrid | None = None, layout=None, truncation: float | None = None,
                 weight_q8: bool = False, max_weight: float = MAX_WEIGHT,
                 prior_weight: float = PRIOR_WEIGHT, stream: int | None = None):
        self._lib = _lib.load()
        self.width, self.height = int(width), int(height)
        self.voxel = float(voxel)
        self.truncation = float(truncation) if truncation is not None else self.voxel * 4
        self.weight_q8 = bool(weight_q8)
        d = _lib.TsdfDesc()
        d.origin[:] = [float(o) for o in origin]
        d.voxel = self.voxel
        d.truncation = self.truncation
        d.max_weight = float(max_weight)
        d.prior_weight = float(prior_weight)
        self._coords = None
        if dense is not None:
            d.dense = 1
            d.dims[:] = [int(x) for x in dense]
            self.dims = tuple(int(x) for x in dense)
            self.count = None
        else:
            if layout is None:
                raise ValueError("a brick pool needs layout = BrickGrid.build()")
            coords = np.ascontiguousarray(layout[0], dtype=np.int32)
            self._coords = coords
            d.dense = 0
            d.coords = coords.ctypes.data_as(C.POINTER(C.c_int32))
            d.count = int(coords.shape[0])
            self.count = int(coords.shape[0])
            self.dims = None
        self.grid = grid
        self.layout = layout
        d.weight_type = _lib.WEIGHT_Q8 if weight_q8 else _lib.WEIGHT_F32
        d.width, d.height = self.width, self.height
        d.stream = stream
        h = C.c_void_p()
        _lib.check(self._lib.l3d_tsdf_create(C.byref(d), C.byref(h)))
        self._handle = h

    def _h(self):
        if self._handle is None:
            raise RuntimeError("TsdfVolume used after destroy()")
        return self._handle

    @property
    def voxels(self) -> int:
        return int(self._lib.l3d_tsdf_voxels(self._h()))

    def integrate(self, view: IntegrationView, depth=None, stereo=None) -> None:
        """integrate (tsdf-volume.ts:240-268): one packed map, from a host array `depth` (H, W)
        u32 or from `stereo`'s filtered map."""
        keep: list = []
        cv = _c_view(view, keep)
        if stereo is not None:
            _lib.check(self._lib.l3d_tsdf_integrate(self._h(), stereo._h(), None, C.byref(cv)))
        else:
            p = np.ascontiguousarray(depth, dtype=np.uint32)
            _lib.check(self._lib.l3d_tsdf_integrate(self._h(), None, _lib.ptr(p), C.byref(cv)))
            keep.append(p)
        if keep:
            self.synchronize()

    def integrate_layer(self, view: IntegrationView, stereo, layer: int) -> None:
        """integrate (tsdf-volume.ts:240-268) of `stereo`'s filter_all map of `layer`: one view
        per launch, the reference's form."""
        keep: list = []
        cv = _c_view(view, keep)
        _lib.check(self._lib.l3d_tsdf_integrate_layer(self._h(), stereo._h(), int(layer), C.byref(cv)))
        if keep:
            self.synchronize()

    def count_updates(self, views: Sequence[IntegrationView], depths=None, stereo=None,
                      layers: Sequence[int] | None = None) -> tuple[int, int, int]:
        """(visible voxel-views, voxel-updates, voxel-views the depth-aware cull keeps) of
        integrating these maps, without integrating them."""
        keep: list = []
        arr = (_lib.IntegrationView * len(views))(*[_c_view(v, keep) for v in views])
        vis, upd, kept = C.c_int64(), C.c_int64(), C.c_int64()
        if stereo is not None:
            lay = np.asarray(layers if layers is not None else range(len(views)), dtype=np.int32)
            _lib.check(self._lib.l3d_tsdf_count_updates(
                self._h(), stereo._h(), lay.ctypes.data_as(C.POINTER(C.c_int32)), None,
                len(views), arr, C.byref(vis), C.byref(upd), C.byref(kept)))
        else:
            p = np.ascontiguousarray(depths, dtype=np.uint32)
            _lib.check(self._lib.l3d_tsdf_count_updates(self._h(), None, None, _lib.ptr(p), len(views),
                                                        arr, C.byref(vis), C.byref(upd), C.byref(kept)))
        return int(vis.value), int(upd.value), int(kept.value)

    def integrate_many(self, views: Sequence[IntegrationView], depths=None, stereo=None,
                       layers: Sequence[int] | None = None) -> None:
        """Integrates many maps in one sweep; equal bit for bit to integrate() in order."""
        keep: list = []
        arr = (_lib.IntegrationView * len(views))(*[_c_view(v, keep) for v in views])
        if stereo is not None:
            lay = np.asarray(layers if layers is not None else range(len(views)), dtype=np.int32)
            _lib.check(self._lib.l3d_tsdf_integrate_many(
                self._h(), stereo._h(), lay.ctypes.data_as(C.POINTER(C.c_int32)), None,
                len(views), arr))
        else:
            p = np.ascontiguousarray(depths, dtype=np.uint32)
            _lib.check(self._lib.l3d_tsdf_integrate_many(self._h(), None, None, _lib.ptr(p),
                                                         len(views), arr))
            keep.append(p)
        if keep:
            self.synchronize()

    def integrate_many_read(self, views: Sequence[IntegrationView], depths=None, stereo=None,
                            layers: Sequence[int] | None = None, out=None, wait: bool = True):
        """integrate_many() then read(), with the read-back overlapped with the sweep.  `out`:
        optional (tsdf, weight) host buffers of voxels elements each (pinned memory, e.g.
        torch's pin_memory(), overlaps fully); returns them shaped like read()'s.  With
        wait=False (`out` required) the call returns once the work is queued
        (l3d_tsdf_integrate_many_read_async): the buffers hold the volume after wait_read()."""
        if not wait and out is None:
            raise ValueError("an asynchronous read-back needs the caller's `out` buffers")
        keep: list = []
        arr = (_lib.IntegrationView * len(views))(*[_c_view(v, keep) for v in views])
        tsdf, weight = out if out is not None else self._host_volume()
        tp = _host_ptr(tsdf, self.voxels, 4)
        wp = _host_ptr(weight, self.voxels, 2 if self.weight_q8 else 4)
        fn = self._lib.l3d_tsdf_integrate_many_read if wait else self._lib.l3d_tsdf_integrate_many_read_async
        if stereo is not None:
            lay = np.asarray(layers if layers is not None else range(len(views)), dtype=np.int32)
            _lib.check(fn(self._h(), stereo._h(), lay.ctypes.data_as(C.POINTER(C.c_int32)), None,
                          len(views), arr, tp, wp))
        else:
            p = np.ascontiguousarray(depths, dtype=np.uint32)
            _lib.check(fn(self._h(), None, None, _lib.ptr(p), len(views), arr, tp, wp))
            keep.append(p)
        return self._shaped(tsdf, weight)

    def wait_read(self) -> None:
        """Blocks until an asynchronous read-back (integrate_many_read(wait=False)) is done."""
        _lib.check(self._lib.l3d_tsdf_wait_read(self._h()))

    def _host_volume(self) -> tuple[np.ndarray, np.ndarray]:
        n = self.voxels
        return (np.empty(n, dtype=np.float32),
                np.empty(n, dtype=np.uint16 if self.weight_q8 else np.float32))

    def _shaped(self, tsdf, weight):
        if self.dims is not None and isinstance(tsdf, np.ndarray):
            X, Y, Z = self.dims
            return tsdf.reshape(Z, Y, X), weight.reshape(Z, Y, X)
        return tsdf, weight

    def read(self) -> tuple[np.ndarray, np.ndarray]:
        """read (tsdf-volume.ts:270-277): (tsdf f32, weight f32 or uint16 Q8.8)."""
        n = self.voxels
        tsdf = np.empty(n, dtype=np.float32)
        weight = np.empty(n, dtype=np.uint16 if self.weight_q8 else np.float32)
        _lib.check(self._lib.l3d_tsdf_read(self._h(), _lib.ptr(tsdf), _lib.ptr(weight)))
        if self.dims is not None:
            X, Y, Z = self.dims
            return tsdf.reshape(Z, Y, X), weight.reshape(Z, Y, X)
        return tsdf, weight

    def reset(self) -> None:
        _lib.check(self._lib.l3d_tsdf_reset(self._h()))

    @property
    def stream(self) -> int:
        s = C.c_void_p()
        _lib.check(self._lib.l3d_tsdf_stream(self._h(), C.byref(s)))
        return s.value or 0

    @property
    def launches(self) -> int:
        return int(self._lib.l3d_tsdf_launches(self._h()))

    def synchronize(self) -> None:
        _lib.check(self._lib.l3d_tsdf_synchronize(self._h()))

    def destroy(self) -> None:
        if self._handle is not None:
            self._lib.l3d_tsdf_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass
