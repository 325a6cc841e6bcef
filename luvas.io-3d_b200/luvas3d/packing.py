"""Host-side decoding of the packed depth format (frontend/src/app/vision/mvs/depth-maps.ts:57-85).

A packed sample is a u32: bits 0-15 f16 depth, 16-21 and 22-27 the octahedral normal (6 bits
each), 28-31 the matching cost quantised to 0-15 (mvs/depth-packing.wgsl.ts:21-33).  Zero means
no depth.  These numpy helpers serve the consumers of the packed maps (fusion, meshing, tests).
"""
from __future__ import annotations

import numpy as np


def half_to_float(bits) -> np.ndarray:
    """halfToFloat (depth-maps.ts:57-60): IEEE half bits -> float32 (vectorised)."""
    return np.asarray(bits, dtype=np.uint32).astype(np.uint16).view(np.float16).astype(np.float32)


def unpack_depth(packed) -> np.ndarray:
    return half_to_float(np.asarray(packed, dtype=np.uint32) & 0xFFFF)


def unpack_cost(packed) -> np.ndarray:
    return (np.asarray(packed, dtype=np.uint32) >> 28).astype(np.uint32)


def unpack_samples(packed) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """unpackDepthSample (depth-maps.ts:66-85) over an array, in float64.

    Returns (valid, depth, normal[..., 3]); invalid entries have depth 0 and normal 0.
    """
    p = np.asarray(packed, dtype=np.uint32)
    d = half_to_float(p & 0xFFFF).astype(np.float64)
    valid = (p != 0) & (d > 0)
    ex = ((p >> 16) & 63).astype(np.float64) / 63 * 2 - 1
    ey = ((p >> 22) & 63).astype(np.float64) / 63 * 2 - 1
    nz = 1 - np.abs(ex) - np.abs(ey)
    fold = nz < 0
    nx = np.where(fold, (1 - np.abs(ey)) * np.where(ex >= 0, 1.0, -1.0), ex)
    ny = np.where(fold, (1 - np.abs(ex)) * np.where(ey >= 0, 1.0, -1.0), ey)
    length = np.sqrt(nx * nx + ny * ny + nz * nz)
    length = np.where(length == 0, 1.0, length)
    n = np.stack([nx / length, ny / length, nz / length], axis=-1)
    n[~valid] = 0
    return valid, np.where(valid, d, 0.0), n
