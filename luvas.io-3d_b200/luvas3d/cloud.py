"""Dense point cloud on the GPU: PointAccumulator and fuseDepthMaps
(frontend/src/app/vision/fusion/point-accumulator.ts:16-147, depth-fusion.ts:9-74) over the
l3d_cloud_* entry points of include/luvas3d.h."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Callable, Sequence

import numpy as np

from . import _lib
from .camera import StereoView
from .stereo import DenseStereo, _c_views


@dataclass
class PointCloud:
    """PointCloud (point-accumulator.ts:1-7), plus the integer cell of each point."""

    positions: np.ndarray   # (n, 3) float32
    normals: np.ndarray     # (n, 3) float32
    colors: np.ndarray      # (n, 3) uint8
    support: np.ndarray     # (n,) uint16: samples merged into the point
    cells: np.ndarray       # (n, 3) int32


@dataclass
class FusionView:
    """FusionView (depth-fusion.ts:8-16)."""

    view: StereoView
    checks: Sequence[int]
    needed: int
    thumb: np.ndarray       # (th, tw, 3) uint8


class PointAccumulator:
    """Averages oriented, coloured samples per cell of `cell` metres on the device."""

    def __init__(self, cell: float, stream: int | None = None):
        self._lib = _lib.load()
        h = C.c_void_p()
        _lib.check(self._lib.l3d_cloud_create(float(cell), stream, C.byref(h)))
        self._handle = h

    def _h(self):
        if self._handle is None:
            raise RuntimeError("PointAccumulator used after destroy()")
        return self._handle

    @property
    def size(self) -> int:
        n = C.c_int64()
        _lib.check(self._lib.l3d_cloud_size(self._h(), C.byref(n)))
        return int(n.value)

    @property
    def cell(self) -> float:
        c = C.c_double()
        _lib.check(self._lib.l3d_cloud_cell(self._h(), C.byref(c)))
        return float(c.value)

    def add(self, x, y, z, nx, ny, nz, r, g, b) -> None:
        self.add_points(np.array([[x, y, z, nx, ny, nz, r, g, b]], dtype=np.float64))

    def add_points(self, samples: np.ndarray) -> None:
        """(n, 9) samples: x y z nx ny nz r g b."""
        s = np.ascontiguousarray(samples, dtype=np.float64).reshape(-1, 9)
        _lib.check(self._lib.l3d_cloud_add_points(self._h(), s.shape[0], _lib.ptr(s)))

    def add_depth_map(self, view: StereoView, thumb: np.ndarray, packed: np.ndarray | None = None,
                      stereo: DenseStereo | None = None) -> None:
        """addDepthMap: a host packed map (H, W) or the stereo handle's last filtered map."""
        rgb = np.ascontiguousarray(thumb, dtype=np.uint8)
        cv = _c_views([view])
        if packed is not None:
            p = np.ascontiguousarray(packed, dtype=np.uint32)
            _lib.check(self._lib.l3d_cloud_add(self._h(), None, _lib.ptr(p), p.shape[1], p.shape[0],
                                               cv, _lib.ptr(rgb), rgb.shape[1], rgb.shape[0]))
        else:
            _lib.check(self._lib.l3d_cloud_add(self._h(), stereo._h(), None, 0, 0, cv, _lib.ptr(rgb),
                                               rgb.shape[1], rgb.shape[0]))

    def coarsen(self, factor: float = 1.4) -> None:
        _lib.check(self._lib.l3d_cloud_coarsen(self._h(), float(factor)))

    def cloud(self, min_support: int = 1) -> PointCloud:
        """cloud(minSupport) (point-accumulator.ts:114-143), ordered by cell.  One read into
        buffers sized for every occupied cell, trimmed to the points returned."""
        k = self.size
        out = PointCloud(np.zeros((k, 3), np.float32), np.zeros((k, 3), np.float32),
                         np.zeros((k, 3), np.uint8), np.zeros(k, np.uint16),
                         np.zeros((k, 3), np.int32))
        n = C.c_int64()
        _lib.check(self._lib.l3d_cloud_read(self._h(), int(min_support), k, C.byref(n),
                                            _lib.ptr(out.positions), _lib.ptr(out.normals),
                                            _lib.ptr(out.colors), _lib.ptr(out.support),
                                            _lib.ptr(out.cells)))
        m = int(n.value)
        return PointCloud(out.positions[:m], out.normals[:m], out.colors[:m], out.support[:m],
                          out.cells[:m])

    @property
    def launches(self) -> int:
        return int(self._lib.l3d_cloud_launches(self._h()))

    def destroy(self) -> None:
        if self._handle is not None:
            self._lib.l3d_cloud_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


def fuse_depth_maps(stereo: DenseStereo, views: Sequence[FusionView], cell: float,
                    cell_budget: int,
                    progress: Callable[[float, str], None] | None = None) -> tuple[PointCloud, float]:
    """fuseDepthMaps (depth-fusion.ts:23-39): consistency-filter every view, add its samples, and
    grow the cell while the cloud holds more than `cell_budget` cells.  The filtered maps stay
    on the device."""
    acc = PointAccumulator(cell)
    try:
        for layer, v in enumerate(views):
            if progress:
                progress(layer / len(views), f"{layer + 1}/{len(views)}")
            stereo.filter(layer, v.checks, v.needed)
            acc.add_depth_map(v.view, v.thumb, stereo=stereo)
            while acc.size > cell_budget:
                acc.coarsen()
        return acc.cloud(), acc.cell
    finally:
        acc.destroy()
