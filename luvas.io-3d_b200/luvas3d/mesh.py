"""Surface extraction on the GPU: extractSurface, computeNormals, removeSmallComponents and
BrickGrid (frontend/src/app/vision/fusion/surface-nets.ts:47-174, mesh.ts:9-87,
tsdf-volume.ts:13-65) over the l3d_mesh_* / l3d_brick_grid_build entry points."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from .tsdf import TsdfVolume


@dataclass
class Mesh:
    """Mesh (mesh.ts:1-6)."""

    positions: np.ndarray   # (V, 3) float32
    normals: np.ndarray     # (V, 3) float32
    indices: np.ndarray     # (3F,) uint32


class DeviceMesh:
    """A mesh held on the device."""

    def __init__(self, handle: C.c_void_p):
        self._lib = _lib.load()
        self._handle = handle

    @property
    def counts(self) -> tuple[int, int]:
        nv, ni = C.c_int64(), C.c_int64()
        _lib.check(self._lib.l3d_mesh_counts(self._handle, C.byref(nv), C.byref(ni)))
        return int(nv.value), int(ni.value)

    def read(self) -> Mesh:
        nv, ni = self.counts
        m = Mesh(np.zeros((nv, 3), np.float32), np.zeros((nv, 3), np.float32), np.zeros(ni, np.uint32))
        _lib.check(self._lib.l3d_mesh_read(self._handle, _lib.ptr(m.positions), _lib.ptr(m.normals),
                                           _lib.ptr(m.indices)))
        return m

    def remove_small_components(self, fraction: float, min_faces: int) -> "DeviceMesh":
        h = C.c_void_p()
        _lib.check(self._lib.l3d_mesh_remove_small_components(self._handle, float(fraction),
                                                              int(min_faces), C.byref(h)))
        return DeviceMesh(h)

    @property
    def launches(self) -> int:
        return int(self._lib.l3d_mesh_launches(self._handle))

    def destroy(self) -> None:
        if self._handle is not None:
            self._lib.l3d_mesh_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


def extract_surface_device(volume, min_weight: float) -> DeviceMesh:
    """extractSurface of a TsdfVolume (in place on the device) or of a host SdfBricks dict
    (origin, voxel, dims, lookup, tsdf, weight)."""
    lib = _lib.load()
    h = C.c_void_p()
    if isinstance(volume, TsdfVolume):
        _lib.check(lib.l3d_tsdf_extract_surface(volume._h(), float(min_weight), C.byref(h)))
        return DeviceMesh(h)
    lk = np.ascontiguousarray(volume["lookup"], np.int32)
    ts = np.ascontiguousarray(volume["tsdf"], np.float32)
    wt = np.ascontiguousarray(volume["weight"], np.float32)
    v = _lib.SdfBricks()
    v.origin[:] = [float(o) for o in volume["origin"]]
    v.voxel = float(volume["voxel"])
    v.dims[:] = [int(d) for d in volume["dims"]]
    v.lookup, v.tsdf, v.weight = lk.ctypes.data, ts.ctypes.data, wt.ctypes.data
    v.bricks = ts.size // 512
    _lib.check(lib.l3d_extract_surface(C.byref(v), float(min_weight), C.byref(h)))
    return DeviceMesh(h)


def extract_surface(volume, min_weight: float, components: tuple[float, int] | None = None) -> Mesh:
    """extractSurface (+ computeNormals), then removeSmallComponents(fraction, min_faces) when
    `components` is given, read back to the host."""
    m = extract_surface_device(volume, min_weight)
    try:
        if components is not None:
            r = m.remove_small_components(*components)
            try:
                return r.read()
            finally:
                r.destroy()
        return m.read()
    finally:
        m.destroy()


def brick_grid(origin, voxel: float, extent, points: np.ndarray, radius: float):
    """BrickGrid(origin, voxel, extent), mark(p, radius) for every point, build() on the
    device: (dims, coords (count, 4) int32, lookup int32 over the grid)."""
    lib = _lib.load()
    o = np.ascontiguousarray(origin, np.float64)
    e = np.ascontiguousarray(extent, np.float64)
    p = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
    dims = np.zeros(3, np.int32)
    count = C.c_int32()
    _lib.check(lib.l3d_brick_grid_build(_lib.ptr(o), float(voxel), _lib.ptr(e), _lib.ptr(p), p.shape[0],
                                        float(radius), _lib.ptr(dims), C.byref(count), None, None))
    coords = np.zeros((count.value, 4), np.int32)
    lookup = np.zeros(int(np.prod(dims.astype(np.int64))), np.int32)
    _lib.check(lib.l3d_brick_grid_build(_lib.ptr(o), float(voxel), _lib.ptr(e), _lib.ptr(p), p.shape[0],
                                        float(radius), _lib.ptr(dims), C.byref(count), _lib.ptr(coords),
                                        _lib.ptr(lookup)))
    return dims, coords, lookup
