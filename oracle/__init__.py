"""ctypes wrapper of the CPU oracle (oracle/oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg, as the checker or the timed CPU baseline.  Nothing in the product imports it.
Parity unpinned: the reference has no CPU implementation or golden vectors for this path; the
known-answer tests in tests/test_oracle.py pin the restatement.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libl3doracle.so")

INIT, INIT_COARSE, PROPAGATE, PACK, CONSISTENCY = range(5)


class StereoArgs(C.Structure):
    _fields_ = [
        ("width", C.c_int32), ("height", C.c_int32), ("n_views", C.c_int32),
        ("views", C.c_void_p), ("images", C.c_void_p),
        ("ref", C.c_int32), ("sources", C.c_void_p), ("n_sources", C.c_int32),
        ("min_depth", C.c_double), ("max_depth", C.c_double),
        ("prior", C.c_void_p),
        ("geometric", C.c_int32), ("iterations", C.c_int32),
        ("win_n", C.c_int32), ("win_dil", C.c_int32), ("pack", C.c_int32),
        ("from_coarse", C.c_int32), ("coarse_hyp", C.c_void_p),
        ("coarse_w", C.c_int32), ("coarse_h", C.c_int32),
        ("needed", C.c_int32), ("threads", C.c_int32),
        ("sizes", C.c_void_p),
        ("compensated", C.c_int32),
    ]


class TsdfDesc(C.Structure):
    _fields_ = [
        ("origin", C.c_double * 3), ("voxel", C.c_double), ("truncation", C.c_double),
        ("max_weight", C.c_double), ("prior_weight", C.c_double),
        ("dense", C.c_int32), ("dims", C.c_int32 * 3), ("coords", C.c_void_p), ("count", C.c_int32),
        ("weight_q8", C.c_int32), ("width", C.c_int32), ("height", C.c_int32),
    ]


class SdfBricks(C.Structure):
    _fields_ = [
        ("origin", C.c_double * 3), ("voxel", C.c_double), ("dims", C.c_int32 * 3),
        ("lookup", C.c_void_p), ("tsdf", C.c_void_p), ("weight", C.c_void_p), ("bricks", C.c_int64),
    ]


class TsdfView(C.Structure):
    _fields_ = [
        ("k", C.c_double * 4), ("R", C.c_double * 9), ("t", C.c_double * 3),
        ("max_depth", C.c_double), ("confidence", C.c_double), ("prior", C.c_void_p),
    ]


_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        lib = C.CDLL(LIB_PATH)
        P = C.c_void_p
        for pre in ("orc32", "orc64"):
            getattr(lib, pre + "_solve").argtypes = [C.POINTER(StereoArgs), P, P, P]
            getattr(lib, pre + "_kernel").argtypes = [C.POINTER(StereoArgs), C.c_int32, C.c_int32,
                                                      C.c_int32, P, P, P, P]
            getattr(lib, pre + "_plane_cost").argtypes = [C.POINTER(StereoArgs), P, P, P]
            getattr(lib, pre + "_tsdf_integrate").argtypes = [C.POINTER(TsdfDesc), C.POINTER(TsdfView),
                                                              P, P, P, C.c_int32]
        lib.orc_tsdf_visible.argtypes = [C.POINTER(TsdfDesc), C.POINTER(TsdfView), P]
        lib.orc_cloud_create.restype = P
        lib.orc_cloud_create.argtypes = [C.c_double]
        lib.orc_cloud_destroy.argtypes = [P]
        lib.orc_cloud_add_point.argtypes = [P, P]
        lib.orc_cloud_add_map.argtypes = [P, P, C.c_int32, C.c_int32, P, P, C.c_int32, C.c_int32]
        lib.orc_cloud_coarsen.argtypes = [P, C.c_double]
        lib.orc_cloud_size.restype = C.c_int32
        lib.orc_cloud_size.argtypes = [P]
        lib.orc_cloud_cell.restype = C.c_double
        lib.orc_cloud_cell.argtypes = [P]
        lib.orc_cloud_read.restype = C.c_int32
        lib.orc_cloud_read.argtypes = [P, C.c_int32, P, P, P, P, P]
        lib.orc_extract_surface.argtypes = [C.POINTER(SdfBricks), C.c_double, P, P, P, P, P]
        lib.orc_remove_small_components.argtypes = [C.c_int64, C.c_int64, P, P, P, C.c_double,
                                                     C.c_int32, P, P, P, P, P]
        lib.orc_brick_grid_dims.argtypes = [C.c_double, P, P]
        lib.orc_brick_grid_mark.argtypes = [P, C.c_double, P, P, P, C.c_int64, C.c_double]
        lib.orc_brick_grid_build.restype = C.c_int32
        lib.orc_brick_grid_build.argtypes = [P, P, P, P]
        for name in ("orc_rgba_to_gray", "orc_downsample_rgb", "orc_downsample_gray"):
            getattr(lib, name).argtypes = [P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, P]
        lib.orc_upsample_depth.argtypes = [P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, P]
        lib.orc64_ncc_grad.argtypes = [C.POINTER(StereoArgs), P, P, P, P, P, P, P, P]
        lib.orc64_tsdf_depth.argtypes = [C.POINTER(TsdfDesc), C.POINTER(TsdfView)] + [P] * 11 + [C.c_int32]
        lib.orc_pack_sample.restype = C.c_uint32
        lib.orc_pack_sample.argtypes = [C.c_float] * 5
        lib.orc_unpack_depth.restype = C.c_float
        lib.orc_unpack_depth.argtypes = [C.c_uint32]
        lib.orc_unpack_normal.argtypes = [C.c_uint32, P]
        lib.orc_pcg.restype = C.c_uint32
        lib.orc_pcg.argtypes = [C.c_uint32]
        lib.orc_expf.restype = C.c_float
        lib.orc_expf.argtypes = [C.c_float]
        lib.orc_sincosf.argtypes = [C.c_float, P, P]
        lib.orc_f32_to_f16.restype = C.c_uint32
        lib.orc_f32_to_f16.argtypes = [C.c_float]
        lib.orc_f16_to_f32.restype = C.c_float
        lib.orc_f16_to_f32.argtypes = [C.c_uint32]
        lib.orc_seed.restype = C.c_uint32
        lib.orc_seed.argtypes = [C.c_int32] * 4
        _lib = lib
    return _lib


def _views_array(views) -> np.ndarray:
    out = np.zeros((len(views), 16), dtype=np.float64)
    for i, v in enumerate(views):
        k = v.intrinsics
        out[i, :4] = (k.fx, k.fy, k.cx, k.cy)
        out[i, 4:13] = np.asarray(v.pose.R, dtype=np.float64).reshape(9)
        out[i, 13:16] = np.asarray(v.pose.t, dtype=np.float64).reshape(3)
    return out


class Stereo:
    """Oracle state for one image set: images, packed depth maps of every view and the hypothesis
    buffers of one reference view, in FP32 (`precision=32`) or FP64.

    Views may differ in size (images of different shapes): images and depth maps are then kept
    concatenated, `depths` is a list of per-view arrays and `hyp`/`cost` take the shape of the
    reference view of the last call."""

    def __init__(self, width, height, views, images, precision: int = 32, window: int = 6,
                 dilation: int = 2, threads: int = 0, compensated: bool = False):
        self.V = len(views)
        self.views = _views_array(views)
        imgs = [np.ascontiguousarray(i, dtype=np.float32) for i in images]
        self.shapes = [im.shape for im in imgs]
        self.uniform = all(sh == (int(height), int(width)) for sh in self.shapes)
        self.W, self.H = int(width), int(height)
        self.sizes = np.ascontiguousarray([[sh[1], sh[0]] for sh in self.shapes], dtype=np.int32)
        self.offsets = np.concatenate([[0], np.cumsum([sh[0] * sh[1] for sh in self.shapes])])
        self.images = np.ascontiguousarray(np.concatenate([im.reshape(-1) for im in imgs]))
        self.dt = np.float32 if precision == 32 else np.float64
        self.pre = "orc32" if precision == 32 else "orc64"
        pmax = max(sh[0] * sh[1] for sh in self.shapes)
        self._hyp = np.zeros(pmax * 4, dtype=self.dt)
        self._cost = np.zeros(pmax, dtype=self.dt)
        self._filtered = np.zeros(pmax, dtype=np.uint32)
        self._depths = np.zeros(int(self.offsets[-1]), dtype=np.uint32)
        self._ref_shape = self.shapes[0]
        self.window, self.dilation, self.threads = window, dilation, threads
        self.compensated = bool(compensated)
        self.coarse = None  # (hyp (h, w, 4) in this precision)

    @property
    def hyp(self):
        h, w = self._ref_shape
        return self._hyp[:h * w * 4].reshape(h, w, 4)

    @hyp.setter
    def hyp(self, value):
        h, w = self._ref_shape
        self._hyp[:h * w * 4] = np.asarray(value, dtype=self.dt).reshape(-1)

    @property
    def cost(self):
        h, w = self._ref_shape
        return self._cost[:h * w].reshape(h, w)

    @cost.setter
    def cost(self, value):
        h, w = self._ref_shape
        self._cost[:h * w] = np.asarray(value, dtype=self.dt).reshape(-1)

    @property
    def filtered(self):
        h, w = self._ref_shape
        return self._filtered[:h * w].reshape(h, w)

    @property
    def depths(self):
        if self.uniform:
            return self._depths.reshape(self.V, self.H, self.W)
        return [self._depths[self.offsets[i]:self.offsets[i + 1]].reshape(self.shapes[i])
                for i in range(self.V)]

    def _args(self, ref, sources, min_depth=0.5, max_depth=3.0, prior=None, geometric=False,
              iterations=3, pack=True, from_coarse=False, needed=0):
        keep = []
        a = StereoArgs()
        a.width, a.height, a.n_views = self.W, self.H, self.V
        a.sizes = None if self.uniform else self.sizes.ctypes.data
        self._ref_shape = self.shapes[int(ref)]
        a.views = self.views.ctypes.data
        a.images = self.images.ctypes.data
        a.ref = int(ref)
        src = np.asarray(list(sources), dtype=np.int32)
        keep.append(src)
        a.sources = src.ctypes.data
        a.n_sources = len(src)
        a.min_depth, a.max_depth = float(min_depth), float(max_depth)
        if prior is not None:
            pr = np.ascontiguousarray(prior, dtype=np.float32)
            keep.append(pr)
            a.prior = pr.ctypes.data
        a.geometric = int(bool(geometric))
        a.iterations = int(iterations)
        a.win_n, a.win_dil = self.window, self.dilation
        a.pack = int(bool(pack))
        if self.coarse is not None:
            ch = np.ascontiguousarray(self.coarse, dtype=self.dt)
            keep.append(ch)
            a.coarse_hyp = ch.ctypes.data
            a.coarse_h, a.coarse_w = ch.shape[0], ch.shape[1]
        a.from_coarse = int(bool(from_coarse))
        a.needed = int(needed)
        a.threads = int(self.threads)
        a.compensated = int(self.compensated)
        return a, keep

    def solve(self, ref, sources, **kw) -> None:
        a, keep = self._args(ref, sources, **kw)
        rc = getattr(load(), self.pre + "_solve")(C.byref(a), self._hyp.ctypes.data,
                                                  self._cost.ctypes.data, self._depths.ctypes.data)
        assert rc == 0, "oracle rejected the arguments"

    def kernel(self, kernel, ref, sources, iteration=0, phase=0, **kw) -> None:
        a, keep = self._args(ref, sources, **kw)
        rc = getattr(load(), self.pre + "_kernel")(C.byref(a), int(kernel), int(iteration),
                                                   int(phase), self._hyp.ctypes.data,
                                                   self._cost.ctypes.data, self._depths.ctypes.data,
                                                   self._filtered.ctypes.data)
        assert rc == 0, "oracle rejected the arguments"

    def filter(self, ref, checks, needed) -> np.ndarray:
        self.kernel(CONSISTENCY, ref, checks, needed=needed)
        return self.filtered.copy()

    def plane_cost(self, ref, sources, planes, **kw):
        a, keep = self._args(ref, sources, **kw)
        pl = np.ascontiguousarray(planes, dtype=self.dt)
        h, w = self._ref_shape
        cost = np.zeros((h, w), dtype=self.dt)
        vc = np.zeros((h, w, 8), dtype=self.dt)
        rc = getattr(load(), self.pre + "_plane_cost")(C.byref(a), pl.ctypes.data, cost.ctypes.data,
                                                       vc.ctypes.data)
        assert rc == 0
        return cost, vc


class NccGrad:
    """FP64 summed-NCC objective of one reference view and its forward-mode (dual-number)
    gradients with respect to per-pixel planes (depth, angle a, angle b) and per-view se(3)
    increments (oracle/grad.cpp)."""

    def __init__(self, views, images, window: int = 6, dilation: int = 2, threads: int = 0):
        self.st = Stereo(images[0].shape[1], images[0].shape[0], views, images, precision=64,
                         window=window, dilation=dilation, threads=threads)

    def __call__(self, ref, sources, planes, deltas=None, weights=None, grad_planes=False,
                 grad_deltas=False):
        """Returns (cost (H, W), grad_planes (H, W, 3) or None, grad_deltas (V, 6) or None) for
        the objective sum(weights * cost) (weights None = ones)."""
        a, keep = self.st._args(ref, sources)
        h, w = self.st._ref_shape
        pl = np.ascontiguousarray(planes, dtype=np.float64).reshape(h, w, 3)
        de = None if deltas is None else np.ascontiguousarray(deltas, dtype=np.float64).reshape(-1, 6)
        wt = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64).reshape(h, w)
        cost = np.zeros((h, w), dtype=np.float64)
        gp = np.zeros((h, w, 3), dtype=np.float64) if grad_planes else None
        gd = np.zeros((self.st.V, 6), dtype=np.float64) if grad_deltas else None
        ptr = lambda x: None if x is None else x.ctypes.data  # noqa: E731
        rc = load().orc64_ncc_grad(C.byref(a), pl.ctypes.data, ptr(de), ptr(wt), cost.ctypes.data,
                                   ptr(gp), ptr(gd), None, None)
        assert rc == 0
        return cost, gp, gd

    def structure(self, ref, sources, planes, deltas=None):
        """(cost, margin, cells) per pixel: margin is the smallest distance (texels) from a
        window sample to a source's border (-1 where a source's cost is the constant 2 or 1),
        cells a hash of the texel cells the samples fall in; the cost is smooth in a parameter
        while a pixel's hash stays the same."""
        a, keep = self.st._args(ref, sources)
        h, w = self.st._ref_shape
        pl = np.ascontiguousarray(planes, dtype=np.float64).reshape(h, w, 3)
        de = None if deltas is None else np.ascontiguousarray(deltas, dtype=np.float64).reshape(-1, 6)
        margin = np.zeros((h, w), dtype=np.float64)
        cells = np.zeros((h, w), dtype=np.uint64)
        cost = np.zeros((h, w), dtype=np.float64)
        rc = load().orc64_ncc_grad(C.byref(a), pl.ctypes.data, None if de is None else de.ctypes.data,
                                   None, cost.ctypes.data, None, None, margin.ctypes.data,
                                   cells.ctypes.data)
        assert rc == 0
        return cost, margin, cells


def extract_surface(origin, voxel, dims, lookup, tsdf, weight, min_weight):
    """extractSurface + computeNormals -> (positions (V, 3) f32, normals (V, 3) f32,
    indices (I,) u32)."""
    lk = np.ascontiguousarray(lookup, dtype=np.int32)
    ts = np.ascontiguousarray(tsdf, dtype=np.float32)
    wt = np.ascontiguousarray(weight, dtype=np.float32)
    v = SdfBricks()
    v.origin[:] = [float(o) for o in origin]
    v.voxel = float(voxel)
    v.dims[:] = [int(d) for d in dims]
    v.lookup, v.tsdf, v.weight = lk.ctypes.data, ts.ctypes.data, wt.ctypes.data
    v.bricks = ts.size // 512
    nv, ni = C.c_int64(), C.c_int64()
    lib = load()
    lib.orc_extract_surface(C.byref(v), float(min_weight), C.byref(nv), C.byref(ni), None, None, None)
    pos = np.zeros((nv.value, 3), np.float32)
    nrm = np.zeros((nv.value, 3), np.float32)
    idx = np.zeros(ni.value, np.uint32)
    lib.orc_extract_surface(C.byref(v), float(min_weight), C.byref(nv), C.byref(ni),
                            pos.ctypes.data, nrm.ctypes.data, idx.ctypes.data)
    return pos, nrm, idx


def remove_small_components(pos, nrm, idx, fraction, min_faces):
    p = np.ascontiguousarray(pos, np.float32)
    n = np.ascontiguousarray(nrm, np.float32)
    i = np.ascontiguousarray(idx, np.uint32)
    op = np.zeros_like(p)
    on = np.zeros_like(n)
    oi = np.zeros_like(i)
    nv, ni = C.c_int64(), C.c_int64()
    load().orc_remove_small_components(p.shape[0], i.size, p.ctypes.data, n.ctypes.data, i.ctypes.data,
                                       float(fraction), int(min_faces), C.byref(nv), C.byref(ni),
                                       op.ctypes.data, on.ctypes.data, oi.ctypes.data)
    return op[:nv.value], on[:nv.value], oi[:ni.value]


def brick_grid(origin, voxel, extent, points, radius):
    """BrickGrid(origin, voxel, extent), mark(points, radius), build() -> (dims, coords, lookup)."""
    lib = load()
    o = np.ascontiguousarray(origin, np.float64)
    e = np.ascontiguousarray(extent, np.float64)
    dims = np.zeros(3, np.int32)
    lib.orc_brick_grid_dims(float(voxel), e.ctypes.data, dims.ctypes.data)
    marks = np.zeros(int(np.prod(dims.astype(np.int64))), np.uint8)
    pts = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
    lib.orc_brick_grid_mark(o.ctypes.data, float(voxel), dims.ctypes.data, marks.ctypes.data,
                            pts.ctypes.data, pts.shape[0], float(radius))
    lookup = np.zeros(marks.size, np.int32)
    count = lib.orc_brick_grid_build(dims.ctypes.data, marks.ctypes.data, None, lookup.ctypes.data)
    coords = np.zeros((count, 4), np.int32)
    lib.orc_brick_grid_build(dims.ctypes.data, marks.ctypes.data, coords.ctypes.data, lookup.ctypes.data)
    return dims, coords, lookup


def rgba_to_gray(rgba, tw, th):
    a = np.ascontiguousarray(rgba, np.uint8)
    out = np.zeros((th, tw), np.uint8)
    load().orc_rgba_to_gray(a.ctypes.data, a.shape[1], a.shape[0], tw, th, out.ctypes.data)
    return out


def downsample_rgb(rgba, tw, th):
    a = np.ascontiguousarray(rgba, np.uint8)
    out = np.zeros((th, tw, 3), np.uint8)
    load().orc_downsample_rgb(a.ctypes.data, a.shape[1], a.shape[0], tw, th, out.ctypes.data)
    return out


def downsample_gray(gray, tw, th):
    a = np.ascontiguousarray(gray, np.uint8)
    out = np.zeros((th, tw), np.uint8)
    load().orc_downsample_gray(a.ctypes.data, a.shape[1], a.shape[0], tw, th, out.ctypes.data)
    return out


def upsample_depth(grid, width, height):
    g = np.ascontiguousarray(grid, np.float32)
    out = np.zeros((height, width), np.float32)
    load().orc_upsample_depth(g.ctypes.data, g.shape[1], g.shape[0], width, height, out.ctypes.data)
    return out


class Cloud:
    """PointAccumulator + addDepthMap restated (oracle/cloud.cpp)."""

    def __init__(self, cell: float):
        self._c = load().orc_cloud_create(float(cell))

    def __del__(self):
        if getattr(self, "_c", None):
            load().orc_cloud_destroy(self._c)
            self._c = None

    def add(self, x, y, z, nx, ny, nz, r, g, b) -> None:
        p = np.array([x, y, z, nx, ny, nz, r, g, b], dtype=np.float64)
        load().orc_cloud_add_point(self._c, p.ctypes.data)

    def add_map(self, packed, view, thumb) -> None:
        """packed (H, W) u32; view a StereoView; thumb (th, tw, 3) uint8."""
        pk = np.ascontiguousarray(packed, dtype=np.uint32)
        v = _views_array([view])[0].copy()
        rgb = np.ascontiguousarray(thumb, dtype=np.uint8)
        load().orc_cloud_add_map(self._c, pk.ctypes.data, pk.shape[1], pk.shape[0], v.ctypes.data,
                                 rgb.ctypes.data, rgb.shape[1], rgb.shape[0])

    def coarsen(self, factor: float = 1.4) -> None:
        load().orc_cloud_coarsen(self._c, float(factor))

    @property
    def size(self) -> int:
        return int(load().orc_cloud_size(self._c))

    @property
    def cell(self) -> float:
        return float(load().orc_cloud_cell(self._c))

    def cloud(self, min_support: int = 1) -> dict:
        lib = load()
        n = lib.orc_cloud_read(self._c, int(min_support), None, None, None, None, None)
        out = {"positions": np.zeros((n, 3), np.float32), "normals": np.zeros((n, 3), np.float32),
               "colors": np.zeros((n, 3), np.uint8), "support": np.zeros(n, np.uint16),
               "cells": np.zeros((n, 3), np.int32)}
        lib.orc_cloud_read(self._c, int(min_support), out["positions"].ctypes.data,
                           out["normals"].ctypes.data, out["colors"].ctypes.data,
                           out["support"].ctypes.data, out["cells"].ctypes.data)
        return out


def tsdf_depth(desc, view_kw: dict, packed, depth, tsdf_in, weight_in, grad_tsdf=None,
               grad_weight=None, threads=0):
    """FP64 differentiable TSDF integration of one view (oracle/grad.cpp).  weight_in is in units
    (Q8.8 volumes: value / 256).  Returns (tsdf_out, weight_out, grad_depth, grad_tsdf_in,
    grad_weight_in); the gradients are None without grad_tsdf."""
    v, keep = tsdf_view(**view_kw)
    pk = np.ascontiguousarray(packed, dtype=np.uint32).reshape(-1)
    dp = np.ascontiguousarray(depth, dtype=np.float64).reshape(-1)
    t0 = np.ascontiguousarray(tsdf_in, dtype=np.float64).reshape(-1)
    w0 = np.ascontiguousarray(weight_in, dtype=np.float64).reshape(-1)
    t1 = np.empty_like(t0)
    w1 = np.empty_like(w0)
    gd = gt0 = gw0 = None
    gT = gW = None
    if grad_tsdf is not None:
        gT = np.ascontiguousarray(grad_tsdf, dtype=np.float64).reshape(-1)
        gW = None if grad_weight is None else np.ascontiguousarray(grad_weight, dtype=np.float64).reshape(-1)
        gd = np.zeros_like(dp)
        gt0 = np.empty_like(t0)
        gw0 = np.empty_like(w0)
    ptr = lambda a: None if a is None else a.ctypes.data  # noqa: E731
    rc = load().orc64_tsdf_depth(C.byref(desc), C.byref(v), ptr(pk), ptr(dp), ptr(t0), ptr(w0),
                                 ptr(t1), ptr(w1), ptr(gT), ptr(gW), ptr(gd), ptr(gt0), ptr(gw0),
                                 int(threads))
    assert rc == 0
    return t1, w1, gd, gt0, gw0


def tsdf_desc(width, height, voxel, origin, truncation, dense=None, coords=None,
              weight_q8=False, max_weight=96.0, prior_weight=0.12):
    d = TsdfDesc()
    d.origin[:] = [float(o) for o in origin]
    d.voxel, d.truncation = float(voxel), float(truncation)
    d.max_weight, d.prior_weight = float(max_weight), float(prior_weight)
    keep = []
    if dense is not None:
        d.dense = 1
        d.dims[:] = [int(x) for x in dense]
    else:
        c = np.ascontiguousarray(coords, dtype=np.int32)
        keep.append(c)
        d.dense = 0
        d.coords = c.ctypes.data
        d.count = c.shape[0]
    d.weight_q8 = int(bool(weight_q8))
    d.width, d.height = int(width), int(height)
    return d, keep


def tsdf_view(k, R, t, max_depth, confidence=0.0, prior=None):
    v = TsdfView()
    v.k[:] = [float(x) for x in k]
    v.R[:] = [float(x) for x in np.asarray(R, dtype=np.float64).reshape(9)]
    v.t[:] = [float(x) for x in np.asarray(t, dtype=np.float64).reshape(3)]
    v.max_depth, v.confidence = float(max_depth), float(confidence)
    keep = []
    if prior is not None:
        p = np.ascontiguousarray(prior, dtype=np.float32)
        keep.append(p)
        v.prior = p.ctypes.data
    return v, keep


class Tsdf:
    """Oracle TSDF volume (f32 tsdf; f32 or Q8.8 uint16 weights; FP64 with precision=64)."""

    def __init__(self, width, height, voxel, origin, truncation, dense=None, coords=None,
                 weight_q8=False, max_weight=96.0, prior_weight=0.12, precision=32, threads=0):
        self.desc, self._keep = tsdf_desc(width, height, voxel, origin, truncation, dense, coords,
                                          weight_q8, max_weight, prior_weight)
        n = int(np.prod(dense)) if dense is not None else int(np.asarray(coords).shape[0]) * 512
        self.dt = np.float32 if precision == 32 else np.float64
        self.pre = "orc32" if precision == 32 else "orc64"
        self.tsdf = np.ones(n, dtype=self.dt)
        self.weight = np.zeros(n, dtype=np.uint16 if weight_q8 else self.dt)
        self.threads = threads

    def integrate(self, view_kw: dict, depth: np.ndarray) -> None:
        v, keep = tsdf_view(**view_kw)
        d = np.ascontiguousarray(depth, dtype=np.uint32)
        rc = getattr(load(), self.pre + "_tsdf_integrate")(C.byref(self.desc), C.byref(v), d.ctypes.data,
                                                           self.tsdf.ctypes.data,
                                                           self.weight.ctypes.data, self.threads)
        assert rc == 0

    def visible(self, view_kw: dict) -> np.ndarray:
        v, keep = tsdf_view(**view_kw)
        if self.desc.dense:
            nb = [(int(x) + 7) // 8 for x in self.desc.dims]
            out = np.zeros(nb[0] * nb[1] * nb[2], dtype=np.uint8)
        else:
            out = np.zeros(self.desc.count, dtype=np.uint8)
        load().orc_tsdf_visible(C.byref(self.desc), C.byref(v), out.ctypes.data)
        return out


def pack_sample(depth, n, cost) -> int:
    return int(load().orc_pack_sample(float(depth), float(n[0]), float(n[1]), float(n[2]), float(cost)))


def unpack_normal(packed) -> np.ndarray:
    out = np.zeros(3, dtype=np.float32)
    load().orc_unpack_normal(int(packed), out.ctypes.data)
    return out


def expf(x) -> float:
    return float(load().orc_expf(float(x)))


def sincosf(a):
    s = C.c_float()
    c = C.c_float()
    load().orc_sincosf(float(a), C.byref(s), C.byref(c))
    return s.value, c.value
