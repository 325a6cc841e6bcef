"""PatchMatch multi-view stereo: the host-side mirror of DenseStereo and the StereoMethod registry.

Mirrors frontend/src/app/vision/mvs/dense-stereo.ts (class DenseStereo, SolveOptions,
StereoOptions, CoarseLevel) and frontend/src/app/vision/mvs/methods/ (STEREO_METHODS with
'single-scale' and 'coarse-to-fine').  Every call goes through libluvas3d.so; the device work is
the CUDA kernels of the library.  Names follow the reference in snake_case.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Callable, Sequence

import numpy as np

from . import _lib
from .camera import StereoView, scale_intrinsics

MAX_SOURCES = _lib.MAX_SOURCES


@dataclass
class SolveOptions:
    """SolveOptions (dense-stereo.ts:16-29)."""

    sources: Sequence[int]
    min_depth: float
    max_depth: float
    prior: np.ndarray | None = None       # width * height metres, 0 = none
    geometric: bool = False
    iterations: int = 3
    from_coarse: bool = False
    pack: bool = True


@dataclass
class StereoOptions:
    """StereoOptions (dense-stereo.ts:38-42) plus the device layout choices of this library."""

    coarse: "DenseStereo | None" = None
    depth_maps: bool = True
    storage: int = _lib.DTYPE_F32
    form: int = _lib.FORM_PLAIN
    window: int = 6
    dilation: int = 2
    stream: int | None = None              # cudaStream_t as an integer, or None
    compensated: bool = False              # fast/exact forms: Neumaier-compensated window sums


def _c_views(views: Sequence[StereoView]):
    arr = (_lib.View * len(views))()
    for i, v in enumerate(views):
        k = v.intrinsics
        arr[i].intrinsics = _lib.Intrinsics(k.fx, k.fy, k.cx, k.cy)
        R = np.asarray(v.pose.R, dtype=np.float64).reshape(9)
        t = np.asarray(v.pose.t, dtype=np.float64).reshape(3)
        arr[i].pose.R[:] = list(R)
        arr[i].pose.t[:] = list(t)
    return arr


class _SolveArgs:
    """Keeps the ctypes buffers of one SolveOpts alive."""

    def __init__(self, o: SolveOptions, pixels: int):
        self.sources = (C.c_int32 * max(1, len(o.sources)))(*[int(s) for s in o.sources])
        self.prior = None
        if o.prior is not None:
            self.prior = np.ascontiguousarray(o.prior, dtype=np.float32).reshape(-1)
            if self.prior.size != pixels:
                raise ValueError(f"prior has {self.prior.size} values, expected {pixels}")
        self.c = _lib.SolveOpts(
            self.sources, len(o.sources), float(o.min_depth), float(o.max_depth),
            self.prior.ctypes.data_as(C.POINTER(C.c_float)) if self.prior is not None else None,
            int(bool(o.geometric)), int(o.iterations), int(bool(o.from_coarse)), int(bool(o.pack)))


class DenseStereo:
    """GPU PatchMatch for every keyframe (DenseStereo, dense-stereo.ts:61-370).

    All views' images live in one device array and all packed depth maps (u32 per pixel) in one
    device buffer, so the geometric pass and the consistency filter can read any neighbour.
    """

    def __init__(self, width: int, height: int, views: Sequence[StereoView],
                 options: StereoOptions | None = None, sizes: Sequence[tuple[int, int]] | None = None):
        """sizes: per-view (width, height) when the views differ in size (width/height are then
        only a default); None gives every view width x height as in the reference."""
        self._lib = _lib.load()
        o = options or StereoOptions()
        self.width = int(width)
        self.height = int(height)
        self.views = list(views)
        self.sizes = ([(int(w), int(h)) for w, h in sizes] if sizes is not None
                      else [(self.width, self.height)] * len(self.views))
        if len(self.sizes) != len(self.views):
            raise ValueError("one size per view")
        self._hyp_ref = 0
        self._filtered_ref = 0
        self.options = o
        copts = _lib.StereoOpts()
        self._lib.l3d_stereo_opts_default(C.byref(copts))
        copts.coarse = o.coarse._handle if o.coarse is not None else None
        copts.depth_maps = int(bool(o.depth_maps))
        copts.storage = int(o.storage)
        copts.form = int(o.form)
        copts.window = int(o.window)
        copts.dilation = int(o.dilation)
        copts.stream = o.stream
        copts.compensated = int(bool(o.compensated))
        self._coarse = o.coarse  # the coarse level must outlive this one
        h = C.c_void_p()
        cviews = _c_views(self.views)
        csizes = (C.c_int32 * (2 * len(self.views)))(*[v for wh in self.sizes for v in wh])
        _lib.check(self._lib.l3d_stereo_create_sized(len(self.views), cviews, csizes,
                                                     C.byref(copts), C.byref(h)))
        self._handle = h

    @property
    def pixels(self) -> int:
        return self.width * self.height

    def shape(self, layer: int) -> tuple[int, int]:
        """(height, width) of one view."""
        if not 0 <= int(layer) < len(self.sizes):
            raise _lib.L3dError(_lib.L3D_EINVAL, f"layer {layer} out of range [0, {len(self.sizes)})")
        w, h = self.sizes[int(layer)]
        return h, w

    def _h(self):
        if self._handle is None:
            raise RuntimeError("DenseStereo used after destroy()")
        return self._handle

    def set_image(self, layer: int, gray: np.ndarray) -> None:
        """setImage (dense-stereo.ts:175-182); u8 (r8unorm), float32, float16 or bfloat16 bits."""
        a = np.ascontiguousarray(gray)
        h, w = self.shape(layer)
        if a.shape[-2:] != (h, w) and a.size != h * w:
            raise ValueError(f"image shape {a.shape} does not match {h}x{w}")
        dtype = {np.dtype(np.uint8): _lib.DTYPE_U8, np.dtype(np.float32): _lib.DTYPE_F32,
                 np.dtype(np.float16): _lib.DTYPE_F16}.get(a.dtype)
        if dtype is None:
            raise TypeError(f"unsupported image dtype {a.dtype}")
        _lib.check(self._lib.l3d_stereo_set_image(self._h(), int(layer), dtype, _lib.ptr(a), 0))

    def set_image_device(self, layer: int, data_ptr: int, dtype: int, row_stride: int = 0) -> None:
        """Uploads from a host pointer of the given library dtype (pinned memory stays async)."""
        _lib.check(self._lib.l3d_stereo_set_image(self._h(), int(layer), int(dtype),
                                                  C.c_void_p(data_ptr), int(row_stride)))

    def solve(self, ref: int, options: SolveOptions) -> None:
        """solve (dense-stereo.ts:185-239): init, red/black iterations, pack."""
        h, w = self.shape(ref)
        args = _SolveArgs(options, h * w)
        _lib.check(self._lib.l3d_stereo_solve(self._h(), int(ref), C.byref(args.c)))
        self._hyp_ref = int(ref)
        if args.prior is not None:
            self.synchronize()  # the prior may be pinned; keep it alive until copied

    def solve_all(self, refs: Sequence[int], options: Sequence[SolveOptions]) -> None:
        """The photometric stage for many reference views in one call."""
        args = [_SolveArgs(o, int(np.prod(self.shape(r)))) for r, o in zip(refs, options)]
        arr = (_lib.SolveOpts * len(args))(*[a.c for a in args])
        crefs = (C.c_int32 * len(refs))(*[int(r) for r in refs])
        _lib.check(self._lib.l3d_stereo_solve_all(self._h(), len(refs), crefs, arr))
        if any(a.prior is not None for a in args):
            self.synchronize()

    def dispatch(self, kernel: int, ref: int, options: SolveOptions, iteration: int = 0,
                 phase: int = 0) -> None:
        """One kernel over the whole image (the unit DenseStereo.sliced submits)."""
        args = _SolveArgs(options, int(np.prod(self.shape(ref))))
        _lib.check(self._lib.l3d_stereo_dispatch(self._h(), int(kernel), int(ref), C.byref(args.c),
                                                 int(iteration), int(phase)))
        self._hyp_ref = int(ref)
        if args.prior is not None:
            self.synchronize()

    @property
    def hypotheses(self) -> np.ndarray:
        """The current per-pixel planes (dense-stereo.ts:242-244), read back: (H, W, 4)."""
        hyp = np.empty(self.shape(self._hyp_ref) + (4,), dtype=np.float32)
        _lib.check(self._lib.l3d_stereo_read_hyp(self._h(), _lib.ptr(hyp), None))
        return hyp

    def read_hypotheses(self) -> tuple[np.ndarray, np.ndarray]:
        shape = self.shape(self._hyp_ref)
        hyp = np.empty(shape + (4,), dtype=np.float32)
        cost = np.empty(shape, dtype=np.float32)
        _lib.check(self._lib.l3d_stereo_read_hyp(self._h(), _lib.ptr(hyp), _lib.ptr(cost)))
        return hyp, cost

    def read_hypotheses_layer(self, layer: int) -> tuple[np.ndarray, np.ndarray]:
        shape = self.shape(layer)
        hyp = np.empty(shape + (4,), dtype=np.float32)
        cost = np.empty(shape, dtype=np.float32)
        _lib.check(self._lib.l3d_stereo_read_hyp_layer(self._h(), int(layer), _lib.ptr(hyp),
                                                       _lib.ptr(cost)))
        return hyp, cost

    def write_hypotheses(self, hyp: np.ndarray | None, cost: np.ndarray | None) -> None:
        h = None if hyp is None else np.ascontiguousarray(hyp, dtype=np.float32)
        c = None if cost is None else np.ascontiguousarray(cost, dtype=np.float32)
        _lib.check(self._lib.l3d_stereo_write_hyp(self._h(), _lib.ptr(h), _lib.ptr(c)))
        self.synchronize()

    def write_depth_map(self, ref: int, packed: np.ndarray) -> None:
        p = np.ascontiguousarray(packed, dtype=np.uint32)
        _lib.check(self._lib.l3d_stereo_write_depth(self._h(), int(ref), _lib.ptr(p)))
        self.synchronize()

    def filter(self, ref: int, sources: Sequence[int], needed: int) -> None:
        """filter (dense-stereo.ts:250-263): consistency check of depths[ref] into `filtered`."""
        src = (C.c_int32 * max(1, len(sources)))(*[int(s) for s in sources])
        _lib.check(self._lib.l3d_stereo_filter(self._h(), int(ref), src, len(sources), int(needed)))
        self._filtered_ref = int(ref)

    def filter_all(self, refs: Sequence[int], checks: Sequence[Sequence[int]],
                   needed: Sequence[int]) -> None:
        """filter() for many views into per-view filtered maps."""
        n = len(refs)
        table = np.full((n, MAX_SOURCES), -1, dtype=np.int32)
        for i, c in enumerate(checks):
            c = list(c)[:MAX_SOURCES]
            table[i, :len(c)] = c
        r = np.asarray(refs, dtype=np.int32)
        nd = np.asarray(needed, dtype=np.int32)
        _lib.check(self._lib.l3d_stereo_filter_all(
            self._h(), n, r.ctypes.data_as(C.POINTER(C.c_int32)),
            table.ctypes.data_as(C.POINTER(C.c_int32)), nd.ctypes.data_as(C.POINTER(C.c_int32))))

    def filtered_map(self, ref: int, sources: Sequence[int], needed: int) -> np.ndarray:
        """filteredMap (dense-stereo.ts:301-306): filter, then read back (H, W) u32."""
        self.filter(ref, sources, needed)
        return self.read_filtered()

    def read_filtered(self) -> np.ndarray:
        out = np.empty(self.shape(self._filtered_ref), dtype=np.uint32)
        _lib.check(self._lib.l3d_stereo_read_filtered(self._h(), _lib.ptr(out)))
        return out

    def read_filtered_layer(self, layer: int) -> np.ndarray:
        out = np.empty(self.shape(layer), dtype=np.uint32)
        _lib.check(self._lib.l3d_stereo_read_filtered_layer(self._h(), int(layer), _lib.ptr(out)))
        return out

    def read_filtered_all_async(self, out) -> None:
        """Queues the copy of every view's filter_all map (concatenated in layer order) into the
        host buffer `out` (u32 or i32, at least the views' total pixels; pinned memory, e.g. a
        pinned torch tensor, overlaps with other work); `out` holds them after synchronize()."""
        total = int(sum(w * h for w, h in self.sizes))
        if isinstance(out, np.ndarray):
            ok, addr = out.flags.c_contiguous and out.size >= total and out.itemsize == 4, out.ctypes.data
        else:
            ok = (not out.is_cuda) and out.is_contiguous() and out.numel() >= total and out.element_size() == 4
            addr = out.data_ptr()
        if not ok:
            raise ValueError(f"host buffer must be contiguous with >= {total} 4-byte elements")
        _lib.check(self._lib.l3d_stereo_read_filtered_all_async(self._h(), C.c_void_p(addr)))

    def depth_map(self, ref: int) -> np.ndarray:
        """depthMap (dense-stereo.ts:309-312): raw packed map of one view, (H, W) u32."""
        out = np.empty(self.shape(ref), dtype=np.uint32)
        _lib.check(self._lib.l3d_stereo_read_depth(self._h(), int(ref), _lib.ptr(out)))
        return out

    def plane_cost(self, ref: int, options: SolveOptions, planes: np.ndarray,
                   view_costs: bool = False):
        """hypothesis_cost of given planes (H, W, 4) at every pixel of view `ref`."""
        shape = self.shape(ref)
        args = _SolveArgs(options, shape[0] * shape[1])
        pl = np.ascontiguousarray(planes, dtype=np.float32)
        cost = np.empty(shape, dtype=np.float32)
        vc = np.empty(shape + (MAX_SOURCES,), dtype=np.float32) if view_costs else None
        _lib.check(self._lib.l3d_stereo_plane_cost(self._h(), int(ref), C.byref(args.c),
                                                   _lib.ptr(pl), _lib.ptr(cost), _lib.ptr(vc)))
        return (cost, vc) if view_costs else cost

    def buffers(self) -> _lib.StereoBuffers:
        b = _lib.StereoBuffers()
        _lib.check(self._lib.l3d_stereo_buffers_get(self._h(), C.byref(b)))
        return b

    @property
    def stream(self) -> int:
        s = C.c_void_p()
        _lib.check(self._lib.l3d_stereo_stream(self._h(), C.byref(s)))
        return s.value or 0

    @property
    def launches(self) -> int:
        return int(self._lib.l3d_stereo_launches(self._h()))

    @property
    def variant(self) -> int:
        """Batched-form kernel variant: texture-sampled window rows + 8 x quad lane mapping
        + 16 x texture gathers with exact weights + 32 x the window in shared memory."""
        return int(self._lib.l3d_stereo_variant(self._h()))

    @variant.setter
    def variant(self, v: int) -> None:
        _lib.check(self._lib.l3d_stereo_set_variant(self._h(), int(v)))

    def autotune(self, refs: Sequence[int], options: Sequence[SolveOptions]) -> tuple[int, float]:
        """Times each variant on up to three iterations of this batch; keeps the fastest."""
        args = [_SolveArgs(o, int(np.prod(self.shape(r)))) for r, o in zip(refs, options)]
        arr = (_lib.SolveOpts * len(args))(*[a.c for a in args])
        crefs = (C.c_int32 * len(refs))(*[int(r) for r in refs])
        best, ms = C.c_int32(), C.c_float()
        _lib.check(self._lib.l3d_stereo_autotune(self._h(), len(refs), crefs, arr, C.byref(best),
                                                 C.byref(ms)))
        return best.value, ms.value

    def set_graphs(self, enable: bool) -> None:
        """Replay batched solves from CUDA graphs (fast form)."""
        _lib.check(self._lib.l3d_stereo_set_graphs(self._h(), int(bool(enable))))

    def synchronize(self) -> None:
        _lib.check(self._lib.l3d_stereo_synchronize(self._h()))

    def destroy(self) -> None:
        """destroy (dense-stereo.ts:357-370)."""
        if self._handle is not None:
            self._lib.l3d_stereo_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


# ---- stereo methods (mvs/methods/) -------------------------------------------------------

@dataclass
class StereoInput:
    """StereoInput (methods/stereo-method.ts:4-18)."""

    width: int
    height: int
    views: Sequence[StereoView]
    sources: Sequence[Sequence[int]]
    ranges: Sequence[tuple[float, float]]
    gray: Callable[[int, int, int], np.ndarray]
    prior: Callable[[int, int, int], np.ndarray | None] = lambda layer, w, h: None


@dataclass
class StereoSettings:
    """StereoSettings (methods/stereo-method.ts:20-24)."""

    iterations: int
    fine_iterations: int = 0
    options: StereoOptions = field(default_factory=StereoOptions)


class StereoRun:
    """StereoRun (methods/stereo-method.ts:34-39)."""

    def __init__(self, stereo: DenseStereo, solve: Callable[[int], None],
                 destroy: Callable[[], None]):
        self.stereo = stereo
        self._solve = solve
        self._destroy = destroy

    def solve(self, layer: int) -> None:
        self._solve(layer)

    def destroy(self) -> None:
        self._destroy()


def upload_images(stereo: DenseStereo, inp: StereoInput) -> None:
    """uploadImages (methods/stereo-method.ts:27-31)."""
    for layer in range(len(inp.views)):
        stereo.set_image(layer, inp.gray(layer, stereo.width, stereo.height))


def _single_scale(inp: StereoInput, settings: StereoSettings) -> StereoRun:
    """single-scale (methods/single-scale.ts:5-27)."""
    stereo = DenseStereo(inp.width, inp.height, inp.views, settings.options)
    try:
        upload_images(stereo, inp)
    except Exception:
        stereo.destroy()
        raise

    def solve(layer: int) -> None:
        stereo.solve(layer, SolveOptions(
            sources=inp.sources[layer], min_depth=inp.ranges[layer][0],
            max_depth=inp.ranges[layer][1], prior=inp.prior(layer, inp.width, inp.height),
            geometric=False, iterations=settings.iterations))

    return StereoRun(stereo, solve, stereo.destroy)


def _coarse_to_fine(inp: StereoInput, settings: StereoSettings) -> StereoRun:
    """coarse-to-fine (methods/coarse-to-fine.ts:9-68): half resolution first, then full
    resolution seeded by the coarse planes."""
    cw, ch = round(inp.width / 2), round(inp.height / 2)
    coarse_views = [StereoView(scale_intrinsics(v.intrinsics, cw / inp.width, ch / inp.height), v.pose)
                    for v in inp.views]
    copts = StereoOptions(depth_maps=False, storage=settings.options.storage,
                          form=settings.options.form, window=settings.options.window,
                          dilation=settings.options.dilation,
                          compensated=settings.options.compensated)
    coarse = DenseStereo(cw, ch, coarse_views, copts)
    fopts = StereoOptions(coarse=coarse, storage=settings.options.storage, form=settings.options.form,
                          window=settings.options.window, dilation=settings.options.dilation,
                          compensated=settings.options.compensated)
    stereo = DenseStereo(inp.width, inp.height, inp.views, fopts)
    try:
        upload_images(coarse, inp)
        upload_images(stereo, inp)
    except Exception:
        stereo.destroy()
        coarse.destroy()
        raise

    def solve(layer: int) -> None:
        lo, hi = inp.ranges[layer]
        coarse.solve(layer, SolveOptions(sources=inp.sources[layer], min_depth=lo, max_depth=hi,
                                         prior=inp.prior(layer, cw, ch), geometric=False,
                                         iterations=settings.iterations, pack=False))
        stereo.solve(layer, SolveOptions(sources=inp.sources[layer], min_depth=lo, max_depth=hi,
                                         prior=None, geometric=False,
                                         iterations=settings.fine_iterations, from_coarse=True))

    def destroy() -> None:
        # the fine level reads the coarse planes: release them together
        stereo.destroy()
        coarse.destroy()

    return StereoRun(stereo, solve, destroy)


class StereoMethod:
    """StereoMethod (methods/stereo-method.ts:42-44)."""

    def __init__(self, create: Callable[[StereoInput, StereoSettings], StereoRun]):
        self.create = create


# STEREO_METHODS (methods/index.ts:7-10)
STEREO_METHODS: dict[str, StereoMethod] = {
    "single-scale": StereoMethod(_single_scale),
    "coarse-to-fine": StereoMethod(_coarse_to_fine),
}
