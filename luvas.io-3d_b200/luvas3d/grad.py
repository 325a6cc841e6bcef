"""Differentiable multi-view NCC cost and TSDF integration, for plane and pose polishing.

torch.autograd.Function wrappers over the adjoint entry points of include/luvas3d.h
(l3d_ncc_forward / l3d_ncc_backward, l3d_tsdf_forward_depth / l3d_tsdf_backward).  The reference
scanner has no gradients; its PatchMatch stops at the discrete search.  These functions give
the gradients that polish the planes it finds, and the camera poses, afterwards.

Tensors are CUDA tensors; the kernels run on torch's current stream.

NCC objective of a reference view: per pixel, the sum over the sources of view_cost
(mvs/patchmatch.wgsl.ts:130-159), the bilateral-weighted 1 - NCC over the handle's window.
  planes  (H, W, 3) float32: z-depth d and normal angles (a, b),
          n = (sin a cos b, sin b, -cos a cos b)
  deltas  (V, 6) float32 se(3) increments (v, w) of every view's pose:
          X -> Exp(w) (R X + t) + v with (R, t) the handle's pose
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Sequence

import numpy as np
import torch

from . import _lib
from .stereo import DenseStereo
from .tsdf import IntegrationView, TsdfVolume, _c_view


# cudaStreamLegacy: the legacy default stream named explicitly (a NULL stream would mean the
# handle's own stream to the C ABI, which does not synchronise with torch's default stream)
_LEGACY_STREAM = 1


def _stream() -> C.c_void_p:
    """torch's current stream as a cudaStream_t for the C ABI."""
    s = torch.cuda.current_stream().cuda_stream
    return C.c_void_p(s if s else _LEGACY_STREAM)


def _ptr(t: torch.Tensor | None):
    return None if t is None else C.c_void_p(t.data_ptr())


def _check_cuda(name: str, t: torch.Tensor, dtype=None, shape=None) -> None:
    if not t.is_cuda or not t.is_contiguous():
        raise ValueError(f"{name} must be a contiguous CUDA tensor")
    if dtype is not None and t.dtype != dtype:
        raise ValueError(f"{name} must be {dtype}, got {t.dtype}")
    if shape is not None and tuple(t.shape) != tuple(shape):
        raise ValueError(f"{name} must have shape {tuple(shape)}, got {tuple(t.shape)}")


# ------------------------------------------------------------------ planes ------------------

def planes_from_hypotheses(hyp) -> torch.Tensor:
    """(H, W, 4) hypotheses (normal xyz, depth) -> (H, W, 3) planes (depth, a, b)."""
    h = torch.as_tensor(np.asarray(hyp) if not isinstance(hyp, torch.Tensor) else hyp,
                        dtype=torch.float64)
    n = h[..., :3]
    n = n / n.norm(dim=-1, keepdim=True).clamp_min(1e-12)
    b = torch.asin(n[..., 1].clamp(-1.0, 1.0))
    a = torch.atan2(n[..., 0], -n[..., 2])
    return torch.stack([h[..., 3], a, b], dim=-1).to(torch.float32)


def normals_from_planes(planes: torch.Tensor) -> torch.Tensor:
    a, b = planes[..., 1], planes[..., 2]
    return torch.stack([torch.sin(a) * torch.cos(b), torch.sin(b), -torch.cos(a) * torch.cos(b)], -1)


# ------------------------------------------------------------------ NCC ---------------------

def _sources(ref: int, sources: Sequence[int]):
    src = np.ascontiguousarray(list(sources), dtype=np.int32)
    if not 1 <= src.size <= _lib.MAX_SOURCES:
        raise ValueError(f"1..{_lib.MAX_SOURCES} sources, got {src.size}")
    return src


def _ncc_call(stereo: DenseStereo, ref: int, sources, planes, deltas, grad_cost, want_planes,
              want_deltas):
    h, w = stereo.shape(ref)
    _check_cuda("planes", planes, torch.float32, (h, w, 3))
    if deltas is not None:
        _check_cuda("deltas", deltas, torch.float32, (len(stereo.sizes), 6))
    src = _sources(ref, sources)
    cost = torch.empty((h, w), dtype=torch.float32, device=planes.device)
    gp = torch.empty_like(planes) if want_planes else None
    gd = torch.zeros((len(stereo.sizes), 6), dtype=torch.float64, device=planes.device) if want_deltas else None
    lib = _lib.load()
    sp = src.ctypes.data_as(C.POINTER(C.c_int32))
    if gp is None and gd is None:
        _lib.check(lib.l3d_ncc_forward(stereo._h(), int(ref), sp, int(src.size), _ptr(planes),
                                       _ptr(deltas), _ptr(cost), _stream()))
    else:
        if grad_cost is not None:
            _check_cuda("grad_cost", grad_cost, torch.float32, (h, w))
        _lib.check(lib.l3d_ncc_backward(stereo._h(), int(ref), sp, int(src.size), _ptr(planes),
                                        _ptr(deltas), _ptr(grad_cost), _ptr(cost), _ptr(gp),
                                        _ptr(gd), _stream()))
    return cost, gp, gd


class NccCost(torch.autograd.Function):
    """Per-pixel summed NCC cost of one reference view; the backward pass recomputes the warped
    window samples (nothing but the inputs is saved)."""

    @staticmethod
    def forward(ctx, planes, deltas, stereo, ref, sources):
        cost, _, _ = _ncc_call(stereo, ref, sources, planes, deltas, None, False, False)
        ctx.stereo, ctx.ref, ctx.sources = stereo, ref, sources
        ctx.save_for_backward(planes, deltas)
        return cost

    @staticmethod
    def backward(ctx, grad_cost):
        planes, deltas = ctx.saved_tensors
        want_p = ctx.needs_input_grad[0]
        want_d = deltas is not None and ctx.needs_input_grad[1]
        if not (want_p or want_d):
            return None, None, None, None, None
        _, gp, gd = _ncc_call(ctx.stereo, ctx.ref, ctx.sources, planes, deltas,
                              grad_cost.contiguous().to(torch.float32), want_p, want_d)
        return gp, (gd.to(torch.float32) if want_d else None), None, None, None


def ncc_cost(stereo: DenseStereo, ref: int, sources: Sequence[int], planes: torch.Tensor,
             deltas: torch.Tensor | None = None) -> torch.Tensor:
    """(H, W) summed NCC cost of view `ref` over `sources`, differentiable in planes and deltas."""
    return NccCost.apply(planes, deltas, stereo, int(ref), tuple(int(s) for s in sources))


def ncc_value_and_grad(stereo: DenseStereo, ref: int, sources: Sequence[int], planes: torch.Tensor,
                       deltas: torch.Tensor | None = None, weights: torch.Tensor | None = None,
                       grad_deltas: torch.Tensor | None = None):
    """One pass: cost (H, W) and the gradients of sum(weights * cost) (weights None = ones) with
    respect to planes (H, W, 3) and, when grad_deltas (V, 6 float64) is given, the deltas (added
    into grad_deltas).  Returns (cost, grad_planes)."""
    h, w = stereo.shape(ref)
    _check_cuda("planes", planes, torch.float32, (h, w, 3))
    if deltas is not None:
        _check_cuda("deltas", deltas, torch.float32, (len(stereo.sizes), 6))
    if grad_deltas is not None:
        _check_cuda("grad_deltas", grad_deltas, torch.float64, (len(stereo.sizes), 6))
    if weights is not None:
        _check_cuda("weights", weights, torch.float32, (h, w))
    src = _sources(ref, sources)
    cost = torch.empty((h, w), dtype=torch.float32, device=planes.device)
    gp = torch.empty_like(planes)
    _lib.check(_lib.load().l3d_ncc_backward(
        stereo._h(), int(ref), src.ctypes.data_as(C.POINTER(C.c_int32)), int(src.size),
        _ptr(planes), _ptr(deltas), _ptr(weights), _ptr(cost), _ptr(gp), _ptr(grad_deltas),
        _stream()))
    return cost, gp


# ------------------------------------------------------------------ TSDF --------------------

def _view_struct(view: IntegrationView, keep: list):
    v = IntegrationView(view.intrinsics, view.pose, view.max_depth, None, view.confidence)
    return _c_view(v, keep)


class TsdfIntegrateDepth(torch.autograd.Function):
    """Out-of-place TSDF integration of one view with an FP32 depth map; differentiable in the
    depth map and the volume state before the update (tsdf and, for f32 weights, weight)."""

    @staticmethod
    def forward(ctx, depth, tsdf, weight, volume, view, packed, prior):
        keep: list = []
        cv = _view_struct(view, keep)
        h, w = depth.shape
        tsdf_out = torch.empty_like(tsdf)
        weight_out = torch.empty_like(weight)
        _lib.check(_lib.load().l3d_tsdf_forward_depth(
            volume._h(), C.byref(cv), int(w), int(h), _ptr(packed), _ptr(depth), _ptr(prior),
            _ptr(tsdf), _ptr(weight), _ptr(tsdf_out), _ptr(weight_out), _stream()))
        ctx.volume, ctx.view = volume, view
        ctx.save_for_backward(depth, tsdf, weight, packed, prior)
        if volume.weight_q8:
            ctx.mark_non_differentiable(weight_out)
        return tsdf_out, weight_out

    @staticmethod
    def backward(ctx, g_tsdf, g_weight):
        depth, tsdf, weight, packed, prior = ctx.saved_tensors
        volume = ctx.volume
        keep: list = []
        cv = _view_struct(ctx.view, keep)
        h, w = depth.shape
        if g_tsdf is None:
            g_tsdf = torch.zeros_like(tsdf)
        g_tsdf = g_tsdf.contiguous()
        gw = None
        if not volume.weight_q8 and g_weight is not None:
            gw = g_weight.contiguous()
        grad_depth = torch.zeros_like(depth) if ctx.needs_input_grad[0] else None
        grad_tsdf = torch.empty_like(tsdf) if ctx.needs_input_grad[1] else None
        grad_weight = (torch.empty_like(weight) if (ctx.needs_input_grad[2] and not volume.weight_q8)
                       else None)
        if grad_depth is not None or grad_tsdf is not None or grad_weight is not None:
            _lib.check(_lib.load().l3d_tsdf_backward(
                volume._h(), C.byref(cv), int(w), int(h), _ptr(packed), _ptr(depth), _ptr(prior),
                _ptr(tsdf), _ptr(weight), _ptr(g_tsdf), _ptr(gw), _ptr(grad_depth),
                _ptr(grad_tsdf), _ptr(grad_weight), _stream()))
        return grad_depth, grad_tsdf, grad_weight, None, None, None, None


def integrate_depth(volume: TsdfVolume, view: IntegrationView, packed: torch.Tensor,
                    depth: torch.Tensor, tsdf: torch.Tensor, weight: torch.Tensor,
                    prior: torch.Tensor | None = None):
    """(tsdf_out, weight_out) after integrating `view` with depths from `depth` (H, W float32);
    `packed` (H, W, 4-byte integers holding the packed samples) gives validity, normals and
    costs.  tsdf / weight are flat volume tensors laid out like the handle's volume
    (float32; weights float32, or 2-byte Q8.8 for a Q8 volume).  The handle's own volume is not
    touched."""
    h, w = depth.shape
    _check_cuda("depth", depth, torch.float32)
    _check_cuda("packed", packed, shape=(h, w))
    if packed.element_size() != 4:
        raise ValueError("packed must hold 4-byte packed samples")
    n = volume.voxels
    _check_cuda("tsdf", tsdf, torch.float32, (n,))
    _check_cuda("weight", weight, shape=(n,))
    if weight.element_size() != (2 if volume.weight_q8 else 4):
        raise ValueError("weight element size does not match the volume's weight type")
    if prior is not None:
        _check_cuda("prior", prior, torch.float32, (h, w))
    return TsdfIntegrateDepth.apply(depth, tsdf, weight, volume, view, packed, prior)


# ------------------------------------------------------------------ polishing ---------------

@dataclass
class PolishResult:
    planes: list                     # per reference view, (H, W, 3) float32 tensors
    deltas: torch.Tensor             # (V, 6) float32
    losses: list = field(default_factory=list)
    ms_per_step: float = 0.0


def polish(stereo: DenseStereo, refs: Sequence[int], sources: Sequence[Sequence[int]],
           planes: Sequence[torch.Tensor], steps: int = 20, lr_depth: float = 2e-3,
           lr_angle: float = 1e-2, lr_trans: float = 5e-4, lr_rot: float = 5e-4,
           fixed: Sequence[int] = (0,), weights: Sequence[torch.Tensor] | None = None,
           refine_planes: bool = True, refine_poses: bool = True) -> PolishResult:
    """Adam on the planes of `refs` and on every view's pose increment, minimising the mean over
    the reference views of the weighted mean per-pixel NCC cost.  Views in `fixed` keep their
    pose (they fix the gauge).  Each step is one gradient pass per reference view."""
    dev = planes[0].device
    V = len(stereo.sizes)
    depth = [p[..., :1].clone().requires_grad_(refine_planes) for p in planes]
    angle = [p[..., 1:].clone().requires_grad_(refine_planes) for p in planes]
    dv = torch.zeros((V, 3), dtype=torch.float32, device=dev, requires_grad=refine_poses)
    dw = torch.zeros((V, 3), dtype=torch.float32, device=dev, requires_grad=refine_poses)
    groups = []
    if refine_planes:
        groups += [{"params": depth, "lr": lr_depth}, {"params": angle, "lr": lr_angle}]
    if refine_poses:
        groups += [{"params": [dv], "lr": lr_trans}, {"params": [dw], "lr": lr_rot}]
    opt = torch.optim.Adam(groups)
    keep = torch.ones(V, 1, device=dev)
    for f in fixed:
        keep[int(f)] = 0.0
    if weights is None:
        weights = [torch.ones(p.shape[:2], dtype=torch.float32, device=dev) for p in planes]
    scale = [w / (w.sum().clamp_min(1.0) * len(refs)) for w in weights]
    out = PolishResult(planes=[], deltas=torch.zeros(V, 6, device=dev))
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    start.record()
    for step in range(steps + 1):
        with torch.no_grad():
            deltas = torch.cat([dv, dw], 1).contiguous()
            gd = torch.zeros((V, 6), dtype=torch.float64, device=dev)
            loss = torch.zeros((), dtype=torch.float64, device=dev)
            grads = []
            for i, r in enumerate(refs):
                pl = torch.cat([depth[i], angle[i]], -1).contiguous()
                cost, gp = ncc_value_and_grad(stereo, r, sources[i], pl, deltas, scale[i].contiguous(),
                                              gd if refine_poses else None)
                loss += (cost.double() * scale[i]).sum()
                grads.append(gp)
        out.losses.append(loss)
        if step == steps:
            break
        opt.zero_grad(set_to_none=False)
        if refine_planes:
            for i in range(len(refs)):
                depth[i].grad = grads[i][..., :1].contiguous()
                angle[i].grad = grads[i][..., 1:].contiguous()
        if refine_poses:
            g = gd.to(torch.float32) * keep
            dv.grad = g[:, :3].contiguous()
            dw.grad = g[:, 3:].contiguous()
        opt.step()
    end.record()
    torch.cuda.synchronize()
    out.ms_per_step = start.elapsed_time(end) / max(1, steps + 1)
    out.losses = [float(l) for l in out.losses]
    with torch.no_grad():
        out.planes = [torch.cat([d, a], -1).detach().contiguous() for d, a in zip(depth, angle)]
        out.deltas = torch.cat([dv, dw], 1).detach().contiguous()
    return out


def apply_deltas(views, deltas) -> list:
    """Poses after the increments: R' = Exp(w) R, t' = Exp(w) t + v (FP64 on the host)."""
    from .camera import Pose, StereoView
    d = np.asarray(deltas.detach().cpu() if isinstance(deltas, torch.Tensor) else deltas,
                   dtype=np.float64).reshape(-1, 6)
    out = []
    for v, (vx, vy, vz, wx, wy, wz) in zip(views, d):
        E = so3_exp(np.array([wx, wy, wz]))
        R = E @ np.asarray(v.pose.R, dtype=np.float64)
        t = E @ np.asarray(v.pose.t, dtype=np.float64) + np.array([vx, vy, vz])
        out.append(StereoView(v.intrinsics, Pose(R, t)))
    return out


def so3_exp(w: np.ndarray) -> np.ndarray:
    th = float(np.linalg.norm(w))
    K = np.array([[0, -w[2], w[1]], [w[2], 0, -w[0]], [-w[1], w[0], 0]], dtype=np.float64)
    if th < 1e-8:
        return np.eye(3) + K + 0.5 * K @ K
    return np.eye(3) + np.sin(th) / th * K + (1 - np.cos(th)) / th ** 2 * K @ K
