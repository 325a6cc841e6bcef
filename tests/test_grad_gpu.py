"""Gradient kernels (grad.cu, the adjoint in tsdf.cu) against the FP64 dual-number oracle and
central differences, through the C ABI and the torch.autograd wrappers.

Tolerances: per-pixel gradients within 1e-3 relative (to the larger of |g| and the median |g|)
on at least 99.5% of the pixels whose windows stay half a texel inside every source; the rest
are samples that FP32 and FP64 place in different texel cells (the bilinear interpolant has a
kink at every texel edge).  Pose gradients, sums over all pixels, within 1e-3 of their block's
norm.  NCC cost within 1e-4 per source.
"""
import numpy as np
import pytest

import oracle
from helpers import arc_workload

torch = pytest.importorskip("torch")

from luvas3d import (DTYPE_F16, FORM_FAST, DenseStereo, IntegrationView, StereoOptions,  # noqa: E402
                     TsdfVolume)
from luvas3d import grad as G  # noqa: E402

pytestmark = pytest.mark.gpu

SOURCES = [1, 2, 3]
H_STEP = 1e-4


def _rel(err, g):
    return np.abs(err) / np.maximum(np.abs(g), np.median(np.abs(g)))


@pytest.fixture(scope="module")
def scene():
    views, imgs, truth, _ = arc_workload(n=4, W=128, H=96, f=112.0, step_deg=6.0, seed=5)
    rng = np.random.default_rng(0)
    d = np.where(truth[0] > 0, truth[0], 2.0)
    planes = np.stack([d, rng.uniform(-0.3, 0.3, d.shape), rng.uniform(-0.3, 0.3, d.shape)], -1)
    planes = planes.astype(np.float32)
    deltas = rng.normal(scale=1e-3, size=(4, 6)).astype(np.float32)
    s = DenseStereo(128, 96, views)
    for i, im in enumerate(imgs):
        s.set_image(i, im)
    o = oracle.NccGrad(views, imgs)
    _, margin, _ = o.structure(0, SOURCES, planes.astype(np.float64), deltas.astype(np.float64))
    return views, imgs, planes, deltas, s, o, margin > 0.5


def _cuda(a):
    return torch.tensor(np.ascontiguousarray(a), device="cuda")


def test_ncc_cost_matches_fp64_oracle(scene):
    """FP32 cost against the FP64 objective: as close as the reference's own FP32 arithmetic
    (the FP32 oracle) comes on the same planes.  On this finely textured scene that is 1e-4 per
    source on 99% of the pixels; FP32 rounding of the window sums, amplified where a window has
    little variance, leaves a tail of a few 1e-3."""
    views, imgs, planes, deltas, s, o, valid = scene
    cost = G.ncc_cost(s, 0, SOURCES, _cuda(planes), _cuda(deltas)).cpu().numpy()
    want, _, _ = o(0, SOURCES, planes, deltas)
    err = np.abs(cost - want)[valid]
    # the reference arithmetic's own spread on the same planes (no pose increments)
    a, b = planes[..., 1].astype(np.float64), planes[..., 2].astype(np.float64)
    n = np.stack([np.sin(a) * np.cos(b), np.sin(b), -np.cos(a) * np.cos(b)], -1)
    pl4 = np.concatenate([n, planes[..., :1]], -1)
    c32, v32 = oracle.Stereo(128, 96, views, imgs, 32).plane_cost(
        0, SOURCES, pl4.astype(np.float32), min_depth=0.1, max_depth=10.0)
    c64, v64 = oracle.Stereo(128, 96, views, imgs, 64).plane_cost(
        0, SOURCES, pl4.astype(np.float32).astype(np.float64), min_depth=0.1, max_depth=10.0)
    ok = (v64[..., :3] < 1.5).all(-1) & (v64[..., :3] > 0).all(-1) & (c64 < 2)
    ref_err = np.abs(v32[..., :3].sum(-1) - v64[..., :3].sum(-1))[ok]
    assert np.mean(err <= 1e-4 * len(SOURCES)) >= 0.99, np.percentile(err, 99.9)
    assert err.max() <= 2 * ref_err.max() + 1e-4, (err.max(), ref_err.max())
    # pixels without a valid plane or window keep the constants exactly
    np.testing.assert_array_equal(cost[want == 2.0 * len(SOURCES)], 2.0 * len(SOURCES))


def test_ncc_plane_gradient_matches_fp64_oracle(scene):
    views, imgs, planes, deltas, s, o, valid = scene
    cost, gp = G.ncc_value_and_grad(s, 0, SOURCES, _cuda(planes), _cuda(deltas))
    gp = gp.cpu().numpy()
    want_cost, want, _ = o(0, SOURCES, planes, deltas, grad_planes=True)
    for j in range(3):
        rel = _rel(gp[..., j][valid] - want[..., j][valid], want[..., j][valid])
        assert np.mean(rel < 1e-3) >= 0.995, (j, np.percentile(rel, 99.5))
    # a pixel whose every source costs the constant 2 has no gradient
    assert np.all(gp[want_cost == 2.0 * len(SOURCES)] == 0)


def test_ncc_pose_gradient_matches_fp64_oracle(scene):
    views, imgs, planes, deltas, s, o, valid = scene
    w = valid.astype(np.float32)
    gd = torch.zeros((4, 6), dtype=torch.float64, device="cuda")
    G.ncc_value_and_grad(s, 0, SOURCES, _cuda(planes), _cuda(deltas), _cuda(w), gd)
    got = gd.cpu().numpy()
    _, _, want = o(0, SOURCES, planes, deltas, weights=w, grad_deltas=True)
    for v in range(4):
        for b in range(2):
            blk = slice(3 * b, 3 * b + 3)
            err = np.linalg.norm(got[v, blk] - want[v, blk]) / np.linalg.norm(want[v, blk])
            assert err < 1e-3, (v, b, got[v, blk], want[v, blk])


def test_ncc_gradient_matches_central_differences(scene):
    """The GPU adjoint against central differences (h = 1e-4) of the FP64 objective, where the
    objective is smooth over the step."""
    views, imgs, planes, deltas, s, o, valid = scene
    _, gp = G.ncc_value_and_grad(s, 0, SOURCES, _cuda(planes), _cuda(deltas))
    gp = gp.cpu().numpy()
    p64, d64 = planes.astype(np.float64), deltas.astype(np.float64)
    for j in range(3):
        pp, pm = p64.copy(), p64.copy()
        pp[..., j] += H_STEP
        pm[..., j] -= H_STEP
        cp, _, hp = o.structure(0, SOURCES, pp, d64)
        cm, _, hm = o.structure(0, SOURCES, pm, d64)
        smooth = valid & (hp == hm)
        fd = (cp - cm) / (2 * H_STEP)
        rel = _rel(gp[..., j][smooth] - fd[smooth], fd[smooth])
        assert np.mean(rel < 1e-3) >= 0.995, (j, np.percentile(rel, 99.5))


def test_autograd_function_matches_fused_call(scene):
    views, imgs, planes, deltas, s, o, valid = scene
    w = _cuda(valid.astype(np.float32))
    pl = _cuda(planes).requires_grad_(True)
    de = _cuda(deltas).requires_grad_(True)
    cost = G.ncc_cost(s, 0, SOURCES, pl, de)
    (cost * w).sum().backward()
    gd = torch.zeros((4, 6), dtype=torch.float64, device="cuda")
    c2, gp = G.ncc_value_and_grad(s, 0, SOURCES, _cuda(planes), _cuda(deltas), w, gd)
    torch.testing.assert_close(cost.detach(), c2, rtol=0, atol=0)
    torch.testing.assert_close(pl.grad, gp, rtol=0, atol=0)
    torch.testing.assert_close(de.grad, gd.float(), rtol=1e-5, atol=1e-3)


def test_ncc_gradient_f16_storage(scene):
    """FP16 image storage: the same kernels read half texels; checked against the oracle on the
    FP16-rounded images."""
    views, imgs, planes, deltas, _, _, valid = scene
    s16 = DenseStereo(128, 96, views, StereoOptions(storage=DTYPE_F16, form=FORM_FAST))
    for i, im in enumerate(imgs):
        s16.set_image(i, im)
    rounded = [im.astype(np.float16).astype(np.float32) for im in imgs]
    o16 = oracle.NccGrad(views, rounded)
    _, gp = G.ncc_value_and_grad(s16, 0, SOURCES, _cuda(planes), _cuda(deltas))
    _, want, _ = o16(0, SOURCES, planes, deltas, grad_planes=True)
    gp = gp.cpu().numpy()
    for j in range(3):
        rel = _rel(gp[..., j][valid] - want[..., j][valid], want[..., j][valid])
        assert np.mean(rel < 1e-3) >= 0.99, (j, np.percentile(rel, 99))


def test_ncc_rejects_bad_arguments(scene):
    views, imgs, planes, deltas, s, o, valid = scene
    with pytest.raises(Exception):
        G.ncc_cost(s, 0, [0, 1], _cuda(planes))           # reference listed as a source
    with pytest.raises(Exception):
        G.ncc_cost(s, 9, SOURCES, _cuda(planes))          # layer out of range
    with pytest.raises(ValueError):
        G.ncc_cost(s, 0, SOURCES, _cuda(planes[:10]))     # wrong plane shape


# ------------------------------------------------------------------ TSDF --------------------

@pytest.fixture(scope="module")
def tsdf_case():
    views, imgs, truth, _ = arc_workload(n=3, W=96, H=72, f=84.0, step_deg=6.0, seed=5)
    W, H = 96, 72
    rng = np.random.default_rng(1)
    packed = np.zeros((H, W), dtype=np.uint32)
    for y, x in zip(*np.nonzero(truth[0] > 0)):
        packed[y, x] = oracle.pack_sample(truth[0][y, x], (0.0, 0.0, -1.0), rng.uniform(0, 0.9))
    unpacked = np.vectorize(lambda p: oracle.load().orc_unpack_depth(int(p)))(packed).astype(np.float32)
    depth = (unpacked + rng.uniform(-0.003, 0.003, unpacked.shape) * (unpacked > 0)).astype(np.float32)
    dims = (48, 40, 48)
    n = int(np.prod(dims))
    t0 = rng.uniform(-1, 1, n).astype(np.float32)
    w0 = rng.uniform(0, 3, n).astype(np.float32)
    gT = rng.normal(size=n).astype(np.float32)
    gW = rng.normal(size=n).astype(np.float32)
    k = views[0].intrinsics
    vk = dict(k=(k.fx, k.fy, k.cx, k.cy), R=views[0].pose.R, t=views[0].pose.t, max_depth=5.0,
              confidence=1.5)
    iv = IntegrationView(k, views[0].pose, 5.0, None, 1.5)
    return views, packed, unpacked, depth, dims, t0, w0, gT, gW, vk, iv


def _volume(dims, q8=False):
    return TsdfVolume(96, 72, 0.05, (-1.2, -1.0, -1.2), dense=dims, truncation=0.15, weight_q8=q8)


@pytest.mark.parametrize("q8", [False, True])
def test_tsdf_forward_depth_equals_integrate(tsdf_case, q8):
    """With the packed depths as the FP32 map, the out-of-place update equals the handle's own
    integrate bit for bit."""
    views, packed, unpacked, depth, dims, t0, w0, gT, gW, vk, iv = tsdf_case
    vol = _volume(dims, q8)
    vol.integrate(iv, depth=packed)
    want_t, want_w = vol.read()
    n = vol.voxels
    t_in = torch.ones(n, device="cuda")
    w_in = torch.zeros(n, dtype=torch.int16 if q8 else torch.float32, device="cuda")
    t1, w1 = G.integrate_depth(vol, iv, _cuda(packed.view(np.int32)), _cuda(unpacked), t_in, w_in)
    assert np.array_equal(t1.cpu().numpy().view(np.uint32), want_t.reshape(-1).view(np.uint32))
    got_w = w1.cpu().numpy()
    assert np.array_equal(got_w.view(np.uint16) if q8 else got_w.view(np.uint32),
                          want_w.reshape(-1).view(np.uint16 if q8 else np.uint32))


def test_tsdf_backward_matches_fp64_oracle(tsdf_case):
    views, packed, unpacked, depth, dims, t0, w0, gT, gW, vk, iv = tsdf_case
    vol = _volume(dims)
    dt = _cuda(depth).requires_grad_(True)
    tt = _cuda(t0).requires_grad_(True)
    wt = _cuda(w0).requires_grad_(True)
    t1, w1 = G.integrate_depth(vol, iv, _cuda(packed.view(np.int32)), dt, tt, wt)
    ((t1 * _cuda(gT)).sum() + (w1 * _cuda(gW)).sum()).backward()
    desc, keep = oracle.tsdf_desc(96, 72, 0.05, (-1.2, -1.0, -1.2), 0.15, dense=dims)
    wt1, ww1, gd, gt0, gw0 = oracle.tsdf_depth(desc, vk, packed, depth.astype(np.float64), t0, w0, gT, gW)
    np.testing.assert_allclose(t1.detach().cpu().numpy(), wt1, atol=1e-5)
    np.testing.assert_allclose(w1.detach().cpu().numpy(), ww1, rtol=1e-5, atol=1e-5)
    got = dt.grad.cpu().numpy().reshape(-1)
    nz = gd != 0
    assert nz.sum() > 1000
    rel = _rel(got[nz] - gd[nz], gd[nz])
    assert np.mean(rel < 1e-3) >= 0.995, np.percentile(rel, 99.5)
    np.testing.assert_allclose(tt.grad.cpu().numpy(), gt0, rtol=1e-4, atol=1e-5)
    np.testing.assert_allclose(wt.grad.cpu().numpy(), gw0, rtol=1e-4, atol=1e-5)


def test_tsdf_autograd_chains_two_views(tsdf_case):
    """Two integrations in a row: the depth gradient of the first view flows back through the
    second update (T and W of the intermediate volume)."""
    views, packed, unpacked, depth, dims, t0, w0, gT, gW, vk, iv = tsdf_case
    k = views[1].intrinsics
    iv2 = IntegrationView(k, views[1].pose, 5.0, None, 1.5)
    vk2 = dict(k=(k.fx, k.fy, k.cx, k.cy), R=views[1].pose.R, t=views[1].pose.t, max_depth=5.0,
               confidence=1.5)
    vol = _volume(dims)
    d1 = _cuda(depth).requires_grad_(True)
    d2 = _cuda(depth[:, ::-1].copy()).requires_grad_(True)
    pk = _cuda(packed.view(np.int32))
    pk2 = _cuda(packed[:, ::-1].copy().view(np.int32))
    t1, w1 = G.integrate_depth(vol, iv, pk, d1, _cuda(t0), _cuda(w0))
    t2, w2 = G.integrate_depth(vol, iv2, pk2, d2, t1, w1)
    (t2 * _cuda(gT)).sum().backward()
    desc, keep = oracle.tsdf_desc(96, 72, 0.05, (-1.2, -1.0, -1.2), 0.15, dense=dims)
    a_t1, a_w1, _, _, _ = oracle.tsdf_depth(desc, vk, packed, depth.astype(np.float64), t0, w0)
    _, _, gd2, gt1, gw1 = oracle.tsdf_depth(desc, vk2, packed[:, ::-1].copy(),
                                            depth[:, ::-1].astype(np.float64), a_t1, a_w1, gT, None)
    _, _, gd1, _, _ = oracle.tsdf_depth(desc, vk, packed, depth.astype(np.float64), t0, w0, gt1, gw1)
    for got, want in ((d1.grad, gd1), (d2.grad, gd2)):
        got = got.cpu().numpy().reshape(-1)
        nz = want != 0
        rel = _rel(got[nz] - want[nz], want[nz])
        assert np.mean(rel < 1e-3) >= 0.995, np.percentile(rel, 99.5)
