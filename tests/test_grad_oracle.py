"""The FP64 gradient oracle (oracle/grad.cpp) against central differences of its own objective.

The oracle's derivatives come from forward-mode dual numbers over a direct FP64 restatement of
the NCC objective and of the TSDF update.  Central differences use h = 1e-4 (metres for depth and
translation, radians for angles and rotation).  The NCC objective is only piecewise smooth:
bilinear sampling has a kink at every texel edge and a window that leaves an image jumps to the
constant cost 2.  A difference quotient is therefore compared only where the objective is smooth
over [x - h, x + h]: every window sample stays in its texel cell (the oracle reports a hash of
the cells) and at least half a texel inside every source.  Along those the dual-number
derivative must match the difference quotient to 1e-3 relative.
"""
import numpy as np
import pytest

import oracle
from helpers import arc_workload

H_STEP = 1e-4
SOURCES = [1, 2, 3]


@pytest.fixture(scope="module")
def scene():
    views, imgs, truth, _ = arc_workload(n=4, W=128, H=96, f=112.0, step_deg=6.0, seed=5)
    rng = np.random.default_rng(0)
    d = np.where(truth[0] > 0, truth[0], 2.0)
    planes = np.stack([d, rng.uniform(-0.3, 0.3, d.shape), rng.uniform(-0.3, 0.3, d.shape)], -1)
    deltas = rng.normal(scale=1e-3, size=(4, 6))
    return views, imgs, planes, deltas


def _rel(err, g):
    """Error relative to the larger of |g| and the median |g| (tiny gradients are not a scale)."""
    return np.abs(err) / np.maximum(np.abs(g), np.median(np.abs(g)))


def test_oracle_cost_equals_plane_cost_oracle(scene):
    """The objective is the existing FP64 oracle's view_cost summed over the sources."""
    views, imgs, planes, _ = scene
    g = oracle.NccGrad(views, imgs)
    c, _, _ = g(0, SOURCES, planes)
    st = oracle.Stereo(128, 96, views, imgs, precision=64)
    a, b = planes[..., 1], planes[..., 2]
    n = np.stack([np.sin(a) * np.cos(b), np.sin(b), -np.cos(a) * np.cos(b)], -1)
    hyp_cost, vc = st.plane_cost(0, SOURCES, np.concatenate([n, planes[..., :1]], -1),
                                 min_depth=0.1, max_depth=10.0)
    ok = hyp_cost < 2.0
    assert ok.mean() > 0.5
    np.testing.assert_allclose(c[ok], vc[..., :3].sum(-1)[ok], atol=1e-9)


def test_plane_gradient_matches_central_differences(scene):
    views, imgs, planes, deltas = scene
    g = oracle.NccGrad(views, imgs)
    _, margin, _ = g.structure(0, SOURCES, planes, deltas)
    valid = margin > 0.5
    _, gp, _ = g(0, SOURCES, planes, deltas, grad_planes=True)
    for j, name in enumerate(["depth", "angle a", "angle b"]):
        pp, pm = planes.copy(), planes.copy()
        pp[..., j] += H_STEP
        pm[..., j] -= H_STEP
        cp, _, hp = g.structure(0, SOURCES, pp, deltas)
        cm, _, hm = g.structure(0, SOURCES, pm, deltas)
        smooth = valid & (hp == hm)
        assert smooth.sum() > 0.5 * valid.sum(), name
        fd = (cp - cm) / (2 * H_STEP)
        rel = _rel(fd[smooth] - gp[..., j][smooth], gp[..., j][smooth])
        assert rel.max() < 1e-3, f"{name}: max relative error {rel.max():.2e}"


def test_pose_gradient_matches_central_differences(scene):
    views, imgs, planes, deltas = scene
    g = oracle.NccGrad(views, imgs)
    _, margin, _ = g.structure(0, SOURCES, planes, deltas)
    valid = margin > 0.5
    for v in range(4):
        for j in range(6):
            dp, dm = deltas.copy(), deltas.copy()
            dp[v, j] += H_STEP
            dm[v, j] -= H_STEP
            cp, _, hp = g.structure(0, SOURCES, planes, dp)
            cm, _, hm = g.structure(0, SOURCES, planes, dm)
            w = (valid & (hp == hm)).astype(np.float64)
            fd = ((cp - cm) * w).sum() / (2 * H_STEP)
            _, _, gd = g(0, SOURCES, planes, deltas, weights=w, grad_deltas=True)
            # scale: the view's gradient block (translation or rotation) of the same weights
            block = gd[v, 3 * (j // 3):3 * (j // 3) + 3]
            err = abs(fd - gd[v, j]) / np.linalg.norm(block)
            assert err < 1e-3, f"view {v} parameter {j}: {fd} vs {gd[v, j]} ({err:.2e})"


def test_gradient_directional_derivative(scene):
    """Along the gradient over all valid pixels, kinks included: the kink errors average out."""
    views, imgs, planes, deltas = scene
    g = oracle.NccGrad(views, imgs)
    _, margin, _ = g.structure(0, SOURCES, planes, deltas)
    w = (margin > 0.5).astype(np.float64)
    _, gp, _ = g(0, SOURCES, planes, deltas, weights=w, grad_planes=True)
    r = gp / np.abs(gp).max()
    cp, _, _ = g(0, SOURCES, planes + H_STEP * r, deltas)
    cm, _, _ = g(0, SOURCES, planes - H_STEP * r, deltas)
    fd = ((cp - cm) * w).sum() / (2 * H_STEP)
    an = (gp * r).sum()
    assert abs(fd - an) / abs(an) < 1e-3


@pytest.fixture(scope="module")
def tsdf_case():
    views, imgs, truth, _ = arc_workload(n=3, W=96, H=72, f=84.0, step_deg=6.0, seed=5)
    W, H = 96, 72
    rng = np.random.default_rng(1)
    packed = np.zeros((H, W), dtype=np.uint32)
    for y, x in zip(*np.nonzero(truth[0] > 0)):
        packed[y, x] = oracle.pack_sample(truth[0][y, x], (0.0, 0.0, -1.0), rng.uniform(0, 0.9))
    depth = np.vectorize(lambda p: oracle.load().orc_unpack_depth(int(p)))(packed).astype(np.float64)
    depth += rng.uniform(-0.003, 0.003, depth.shape) * (depth > 0)
    dims = (48, 40, 48)
    desc, keep = oracle.tsdf_desc(W, H, 0.05, (-1.2, -1.0, -1.2), 0.15, dense=dims)
    n = int(np.prod(dims))
    t0, w0 = rng.uniform(-1, 1, n), rng.uniform(0, 3, n)
    k = views[0].intrinsics
    vk = dict(k=(k.fx, k.fy, k.cx, k.cy), R=views[0].pose.R, t=views[0].pose.t, max_depth=5.0,
              confidence=1.5)
    gT, gW = rng.normal(size=n), rng.normal(size=n)
    return desc, keep, vk, packed, depth, t0, w0, gT, gW


def test_tsdf_depth_gradient_matches_central_differences(tsdf_case):
    desc, _, vk, packed, depth, t0, w0, gT, gW = tsdf_case
    _, _, gd, _, _ = oracle.tsdf_depth(desc, vk, packed, depth, t0, w0, gT, gW)
    assert (gd != 0).sum() > 1000
    r = (gd / np.abs(gd).max()).reshape(depth.shape)
    tp, wp = oracle.tsdf_depth(desc, vk, packed, depth + H_STEP * r, t0, w0)[:2]
    tm, wm = oracle.tsdf_depth(desc, vk, packed, depth - H_STEP * r, t0, w0)[:2]
    # a voxel whose update starts or stops inside the step jumps; leave those out
    jump = (wp == w0) != (wm == w0)
    assert jump.sum() < 20
    gT2, gW2 = gT * ~jump, gW * ~jump
    _, _, gd2, _, _ = oracle.tsdf_depth(desc, vk, packed, depth, t0, w0, gT2, gW2)
    fd = ((gT2 * (tp - tm)).sum() + (gW2 * (wp - wm)).sum()) / (2 * H_STEP)
    an = (gd2 * r.reshape(-1)).sum()
    assert abs(fd - an) / abs(an) < 1e-3


def test_tsdf_state_gradient_matches_central_differences(tsdf_case):
    desc, _, vk, packed, depth, t0, w0, gT, gW = tsdf_case
    _, _, _, gt0, gw0 = oracle.tsdf_depth(desc, vk, packed, depth, t0, w0, gT, gW)
    s = np.random.default_rng(2).normal(size=t0.size)

    def L(tt, ww):
        t1, w1 = oracle.tsdf_depth(desc, vk, packed, depth, tt, ww)[:2]
        return (gT * t1).sum() + (gW * w1).sum()

    fd_t = (L(t0 + H_STEP * s, w0) - L(t0 - H_STEP * s, w0)) / (2 * H_STEP)
    fd_w = (L(t0, w0 + H_STEP * s) - L(t0, w0 - H_STEP * s)) / (2 * H_STEP)
    assert abs(fd_t - (gt0 * s).sum()) / abs(fd_t) < 1e-3
    assert abs(fd_w - (gw0 * s).sum()) / abs(fd_w) < 1e-3


def test_tsdf_forward_equals_integrate_oracle(tsdf_case):
    """With the packed depths, the differentiable update is the FP64 integrate oracle's."""
    desc, _, vk, packed, _, t0, w0, _, _ = tsdf_case
    depth = np.vectorize(lambda p: oracle.load().orc_unpack_depth(int(p)))(packed).astype(np.float64)
    t1, w1 = oracle.tsdf_depth(desc, vk, packed, depth, t0, w0)[:2]
    o = oracle.Tsdf(96, 72, 0.05, (-1.2, -1.0, -1.2), 0.15, dense=(48, 40, 48), precision=64)
    o.tsdf[:] = t0
    o.weight[:] = w0
    o.integrate(vk, packed)
    np.testing.assert_allclose(t1, o.tsdf, atol=1e-12)
    np.testing.assert_allclose(w1, o.weight, atol=1e-12)
