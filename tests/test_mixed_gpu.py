"""Views of different image sizes (the batching configuration mixes 480x360 ... 1280x960).

The plain form stays bit-exact against the oracle with per-view sizes; the fast form's batch
equals its views solved one by one; the TSDF sweep over maps of different sizes equals the
per-view integrations.
"""
import numpy as np
import pytest

import oracle
from helpers import assert_bit_equal
from luvas3d import (DTYPE_F16, FORM_FAST, DenseStereo, IntegrationView, SolveOptions,
                     StereoOptions, TsdfVolume, scenes)
from luvas3d.camera import Intrinsics, StereoView, look_at

pytestmark = pytest.mark.gpu

SIZES = [(160, 120), (96, 72), (200, 150), (128, 96), (112, 84)]


@pytest.fixture(scope="module")
def mixed():
    views = []
    for s, (W, H) in enumerate(SIZES):
        a = np.radians(5.0 * (s - 2))
        k = Intrinsics(0.875 * W, 0.875 * W, W / 2, H / 2)
        views.append(StereoView(k, look_at((2.5 * np.sin(a), 0.3, 2.5 * np.cos(a)), (0, -0.3, 0))))
    imgs, truth = scenes.render_sphere(views, SIZES, seed=13)
    srcs = [[j for j in range(5) if j != i] for i in range(5)]
    return views, imgs, truth, srcs


def test_plain_mixed_sizes_bit_exact(mixed):
    views, imgs, truth, srcs = mixed
    o = oracle.Stereo(0, 0, views, imgs, 32)
    s = DenseStereo(0, 0, views, sizes=SIZES)
    for i, im in enumerate(imgs):
        s.set_image(i, im)
    for r in range(5):
        o.solve(r, srcs[r], min_depth=0.5, max_depth=5.0, iterations=2)
        s.solve(r, SolveOptions(srcs[r], 0.5, 5.0, iterations=2))
        hyp, cost = s.read_hypotheses()
        assert hyp.shape == (SIZES[r][1], SIZES[r][0], 4)
        assert_bit_equal(hyp, o.hyp, f"view {r} hyp")
        assert_bit_equal(cost, o.cost, f"view {r} cost")
    for r in range(5):
        assert_bit_equal(s.depth_map(r), o.depths[r], f"view {r} packed")
        assert_bit_equal(s.filtered_map(r, srcs[r], 2), o.filter(r, srcs[r], 2), f"view {r} filtered")


def test_fast_mixed_sizes_batch_equals_single(mixed):
    views, imgs, truth, srcs = mixed
    a = DenseStereo(0, 0, views, StereoOptions(form=FORM_FAST, storage=DTYPE_F16), sizes=SIZES)
    b = DenseStereo(0, 0, views, StereoOptions(form=FORM_FAST, storage=DTYPE_F16), sizes=SIZES)
    for i, im in enumerate(imgs):
        a.set_image(i, im)
        b.set_image(i, im)
    opts = [SolveOptions(srcs[r], 0.5, 5.0, iterations=3) for r in range(5)]
    a.solve_all(range(5), opts)
    for r in range(5):
        b.solve(r, opts[r])
        assert_bit_equal(a.read_hypotheses_layer(r)[0], b.read_hypotheses()[0], f"view {r}")
        assert_bit_equal(a.depth_map(r), b.depth_map(r), f"view {r} packed")
        d = a.read_hypotheses_layer(r)[0][..., 3]
        m = truth[r] > 0
        assert np.median(np.abs(d[m] - truth[r][m]) / truth[r][m]) < 0.01


def test_tsdf_sweep_over_mixed_sizes(mixed):
    views, imgs, truth, srcs = mixed
    s = DenseStereo(0, 0, views, StereoOptions(form=FORM_FAST, storage=DTYPE_F16), sizes=SIZES)
    for i, im in enumerate(imgs):
        s.set_image(i, im)
    s.solve_all(range(5), [SolveOptions(srcs[r], 0.5, 5.0, iterations=3) for r in range(5)])
    s.filter_all(range(5), srcs, [2] * 5)
    dims, voxel, origin = (48, 40, 48), 0.05, (-1.2, -1.0, -1.2)
    iv = [IntegrationView(v.intrinsics, v.pose, 5.0) for v in views]
    sweep = TsdfVolume(200, 150, voxel, origin, dense=dims, truncation=0.15, weight_q8=True)
    sweep.integrate_many(iv, stereo=s, layers=list(range(5)))
    t_s, w_s = sweep.read()
    want_t = np.ones(int(np.prod(dims)), dtype=np.float32)
    want_w = np.zeros(int(np.prod(dims)), dtype=np.uint16)
    for r, v in enumerate(views):
        W, H = SIZES[r]
        m = s.read_filtered_layer(r)
        o = oracle.Tsdf(W, H, voxel, origin, 0.15, dense=dims, weight_q8=True)
        o.tsdf[:] = want_t
        o.weight[:] = want_w
        k = v.intrinsics
        o.integrate(dict(k=(k.fx, k.fy, k.cx, k.cy), R=v.pose.R, t=v.pose.t, max_depth=5.0), m)
        want_t, want_w = o.tsdf.copy(), o.weight.copy()
    assert_bit_equal(t_s.reshape(-1), want_t, "tsdf")
    assert_bit_equal(w_s.reshape(-1), want_w, "weight")
    assert (want_w > 0).sum() > 1000
    # every view's filtered map in one asynchronous copy equals the per-layer reads
    import torch
    out = torch.empty(sum(w * h for w, h in SIZES), dtype=torch.int32).pin_memory()
    s.read_filtered_all_async(out)
    s.synchronize()
    off = 0
    for r, (W, H) in enumerate(SIZES):
        assert np.array_equal(out.numpy()[off:off + W * H].view(np.uint32).reshape(H, W),
                              s.read_filtered_layer(r)), f"view {r}"
        off += W * H
    with pytest.raises(ValueError):
        s.read_filtered_all_async(np.empty(3, np.uint32))


def test_view_sizes_are_reported(mixed):
    views, imgs, truth, srcs = mixed
    s = DenseStereo(0, 0, views, sizes=SIZES)
    import ctypes as C
    from luvas3d import _lib
    w, h = C.c_int32(), C.c_int32()
    for i, (W, H) in enumerate(SIZES):
        _lib.check(_lib.load().l3d_stereo_view_size(s._h(), i, C.byref(w), C.byref(h)))
        assert (w.value, h.value) == (W, H)
    with pytest.raises(ValueError):
        s.set_image(0, imgs[1])
