"""PatchMatch parity: the CUDA kernels through the C ABI against the FP32 oracle.

The plain FP32 form follows the oracle's operation order, so every comparison here is bit-exact:
per-function (hypothesis cost of fixed planes), one kernel from an identical state, and whole
solves (which a single flipped argmin would break).  Tolerances of the path (depth 1e-3 relative
on >= 99.5 % of valid pixels, NCC cost 1e-4, TSDF 1e-5) are therefore met with margin zero.
"""
import numpy as np
import pytest

import oracle
from helpers import arc_workload, assert_bit_equal
from luvas3d import (KERNEL_INIT, KERNEL_INIT_COARSE, KERNEL_PACK, KERNEL_PROPAGATE, DenseStereo,
                     L3dError, SolveOptions, StereoOptions, scenes)
from luvas3d.camera import scale_intrinsics, StereoView

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def arc():
    return arc_workload()


@pytest.fixture(scope="module")
def small():
    return scenes.small()


def gpu_stereo(views, imgs, W, H, **kw):
    s = DenseStereo(W, H, views, StereoOptions(**kw))
    for i, im in enumerate(imgs):
        s.set_image(i, np.asarray(im, dtype=np.float32))
    return s


def test_plane_cost_bit_exact(arc):
    views, imgs, truth, srcs = arc
    W, H = 160, 120
    rng = np.random.default_rng(0)
    planes = np.zeros((H, W, 4), dtype=np.float32)
    n = rng.normal(size=(H, W, 3)) * 0.3 + np.array([0, 0, -1.0])
    planes[..., :3] = n / np.linalg.norm(n, axis=-1, keepdims=True)
    planes[..., 3] = rng.uniform(1.0, 2.5, size=(H, W))
    o = oracle.Stereo(W, H, views, imgs, 32)
    want, want_vc = o.plane_cost(2, srcs[2], planes, min_depth=0.5, max_depth=5.0)
    s = gpu_stereo(views, imgs, W, H)
    got, got_vc = s.plane_cost(2, SolveOptions(srcs[2], 0.5, 5.0), planes, view_costs=True)
    assert_bit_equal(got, want.astype(np.float32), "hypothesis cost")
    assert_bit_equal(got_vc, want_vc.astype(np.float32), "per-view cost")
    assert (want < 1).mean() > 0.2  # the planes are not all rejected


def test_u8_images_are_r8unorm(arc):
    views, imgs, truth, srcs = arc
    W, H = 160, 120
    u8 = [np.clip(np.rint(im * 255), 0, 255).astype(np.uint8) for im in imgs]
    f32 = [(u.astype(np.float32) / np.float32(255)) for u in u8]
    o = oracle.Stereo(W, H, views, f32, 32)
    o.solve(2, srcs[2], min_depth=0.5, max_depth=5.0, iterations=1)
    s = DenseStereo(W, H, views)
    for i, im in enumerate(u8):
        s.set_image(i, im)
    s.solve(2, SolveOptions(srcs[2], 0.5, 5.0, iterations=1))
    hyp, cost = s.read_hypotheses()
    assert_bit_equal(hyp, o.hyp, "hyp")
    assert_bit_equal(s.depth_map(2), o.depths[2], "packed")


def test_each_kernel_from_an_identical_state(arc):
    views, imgs, truth, srcs = arc
    W, H = 160, 120
    o = oracle.Stereo(W, H, views, imgs, 32)
    s = gpu_stereo(views, imgs, W, H)
    opts = SolveOptions(srcs[2], 0.5, 5.0)
    kw = dict(min_depth=0.5, max_depth=5.0)
    o.kernel(oracle.INIT, 2, srcs[2], **kw)
    s.dispatch(KERNEL_INIT, 2, opts)
    hyp, cost = s.read_hypotheses()
    assert_bit_equal(hyp, o.hyp, "init hyp")
    assert_bit_equal(cost, o.cost, "init cost")
    for it, phase in ((0, 0), (0, 1), (1, 0), (2, 1)):
        # start both from the oracle's state so each step is checked on its own
        s.write_hypotheses(o.hyp, o.cost)
        o.kernel(oracle.PROPAGATE, 2, srcs[2], iteration=it, phase=phase, **kw)
        s.dispatch(KERNEL_PROPAGATE, 2, opts, iteration=it, phase=phase)
        hyp, cost = s.read_hypotheses()
        assert_bit_equal(hyp, o.hyp, f"propagate it {it} phase {phase}")
        assert_bit_equal(cost, o.cost, f"propagate cost it {it} phase {phase}")
    o.kernel(oracle.PACK, 2, srcs[2], **kw)
    s.dispatch(KERNEL_PACK, 2, opts)
    assert_bit_equal(s.depth_map(2), o.depths[2], "pack")


@pytest.mark.parametrize("iterations", [1, 4])
def test_whole_solve_bit_exact_arc(arc, iterations):
    views, imgs, truth, srcs = arc
    W, H = 160, 120
    o = oracle.Stereo(W, H, views, imgs, 32)
    o.solve(2, srcs[2], min_depth=0.5, max_depth=5.0, iterations=iterations)
    s = gpu_stereo(views, imgs, W, H)
    s.solve(2, SolveOptions(srcs[2], 0.5, 5.0, iterations=iterations))
    hyp, cost = s.read_hypotheses()
    assert_bit_equal(hyp, o.hyp, "hyp")
    assert_bit_equal(cost, o.cost, "cost")
    assert_bit_equal(s.depth_map(2), o.depths[2], "packed depth")
    # and the result is a reconstruction: median relative depth error on the surface
    tr = truth[2]
    m = tr > 0
    rel = np.abs(hyp[..., 3] - tr) / np.where(m, tr, 1)
    if iterations == 4:
        assert np.median(rel[m]) < 0.004


def test_small_workload_all_views_then_filter(small):
    """The 8-view 320x240 workload: every view solved (3 iterations, 4 sources), then the
    consistency filter of every view; packed and filtered maps bit-exact."""
    w = small
    o = oracle.Stereo(w.width, w.height, w.views, w.images, 32)
    s = gpu_stereo(w.views, w.images, w.width, w.height)
    for r in range(len(w.views)):
        lo, hi = w.ranges[r]
        o.solve(r, w.sources[r], min_depth=lo, max_depth=hi, iterations=w.iterations)
        s.solve(r, SolveOptions(w.sources[r], lo, hi, iterations=w.iterations))
        hyp, cost = s.read_hypotheses()
        assert_bit_equal(hyp, o.hyp, f"view {r} hyp")
        assert_bit_equal(cost, o.cost, f"view {r} cost")
    for r in range(len(w.views)):
        assert_bit_equal(s.depth_map(r), o.depths[r], f"view {r} packed")
        want = o.filter(r, w.sources[r], w.needed[r])
        got = s.filtered_map(r, w.sources[r], w.needed[r])
        assert_bit_equal(got, want, f"view {r} filtered")
        assert np.array_equal(got != 0, want != 0)  # valid-pixel mask


def test_geometric_pass_bit_exact(arc):
    views, imgs, truth, srcs = arc
    W, H = 160, 120
    o = oracle.Stereo(W, H, views, imgs, 32)
    s = gpu_stereo(views, imgs, W, H)
    for r in range(len(views)):
        o.solve(r, srcs[r], min_depth=0.5, max_depth=5.0, iterations=2)
        s.solve(r, SolveOptions(srcs[r], 0.5, 5.0, iterations=2))
    # ACMM pass: views in order, each reading the maps packed so far (Gauss-Seidel)
    for r in range(len(views)):
        o.solve(r, srcs[r], min_depth=0.5, max_depth=5.0, iterations=1, geometric=True)
        s.solve(r, SolveOptions(srcs[r], 0.5, 5.0, iterations=1, geometric=True))
        hyp, cost = s.read_hypotheses()
        assert_bit_equal(hyp, o.hyp, f"geometric view {r}")
        assert_bit_equal(cost, o.cost, f"geometric cost {r}")
    for r in range(len(views)):
        assert_bit_equal(s.depth_map(r), o.depths[r], f"geometric packed {r}")


def test_prior_competes_in_init(arc):
    views, imgs, truth, srcs = arc
    W, H = 160, 120
    prior = np.where(np.arange(W * H).reshape(H, W) % 3 == 0, truth[2] * 1.01, 0).astype(np.float32)
    o = oracle.Stereo(W, H, views, imgs, 32)
    o.solve(2, srcs[2], min_depth=0.5, max_depth=5.0, iterations=1, prior=prior)
    s = gpu_stereo(views, imgs, W, H)
    s.solve(2, SolveOptions(srcs[2], 0.5, 5.0, iterations=1, prior=prior))
    hyp, cost = s.read_hypotheses()
    assert_bit_equal(hyp, o.hyp, "hyp with prior")
    assert_bit_equal(cost, o.cost, "cost with prior")


def test_coarse_to_fine_bit_exact(arc):
    """coarse-to-fine (methods/coarse-to-fine.ts:9-68): half-resolution planes seed init_coarse."""
    views, imgs, truth, srcs = arc
    W, H = 160, 120
    cw, ch = 80, 60
    cviews = [StereoView(scale_intrinsics(v.intrinsics, cw / W, ch / H), v.pose) for v in views]
    cimgs = [im.reshape(ch, 2, cw, 2).mean(axis=(1, 3)).astype(np.float32) for im in imgs]
    oc = oracle.Stereo(cw, ch, cviews, cimgs, 32)
    oc.solve(2, srcs[2], min_depth=0.5, max_depth=5.0, iterations=2, pack=False)
    of = oracle.Stereo(W, H, views, imgs, 32)
    of.coarse = oc.hyp.copy()
    of.solve(2, srcs[2], min_depth=0.5, max_depth=5.0, iterations=1, from_coarse=True)
    coarse = DenseStereo(cw, ch, cviews, StereoOptions(depth_maps=False))
    for i, im in enumerate(cimgs):
        coarse.set_image(i, im)
    fine = DenseStereo(W, H, views, StereoOptions(coarse=coarse))
    for i, im in enumerate(imgs):
        fine.set_image(i, im)
    coarse.solve(2, SolveOptions(srcs[2], 0.5, 5.0, iterations=2, pack=False))
    ch_hyp, _ = coarse.read_hypotheses()
    assert_bit_equal(ch_hyp, oc.hyp, "coarse planes")
    fine.solve(2, SolveOptions(srcs[2], 0.5, 5.0, iterations=1, from_coarse=True))
    hyp, cost = fine.read_hypotheses()
    assert_bit_equal(hyp, of.hyp, "fine hyp")
    assert_bit_equal(fine.depth_map(2), of.depths[2], "fine packed")
    fine.dispatch(KERNEL_INIT_COARSE, 2, SolveOptions(srcs[2], 0.5, 5.0))
    of.kernel(oracle.INIT_COARSE, 2, srcs[2], min_depth=0.5, max_depth=5.0)
    assert_bit_equal(fine.read_hypotheses()[0], of.hyp, "init_coarse alone")


def test_dense_window_bit_exact(arc):
    views, imgs, truth, srcs = arc
    W, H = 160, 120
    o = oracle.Stereo(W, H, views, imgs, 32, window=11, dilation=1)
    o.solve(2, srcs[2], min_depth=0.5, max_depth=5.0, iterations=1)
    s = gpu_stereo(views, imgs, W, H, window=11, dilation=1)
    s.solve(2, SolveOptions(srcs[2], 0.5, 5.0, iterations=1))
    hyp, cost = s.read_hypotheses()
    assert_bit_equal(hyp, o.hyp, "11x11 hyp")
    assert_bit_equal(cost, o.cost, "11x11 cost")


@pytest.mark.parametrize("W,H,n_src", [(161, 97, 1), (33, 17, 2), (7, 5, 3)])
def test_ragged_sizes_and_few_sources(W, H, n_src):
    views, imgs, truth, srcs = arc_workload(n=4, W=W, H=H, f=W * 0.875)
    o = oracle.Stereo(W, H, views, imgs, 32)
    s = gpu_stereo(views, imgs, W, H)
    src = srcs[1][:n_src]
    o.solve(1, src, min_depth=0.5, max_depth=5.0, iterations=2)
    s.solve(1, SolveOptions(src, 0.5, 5.0, iterations=2))
    hyp, cost = s.read_hypotheses()
    assert_bit_equal(hyp, o.hyp, "hyp")
    assert_bit_equal(s.depth_map(1), o.depths[1], "packed")
    want = o.filter(1, src, 1)
    assert_bit_equal(s.filtered_map(1, src, 1), want, "filtered")


def test_no_sources_is_a_no_op(arc):
    views, imgs, truth, srcs = arc
    s = gpu_stereo(views, imgs, 160, 120)
    before = s.launches
    s.solve(2, SolveOptions([], 0.5, 5.0, iterations=3))
    assert s.launches == before


def test_errors_are_reported(arc):
    views, imgs, truth, srcs = arc
    s = gpu_stereo(views, imgs, 160, 120)
    with pytest.raises(L3dError):
        s.solve(9, SolveOptions([0], 0.5, 5.0))
    with pytest.raises(L3dError):
        s.solve(0, SolveOptions([7], 0.5, 5.0))
    with pytest.raises(L3dError):
        s.solve(0, SolveOptions([1], 5.0, 0.5))
    with pytest.raises(L3dError):
        s.solve(0, SolveOptions([1], 0.5, 5.0, from_coarse=True))
    one = DenseStereo(160, 120, views, StereoOptions(depth_maps=False))
    with pytest.raises(L3dError):
        one.solve(1, SolveOptions([0], 0.5, 5.0, pack=True))
    s.destroy()
    with pytest.raises(RuntimeError):
        s.solve(0, SolveOptions([1], 0.5, 5.0))
