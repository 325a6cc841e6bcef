"""The exact batched form (L3D_FORM_EXACT) against the FP32 oracle, bit for bit.

The exact form runs every reference view of a batch in one launch per kernel, like the fast form,
but evaluates the multi-view NCC with the plain form's arithmetic: FP32 texels fetched as texture
gathers (the four texels of each bilinear footprint), exact bilinear weights, per-sample
homogeneous coordinates with an IEEE reciprocal, raw-value window sums.  Its batched solves
therefore equal the oracle's per-view solves of patchmatch.wgsl.ts (init 255-289, propagate
349-423, pack 425-433) bit for bit, and with compensated sums they equal the oracle's compensated
mode bit for bit.  A wrong gather component order, footprint or clamp would break every one of
these equalities.
"""
import numpy as np
import pytest

import oracle
from helpers import arc_workload, assert_bit_equal
from luvas3d import (FORM_EXACT, FORM_PLAIN, KERNEL_INIT, KERNEL_PACK, KERNEL_PROPAGATE,
                     DenseStereo, SolveOptions, StereoOptions, scale_intrinsics, scenes)
from luvas3d.camera import Intrinsics, StereoView, look_at

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def arc():
    return arc_workload()


@pytest.fixture(scope="module")
def small():
    return scenes.small()


def exact_stereo(views, imgs, W, H, compensated=False, sizes=None, **kw):
    s = DenseStereo(W, H, views, StereoOptions(form=FORM_EXACT, compensated=compensated, **kw),
                    sizes=sizes)
    for i, im in enumerate(imgs):
        s.set_image(i, np.asarray(im, dtype=np.float32))
    return s


@pytest.mark.parametrize("compensated", [False, True])
def test_plane_cost_bit_exact(arc, compensated):
    views, imgs, truth, srcs = arc
    W, H = 160, 120
    rng = np.random.default_rng(1)
    planes = np.zeros((H, W, 4), dtype=np.float32)
    n = rng.normal(size=(H, W, 3)) * 0.3 + np.array([0, 0, -1.0])
    planes[..., :3] = n / np.linalg.norm(n, axis=-1, keepdims=True)
    planes[..., 3] = rng.uniform(1.0, 2.5, size=(H, W))
    o = oracle.Stereo(W, H, views, imgs, 32, compensated=compensated)
    want, _ = o.plane_cost(2, srcs[2], planes, min_depth=0.5, max_depth=5.0)
    s = exact_stereo(views, imgs, W, H, compensated)
    got = s.plane_cost(2, SolveOptions(srcs[2], 0.5, 5.0), planes)
    assert_bit_equal(got, want.astype(np.float32), "hypothesis cost")
    assert (want < 1).mean() > 0.2  # the planes are not all rejected
    assert (want == 2).mean() > 0.01  # and some windows leave a source image


@pytest.mark.parametrize("compensated,variant", [(False, 14), (False, 6), (True, 14)])
def test_batched_solve_equals_oracle_per_view(small, compensated, variant):
    """The 8-view 320x240 workload (4 sources, 3 iterations) solved in one batch: every view's
    planes, costs and packed map equal the oracle's per-view solve."""
    w = small
    o = oracle.Stereo(w.width, w.height, w.views, w.images, 32, compensated=compensated)
    s = exact_stereo(w.views, w.images, w.width, w.height, compensated)
    s.variant = variant
    refs = list(range(len(w.views)))
    opts = [SolveOptions(w.sources[r], w.ranges[r][0], w.ranges[r][1], iterations=w.iterations)
            for r in refs]
    s.solve_all(refs, opts)
    for r in refs:
        o.solve(r, w.sources[r], min_depth=w.ranges[r][0], max_depth=w.ranges[r][1],
                iterations=w.iterations)
        hyp, cost = s.read_hypotheses_layer(r)
        assert_bit_equal(hyp, o.hyp, f"view {r} hyp")
        assert_bit_equal(cost, o.cost, f"view {r} cost")
    for r in refs:
        assert_bit_equal(s.depth_map(r), o.depths[r], f"view {r} packed")
    s.destroy()


def test_graph_replay_equals_oracle(arc):
    views, imgs, truth, srcs = arc
    W, H = 160, 120
    s = exact_stereo(views, imgs, W, H)
    s.set_graphs(True)
    opts = [SolveOptions(srcs[r], 0.5, 5.0, iterations=2) for r in range(5)]
    s.solve_all(range(5), opts)
    s.solve_all(range(5), opts)  # the replay of the captured graph
    o = oracle.Stereo(W, H, views, imgs, 32)
    for r in range(5):
        o.solve(r, srcs[r], min_depth=0.5, max_depth=5.0, iterations=2)
        hyp, cost = s.read_hypotheses_layer(r)
        assert_bit_equal(hyp, o.hyp, f"view {r} hyp")
        assert_bit_equal(cost, o.cost, f"view {r} cost")


def test_each_kernel_from_an_identical_state(arc):
    views, imgs, truth, srcs = arc
    W, H = 160, 120
    o = oracle.Stereo(W, H, views, imgs, 32)
    s = exact_stereo(views, imgs, W, H)
    opts = SolveOptions(srcs[2], 0.5, 5.0)
    kw = dict(min_depth=0.5, max_depth=5.0)
    o.kernel(oracle.INIT, 2, srcs[2], **kw)
    s.dispatch(KERNEL_INIT, 2, opts)
    hyp, cost = s.read_hypotheses()
    assert_bit_equal(hyp, o.hyp, "init hyp")
    assert_bit_equal(cost, o.cost, "init cost")
    for it, phase in ((0, 0), (0, 1), (1, 0), (3, 1)):
        s.write_hypotheses(o.hyp, o.cost)
        o.kernel(oracle.PROPAGATE, 2, srcs[2], iteration=it, phase=phase, **kw)
        s.dispatch(KERNEL_PROPAGATE, 2, opts, iteration=it, phase=phase)
        hyp, cost = s.read_hypotheses()
        assert_bit_equal(hyp, o.hyp, f"propagate it {it} phase {phase}")
        assert_bit_equal(cost, o.cost, f"propagate cost it {it} phase {phase}")
    o.kernel(oracle.PACK, 2, srcs[2], **kw)
    s.dispatch(KERNEL_PACK, 2, opts)
    assert_bit_equal(s.depth_map(2), o.depths[2], "pack")


def test_geometric_pass_and_prior_bit_exact(arc):
    """Per-view solves (the reference's Gauss-Seidel order): a photometric pass with a phone
    prior, then a geometric pass that reads every source's packed map."""
    views, imgs, truth, srcs = arc
    W, H = 160, 120
    o = oracle.Stereo(W, H, views, imgs, 32)
    s = exact_stereo(views, imgs, W, H)
    prior = np.where(truth[1] > 0, truth[1] * 1.02, 0).astype(np.float32)
    for r in range(5):
        pr = prior if r == 1 else None
        o.solve(r, srcs[r], min_depth=0.5, max_depth=5.0, iterations=2, prior=pr)
        s.solve(r, SolveOptions(srcs[r], 0.5, 5.0, iterations=2, prior=pr))
        hyp, cost = s.read_hypotheses()
        assert_bit_equal(hyp, o.hyp, f"view {r} photometric hyp")
    for r in range(5):
        o.solve(r, srcs[r], min_depth=0.5, max_depth=5.0, iterations=1, geometric=True)
        s.solve(r, SolveOptions(srcs[r], 0.5, 5.0, iterations=1, geometric=True))
        hyp, cost = s.read_hypotheses()
        assert_bit_equal(hyp, o.hyp, f"view {r} geometric hyp")
        assert_bit_equal(cost, o.cost, f"view {r} geometric cost")
    for r in range(5):
        assert_bit_equal(s.depth_map(r), o.depths[r], f"view {r} packed")
        assert_bit_equal(s.filtered_map(r, srcs[r], 2), o.filter(r, srcs[r], 2), f"view {r} filtered")


def test_mixed_and_ragged_sizes_bit_exact():
    """Views of different (odd) sizes in one batch, including windows that graze image edges."""
    sizes = [(161, 97), (96, 72), (33, 17), (128, 96), (7, 5)]
    views = []
    for s_, (W, H) in enumerate(sizes):
        a = np.radians(5.0 * (s_ - 2))
        k = Intrinsics(0.875 * W, 0.875 * W, W / 2, H / 2)
        views.append(StereoView(k, look_at((2.5 * np.sin(a), 0.3, 2.5 * np.cos(a)), (0, -0.3, 0))))
    imgs, _ = scenes.render_sphere(views, sizes, seed=5)
    srcs = [[j for j in range(5) if j != i][: 1 + i % 3] for i in range(5)]
    o = oracle.Stereo(0, 0, views, imgs, 32)
    s = exact_stereo(views, imgs, 0, 0, sizes=sizes)
    opts = [SolveOptions(srcs[r], 0.5, 5.0, iterations=2) for r in range(5)]
    s.solve_all(range(5), opts)
    for r in range(5):
        o.solve(r, srcs[r], min_depth=0.5, max_depth=5.0, iterations=2)
        hyp, cost = s.read_hypotheses_layer(r)
        assert hyp.shape == (sizes[r][1], sizes[r][0], 4)
        assert_bit_equal(hyp, o.hyp, f"view {r} hyp")
        assert_bit_equal(cost, o.cost, f"view {r} cost")


def test_coarse_to_fine_equals_plain_form(arc):
    """init_coarse (patchmatch.wgsl.ts:296-333): the exact form's coarse start equals the plain
    form's, which is bit-exact against the oracle."""
    views, imgs, truth, srcs = arc
    W, H = 160, 120
    cw, ch = W // 2, H // 2
    cviews = [StereoView(scale_intrinsics(v.intrinsics, cw / W, ch / H), v.pose) for v in views]

    def levels(form):
        c = DenseStereo(cw, ch, cviews, StereoOptions(depth_maps=False, form=form))
        f = DenseStereo(W, H, views, StereoOptions(coarse=c, form=form))
        for i, im in enumerate(imgs):
            c.set_image(i, np.ascontiguousarray(im[::2, ::2]))
            f.set_image(i, im)
        return c, f

    c1, f1 = levels(FORM_EXACT)
    c2, f2 = levels(FORM_PLAIN)
    for r in range(5):
        co = SolveOptions(srcs[r], 0.5, 5.0, iterations=2, pack=False)
        fo = SolveOptions(srcs[r], 0.5, 5.0, iterations=1, from_coarse=True)
        c1.solve(r, co)
        f1.solve(r, fo)
        c2.solve(r, co)
        f2.solve(r, fo)
        got, gc = f1.read_hypotheses()
        want, wc = f2.read_hypotheses()
        assert_bit_equal(got, want, f"view {r} hyp")
        assert_bit_equal(gc, wc, f"view {r} cost")
