"""The fast PatchMatch form (FP16/BF16 image storage, texture-filtered samples, batched views).

It is not bit-exact by design (hardware bilinear weights, FP16/BF16 storage, approximate
reciprocals), so it is checked the way a precision change is checked: the NCC cost of fixed
planes against the FP64 oracle, depth accuracy against ground truth next to the plain FP32 form,
and determinism (a batch equals its views solved one at a time).
"""
import numpy as np
import pytest

import oracle
from helpers import arc_workload, assert_bit_equal
from luvas3d import (DTYPE_BF16, DTYPE_F16, DTYPE_F32, DTYPE_U8, FORM_FAST, FORM_PLAIN, DenseStereo,
                     L3dError, SolveOptions, StereoOptions, packing)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def arc():
    return arc_workload(n=5, W=256, H=192, f=224.0)


def make(views, imgs, W, H, form=FORM_FAST, storage=DTYPE_F16):
    s = DenseStereo(W, H, views, StereoOptions(form=form, storage=storage))
    for i, im in enumerate(imgs):
        s.set_image(i, np.asarray(im, dtype=np.float32))
    return s


@pytest.mark.parametrize("storage", [DTYPE_F16, DTYPE_BF16, DTYPE_F32, DTYPE_U8])
def test_fixed_plane_cost_close_to_fp64(arc, storage):
    views, imgs, truth, srcs = arc
    W, H = 256, 192
    # planes of the true surface (depth from the ray cast, normal facing the camera)
    planes = np.zeros((H, W, 4), dtype=np.float32)
    planes[..., 2] = -1.0
    planes[..., 3] = np.where(truth[2] > 0, truth[2], 1.0)
    o = oracle.Stereo(W, H, views, imgs, 64)
    want, _ = o.plane_cost(2, srcs[2], planes.astype(np.float64), min_depth=0.5, max_depth=5.0)
    s = make(views, imgs, W, H, storage=storage)
    got = s.plane_cost(2, SolveOptions(srcs[2], 0.5, 5.0), planes)
    valid = (want < 1.5) & (got < 1.5)
    assert valid.mean() > 0.7
    assert np.array_equal(want >= 1.5, got >= 1.5) or np.mean((want >= 1.5) != (got >= 1.5)) < 0.01
    err = np.abs(got[valid] - want[valid])
    p99 = np.percentile(err, 99)
    print(f"storage {storage}: cost error vs FP64 max {err.max():.2e} p99 {p99:.2e} "
          f"median {np.median(err):.2e}")
    # U8 (the reference's r8unorm textures) is limited by the 1/255 quantization of the inputs
    tol = {DTYPE_F32: 2e-3, DTYPE_F16: 5e-3, DTYPE_BF16: 2e-2, DTYPE_U8: 1.5e-2}[storage]
    assert p99 < tol


def depth_stats(hyp, truth):
    m = truth > 0
    rel = np.abs(hyp[..., 3] - truth) / np.where(m, truth, 1)
    return np.median(rel[m]), (rel[m] < 0.01).mean()


@pytest.mark.parametrize("storage", [DTYPE_F16, DTYPE_BF16, DTYPE_U8])
def test_fast_depth_accuracy_matches_plain(arc, storage):
    views, imgs, truth, srcs = arc
    W, H = 256, 192
    plain = make(views, imgs, W, H, form=FORM_PLAIN, storage=DTYPE_F32)
    fast = make(views, imgs, W, H, storage=storage)
    opts = SolveOptions(srcs[2], 0.5, 5.0, iterations=5)
    plain.solve(2, opts)
    fast.solve(2, opts)
    pm, pf = depth_stats(plain.read_hypotheses()[0], truth[2])
    fm, ff = depth_stats(fast.read_hypotheses()[0], truth[2])
    print(f"plain median {pm:.2e} within1% {pf:.3f} | fast({storage}) median {fm:.2e} within1% {ff:.3f}")
    assert fm < max(1.25 * pm, pm + 3e-4)
    assert ff > pf - 0.03
    # packed maps valid on a similar share of pixels
    vp = (plain.depth_map(2) != 0).mean()
    vf = (fast.depth_map(2) != 0).mean()
    assert abs(vp - vf) < 0.05


@pytest.mark.parametrize("variant", [6, 14, 4, 12, 3, 11, 2, 10, 38, 46])
def test_every_variant_keeps_accuracy(arc, variant):
    """Kernel variants split the window rows between the texture unit and software bilinear on
    the LSU path, map hardware quads to rows or 2x2 blocks and keep the window in shared memory
    (+32); accuracy must not change."""
    views, imgs, truth, srcs = arc
    W, H = 256, 192
    plain = make(views, imgs, W, H, form=FORM_PLAIN, storage=DTYPE_F32)
    fast = make(views, imgs, W, H)
    fast.variant = variant
    assert fast.variant == variant
    opts = SolveOptions(srcs[2], 0.5, 5.0, iterations=5)
    plain.solve(2, opts)
    fast.solve(2, opts)
    pm, pf = depth_stats(plain.read_hypotheses()[0], truth[2])
    fm, ff = depth_stats(fast.read_hypotheses()[0], truth[2])
    print(f"variant {variant}: fast median {fm:.2e} within1% {ff:.3f} (plain {pm:.2e} {pf:.3f})")
    assert fm < max(1.25 * pm, pm + 3e-4)
    assert ff > pf - 0.03
    planes = np.zeros((H, W, 4), dtype=np.float32)
    planes[..., 2] = -1.0
    planes[..., 3] = np.where(truth[2] > 0, truth[2], 1.0)
    o = oracle.Stereo(W, H, views, imgs, 64)
    want, _ = o.plane_cost(2, srcs[2], planes.astype(np.float64), min_depth=0.5, max_depth=5.0)
    got = fast.plane_cost(2, SolveOptions(srcs[2], 0.5, 5.0), planes)
    valid = (want < 1.5) & (got < 1.5)
    assert np.percentile(np.abs(got[valid] - want[valid]), 99) < 5e-3


@pytest.mark.parametrize("storage,compensated,variant", [
    (DTYPE_F16, False, 14), (DTYPE_F16, False, 6), (DTYPE_F32, False, 30), (DTYPE_F32, True, 30),
    (DTYPE_F16, True, 14), (DTYPE_U8, False, 14)])
def test_shared_window_equals_register_window(arc, storage, compensated, variant):
    """+32 keeps the reference window in shared memory instead of registers; the arithmetic is the
    same, so a solve (init and every propagate colour) equals the register variant bit for bit."""
    views, imgs, truth, srcs = arc
    W, H = 256, 192
    out = []
    for v in (variant, variant | 32):
        s = DenseStereo(W, H, views, StereoOptions(form=FORM_FAST, storage=storage,
                                                   compensated=compensated))
        for i, im in enumerate(imgs):
            s.set_image(i, np.asarray(im, dtype=np.float32))
        s.variant = v
        assert s.variant == v
        s.solve_all([1, 2, 3], [SolveOptions(srcs[r], 0.5, 5.0, iterations=3) for r in (1, 2, 3)])
        out.append([a for r in (1, 2, 3) for a in s.read_hypotheses_layer(r)])
    for i, (a, b) in enumerate(zip(*out)):
        assert_bit_equal(b, a, f"view {i // 2 + 1} {'cost' if i % 2 else 'hypotheses'}")


def test_variant_validation(arc):
    views, imgs, truth, srcs = arc
    fast = make(views, imgs, 256, 192)
    for bad in (5, 1, 7, 16, -1, 36, 44, 64, 110, 128):
        with pytest.raises(L3dError):
            fast.variant = bad
    bf16 = make(views, imgs, 256, 192, storage=DTYPE_BF16)
    with pytest.raises(L3dError):
        bf16.variant = 46
    plain = make(views, imgs, 256, 192, form=FORM_PLAIN, storage=DTYPE_F32)
    with pytest.raises(L3dError):
        plain.variant = 6


def test_batch_equals_single_views(arc):
    views, imgs, truth, srcs = arc
    W, H = 256, 192
    a = make(views, imgs, W, H)
    b = make(views, imgs, W, H)
    opts = [SolveOptions(srcs[r], 0.5, 5.0, iterations=3) for r in range(5)]
    a.solve_all(list(range(5)), opts)
    for r in range(5):
        b.solve(r, opts[r])
        hb, cb = b.read_hypotheses()
        ha, ca = a.read_hypotheses_layer(r)
        assert_bit_equal(ha, hb, f"view {r} hyp")
        assert_bit_equal(ca, cb, f"view {r} cost")
        assert_bit_equal(a.depth_map(r), b.depth_map(r), f"view {r} packed")


def test_mixed_iterations_and_pack_flags(arc):
    views, imgs, truth, srcs = arc
    W, H = 256, 192
    a = make(views, imgs, W, H)
    b = make(views, imgs, W, H)
    opts = [SolveOptions(srcs[r], 0.5, 5.0, iterations=1 + r % 3, pack=r != 1) for r in range(5)]
    a.solve_all(list(range(5)), opts)
    for r in range(5):
        b.solve(r, opts[r])
        assert_bit_equal(a.read_hypotheses_layer(r)[0], b.read_hypotheses()[0], f"view {r}")
    assert np.all(a.depth_map(1) == 0)


def test_geometric_batch_runs_and_keeps_accuracy(arc):
    views, imgs, truth, srcs = arc
    W, H = 256, 192
    a = make(views, imgs, W, H)
    refs = list(range(5))
    a.solve_all(refs, [SolveOptions(srcs[r], 0.5, 5.0, iterations=4) for r in refs])
    before = depth_stats(a.read_hypotheses_layer(2)[0], truth[2])
    a.solve_all(refs, [SolveOptions(srcs[r], 0.5, 5.0, iterations=1, geometric=True) for r in refs])
    after = depth_stats(a.read_hypotheses_layer(2)[0], truth[2])
    print("photometric", before, "geometric", after)
    assert after[0] < before[0] * 1.5 + 1e-4


def test_fast_form_rejections(arc):
    views, imgs, truth, srcs = arc
    with pytest.raises(L3dError):
        DenseStereo(64, 48, views, StereoOptions(form=FORM_FAST, storage=DTYPE_F16, window=11,
                                                 dilation=1))
    s = make(views, [im[:48, :64] for im in imgs], 64, 48)
    with pytest.raises(L3dError):
        s.solve_all([0, 0], [SolveOptions([1], 0.5, 5.0)] * 2)


def test_graph_replay_equals_direct_launches(arc):
    views, imgs, truth, srcs = arc
    W, H = 256, 192
    a = make(views, imgs, W, H)
    b = make(views, imgs, W, H)
    b.set_graphs(True)
    opts = [SolveOptions(srcs[r], 0.5, 5.0, iterations=3) for r in range(5)]
    a.solve_all(list(range(5)), opts)
    for _ in range(3):  # capture, then replays
        b.solve_all(list(range(5)), opts)
    for r in range(5):
        assert_bit_equal(b.read_hypotheses_layer(r)[0], a.read_hypotheses_layer(r)[0], f"view {r}")
        assert_bit_equal(b.depth_map(r), a.depth_map(r), f"packed {r}")
    # a different request is captured separately
    opts2 = [SolveOptions(srcs[r], 0.5, 5.0, iterations=2) for r in range(5)]
    a.solve_all(list(range(5)), opts2)
    b.solve_all(list(range(5)), opts2)
    assert_bit_equal(b.read_hypotheses_layer(1)[0], a.read_hypotheses_layer(1)[0], "second graph")
    b.set_graphs(False)
    with pytest.raises(L3dError):
        make(views, imgs, W, H, form=FORM_PLAIN, storage=DTYPE_F32).set_graphs(True)


def test_autotune_picks_a_valid_variant(arc):
    views, imgs, truth, srcs = arc
    s = make(views, imgs, 256, 192)
    opts = [SolveOptions(srcs[r], 0.5, 5.0, iterations=3) for r in range(5)]
    best, ms = s.autotune(list(range(5)), opts)
    assert best in (6, 14, 4, 12, 38, 46) and s.variant == best and ms > 0
