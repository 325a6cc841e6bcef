"""Properties at the benchmark's full size: the scan workload (48 views of 640x480, 8 sources,
5 iterations, TSDF 512^3 at 4 mm).

The oracle cannot solve this size in test time, so these check relations that hold at any size:
the exact batched form equals the plain per-view form bit for bit; the fast form's depth
accuracy against the rendered ground truth equals the plain form's; a batched solve equals its
views solved one by one; the batched consistency filter equals the per-view filter; the
many-view TSDF sweep (with and without the overlapped read-back) and the one-view-per-launch
integration of the batched maps equal the per-view integrations, and the FP32 oracle's
integration of the same maps (which does run in test time), bit for bit; and the equal-accuracy
forms (fast form with FP32 gathers, exact form) keep the plain form's accuracy against the
ground truth, batched or one by one.
"""
import numpy as np
import pytest

import oracle
from helpers import assert_bit_equal
from luvas3d import (DTYPE_F16, DTYPE_F32, FORM_EXACT, FORM_FAST, FORM_PLAIN, DenseStereo, IntegrationView,
                     SolveOptions, StereoOptions, TsdfVolume, scenes)
from luvas3d.packing import unpack_depth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scan():
    w = scenes.scan()
    refs = list(range(len(w.views)))
    opts = [SolveOptions(w.sources[r], w.ranges[r][0], w.ranges[r][1], iterations=w.iterations)
            for r in refs]
    return w, refs, opts


def solved(w, refs, opts, form, storage):
    s = DenseStereo(w.width, w.height, w.views, StereoOptions(storage=storage, form=form))
    for i, im in enumerate(w.images):
        s.set_image(i, im)
    s.solve_all(refs, opts)
    return s


def accuracy(s, w, refs):
    errs, surf, valid = [], 0, 0
    for r in refs:
        packed = s.depth_map(r)
        t = w.truth[r]
        m = t > 0
        ok = m & (packed != 0)
        surf += int(m.sum())
        valid += int(ok.sum())
        errs.append(np.abs(unpack_depth(packed[ok]) - t[ok]) / t[ok])
    e = np.concatenate(errs)
    return valid / surf, float(np.median(e)), float(np.mean(e < 0.01))


@pytest.fixture(scope="module")
def fast(scan):
    w, refs, opts = scan
    s = solved(w, refs, opts, FORM_FAST, DTYPE_F16)
    yield s
    s.destroy()


def test_fast_form_keeps_the_plain_forms_accuracy(scan, fast):
    w, refs, opts = scan
    plain = solved(w, refs, opts, FORM_PLAIN, DTYPE_F32)
    vp, mp, fp = accuracy(plain, w, refs)
    vf, mf, ff = accuracy(fast, w, refs)
    plain.destroy()
    print(f"plain: valid {vp:.4f} median {mp:.5f} within1% {fp:.4f}; "
          f"fast: valid {vf:.4f} median {mf:.5f} within1% {ff:.4f}")
    assert abs(vf - vp) < 0.005
    assert mf < mp * 1.05 and ff > fp - 0.01
    assert mp < 0.006          # the scene is solvable: median error under 0.6 %


def test_batch_equals_views_one_by_one(scan, fast):
    w, refs, opts = scan
    one = DenseStereo(w.width, w.height, w.views, StereoOptions(storage=DTYPE_F16, form=FORM_FAST))
    for i, im in enumerate(w.images):
        one.set_image(i, im)
    for r in (0, 17, 47):
        one.solve_all([r], [opts[r]])
        assert_bit_equal(one.read_hypotheses_layer(r)[0], fast.read_hypotheses_layer(r)[0],
                         f"view {r} hypotheses")
    one.destroy()


def test_filter_all_equals_per_view_filter(scan, fast):
    w, refs, opts = scan
    fast.filter_all(refs, w.sources, w.needed)
    for r in (0, 23, 47):
        got = fast.read_filtered_layer(r)
        fast.filter(r, w.sources[r], w.needed[r])
        assert_bit_equal(got, fast.read_filtered(), f"view {r} filtered map")
        if r >= 12:   # the first views, 0.2-0.4 m from the sphere, match too little to keep
            assert (got != 0).mean() > 0.3


def test_tsdf_sweep_equals_per_view_integration(scan, fast):
    w, refs, opts = scan
    fast.filter_all(refs, w.sources, w.needed)
    views = [IntegrationView(v.intrinsics, v.pose, w.ranges[i][1]) for i, v in enumerate(w.views)]

    def volume():
        return TsdfVolume(w.width, w.height, w.tsdf_voxel, w.tsdf_origin, dense=w.tsdf_dims,
                          truncation=w.tsdf_truncation, weight_q8=True)

    a, b, c, d = volume(), volume(), volume(), volume()
    for i, r in enumerate(refs):
        a.integrate(views[i], depth=fast.read_filtered_layer(r))
        d.integrate_layer(views[i], fast, r)
    b.integrate_many(views, stereo=fast, layers=refs)
    ta, wa = a.read()
    tb, wb = b.read()
    assert_bit_equal(tb, ta, "tsdf")
    assert_bit_equal(wb, wa, "weight")
    tc, wc = c.integrate_many_read(views, stereo=fast, layers=refs)
    assert_bit_equal(tc, ta, "tsdf (read-back overlapped)")
    assert_bit_equal(wc, wa, "weight (read-back overlapped)")
    td, wd = d.read()
    assert_bit_equal(td, ta, "tsdf (one view per launch from the batched maps)")
    assert_bit_equal(wd, wa, "weight (one view per launch from the batched maps)")
    assert (wa > 0).mean() > 0.05
    for v in (a, b, c, d):
        v.destroy()
    # the FP32 oracle integrating the same 48 maps into the same 512^3 volume (all host cores)
    o = oracle.Tsdf(w.width, w.height, w.tsdf_voxel, w.tsdf_origin, w.tsdf_truncation,
                    dense=w.tsdf_dims, weight_q8=True)
    for i, r in enumerate(refs):
        k = w.views[i].intrinsics
        o.integrate(dict(k=(k.fx, k.fy, k.cx, k.cy), R=w.views[i].pose.R, t=w.views[i].pose.t,
                         max_depth=w.ranges[i][1]), fast.read_filtered_layer(r))
    assert_bit_equal(tb.reshape(-1), o.tsdf.reshape(-1), "tsdf against the oracle")
    assert_bit_equal(wb.reshape(-1), o.weight.reshape(-1), "weight against the oracle")


@pytest.mark.parametrize("form,storage,variant", [(FORM_FAST, DTYPE_F32, 30), (FORM_EXACT, DTYPE_F32, 14)])
def test_equal_accuracy_forms_at_full_size(scan, form, storage, variant):
    w, refs, opts = scan
    s = DenseStereo(w.width, w.height, w.views, StereoOptions(storage=storage, form=form))
    for i, im in enumerate(w.images):
        s.set_image(i, im)
    s.variant = variant
    s.solve_all(refs, opts)
    v, m, f = accuracy(s, w, refs)
    print(f"form {form} variant {variant}: valid {v:.4f} median {m:.5f} within1% {f:.4f}")
    assert m < 0.006 and v > 0.99
    one = DenseStereo(w.width, w.height, w.views, StereoOptions(storage=storage, form=form))
    for i, im in enumerate(w.images):
        one.set_image(i, im)
    one.variant = variant
    for r in (5, 30):
        one.solve_all([r], [opts[r]])
        assert_bit_equal(one.read_hypotheses_layer(r)[0], s.read_hypotheses_layer(r)[0],
                         f"view {r} hypotheses")
    one.destroy()
    s.destroy()


def test_exact_form_equals_plain_form_at_full_size(scan):
    """The exact batched form (all 48 views per launch, CUDA graphs) and the plain per-view form
    compute the FP32 oracle's arithmetic, so at the benchmark's size too their packed depth maps
    agree bit for bit for every view, and their planes and costs for the views checked."""
    w, refs, opts = scan
    exact = solved(w, refs, opts, FORM_EXACT, DTYPE_F32)
    exact.set_graphs(True)
    exact.solve_all(refs, opts)  # a replayed graph gives the same solve
    plain = solved(w, refs, opts, FORM_PLAIN, DTYPE_F32)
    for r in refs:
        assert np.array_equal(exact.depth_map(r), plain.depth_map(r)), f"view {r} packed map"
    for r in (0, 17, 47):
        plain.solve(r, opts[r])
        hp, cp = plain.read_hypotheses()
        hx, cx = exact.read_hypotheses_layer(r)
        assert_bit_equal(hx, hp, f"view {r} hypotheses")
        assert_bit_equal(cx, cp, f"view {r} costs")
    exact.destroy()
    plain.destroy()


def test_plain_form_equals_the_fp32_oracle_at_full_size(scan):
    """Two of the scan's views solved at full size (640x480, 8 sources, 5 iterations) by the
    plain form and by the FP32 oracle (all host cores, a few seconds per view): planes, costs and
    packed maps bit for bit."""
    w, refs, opts = scan
    plain = DenseStereo(w.width, w.height, w.views, StereoOptions(storage=DTYPE_F32, form=FORM_PLAIN))
    for i, im in enumerate(w.images):
        plain.set_image(i, im)
    o = oracle.Stereo(w.width, w.height, w.views, w.images, 32)
    for r in (12, 40):
        plain.solve(r, opts[r])
        o.solve(r, w.sources[r], min_depth=w.ranges[r][0], max_depth=w.ranges[r][1],
                iterations=w.iterations)
        hp, cp = plain.read_hypotheses()
        assert_bit_equal(hp, o.hyp, f"view {r} planes")
        assert_bit_equal(cp, o.cost, f"view {r} costs")
        assert np.array_equal(plain.depth_map(r), o.depths[r]), f"view {r} packed map"
    plain.destroy()
