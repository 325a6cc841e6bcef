"""Coarse-to-fine start in the fast form (init_coarse, patchmatch.wgsl.ts:296-333): a batched
fine solve seeded by the coarse level's batched planes equals the per-view coarse-to-fine
schedule of methods/coarse-to-fine.ts bit for bit, and the coarse start keeps the accuracy."""
import numpy as np
import pytest

from helpers import arc_workload
from luvas3d import (DTYPE_F16, FORM_FAST, STEREO_METHODS, DenseStereo, L3dError, SolveOptions,
                     StereoOptions, scale_intrinsics)
from luvas3d.camera import StereoView
from luvas3d.stereo import StereoInput, StereoSettings

pytestmark = pytest.mark.gpu

W, H = 160, 120


@pytest.fixture(scope="module")
def scene():
    return arc_workload(n=5, W=W, H=H, f=140.0)


def _levels(views, imgs):
    cw, ch = W // 2, H // 2
    cviews = [StereoView(scale_intrinsics(v.intrinsics, cw / W, ch / H), v.pose) for v in views]
    coarse = DenseStereo(cw, ch, cviews, StereoOptions(depth_maps=False, storage=DTYPE_F16, form=FORM_FAST))
    fine = DenseStereo(W, H, views, StereoOptions(coarse=coarse, storage=DTYPE_F16, form=FORM_FAST))
    for i, im in enumerate(imgs):
        coarse.set_image(i, im[::2, ::2].copy())
        fine.set_image(i, im)
    return coarse, fine


def test_batched_coarse_to_fine_equals_per_view(scene):
    views, imgs, truth, srcs = scene
    co = [SolveOptions(srcs[r], 0.5, 5.0, iterations=3, pack=False) for r in range(5)]
    fo = [SolveOptions(srcs[r], 0.5, 5.0, iterations=2, from_coarse=True) for r in range(5)]
    c1, f1 = _levels(views, imgs)
    c1.solve_all(range(5), co)
    f1.solve_all(range(5), fo)
    c2, f2 = _levels(views, imgs)
    for r in range(5):
        c2.solve(r, co[r])
        f2.solve(r, fo[r])
        got, _ = f1.read_hypotheses_layer(r)
        want, _ = f2.read_hypotheses()
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), f"view {r}"
        d = got[..., 3]
        m = truth[r] > 0
        assert np.median(np.abs(d[m] - truth[r][m]) / truth[r][m]) < 0.01


def test_coarse_start_is_used(scene):
    """The fine level started from the coarse planes differs from a random start."""
    views, imgs, truth, srcs = scene
    c, f = _levels(views, imgs)
    c.solve(0, SolveOptions(srcs[0], 0.5, 5.0, iterations=3, pack=False))
    f.solve(0, SolveOptions(srcs[0], 0.5, 5.0, iterations=0, from_coarse=True))
    seeded, _ = f.read_hypotheses()
    f.solve(0, SolveOptions(srcs[0], 0.5, 5.0, iterations=0))
    random, _ = f.read_hypotheses()
    m = truth[0] > 0
    err_seeded = np.median(np.abs(seeded[..., 3][m] - truth[0][m]) / truth[0][m])
    err_random = np.median(np.abs(random[..., 3][m] - truth[0][m]) / truth[0][m])
    assert err_seeded < 0.5 * err_random


def test_coarse_state_errors(scene):
    views, imgs, truth, srcs = scene
    c, f = _levels(views, imgs)
    with pytest.raises(L3dError):      # no batched coarse planes yet
        f.solve_all([0, 1], [SolveOptions(srcs[r], 0.5, 5.0, iterations=1, from_coarse=True) for r in (0, 1)])
    c.solve(1, SolveOptions(srcs[1], 0.5, 5.0, iterations=1, pack=False))
    with pytest.raises(L3dError):      # the coarse planes are of another view
        f.solve(0, SolveOptions(srcs[0], 0.5, 5.0, iterations=1, from_coarse=True))


def test_coarse_to_fine_method_in_the_fast_form(scene):
    views, imgs, truth, srcs = scene
    inp = StereoInput(W, H, views, srcs, [(0.5, 5.0)] * 5, gray=lambda layer, w, h: imgs[layer] if w == W else imgs[layer][::2, ::2].copy())
    run = STEREO_METHODS["coarse-to-fine"].create(
        inp, StereoSettings(iterations=3, fine_iterations=2,
                            options=StereoOptions(storage=DTYPE_F16, form=FORM_FAST)))
    try:
        run.solve(2)
        hyp = run.stereo.hypotheses
        m = truth[2] > 0
        assert np.median(np.abs(hyp[..., 3][m] - truth[2][m]) / truth[2][m]) < 0.01
    finally:
        run.destroy()
