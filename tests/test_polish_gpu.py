"""Gradient-based plane and pose polishing after PatchMatch: the differentiation configuration
(24 views of 640x480 of the sphere scene, poses perturbed by 5 mm / 0.3 deg, 20 Adam steps).

Two starting points:
  - planes from PatchMatch solved with the perturbed poses: the per-pixel planes have already
    absorbed most of the pose error, the polish lowers the cost but hardly moves the poses;
  - planes of the true geometry (PatchMatch solved with the true poses, as a depth prior would
    give) with the perturbed poses: the polish pulls the poses towards the truth.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from luvas3d import DTYPE_F16, FORM_FAST, DenseStereo, SolveOptions, StereoOptions, scenes  # noqa: E402
from luvas3d import grad as G  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def workload():
    w = scenes.polish()
    st = DenseStereo(w.width, w.height, w.views)
    for i, im in enumerate(w.images):
        st.set_image(i, im)
    return w, st


def _planes(w, views):
    refs = list(range(len(w.views)))
    pm = DenseStereo(w.width, w.height, views, StereoOptions(storage=DTYPE_F16, form=FORM_FAST))
    for i, im in enumerate(w.images):
        pm.set_image(i, im)
    pm.solve_all(refs, [SolveOptions(w.sources[r], w.ranges[r][0], w.ranges[r][1],
                                     iterations=w.iterations) for r in refs])
    planes, weights = [], []
    for r in refs:
        hyp, cost = pm.read_hypotheses_layer(r)
        planes.append(G.planes_from_hypotheses(hyp).cuda().contiguous())
        weights.append(torch.tensor((cost < 0.5).astype(np.float32), device="cuda"))
    pm.destroy()
    return planes, weights


def _polish(w, st, views_for_planes):
    planes, weights = _planes(w, views_for_planes)
    res = G.polish(st, list(range(len(w.views))), w.sources, planes, steps=20, weights=weights)
    before = scenes.relative_pose_errors(w.views, w.true_views)
    after = scenes.relative_pose_errors(G.apply_deltas(w.views, res.deltas), w.true_views)
    return res, before, after


def test_polish_from_patchmatch_planes_lowers_the_cost(workload):
    w, st = workload
    res, before, after = _polish(w, st, w.views)
    assert len(res.losses) == 21 and all(np.isfinite(res.losses))
    assert res.losses[-1] < res.losses[0] - 0.02
    assert torch.count_nonzero(res.deltas[0]) == 0      # view 0 fixes the gauge


def test_polish_against_true_geometry_recovers_poses(workload):
    w, st = workload
    res, (rot0, tr0), (rot1, tr1) = _polish(w, st, w.true_views)
    assert res.losses[-1] < res.losses[0]
    assert tr1.mean() < 0.6 * tr0.mean(), (tr0.mean(), tr1.mean())
    assert rot1.mean() < 0.9 * rot0.mean(), (rot0.mean(), rot1.mean())
