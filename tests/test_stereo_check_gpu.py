"""The reference's own stereo self-test, restated on this repository's synthetic scene.

frontend/tools/verify/stereo-check.ts:11-74 renders five views 10 degrees apart on a ring around
its scene (640x360), solves the middle view against the other four (depths 0.1-2 m, 5
iterations, no prior, photometric pass) and requires more than 60 % of the surface pixels to
keep a packed depth with a median relative error under 0.4 %.  Its scene needs WebGL; here the
same check runs on the seeded sphere scene, through both forms.
"""
import numpy as np
import pytest

from luvas3d import (DTYPE_F16, DTYPE_F32, FORM_FAST, FORM_PLAIN, DenseStereo, SolveOptions,
                     StereoOptions, scenes)
from luvas3d.camera import Intrinsics, StereoView, look_at
from luvas3d.packing import unpack_depth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ring():
    k = Intrinsics(560.0, 560.0, 320.0, 180.0)
    views = []
    for step in (-2, -1, 0, 1, 2):
        a = np.radians(10.0 * step)
        views.append(StereoView(k, look_at((1.7 * np.sin(a), 0.2, 1.7 * np.cos(a)), (0.0, 0.0, 0.0))))
    imgs, truth = scenes.render_sphere(views, [(640, 360)] * 5, seed=21)
    return views, imgs, truth


@pytest.mark.parametrize("form,storage", [(FORM_PLAIN, DTYPE_F32), (FORM_FAST, DTYPE_F16)])
def test_patchmatch_recovers_depth_on_true_poses(ring, form, storage):
    views, imgs, truth = ring
    s = DenseStereo(640, 360, views, StereoOptions(form=form, storage=storage))
    for i, im in enumerate(imgs):
        s.set_image(i, im)
    s.solve(2, SolveOptions([0, 1, 3, 4], 0.1, 2.0, iterations=5))
    packed = s.depth_map(2)
    s.destroy()
    t = truth[2]
    covered = t > 0
    valid = covered & (packed != 0)
    err = np.abs(unpack_depth(packed[valid]) - t[valid]) / t[valid]
    frac, median = valid.sum() / covered.sum(), float(np.median(err))
    print(f"form {form}: {100 * frac:.1f} % of surface pixels valid, median {100 * median:.3f} %, "
          f"p90 {100 * np.percentile(err, 90):.2f} %")
    assert frac > 0.6 and median < 0.004
