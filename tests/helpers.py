"""Shared test workloads (small enough for the oracle to finish in seconds)."""
import numpy as np

from luvas3d import scenes
from luvas3d.camera import Intrinsics, StereoView, look_at


def arc_workload(n=5, W=160, H=120, f=140.0, step_deg=5.0, seed=7):
    """Cameras on an arc looking at the sphere scene (the geometry of the reference's
    stereo self-test, frontend/tools/verify/stereo-check.ts:14-31, on this repo's scene)."""
    k = Intrinsics(f, f, W / 2, H / 2)
    views = []
    for s in range(n):
        a = np.radians(step_deg * (s - n // 2))
        views.append(StereoView(k, look_at((2.5 * np.sin(a), 0.3, 2.5 * np.cos(a)), (0, -0.3, 0))))
    imgs, truth = scenes.render_sphere(views, [(W, H)] * n, seed)
    srcs = [[j for j in range(n) if j != i] for i in range(n)]
    return views, imgs, truth, srcs


def bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint32) if a.dtype == np.float32 else a


def assert_bit_equal(got, want, what=""):
    g, w = bits(got), bits(want)
    if not np.array_equal(g, w):
        diff = np.argwhere(g != w)
        raise AssertionError(f"{what}: {len(diff)} of {g.size} entries differ; first at "
                             f"{diff[0].tolist()}: {got[tuple(diff[0])]} vs {want[tuple(diff[0])]}")
