"""The dense-cloud oracle (oracle/cloud.cpp) against the reference's own accumulator tests
(frontend/src/app/vision/fusion/fusion.spec.ts:86-107) and an independent numpy decode of a
depth map (luvas3d/packing.py)."""
import numpy as np

import oracle
from helpers import arc_workload
from luvas3d.packing import unpack_samples


def test_averages_per_cell_and_merges_when_coarsened():
    """fusion.spec.ts:87-101."""
    a = oracle.Cloud(0.01)
    a.add(0.001, 0.001, 0.001, 0, 0, 1, 100, 0, 0)
    a.add(0.003, 0.003, 0.003, 0, 0, 1, 200, 0, 0)
    a.add(0.015, 0.001, 0.001, 1, 0, 0, 0, 50, 0)
    c = a.cloud()
    assert len(c["support"]) == 2
    first = list(c["support"]).index(2)
    assert abs(c["positions"][first, 0] - 0.002) < 5e-7
    assert c["colors"][first, 0] == 150
    a.coarsen(2)
    c = a.cloud()
    assert len(c["support"]) == 1 and c["support"][0] == 3


def test_grows_past_its_initial_capacity():
    """fusion.spec.ts:103-107."""
    a = oracle.Cloud(0.001)
    for i in range(100000):
        a.add(i * 0.002, 0, 0, 0, 1, 0, 1, 2, 3)
    assert a.size == 100000


def _packed_map():
    views, imgs, truth, _ = arc_workload(n=1, W=48, H=36, f=42.0, seed=3)
    rng = np.random.default_rng(4)
    p = np.zeros((36, 48), dtype=np.uint32)
    for y, x in zip(*np.nonzero(truth[0] > 0)):
        n = rng.normal(size=3) * 0.3 + np.array([0, 0, -1.0])
        p[y, x] = oracle.pack_sample(truth[0][y, x], n / np.linalg.norm(n), rng.uniform(0, 0.9))
    return views[0], p


def test_add_map_matches_an_independent_decode():
    """With cells far smaller than the point spacing every sample is its own point: the cloud is
    the decoded depth map in world coordinates (depth-fusion.ts:42-74)."""
    view, packed = _packed_map()
    thumb = (np.arange(24 * 18 * 3) % 251).astype(np.uint8).reshape(18, 24, 3)
    a = oracle.Cloud(1e-5)
    a.add_map(packed, view, thumb)
    c = a.cloud()
    valid, d, n = unpack_samples(packed)
    assert len(c["support"]) == valid.sum() > 500
    k = view.intrinsics
    R, t = np.asarray(view.pose.R), np.asarray(view.pose.t)
    ys, xs = np.nonzero(valid)
    cam = np.stack([(xs - k.cx) / k.fx * d[ys, xs], (ys - k.cy) / k.fy * d[ys, xs], d[ys, xs]], -1)
    world = (cam - t) @ R                      # R^T (x - t)
    normals = n[ys, xs] @ R
    colors = thumb[np.minimum(17, ((ys + 0.5) * 0.5).astype(int)),
                   np.minimum(23, ((xs + 0.5) * 0.5).astype(int))]
    cells = np.floor(world / 1e-5).astype(np.int64)
    got = {tuple(cl): i for i, cl in enumerate(c["cells"].astype(np.int64))}
    idx = np.array([got[tuple(cl)] for cl in cells])
    np.testing.assert_allclose(c["positions"][idx], world, rtol=1e-6, atol=1e-7)
    np.testing.assert_allclose(c["normals"][idx], normals / np.linalg.norm(normals, axis=1, keepdims=True),
                               atol=1e-6)
    np.testing.assert_array_equal(c["colors"][idx], colors)
    assert np.all(c["support"] == 1)
