"""Dense point cloud on the GPU (csrc/cloud.cu) against the oracle: the reference's accumulator
tests through l3d_cloud_add_points, and depth-map fusion of a solved, filtered scan.

The device sums in FP64 and the reference in f32, and the device table is filled in parallel, so
points are compared cell by cell (the cloud is returned ordered by cell): the same cells, the
same support, positions within 1e-5 m, normals within 1e-4, colours within one step."""
import numpy as np
import pytest

import oracle
from helpers import arc_workload
from luvas3d import DenseStereo, SolveOptions
from luvas3d.cloud import FusionView, PointAccumulator, fuse_depth_maps

pytestmark = pytest.mark.gpu


def test_averages_per_cell_and_merges_when_coarsened():
    """fusion.spec.ts:87-101 on the device."""
    a = PointAccumulator(0.01)
    a.add(0.001, 0.001, 0.001, 0, 0, 1, 100, 0, 0)
    a.add(0.003, 0.003, 0.003, 0, 0, 1, 200, 0, 0)
    a.add(0.015, 0.001, 0.001, 1, 0, 0, 0, 50, 0)
    c = a.cloud()
    assert len(c.support) == 2
    first = list(c.support).index(2)
    assert abs(c.positions[first, 0] - 0.002) < 5e-7
    assert c.colors[first, 0] == 150
    a.coarsen(2)
    c = a.cloud()
    assert len(c.support) == 1 and c.support[0] == 3
    assert abs(a.cell - 0.02) < 1e-15


def test_grows_past_its_initial_capacity():
    """fusion.spec.ts:103-107 on the device (one batch of 100 000 samples)."""
    a = PointAccumulator(0.001)
    s = np.zeros((100000, 9))
    s[:, 0] = np.arange(100000) * 0.002
    s[:, 4], s[:, 6], s[:, 7], s[:, 8] = 1, 1, 2, 3
    a.add_points(s)
    assert a.size == 100000
    c = a.cloud()
    np.testing.assert_array_equal(c.cells[:, 0], np.floor(s[:, 0] / 0.001).astype(np.int32))


def test_many_small_adds_grow_the_table():
    """Adds that fit the host-side bound skip the table read-back; the table still grows in
    time when the bound runs out, and repeated cells are not counted twice."""
    a = PointAccumulator(0.001)
    for b in range(150):
        s = np.zeros((2000, 9))
        s[:, 0] = (np.arange(2000) + b * 1000) * 0.002   # half of each batch repeats the last
        s[:, 4], s[:, 6], s[:, 7], s[:, 8] = 1, 1, 2, 3
        a.add_points(s)
    assert a.size == 151000
    c = a.cloud()
    assert c.support.max() == 2 and int(c.support.sum()) == 300000


def test_rejects_cells_out_of_range():
    a = PointAccumulator(1e-6)
    a.add(2.0, 0, 0, 0, 0, 1, 0, 0, 0)          # 2e6 cells from the origin
    with pytest.raises(Exception):
        _ = a.size


def _compare(got, want):
    gk = {tuple(c): i for i, c in enumerate(got.cells)}
    wk = {tuple(c): i for i, c in enumerate(want["cells"])}
    common = set(gk) & set(wk)
    assert len(common) >= 0.999 * max(len(gk), len(wk)), (len(gk), len(wk), len(common))
    gi = np.array([gk[c] for c in common])
    wi = np.array([wk[c] for c in common])
    same = got.support[gi] == want["support"][wi]
    assert same.mean() >= 0.999
    gi, wi = gi[same], wi[same]
    np.testing.assert_allclose(got.positions[gi], want["positions"][wi], atol=1e-5)
    np.testing.assert_allclose(got.normals[gi], want["normals"][wi], atol=1e-4)
    assert np.abs(got.colors[gi].astype(int) - want["colors"][wi]).max() <= 1


@pytest.fixture(scope="module")
def scan():
    views, imgs, truth, srcs = arc_workload(n=5, W=160, H=120, f=140.0)
    s = DenseStereo(160, 120, views)
    for i, im in enumerate(imgs):
        s.set_image(i, im)
    for r in range(5):
        s.solve(r, SolveOptions(srcs[r], 0.5, 5.0, iterations=3))
    thumbs = [(np.stack([im, im * 0.5, 1 - im], -1)[::2, ::2] * 255).astype(np.uint8) for im in imgs]
    maps = [s.filtered_map(r, srcs[r], 2) for r in range(5)]
    return views, srcs, s, thumbs, maps


@pytest.mark.parametrize("budget", [10 ** 9, 20000])
def test_fuse_depth_maps_matches_oracle(scan, budget):
    views, srcs, s, thumbs, maps = scan
    fv = [FusionView(views[r], srcs[r], 2, thumbs[r]) for r in range(5)]
    cloud, cell = fuse_depth_maps(s, fv, 0.004, budget)
    o = oracle.Cloud(0.004)
    for r in range(5):
        o.add_map(maps[r], views[r], thumbs[r])
        while o.size > budget:
            o.coarsen()
    assert abs(cell - o.cell) < 1e-12
    if budget < 10 ** 9:
        assert cell > 0.004                      # the budget forced coarsening
    assert len(cloud.support) > 5000
    _compare(cloud, o.cloud())


def test_add_from_host_map_equals_add_from_stereo(scan):
    views, srcs, s, thumbs, maps = scan
    a = PointAccumulator(0.003)
    b = PointAccumulator(0.003)
    for r in range(5):
        a.add_depth_map(views[r], thumbs[r], packed=maps[r])
        s.filter(r, srcs[r], 2)
        b.add_depth_map(views[r], thumbs[r], stereo=s)
    ca, cb = a.cloud(min_support=2), b.cloud(min_support=2)
    np.testing.assert_array_equal(ca.cells, cb.cells)
    np.testing.assert_array_equal(ca.support, cb.support)
    np.testing.assert_allclose(ca.positions, cb.positions, atol=1e-6)
