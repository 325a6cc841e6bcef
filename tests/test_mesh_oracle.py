"""The surface-extraction oracle (oracle/mesh.cpp) against the reference's own surface-nets
tests (frontend/src/app/vision/fusion/fusion.spec.ts:35-83)."""
import numpy as np
import pytest

import oracle
from mesh_fixtures import sphere_volume


@pytest.fixture(scope="module")
def mesh():
    v = sphere_volume()
    pos, nrm, idx = oracle.extract_surface(v["origin"], v["voxel"], v["dims"], v["lookup"],
                                           v["tsdf"], v["weight"], 0.5)
    return v, pos, nrm, idx


def test_places_vertices_on_the_zero_level_set(mesh):
    v, pos, nrm, idx = mesh
    assert idx.size // 3 > 5000
    r = np.sqrt((pos.astype(np.float64) ** 2).sum(1))
    assert np.abs(r - v["radius"]).max() < v["voxel"] * 0.35


def test_builds_a_closed_surface_with_outward_normals(mesh):
    v, pos, nrm, idx = mesh
    tri = idx.reshape(-1, 3).astype(np.int64)
    edges = np.concatenate([tri[:, [0, 1]], tri[:, [1, 2]], tri[:, [2, 0]]])
    edges.sort(axis=1)
    _, counts = np.unique(edges, axis=0, return_counts=True)
    assert np.all(counts == 2)
    outward = ((nrm * pos).sum(1) > 0).mean()
    assert outward > 0.99


def test_keeps_the_main_component_and_drops_floaters(mesh):
    v, pos, nrm, idx = mesh
    n0 = pos.shape[0]
    fpos = np.concatenate([pos, np.array([[1, 1, 1], [1.001, 1, 1], [1, 1.001, 1]], np.float32)])
    fnrm = np.concatenate([nrm, np.zeros((3, 3), np.float32)])
    fidx = np.concatenate([idx, np.array([n0, n0 + 1, n0 + 2], np.uint32)])
    p, n, i = oracle.remove_small_components(fpos, fnrm, fidx, 0.01, 10)
    assert i.size == idx.size
    # the same triangles, re-indexed in order of first use
    np.testing.assert_array_equal(p[i], pos[idx])
    np.testing.assert_array_equal(n[i], nrm[idx])
    assert p.shape[0] == n0


def test_brick_grid_marks_the_shell(mesh):
    v = mesh[0]
    count = v["coords"].shape[0]
    assert 0 < count < int(np.prod(v["dims"]))
    lk = v["lookup"]
    assert np.array_equal(np.sort(lk[lk >= 0]), np.arange(count))
