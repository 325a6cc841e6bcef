"""Surface extraction on the GPU (csrc/mesh.cu, csrc/scan.cu) against the oracle, bit for bit:
the reference's sphere test volume (fusion.spec.ts:6-33), a TSDF integrated from depth maps (pool
and dense layouts), component removal, and the brick grid."""
import numpy as np
import pytest

import oracle
from helpers import arc_workload, assert_bit_equal
from luvas3d import IntegrationView, TsdfVolume
from luvas3d import mesh as M
from mesh_fixtures import sphere_volume

pytestmark = pytest.mark.gpu


def _same(got, pos, nrm, idx):
    assert got.positions.shape == pos.shape and got.indices.shape == idx.shape
    assert_bit_equal(got.positions, pos, "positions")
    assert_bit_equal(got.normals, nrm, "normals")
    np.testing.assert_array_equal(got.indices, idx)


@pytest.fixture(scope="module")
def sphere():
    return sphere_volume()


def test_sphere_surface_equals_oracle(sphere):
    v = sphere
    got = M.extract_surface(v, 0.5)
    pos, nrm, idx = oracle.extract_surface(v["origin"], v["voxel"], v["dims"], v["lookup"],
                                           v["tsdf"], v["weight"], 0.5)
    assert idx.size // 3 > 5000
    _same(got, pos, nrm, idx)


def test_components_equal_oracle(sphere):
    v = sphere
    m = M.extract_surface_device(v, 0.5)
    base = m.read()
    for fraction, min_faces in [(0.01, 10), (0.6, 10), (2.0, 10)]:
        r = m.remove_small_components(fraction, min_faces)
        got = r.read()
        r.destroy()
        p, n, i = oracle.remove_small_components(base.positions, base.normals, base.indices,
                                                 fraction, min_faces)
        _same(got, p, n, i)
    m.destroy()


def test_brick_grid_equals_oracle(sphere):
    v = sphere
    rng = np.random.default_rng(0)
    pts = rng.normal(size=(5000, 3)) * 0.05
    extent = [0.2, 0.25, 0.3]
    origin = [-0.1, -0.12, -0.15]
    dims, coords, lookup = M.brick_grid(origin, 0.002, extent, pts, 0.008)
    d2, c2, l2 = oracle.brick_grid(origin, 0.002, extent, pts, 0.008)
    np.testing.assert_array_equal(dims, d2)
    np.testing.assert_array_equal(coords, c2)
    np.testing.assert_array_equal(lookup, l2)


@pytest.fixture(scope="module")
def integrated():
    """A TSDF of 3 depth maps of the sphere scene, as a brick pool and as a dense grid."""
    views, imgs, truth, _ = arc_workload(n=3, W=160, H=120, f=140.0)
    packed = []
    for r in range(3):
        p = np.zeros((120, 160), np.uint32)
        for y, x in zip(*np.nonzero(truth[r] > 0)):
            p[y, x] = oracle.pack_sample(truth[r][y, x], (0.0, 0.0, -1.0), 0.2)
        packed.append(p)
    dims = (64, 48, 64)
    origin, voxel = (-0.8, -1.1, -0.8), 0.025
    ivs = [IntegrationView(v.intrinsics, v.pose, 5.0) for v in views]
    dense = TsdfVolume(160, 120, voxel, origin, dense=dims, truncation=0.1)
    for iv, p in zip(ivs, packed):
        dense.integrate(iv, depth=p)
    nb = [(d + 7) // 8 for d in dims]
    bz, by, bx = np.meshgrid(np.arange(nb[2]), np.arange(nb[1]), np.arange(nb[0]), indexing="ij")
    keep = ((bx + by + bz) % 3 != 0).reshape(-1)          # a pool of two thirds of the bricks
    coords = np.zeros((int(keep.sum()), 4), np.int32)
    coords[:, 0], coords[:, 1], coords[:, 2] = bx.reshape(-1)[keep], by.reshape(-1)[keep], bz.reshape(-1)[keep]
    pool = TsdfVolume(160, 120, voxel, origin, layout=(coords, None, coords.shape[0]), truncation=0.1)
    for iv, p in zip(ivs, packed):
        pool.integrate(iv, depth=p)
    return dict(dense=dense, pool=pool, coords=coords, dims=dims, origin=origin, voxel=voxel)


def test_pool_volume_surface_equals_oracle(integrated):
    pool, coords = integrated["pool"], integrated["coords"]
    got = M.extract_surface(pool, 0.5)
    tsdf, weight = pool.read()
    gdims = coords[:, :3].max(0) + 1
    lookup = np.full(int(np.prod(gdims)), -1, np.int32)
    lookup[(coords[:, 2] * gdims[1] + coords[:, 1]) * gdims[0] + coords[:, 0]] = np.arange(len(coords))
    pos, nrm, idx = oracle.extract_surface(integrated["origin"], integrated["voxel"], gdims, lookup,
                                           tsdf.reshape(-1), weight.reshape(-1).astype(np.float32), 0.5)
    assert idx.size > 3000
    _same(got, pos, nrm, idx)


def test_dense_volume_surface_equals_oracle(integrated):
    """A dense grid is extracted as the pool of all its bricks in dense brick order."""
    dense, dims = integrated["dense"], integrated["dims"]
    got = M.extract_surface(dense, 0.5)
    tsdf, weight = dense.read()
    t3 = tsdf.reshape(dims[2], dims[1], dims[0])
    w3 = weight.reshape(dims[2], dims[1], dims[0]).astype(np.float32)
    nb = [(d + 7) // 8 for d in dims]
    bt = np.ones((nb[2] * 8, nb[1] * 8, nb[0] * 8), np.float32)
    bw = np.zeros_like(bt)
    bt[:dims[2], :dims[1], :dims[0]] = t3
    bw[:dims[2], :dims[1], :dims[0]] = w3
    # brick-major pool: brick (x fastest), then voxel x + 8y + 64z
    pt = bt.reshape(nb[2], 8, nb[1], 8, nb[0], 8).transpose(0, 2, 4, 1, 3, 5).reshape(-1)
    pw = bw.reshape(nb[2], 8, nb[1], 8, nb[0], 8).transpose(0, 2, 4, 1, 3, 5).reshape(-1)
    lookup = np.arange(nb[0] * nb[1] * nb[2], dtype=np.int32)
    pos, nrm, idx = oracle.extract_surface(integrated["origin"], integrated["voxel"], nb, lookup, pt, pw, 0.5)
    assert idx.size > 3000
    _same(got, pos, nrm, idx)
