"""Host side of the multi-GPU split (luvas3d/shard.py), on the CPU: view shards, the all-gather
of packed depth maps and the max-over-ranks timing over a 2-rank gloo process group, and the
z-slab TSDF split (brick pools per rank equal the single-volume result bit for bit)."""
import os
import socket
import tempfile

import numpy as np
import pytest

import oracle
from helpers import arc_workload
from luvas3d import shard
from luvas3d.scenes import ROOM_RESOLUTIONS

torch = pytest.importorskip("torch")


def test_shard_views_cover_every_view_once_and_balance_pixels():
    rng = np.random.default_rng(3)
    sizes = [ROOM_RESOLUTIONS[i] for i in rng.integers(0, 4, size=37)]
    for world in (1, 2, 3, 8):
        shards = shard.shard_views(sizes, world)
        flat = sorted(v for s in shards for v in s)
        assert flat == list(range(37))
        loads = [sum(sizes[v][0] * sizes[v][1] for v in s) for s in shards]
        biggest = max(w * h for w, h in sizes)
        assert max(loads) - min(loads) <= biggest
        assert all(s == sorted(s) for s in shards)
    assert shard.shard_views([(4, 4)] * 3, 5)[3:] == [[], []]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _maps(sizes, v):
    w, h = sizes[v]
    return np.random.default_rng(100 + v).integers(0, 2 ** 32, size=(h, w), dtype=np.uint64).astype(np.uint32)


def _worker(rank, world, port, sizes, out_dir):
    import torch.distributed as dist
    from datetime import timedelta

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        shards = shard.shard_views(sizes, world)
        local = {v: _maps(sizes, v) for v in shards[rank]}
        full = shard.gather_packed_maps(local, sizes, shards, rank)
        np.save(os.path.join(out_dir, f"maps{rank}.npy"), full.numpy().view(np.uint32))
        m = shard.max_over_ranks(10.0 + rank)
        np.save(os.path.join(out_dir, f"max{rank}.npy"), np.array([m]))
    finally:
        dist.destroy_process_group()


def test_gather_packed_maps_and_max_over_two_gloo_ranks():
    import torch.multiprocessing as mp

    sizes = [(13, 7), (20, 9), (5, 5), (16, 12), (9, 11)]
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_worker, args=(2, _free_port(), sizes, d), nprocs=2, join=True,
                           start_method="spawn")
        want = np.concatenate([_maps(sizes, v).reshape(-1) for v in range(len(sizes))])
        for r in range(2):
            np.testing.assert_array_equal(np.load(os.path.join(d, f"maps{r}.npy")), want)
            assert float(np.load(os.path.join(d, f"max{r}.npy"))[0]) == 11.0


def test_slab_bricks_split_evenly():
    assert shard.slab_bricks((64, 64, 64), 3) == [(0, 3), (3, 6), (6, 8)]
    assert shard.slab_bricks((8, 8, 20), 2) == [(0, 2), (2, 3)]


def test_slab_brick_pools_equal_the_dense_volume():
    """Each rank's slab, integrated as a brick pool, equals the dense volume's voxels bit for
    bit (the FP32 integrate oracle, which the TSDF kernels match bit for bit)."""
    views, imgs, truth, _ = arc_workload(n=3, W=96, H=72, f=84.0, step_deg=6.0, seed=5)
    dims = (44, 40, 42)
    args = dict(width=96, height=72, voxel=0.05, origin=(-1.1, -1.0, -1.05), truncation=0.15)
    packed = []
    for r in range(3):
        p = np.zeros((72, 96), dtype=np.uint32)
        for y, x in zip(*np.nonzero(truth[r] > 0)):
            p[y, x] = oracle.pack_sample(truth[r][y, x], (0.0, 0.0, -1.0), 0.2)
        packed.append(p)

    def kw(v):
        k = v.intrinsics
        return dict(k=(k.fx, k.fy, k.cx, k.cy), R=v.pose.R, t=v.pose.t, max_depth=5.0)

    dense = oracle.Tsdf(dense=dims, weight_q8=True, **args)
    for v, p in zip(views, packed):
        dense.integrate(kw(v), p)
    t_d = dense.tsdf.reshape(dims[2], dims[1], dims[0])
    w_d = dense.weight.reshape(dims[2], dims[1], dims[0])
    got_t = np.full_like(t_d, np.nan)
    got_w = np.zeros_like(w_d)
    for z0, z1 in shard.slab_bricks(dims, 3):
        coords = shard.slab_layout(dims, z0, z1)
        pool = oracle.Tsdf(coords=coords, weight_q8=True, **args)
        for v, p in zip(views, packed):
            pool.integrate(kw(v), p)
        shard.pool_to_dense(pool.tsdf, coords, dims, got_t)
        shard.pool_to_dense(pool.weight, coords, dims, got_w)
    assert (w_d > 0).sum() > 1000
    np.testing.assert_array_equal(got_t.view(np.uint32), t_d.view(np.uint32))
    np.testing.assert_array_equal(got_w, w_d)


class OracleScan:
    """ScanSplit backend on the CPU: the FP32 oracle stands in for the device kernels (which
    equal it bit for bit), so the split's host logic runs end to end over gloo ranks."""

    def __init__(self, w, dims, voxel, origin, coords):
        self.w, self.dims, self.voxel, self.origin, self.coords = w, dims, voxel, origin, coords
        self.o = oracle.Stereo(w.width, w.height, w.views, w.images, 32, threads=1)
        self.filtered = {}
        self.pool = None

    def solve(self, views):
        for v in views:
            self.o.solve(v, self.w.sources[v], min_depth=self.w.ranges[v][0],
                         max_depth=self.w.ranges[v][1], iterations=self.w.iterations)

    def packed_maps(self, views):
        return {v: self.o.depths[v] for v in views}

    def set_packed_maps(self, full):
        self.o._depths[:] = full.numpy().view(np.uint32)

    def filter_views(self, views):
        self.filtered.update({v: self.o.filter(v, self.w.sources[v], self.w.needed[v]) for v in views})

    def filtered_maps(self, views):
        return {v: self.filtered[v] for v in views}

    def set_filtered_maps(self, full):
        flat = full.numpy().view(np.uint32)
        n = self.w.width * self.w.height
        self.filtered = {v: flat[v * n:(v + 1) * n].reshape(self.w.height, self.w.width).copy()
                         for v in range(len(self.w.views))}

    def integrate(self):
        if self.coords is None:
            return
        self.pool = oracle.Tsdf(self.w.width, self.w.height, self.voxel, self.origin, 4 * self.voxel,
                                coords=self.coords, weight_q8=True, threads=1)
        for i, v in enumerate(self.w.views):
            k = v.intrinsics
            self.pool.integrate(dict(k=(k.fx, k.fy, k.cx, k.cy), R=v.pose.R, t=v.pose.t,
                                     max_depth=self.w.ranges[i][1]), self.filtered[i])


SPLIT_DIMS, SPLIT_VOXEL, SPLIT_ORIGIN = (48, 40, 20), 0.03, (-0.72, -0.6, 0.3)


def _arc_scan():
    """Five views 5 degrees apart on the sphere scene, 72 x 54, each against the other four."""
    from types import SimpleNamespace

    views, imgs, truth, srcs = arc_workload(n=5, W=72, H=54, f=63.0, step_deg=5.0, seed=9)
    return SimpleNamespace(width=72, height=54, views=views, images=imgs, sources=srcs,
                           ranges=[(0.5, 5.0)] * 5, iterations=3, needed=[2] * 5)


def _split_worker(rank, world, port, out_dir):
    import torch.distributed as dist
    from datetime import timedelta

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        w = _arc_scan()
        coords = shard.slab_pool(SPLIT_DIMS, rank, world)
        backend = OracleScan(w, SPLIT_DIMS, SPLIT_VOXEL, SPLIT_ORIGIN, coords)
        split = shard.ScanSplit(backend, [(w.width, w.height)] * len(w.views), rank, world)
        split.step()
        np.save(os.path.join(out_dir, f"w{world}_filtered{rank}.npy"),
                np.stack([backend.filtered[v] for v in range(len(w.views))]))
        np.save(os.path.join(out_dir, f"w{world}_views{rank}.npy"), np.array(split.views + [-1]))
        if coords is not None:
            t = np.full((SPLIT_DIMS[2], SPLIT_DIMS[1], SPLIT_DIMS[0]), np.nan, dtype=np.float32)
            wt = np.zeros_like(t, dtype=np.uint16)
            shard.pool_to_dense(backend.pool.tsdf, coords, SPLIT_DIMS, t)
            shard.pool_to_dense(backend.pool.weight, coords, SPLIT_DIMS, wt)
            np.save(os.path.join(out_dir, f"w{world}_tsdf{rank}.npy"), t)
            np.save(os.path.join(out_dir, f"w{world}_weight{rank}.npy"), wt)
    finally:
        dist.destroy_process_group()


def test_scan_split_over_two_and_three_gloo_ranks_equals_one_rank():
    """ScanSplit end to end (solve of each rank's views, the all-gather of packed maps, the filter
    of each rank's views, the all-gather of filtered maps, the z-slab TSDF), on 1, 2 and 3 gloo
    ranks: every rank's
    filtered maps and the slabs put together equal the one-rank result bit for bit.  Three ranks
    over a grid of three brick rows, and four views of five dealt by pixel count."""
    import torch.multiprocessing as mp

    with tempfile.TemporaryDirectory() as d:
        for world in (1, 2, 3):
            mp.start_processes(_split_worker, args=(world, _free_port(), d), nprocs=world,
                               join=True, start_method="spawn")
        want_f = np.load(os.path.join(d, "w1_filtered0.npy"))
        want_t = np.load(os.path.join(d, "w1_tsdf0.npy"))
        want_w = np.load(os.path.join(d, "w1_weight0.npy"))
        assert (want_f != 0).mean() > 0.05 and (want_w > 0).sum() > 100
        for world in (2, 3):
            t = np.full_like(want_t, np.nan)
            wt = np.zeros_like(want_w)
            views = []
            for r in range(world):
                np.testing.assert_array_equal(np.load(os.path.join(d, f"w{world}_filtered{r}.npy")), want_f)
                views += [v for v in np.load(os.path.join(d, f"w{world}_views{r}.npy")) if v >= 0]
                p = os.path.join(d, f"w{world}_tsdf{r}.npy")
                if os.path.exists(p):
                    rt, rw = np.load(p), np.load(os.path.join(d, f"w{world}_weight{r}.npy"))
                    m = ~np.isnan(rt)
                    t[m], wt[m] = rt[m], rw[m]
            assert sorted(views) == list(range(5))
            np.testing.assert_array_equal(t.view(np.uint32), want_t.view(np.uint32))
            np.testing.assert_array_equal(wt, want_w)


def test_scan_split_with_a_rank_that_owns_no_view():
    """Six gloo ranks over five views: one rank solves and filters nothing but still takes part in
    both all-gathers, and ends with every view's filtered map, equal to one rank's."""
    import torch.multiprocessing as mp

    with tempfile.TemporaryDirectory() as d:
        for world in (1, 6):
            mp.start_processes(_split_worker, args=(world, _free_port(), d), nprocs=world,
                               join=True, start_method="spawn")
        want_f = np.load(os.path.join(d, "w1_filtered0.npy"))
        owners = [[v for v in np.load(os.path.join(d, f"w6_views{r}.npy")) if v >= 0] for r in range(6)]
        assert sorted(v for o in owners for v in o) == list(range(5))
        assert any(not o for o in owners)
        for r in range(6):
            np.testing.assert_array_equal(np.load(os.path.join(d, f"w6_filtered{r}.npy")), want_f)


def test_empty_slab_ranks_integrate_nothing():
    dims = (16, 16, 16)  # two brick rows along z
    assert shard.slab_pool(dims, 2, 3) is None
    assert shard.slab_pool(dims, 0, 3).shape == (4, 4)
    assert [shard.slab_bricks(dims, 3)[r] for r in range(3)] == [(0, 1), (1, 2), (2, 2)]
