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
