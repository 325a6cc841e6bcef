"""The multi-GPU split driver on the device: ScanSplit over DeviceScan (the library's handles,
the all-gather of packed maps through NCCL on the stereo handle's stream, a brick-pool slab per
rank) in a one-rank NCCL process group.  One GPU holds one rank (ranks whose collectives wait on
each other never share a GPU), so this checks the device side of the split path; the exchange
between several ranks is checked over gloo on the CPU (test_shard.py).  The split's filtered
maps and its slab equal the direct single-handle path (solve_all, filter_all, a dense sweep)
bit for bit."""
import os
import socket
from datetime import timedelta

import numpy as np
import pytest

from helpers import arc_workload, assert_bit_equal
from luvas3d import (DTYPE_F16, FORM_FAST, DenseStereo, IntegrationView, SolveOptions,
                     StereoOptions, TsdfVolume, shard)

pytestmark = pytest.mark.gpu

DIMS, VOXEL, ORIGIN, MU = (48, 40, 24), 0.03, (-0.72, -0.6, 0.25), 0.12


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _stereo(views, imgs, W, H, stream):
    s = DenseStereo(W, H, views, StereoOptions(form=FORM_FAST, storage=DTYPE_F16, stream=stream))
    for i, im in enumerate(imgs):
        s.set_image(i, im)
    s.variant = 46
    return s


def test_scan_split_on_one_nccl_rank_equals_the_direct_path():
    import torch
    import torch.distributed as dist

    W, H = 96, 72
    views, imgs, truth, srcs = arc_workload(n=5, W=W, H=H, f=84.0, step_deg=5.0, seed=9)
    n = len(views)
    opts = [SolveOptions(srcs[r], 0.5, 5.0, iterations=3) for r in range(n)]
    needed = [2] * n
    iviews = [IntegrationView(v.intrinsics, v.pose, 5.0) for v in views]
    stream = torch.cuda.Stream()
    sptr = stream.cuda_stream

    # the direct path: one handle, every view, a dense volume
    direct = _stereo(views, imgs, W, H, sptr)
    direct.solve_all(list(range(n)), opts)
    direct.filter_all(list(range(n)), srcs, needed)
    want_f = [direct.read_filtered_layer(r) for r in range(n)]
    dense = TsdfVolume(W, H, VOXEL, ORIGIN, dense=DIMS, truncation=MU, weight_q8=True, stream=sptr)
    dense.integrate_many(iviews, stereo=direct, layers=list(range(n)))
    want_t, want_w = dense.read()
    assert (want_w > 0).sum() > 100

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(_free_port()))
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=timedelta(seconds=60),
                            device_id=torch.device("cuda", torch.cuda.current_device()))
    try:
        st = _stereo(views, imgs, W, H, sptr)
        coords = shard.slab_pool(DIMS, 0, 1)
        vol = TsdfVolume(W, H, VOXEL, ORIGIN, layout=(coords,), truncation=MU, weight_q8=True,
                         stream=sptr)
        split = shard.ScanSplit(shard.DeviceScan(st, vol, opts, srcs, needed, iviews),
                                [(W, H)] * n, 0, 1, device=torch.device("cuda"))
        split.step()
        st.synchronize()
        vol.synchronize()
        for r in range(n):
            assert np.array_equal(st.read_filtered_layer(r), want_f[r]), f"filtered map {r}"
        pt, pw = vol.read()
        t = np.full((DIMS[2], DIMS[1], DIMS[0]), np.nan, dtype=np.float32)
        w = np.zeros_like(t, dtype=np.uint16)
        shard.pool_to_dense(pt.reshape(-1), coords, DIMS, t)
        shard.pool_to_dense(pw.reshape(-1), coords, DIMS, w)
        assert_bit_equal(t, want_t, "tsdf")
        assert_bit_equal(w, want_w, "weight")
    finally:
        dist.destroy_process_group()
