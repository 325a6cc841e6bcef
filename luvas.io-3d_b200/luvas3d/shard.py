"""Splitting one scan over several GPUs (one process per GPU, torch.distributed).

The photometric stage needs nothing from other views' results, so reference views are dealt out
to ranks with no exchange.  Two steps do exchange data:

  - the geometric pass and the consistency filter read the packed depth maps of neighbouring
    views, which may live on other ranks: `gather_packed_maps` all-gathers every rank's maps
    (4 bytes per pixel, once per pass) so each rank holds all of them;
  - TSDF integration is split by z-slabs of 8^3 bricks: each rank owns the bricks of its slab as
    a brick pool (`slab_layout`, the BrickGrid.build() layout) and integrates every view's
    filtered map into them.  A brick pool addresses voxels by the same integer coordinates as
    the dense grid, so each rank's voxels equal the corresponding voxels of a single-GPU dense
    volume bit for bit, and the slabs need no reduction.

Everything here is host logic over a process group; the device work stays in the library's
kernels.  With the NCCL backend the tensors are CUDA tensors and the gathers cross NVLink; the
tests run the same functions over gloo on the CPU.
"""
from __future__ import annotations

import contextlib
from typing import Sequence

import numpy as np


def shard_views(sizes: Sequence[tuple[int, int]], world: int) -> list[list[int]]:
    """Reference views per rank, balanced by pixel count (largest first onto the least-loaded
    rank; ties go to the lower rank), each rank's list in ascending view order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    load = [0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    order = sorted(range(len(sizes)), key=lambda i: (-sizes[i][0] * sizes[i][1], i))
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += sizes[i][0] * sizes[i][1]
    return [sorted(v) for v in out]


def _offsets(sizes):
    return np.concatenate([[0], np.cumsum([w * h for w, h in sizes])]).astype(np.int64)


def gather_packed_maps(local: dict, sizes: Sequence[tuple[int, int]], shards: list[list[int]],
                       rank: int, group=None, device=None):
    """All-gather packed depth maps.  `local` maps each view this rank owns (shards[rank]) to its
    (H, W) packed map (numpy uint32 or an int32/uint32 tensor).  Returns a flat tensor of every
    view's map concatenated in view order (4-byte integers) on `device`.

    Each rank sends one buffer of its views back to back, padded to the largest shard, so the
    gather moves (world - 1) x (largest shard) x 4 bytes into every rank."""
    import torch
    import torch.distributed as dist

    world = len(shards)
    off = _offsets(sizes)
    counts = [int(sum(sizes[v][0] * sizes[v][1] for v in s)) for s in shards]
    cap = max(1, max(counts))
    send = torch.zeros(cap, dtype=torch.int32, device=device)
    pos = 0
    for v in shards[rank]:
        m = local[v]
        t = (torch.from_numpy(np.ascontiguousarray(m).view(np.int32).reshape(-1))
             if isinstance(m, np.ndarray) else m.reshape(-1).view(torch.int32))
        n = sizes[v][0] * sizes[v][1]
        if t.numel() != n:
            raise ValueError(f"view {v}: map has {t.numel()} pixels, expected {n}")
        send[pos:pos + n] = t.to(send.device)
        pos += n
    recv = [torch.empty(cap, dtype=torch.int32, device=device) for _ in range(world)]
    dist.all_gather(recv, send, group=group)
    full = torch.empty(int(off[-1]), dtype=torch.int32, device=device)
    for r in range(world):
        pos = 0
        for v in shards[r]:
            n = sizes[v][0] * sizes[v][1]
            full[int(off[v]):int(off[v]) + n] = recv[r][pos:pos + n]
            pos += n
    return full


def max_over_ranks(value: float, group=None, device=None) -> float:
    """The largest of every rank's value (the multi-GPU timing rule)."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def slab_bricks(dims: Sequence[int], world: int) -> list[tuple[int, int]]:
    """Brick-row ranges [z0, z1) along z, one per rank, as even as whole bricks allow."""
    nbz = (int(dims[2]) + 7) // 8
    base, extra = divmod(nbz, world)
    out, z = [], 0
    for r in range(world):
        n = base + (1 if r < extra else 0)
        out.append((z, z + n))
        z += n
    return out


def slab_layout(dims: Sequence[int], z0: int, z1: int) -> np.ndarray:
    """Brick-pool coordinates (count x 4 int32: bx, by, bz, 0) of the dense grid's bricks with
    bz in [z0, z1), x fastest then y then z (the order of the dense brick index)."""
    nbx, nby = (int(dims[0]) + 7) // 8, (int(dims[1]) + 7) // 8
    bz, by, bx = np.meshgrid(np.arange(z0, z1), np.arange(nby), np.arange(nbx), indexing="ij")
    coords = np.zeros((bx.size, 4), dtype=np.int32)
    coords[:, 0] = bx.reshape(-1)
    coords[:, 1] = by.reshape(-1)
    coords[:, 2] = bz.reshape(-1)
    return coords


def pool_to_dense(values: np.ndarray, coords: np.ndarray, dims: Sequence[int],
                  out: np.ndarray) -> None:
    """Scatters a brick pool's voxels (count * 512, voxel b*512 + x + 8y + 64z) into a dense
    (Z, Y, X) array, dropping voxels outside the grid."""
    X, Y, Z = (int(d) for d in dims)
    v = values.reshape(-1, 8, 8, 8)  # brick, z, y, x
    for b, (bx, by, bz, _) in enumerate(coords):
        x0, y0, z0 = bx * 8, by * 8, bz * 8
        x1, y1, z1 = min(x0 + 8, X), min(y0 + 8, Y), min(z0 + 8, Z)
        out[z0:z1, y0:y1, x0:x1] = v[b, :z1 - z0, :y1 - y0, :x1 - x0]


def slab_pool(dims: Sequence[int], rank: int, world: int) -> np.ndarray | None:
    """The brick-pool coordinates of rank's z-slab, or None when the slab is empty (more ranks
    than brick rows along z: such a rank integrates nothing)."""
    z0, z1 = slab_bricks(dims, world)[rank]
    return slab_layout(dims, z0, z1) if z1 > z0 else None


class ScanSplit:
    """One scan split over the ranks of a process group: the photometric solve of this rank's
    views (shard_views), one all-gather of every view's packed depth map, the consistency filter
    of this rank's views (it reads every view's packed map), one all-gather of every view's
    filtered map, and the TSDF integration of every view into this rank's z-slab of bricks.
    Each rank's slab equals the same bricks of a single-GPU volume bit for bit, and every rank's
    packed and filtered maps equal the single-GPU maps bit for bit (the batched photometric solve
    of a subset of views equals its views solved alone, and the filter of a view depends only on
    the packed maps).

    `backend` does the device work:
      solve(views)              photometric solve of the given reference views;
      packed_maps(views)        {view: that view's packed map (H, W) or flat}, 4-byte integers;
      set_packed_maps(full)     every view's packed map, concatenated in view order (flat);
      filter_views(views)       consistency filter of the given views;
      filtered_maps(views)      {view: that view's filtered map}, 4-byte integers;
      set_filtered_maps(full)   every view's filtered map, concatenated in view order (flat);
      integrate()               TSDF integration of every view into the rank's slab."""

    def __init__(self, backend, sizes: Sequence[tuple[int, int]], rank: int, world: int,
                 group=None, device=None):
        self.backend = backend
        self.sizes = [(int(a), int(b)) for a, b in sizes]
        self.rank, self.world = int(rank), int(world)
        self.group, self.device = group, device
        self.shards = shard_views(self.sizes, self.world)
        self.views = self.shards[self.rank]

    def solve(self) -> None:
        if self.views:
            self.backend.solve(self.views)

    def exchange(self) -> None:
        ctx = getattr(self.backend, "context", None)
        with (ctx() if ctx else contextlib.nullcontext()):
            local = self.backend.packed_maps(self.views)
            full = gather_packed_maps(local, self.sizes, self.shards, self.rank, self.group,
                                      self.device)
            self.backend.set_packed_maps(full)

    def filter(self) -> None:
        if self.views:
            self.backend.filter_views(self.views)

    def exchange_filtered(self) -> None:
        ctx = getattr(self.backend, "context", None)
        with (ctx() if ctx else contextlib.nullcontext()):
            local = self.backend.filtered_maps(self.views)
            full = gather_packed_maps(local, self.sizes, self.shards, self.rank, self.group,
                                      self.device)
            self.backend.set_filtered_maps(full)

    def integrate(self) -> None:
        self.backend.integrate()

    def step(self) -> None:
        self.solve()
        self.exchange()
        self.filter()
        self.exchange_filtered()
        self.integrate()


class _DeviceArray:
    """A device buffer seen through the CUDA array interface (zero-copy torch views)."""

    def __init__(self, ptr: int, n: int, typestr: str = "<i4"):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": typestr,
                                         "data": (int(ptr), False), "version": 3, "strides": None}


def device_view(ptr: int, n: int):
    """A flat int32 torch tensor over n 4-byte integers of device memory at ptr (no copy)."""
    import torch

    return torch.as_tensor(_DeviceArray(ptr, n), device="cuda")


class DeviceScan:
    """ScanSplit backend over the library's handles: a DenseStereo holding every view's image
    and packed map, and (for a rank with a non-empty slab) a brick-pool TsdfVolume of the slab.
    The exchange (copies and the all-gather) runs on the stereo handle's stream (context())."""

    def __init__(self, stereo, tsdf, options, sources, needed, iviews):
        import torch

        self.stereo, self.tsdf = stereo, tsdf
        self.options, self.sources, self.needed, self.iviews = options, sources, needed, iviews
        self.refs = list(range(len(iviews)))
        self.stream = torch.cuda.ExternalStream(stereo.stream)
        sizes = stereo.sizes
        self.off = _offsets(sizes)
        self.maps = device_view(stereo.buffers().depths, int(self.off[-1]))
        self.filtered = None

    def solve(self, views):
        self.stereo.solve_all(views, [self.options[v] for v in views])

    def packed_maps(self, views):
        return {v: self.maps[int(self.off[v]):int(self.off[v + 1])] for v in views}

    def context(self):
        """The exchange runs on the stereo handle's stream, ordered after its solves."""
        import torch

        return torch.cuda.stream(self.stream)

    def set_packed_maps(self, full):
        self.maps.copy_(full)

    def filter_views(self, views):
        self.stereo.filter_all(views, [self.sources[v] for v in views], [self.needed[v] for v in views])
        if self.filtered is None:  # filtered_all exists after the first filter
            self.filtered = device_view(self.stereo.buffers().filtered_all, int(self.off[-1]))

    def filtered_maps(self, views):
        return {v: self.filtered[int(self.off[v]):int(self.off[v + 1])] for v in views}

    def set_filtered_maps(self, full):
        if self.filtered is None:  # a rank without views: allocate filtered_all by filtering none
            self.stereo.filter_all([0], [self.sources[0]], [self.needed[0]])
            self.filtered = device_view(self.stereo.buffers().filtered_all, int(self.off[-1]))
        self.filtered.copy_(full)

    def integrate(self):
        if self.tsdf is not None:
            self.tsdf.integrate_many(self.iviews, stereo=self.stereo, layers=self.refs)
