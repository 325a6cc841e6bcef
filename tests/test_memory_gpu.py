"""The library's per-device memory pool (l3d_memory_trim, l3d_memory_reserved): trimming hands
the memory of destroyed handles back to the driver and leaves the memory of live handles, which
stay usable."""
import numpy as np
import pytest

from luvas3d import memory_reserved, trim_memory
from luvas3d.cloud import PointAccumulator

pytestmark = pytest.mark.gpu


def samples(n, seed):
    rng = np.random.default_rng(seed)
    s = np.zeros((n, 9))
    s[:, :3] = rng.uniform(-1.0, 1.0, (n, 3))
    s[:, 5] = 1.0
    s[:, 6:] = 0.5
    return s


def test_trim_releases_destroyed_handles_memory_and_keeps_live_handles():
    live = PointAccumulator(0.01)
    live.add_points(samples(1000, 1))
    first = live.cloud()
    big = PointAccumulator(0.0005)
    big.add_points(samples(2_000_000, 2))      # about 2 M cells: a table of 4 M slots, 350 MB
    assert big.size > 1_900_000
    r_big, u_big = memory_reserved()
    assert r_big >= u_big >= 300 << 20

    trim_memory(1 << 40)                        # more than the pool holds: nothing to release
    assert memory_reserved()[0] == r_big

    big.destroy()
    trim_memory(0)
    r, u = memory_reserved()
    assert u <= u_big - (300 << 20)             # the big table and its upload buffer are gone
    assert r <= r_big - (300 << 20)             # and their memory went back to the driver
    assert r >= u > 0                           # the live accumulator's table stays

    again = live.cloud()                        # the live handle still works after the trim
    np.testing.assert_array_equal(again.positions, first.positions)
    live.add_points(samples(1000, 3))
    assert live.size > first.positions.shape[0]
    live.destroy()
