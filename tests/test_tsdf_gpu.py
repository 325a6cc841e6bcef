"""TSDF parity: the CUDA integration kernels through the C ABI against the FP32 oracle.

The per-voxel arithmetic is the oracle's, so tsdf values and weights (f32 or Q8.8 uint16) are
compared bit for bit; the required tolerance (TSDF 1e-5 absolute, integer weights exact) is met
with margin zero.  The many-view sweep must equal the per-view launches in order.
"""
import numpy as np
import pytest

import oracle
from helpers import assert_bit_equal
from luvas3d import BrickGrid, IntegrationView, TsdfVolume, scenes
from luvas3d.camera import Intrinsics, Pose, StereoView, look_at

pytestmark = pytest.mark.gpu


def packed_views(n=6, W=120, H=90, f=105.0, seed=5, cost=0.3):
    """Views around the sphere with exact packed depth maps (normals from the sphere/plane)."""
    k = Intrinsics(f, f, W / 2, H / 2)
    views = []
    for i in range(n):
        a = 2 * np.pi * i / n
        views.append(StereoView(k, look_at((2.2 * np.sin(a), 0.5, 2.2 * np.cos(a)), (0, -0.2, 0))))
    _, truth = scenes.render_sphere(views, [(W, H)] * n, seed)
    maps = []
    rng = np.random.default_rng(seed)
    ys, xs = np.mgrid[0:H, 0:W]
    for v, d in zip(views, truth):
        rays = np.stack([(xs - k.cx) / k.fx, (ys - k.cy) / k.fy, np.ones((H, W))], -1)
        pc = rays * d[..., None]
        pw = (pc - v.pose.t) @ v.pose.R  # R^T (pc - t)
        on_plane = np.abs(pw[..., 1] + 1) < 1e-3
        nw = np.where(on_plane[..., None], np.array([0, 1.0, 0]),
                      pw / np.maximum(np.linalg.norm(pw, axis=-1, keepdims=True), 1e-9))
        nc = nw @ v.pose.R.T
        m = np.zeros((H, W), dtype=np.uint32)
        c = rng.uniform(0, 0.5, size=(H, W)) if cost is None else np.full((H, W), cost)
        for y in range(H):
            for x in range(W):
                if d[y, x] > 0 and (x + 2 * y) % 11:
                    m[y, x] = oracle.pack_sample(d[y, x], nc[y, x], c[y, x])
        maps.append(m)
    return views, maps


@pytest.fixture(scope="module")
def scene():
    return packed_views()


def view_kw(v, max_depth=6.0, confidence=0.0, prior=None):
    k = v.intrinsics
    return dict(k=(k.fx, k.fy, k.cx, k.cy), R=v.pose.R, t=v.pose.t, max_depth=max_depth,
                confidence=confidence, prior=prior)


def gpu_view(v, max_depth=6.0, confidence=0.0, prior=None):
    return IntegrationView(v.intrinsics, v.pose, max_depth, prior, confidence)


@pytest.mark.parametrize("q8", [False, True])
@pytest.mark.parametrize("confidence", [0.0, 2.0])
def test_dense_integrate_bit_exact(scene, q8, confidence):
    views, maps = scene
    W, H = 120, 90
    dims, voxel, origin, mu = (64, 48, 56), 0.04, (-1.28, -1.1, -1.1), 0.12
    o = oracle.Tsdf(W, H, voxel, origin, mu, dense=dims, weight_q8=q8)
    g = TsdfVolume(W, H, voxel, origin, dense=dims, truncation=mu, weight_q8=q8)
    for v, m in zip(views, maps):
        o.integrate(view_kw(v, confidence=confidence), m)
        g.integrate(gpu_view(v, confidence=confidence), depth=m)
    t, w = g.read()
    assert_bit_equal(t.reshape(-1), o.tsdf, "tsdf")
    assert_bit_equal(w.reshape(-1), o.weight, "weight")
    assert (o.weight > 0).sum() > 5000


def test_integrate_many_equals_sequence(scene):
    views, maps = scene
    W, H = 120, 90
    dims, voxel, origin, mu = (64, 48, 56), 0.04, (-1.28, -1.1, -1.1), 0.12
    for q8 in (False, True):
        a = TsdfVolume(W, H, voxel, origin, dense=dims, truncation=mu, weight_q8=q8)
        b = TsdfVolume(W, H, voxel, origin, dense=dims, truncation=mu, weight_q8=q8)
        for v, m in zip(views, maps):
            a.integrate(gpu_view(v, confidence=1.5), depth=m)
        b.integrate_many([gpu_view(v, confidence=1.5) for v in views], depths=np.stack(maps))
        ta, wa = a.read()
        tb, wb = b.read()
        assert_bit_equal(tb, ta, "tsdf")
        assert_bit_equal(wb, wa, "weight")


@pytest.mark.parametrize("layout", ["dense", "ragged", "pool"])
@pytest.mark.parametrize("q8", [False, True])
def test_integrate_many_read_equals_sweep_then_read(scene, layout, q8):
    """The sweep split into voxel ranges with overlapped read-back gives the volume of
    integrate_many + read, bit for bit, into pageable numpy and pinned torch buffers."""
    import torch
    views, maps = scene
    W, H = 120, 90
    iv = [gpu_view(v, confidence=1.5) for v in views]
    if layout == "pool":
        voxel = 0.03
        grid = BrickGrid((-1.3, -1.2, -1.3), voxel, (2.6, 2.4, 2.6))
        rng = np.random.default_rng(2)
        pts = rng.normal(size=(2000, 3))
        pts /= np.linalg.norm(pts, axis=1, keepdims=True)
        for p in pts:
            grid.mark(*p, voxel * 4)
        coords, lookup, count = grid.build()

        def make():
            return TsdfVolume(W, H, voxel, grid.origin, grid=grid, layout=(coords, lookup, count),
                              weight_q8=q8)
    else:
        dims = (64, 48, 56) if layout == "dense" else (37, 21, 29)

        def make():
            return TsdfVolume(W, H, 0.04, (-1.28, -1.1, -1.1), dense=dims, truncation=0.12,
                              weight_q8=q8)
    a, b, c = make(), make(), make()
    a.integrate_many(iv, depths=np.stack(maps))
    ta, wa = a.read()
    tb, wb = b.integrate_many_read(iv, depths=np.stack(maps))
    assert_bit_equal(tb, ta, "tsdf")
    assert_bit_equal(wb, wa, "weight")
    n = c.voxels
    pt = torch.empty(n, dtype=torch.float32).pin_memory()
    pw = torch.empty(n, dtype=torch.int16 if q8 else torch.float32).pin_memory()
    c.integrate_many_read(iv, depths=np.stack(maps), out=(pt, pw))
    assert_bit_equal(pt.numpy().reshape(ta.shape), ta, "tsdf (pinned)")
    assert_bit_equal(pw.numpy().view(wa.dtype).reshape(wa.shape), wa, "weight (pinned)")
    # weight only, then a second sweep on top (the read-back leaves the volume in place)
    _, w2 = b.integrate_many_read(iv, depths=np.stack(maps), out=(None, np.empty_like(wb).reshape(-1)))
    a.integrate_many(iv, depths=np.stack(maps))
    assert_bit_equal(w2.reshape(-1), a.read()[1].reshape(-1), "weight after two sweeps")
    with pytest.raises(ValueError):
        b.integrate_many_read(iv, depths=np.stack(maps), out=(np.empty(3, np.float32), None))


@pytest.mark.parametrize("q8", [False, True])
def test_asynchronous_read_back_is_ordered_before_later_writes(scene, q8):
    """l3d_tsdf_integrate_many_read_async returns before the volume is in host memory; a reset
    and another sweep queued on the same handle right after it wait for its copies on the
    device, so the buffers receive the first scan's volume, and wait_read returns it."""
    import torch
    views, maps = scene
    W, H = 120, 90
    iv = [gpu_view(v, confidence=1.5) for v in views]

    def make():
        return TsdfVolume(W, H, 0.04, (-1.28, -1.1, -1.1), dense=(64, 48, 56), truncation=0.12,
                          weight_q8=q8)
    a, b = make(), make()
    a.integrate_many(iv, depths=np.stack(maps))
    ta, wa = a.read()
    a.reset()
    a.integrate_many(iv[::-1], depths=np.stack(maps[::-1]))  # a different second scan
    tr, wr = a.read()
    n = b.voxels
    outs = [(torch.empty(n, dtype=torch.float32).pin_memory(),
             torch.empty(n, dtype=torch.int16 if q8 else torch.float32).pin_memory()) for _ in range(2)]
    b.integrate_many_read(iv, depths=np.stack(maps), out=outs[0], wait=False)
    b.reset()
    b.integrate_many_read(iv[::-1], depths=np.stack(maps[::-1]), out=outs[1], wait=False)
    b.wait_read()
    for (pt, pw), (t, w), what in zip(outs, ((ta, wa), (tr, wr)), ("first scan", "second scan")):
        assert_bit_equal(pt.numpy().reshape(t.shape), t, f"tsdf ({what})")
        assert_bit_equal(pw.numpy().view(w.dtype).reshape(w.shape), w, f"weight ({what})")
    tb, wb = b.read()
    assert_bit_equal(tb, tr, "tsdf after the reads")
    with pytest.raises(ValueError):
        b.integrate_many_read(iv, depths=np.stack(maps), wait=False)


def test_sweep_of_more_views_than_the_shared_view_table_holds(scene):
    """More than ~200 views in one sweep take the sweep of every quad with the view table in
    global memory; the result still equals the views integrated one at a time."""
    views, maps = scene
    W, H = 120, 90
    reps = 220 // len(views) + 1
    iv = [gpu_view(v, confidence=1.5) for v in views] * reps
    ms = np.stack(list(maps) * reps)
    assert len(iv) > 215

    def make():
        return TsdfVolume(W, H, 0.04, (-1.28, -1.1, -1.1), dense=(64, 48, 56), truncation=0.12,
                          weight_q8=True)
    a, b = make(), make()
    a.integrate_many(iv, depths=ms)
    for v, m in zip(iv, ms):
        b.integrate(v, m)
    ta, wa = a.read()
    tb, wb = b.read()
    assert_bit_equal(ta, tb, "tsdf")
    assert_bit_equal(wa, wb, "weight")


def test_brick_pool_and_prior_bit_exact(scene):
    views, maps = scene
    W, H = 120, 90
    voxel = 0.03
    grid = BrickGrid((-1.3, -1.2, -1.3), voxel, (2.6, 2.4, 2.6))
    rng = np.random.default_rng(1)
    pts = rng.normal(size=(3000, 3))
    pts /= np.linalg.norm(pts, axis=1, keepdims=True)
    for p in pts:
        grid.mark(*p, voxel * 4)
    coords, lookup, count = grid.build()
    assert 0 < count < grid.cells
    prior = np.where(maps[0] == 0, 2.0, 0.0).astype(np.float32)
    o = oracle.Tsdf(W, H, voxel, grid.origin, voxel * 4, coords=coords)
    g = TsdfVolume(W, H, voxel, grid.origin, grid=grid, layout=(coords, lookup, count))
    for i, (v, m) in enumerate(zip(views, maps)):
        pr = prior if i == 0 else None
        o.integrate(view_kw(v, prior=pr), m)
        g.integrate(gpu_view(v, prior=pr), depth=m)
    t, w = g.read()
    assert_bit_equal(t, o.tsdf, "pool tsdf")
    assert_bit_equal(w, o.weight, "pool weight")


def test_ragged_dense_grid(scene):
    views, maps = scene
    W, H = 120, 90
    dims = (37, 21, 29)  # x not a multiple of 4: scalar path; partial bricks at the edges
    o = oracle.Tsdf(W, H, 0.07, (-1.3, -1.0, -1.0), 0.2, dense=dims, weight_q8=True)
    g = TsdfVolume(W, H, 0.07, (-1.3, -1.0, -1.0), dense=dims, truncation=0.2, weight_q8=True)
    for v, m in zip(views, maps):
        o.integrate(view_kw(v), m)
        g.integrate(gpu_view(v), depth=m)
    t, w = g.read()
    assert_bit_equal(t.reshape(-1), o.tsdf, "tsdf")
    assert_bit_equal(w.reshape(-1), o.weight, "weight")


def test_reset_and_empty_maps(scene):
    views, maps = scene
    g = TsdfVolume(120, 90, 0.05, (-1, -1, -1), dense=(40, 40, 40), weight_q8=True)
    g.integrate(gpu_view(views[0]), depth=np.zeros((90, 120), np.uint32))
    t, w = g.read()
    assert np.all(t == 1.0) and np.all(w == 0)
    g.integrate(gpu_view(views[0]), depth=maps[0])
    g.reset()
    t, w = g.read()
    assert np.all(t == 1.0) and np.all(w == 0)


def test_update_count_matches_the_oracle(scene):
    """l3d_tsdf_count_updates: the voxel-updates of integrating the maps equal, per view, the
    voxels whose f32 weight the oracle's integration raises (weights stay below the maximum)."""
    views, maps = scene
    W, H = 120, 90
    dims, voxel, origin, mu = (64, 48, 56), 0.04, (-1.28, -1.1, -1.1), 0.12
    o = oracle.Tsdf(W, H, voxel, origin, mu, dense=dims)
    want = 0
    for v, m in zip(views, maps):
        before = o.weight.copy()
        o.integrate(view_kw(v), m)
        want += int((o.weight != before).sum())
    g = TsdfVolume(W, H, voxel, origin, dense=dims, truncation=mu)
    visible, updates, kept = g.count_updates([gpu_view(v) for v in views], depths=np.stack(maps))
    assert updates == want
    assert want > 5000
    assert visible >= kept >= updates
    assert visible <= len(views) * int(np.prod(dims))
    t, w = g.read()  # counting leaves the volume untouched
    assert np.all(w == 0) and np.all(t == 1)


@pytest.mark.parametrize("q8", [False, True])
def test_sweep_with_prior_and_depth_cull_bit_exact(scene, q8):
    """The sweep and the per-view launches cull bricks by depth (a brick provably behind every
    depth of its footprint by more than the truncation band is skipped); with a phone prior
    filling the holes of one map and a narrow truncation band, both still equal the oracle, which
    visits every voxel of every visible brick."""
    views, maps = scene
    W, H = 120, 90
    dims, voxel, origin, mu = (64, 48, 56), 0.04, (-1.28, -1.1, -1.1), 0.05
    prior = np.where(maps[2] == 0, 1.9, 0.0).astype(np.float32)
    o = oracle.Tsdf(W, H, voxel, origin, mu, dense=dims, weight_q8=q8)
    a = TsdfVolume(W, H, voxel, origin, dense=dims, truncation=mu, weight_q8=q8)
    b = TsdfVolume(W, H, voxel, origin, dense=dims, truncation=mu, weight_q8=q8)
    gv = []
    for i, (v, m) in enumerate(zip(views, maps)):
        pr = prior if i == 2 else None
        o.integrate(view_kw(v, prior=pr), m)
        a.integrate(gpu_view(v, prior=pr), depth=m)
        gv.append(gpu_view(v, prior=pr))
    b.integrate_many(gv, depths=np.stack(maps))
    for g, what in ((a, "per view"), (b, "sweep")):
        t, w = g.read()
        assert_bit_equal(t.reshape(-1), o.tsdf, f"tsdf ({what})")
        assert_bit_equal(w.reshape(-1), o.weight, f"weight ({what})")
