"""Known-answer tests that pin the CPU oracle (no GPU needed).

The reference implements PatchMatch and TSDF integration only as WGSL and holds no golden vectors
for them, so these tests pin the restatement: primitives against independent numpy/Python
computations and IEEE references, scenes with exact answers (a fronto-parallel textured wall at a
known depth, a single voxel updated by hand), the brick layout contract of
frontend/src/app/vision/fusion/fusion.spec.ts:6-33, and FP32-vs-FP64 agreement.
"""
import numpy as np
import pytest

import oracle
from luvas3d import packing, scenes
from luvas3d.camera import Intrinsics, Pose, StereoView, look_at


def pcg_ref(v: int) -> int:
    """patchmatch.wgsl.ts:56-60 in Python integers."""
    state = (v * 747796405 + 2891336453) & 0xFFFFFFFF
    word = (((state >> ((state >> 28) + 4)) ^ state) * 277803737) & 0xFFFFFFFF
    return ((word >> 22) ^ word) & 0xFFFFFFFF


def test_pcg_known_values():
    lib = oracle.load()
    # values of the WGSL hash in 32-bit unsigned arithmetic
    expected = [129708002, 2831084092, 2055130248, 4099845390, 3861530882]
    for v, e in zip((0, 1, 2, 12345, 0xFFFFFFFF), expected):
        assert lib.orc_pcg(v) == e == pcg_ref(v)
    rng = np.random.default_rng(0)
    for v in rng.integers(0, 2**32, size=2000, dtype=np.uint64):
        assert lib.orc_pcg(int(v)) == pcg_ref(int(v))


def test_seed_formula_matches_js():
    """dense-stereo.ts:333: Math.imul(ref + 1, 0x9e3779b1) + iteration*97 + phase*13 + flags*7 >>> 0."""
    lib = oracle.load()

    def js(ref, it, ph, fl):
        m = ((ref + 1) * 0x9E3779B1) & 0xFFFFFFFF
        if m >= 2**31:
            m -= 2**32  # Math.imul returns a signed int32
        return int(m + it * 97 + ph * 13 + fl * 7) & 0xFFFFFFFF

    for ref in (0, 1, 7, 47, 95):
        for it in range(6):
            for ph in (0, 1):
                for fl in (0, 1):
                    assert lib.orc_seed(ref, it, ph, fl) == js(ref, it, ph, fl)


def _ulp_err(got: np.ndarray, exact: np.ndarray) -> np.ndarray:
    exact32 = exact.astype(np.float32)
    ulp = np.spacing(np.abs(exact32)).astype(np.float64)
    return np.abs(got.astype(np.float64) - exact) / ulp


def test_expf_within_two_ulp():
    rng = np.random.default_rng(1)
    xs = np.concatenate([rng.uniform(-87, 0, 20000), rng.uniform(-0.5, 0.5, 5000),
                         rng.uniform(-140.0, -20.0, 5000) * 0.7, rng.uniform(0, 88, 2000),
                         [0.0, -0.0, 1.0, -1.0, -50.0]]).astype(np.float32)
    got = np.array([oracle.expf(x) for x in xs], dtype=np.float32)
    exact = np.exp(xs.astype(np.float64))
    normal = exact >= np.finfo(np.float32).tiny
    assert _ulp_err(got[normal], exact[normal]).max() <= 2.0
    # subnormal results: within one subnormal step
    sub = ~normal
    assert np.all(np.abs(got[sub].astype(np.float64) - exact[sub]) <= 2.0 ** -149 + 1e-300)
    assert oracle.expf(-200.0) == 0.0


def test_sincos_within_two_ulp():
    rng = np.random.default_rng(2)
    xs = np.concatenate([rng.uniform(0, 6.2831853, 20000), [0.0, 1e-8, 3.14159265, 6.2831853,
                                                            1.5707963, 4.712389]]).astype(np.float32)
    s = np.zeros(xs.size)
    c = np.zeros(xs.size)
    for i, x in enumerate(xs):
        s[i], c[i] = oracle.sincosf(x)
    x64 = xs.astype(np.float64)
    for got, exact in ((s, np.sin(x64)), (c, np.cos(x64))):
        err = np.abs(got - exact)
        # relative to the ulp of the result, or absolute near zero crossings
        tol = np.maximum(2 * np.spacing(np.abs(exact).astype(np.float32)).astype(np.float64), 2e-8)
        assert np.all(err <= tol)


def test_f16_conversions_match_ieee():
    lib = oracle.load()
    bits = np.arange(65536, dtype=np.uint32)
    ref = bits.astype(np.uint16).view(np.float16).astype(np.float32)
    got = np.array([lib.orc_f16_to_f32(int(b)) for b in bits], dtype=np.float32)
    finite = np.isfinite(ref)
    assert np.array_equal(got[finite].view(np.uint32), ref[finite].view(np.uint32))
    assert np.all(np.isnan(got[np.isnan(ref)]))
    rng = np.random.default_rng(3)
    xs = np.concatenate([rng.uniform(-70000, 70000, 20000), rng.uniform(-1e-4, 1e-4, 20000),
                         rng.uniform(0, 4, 20000), [0.0, -0.0, 65504, 65519.99, 65520, 1e9,
                                                    2.0**-24, 2.0**-25, 1.5 * 2.0**-25,
                                                    2.0**-14, 5.960464477539063e-08]])
    xs = xs.astype(np.float32)
    with np.errstate(over="ignore"):
        ref16 = xs.astype(np.float16).view(np.uint16).astype(np.uint32)
    got16 = np.array([lib.orc_f32_to_f16(float(x)) for x in xs], dtype=np.uint32)
    assert np.array_equal(got16, ref16)


def _fma32(a, b, c):
    return np.float32(np.float64(np.float32(a)) * np.float64(np.float32(b)) + np.float64(np.float32(c)))


def pack_ref(depth, n, cost) -> int:
    """depth-packing.wgsl.ts:21-33 in numpy float32 (fused multiply-adds emulated exactly)."""
    f = np.float32
    depth, cost = f(depth), f(cost)
    if not depth > 0 or not cost < 1:
        return 0
    nx, ny, nz = (f(x) for x in n)
    s = f(f(abs(nx) + abs(ny)) + abs(nz))
    ex, ey = f(nx / s), f(ny / s)
    if nz < 0:
        sx = f(1) if ex >= 0 else f(-1)
        sy = f(1) if ey >= 0 else f(-1)
        ex, ey = f(f(1 - abs(ey)) * sx), f(f(1 - abs(ex)) * sy)
    cx = min(max(_fma32(ex, 0.5, 0.5), f(0)), f(1))
    cy = min(max(_fma32(ey, 0.5, 0.5), f(0)), f(1))
    qx, qy = int(_fma32(cx, 63, 0.5)), int(_fma32(cy, 63, 0.5))
    c = min(15, int(f(cost * f(15))))
    h = int(np.array([depth], dtype=np.float32).astype(np.float16).view(np.uint16)[0])
    return h | (qx << 16) | (qy << 22) | (c << 28)


def test_pack_matches_independent_restatement_and_round_trips():
    rng = np.random.default_rng(4)
    n = rng.normal(size=(3000, 3))
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    depth = rng.uniform(0.05, 60, 3000)
    cost = rng.uniform(0, 1, 3000)
    for i in range(3000):
        p = oracle.pack_sample(depth[i], n[i], cost[i])
        assert p == pack_ref(depth[i], n[i], cost[i])
        assert p >> 28 == min(15, int(np.float32(np.float32(cost[i]) * np.float32(15))))
        d = packing.unpack_depth(np.uint32(p))
        assert abs(float(d) - depth[i]) <= depth[i] * 2.0**-11
        m = oracle.unpack_normal(p)
        assert np.degrees(np.arccos(np.clip(m @ n[i], -1, 1))) < 4.0
    # empty samples
    assert oracle.pack_sample(0.0, (0, 0, -1), 0.1) == 0
    assert oracle.pack_sample(-1.0, (0, 0, -1), 0.1) == 0
    assert oracle.pack_sample(1.0, (0, 0, -1), 1.0) == 0
    assert oracle.pack_sample(1.0, (0, 0, -1), float("nan")) == 0


def test_python_decode_matches_oracle():
    rng = np.random.default_rng(5)
    packed = rng.integers(1, 2**32, size=2000, dtype=np.uint64).astype(np.uint32)
    packed = (packed & ~np.uint32(0xFFFF)) | np.uint32(0x3C00)  # depth 1.0
    valid, d, nrm = packing.unpack_samples(packed)
    assert valid.all() and np.all(d == 1.0)
    for p, m in zip(packed, nrm):
        assert np.allclose(oracle.unpack_normal(int(p)), m, atol=2e-7)


def wall_scene(n_views=5, step=0.06, W=160, H=120, f=140.0):
    """Cameras at z = 0 looking at -z onto the room's back wall (z = -1.5): every pixel sees a
    fronto-parallel textured plane at depth exactly 1.5 m."""
    k = Intrinsics(f, f, W / 2, H / 2)
    views = []
    for i in range(n_views):
        x = (i - n_views // 2) * step
        views.append(StereoView(k, look_at((x, 0.0, 0.0), (x, 0.0, -1.0))))
    imgs, truth = scenes.render_room(views, [(W, H)] * n_views, np.zeros((0, 6)), seed=11)
    return views, imgs, truth


def test_wall_truth_is_exact():
    views, imgs, truth = wall_scene()
    assert np.allclose(truth[2], 1.5, atol=1e-6)


def test_plane_cost_of_the_true_wall_is_low():
    views, imgs, truth = wall_scene()
    W, H = 160, 120
    o = oracle.Stereo(W, H, views, imgs, 32)
    planes = np.zeros((H, W, 4), dtype=np.float32)
    planes[..., 2] = -1.0
    planes[..., 3] = 1.5
    cost, vc = o.plane_cost(2, [0, 1, 3, 4], planes, min_depth=0.5, max_depth=5.0)
    inner = (slice(10, H - 10), slice(20, W - 20))
    assert np.median(cost[inner]) < 0.05
    planes[..., 3] = 2.0
    wrong, _ = o.plane_cost(2, [0, 1, 3, 4], planes, min_depth=0.5, max_depth=5.0)
    assert np.median(wrong[inner]) > 0.3
    # outside the depth range or back-facing: INVALID (2)
    planes[..., 3] = 6.0
    c, _ = o.plane_cost(2, [0, 1, 3, 4], planes, min_depth=0.5, max_depth=5.0)
    assert np.all(c == 2.0)
    planes[..., 2] = 1.0
    planes[..., 3] = 1.5
    c, _ = o.plane_cost(2, [0, 1, 3, 4], planes, min_depth=0.5, max_depth=5.0)
    assert np.all(c == 2.0)


def test_solve_recovers_the_wall_depth():
    views, imgs, truth = wall_scene()
    W, H = 160, 120
    o = oracle.Stereo(W, H, views, imgs, 32)
    o.solve(2, [0, 1, 3, 4], min_depth=0.5, max_depth=5.0, iterations=4)
    d = o.hyp[..., 3]
    rel = np.abs(d - 1.5) / 1.5
    # border columns lose sources to the frame edge; the interior converges
    assert np.median(rel) < 0.004
    assert (rel < 0.01).mean() > 0.8
    packed = o.depths[2]
    assert (packed != 0).mean() > 0.8


def test_fp32_and_fp64_oracles_agree_on_fixed_planes():
    views, imgs, truth = wall_scene()
    W, H = 160, 120
    rng = np.random.default_rng(6)
    planes = np.zeros((H, W, 4))
    n = rng.normal(size=(H, W, 3)) * 0.2 + np.array([0, 0, -1.0])
    planes[..., :3] = n / np.linalg.norm(n, axis=-1, keepdims=True)
    planes[..., 3] = rng.uniform(1.3, 1.7, size=(H, W))
    o32 = oracle.Stereo(W, H, views, imgs, 32)
    o64 = oracle.Stereo(W, H, views, imgs, 64)
    c32, _ = o32.plane_cost(2, [0, 1, 3, 4], planes.astype(np.float32), min_depth=0.5, max_depth=5.0)
    c64, _ = o64.plane_cost(2, [0, 1, 3, 4], planes.astype(np.float32).astype(np.float64),
                            min_depth=0.5, max_depth=5.0)
    valid = (c64 < 1.5) & (c32 < 1.5)
    assert valid.mean() > 0.8
    err = np.abs(c32[valid] - c64[valid])
    # FP32 rounding in the NCC sums; windows with little texture amplify it (small variance)
    assert np.percentile(err, 99.9) < 1e-4
    assert err.max() < 1e-3


def test_compensated_sums_are_a_distinct_arithmetic_closer_to_fp64():
    """The compensated mode (Neumaier sums of the window terms) changes some FP32 costs in their
    last bits, agrees with the plain sums to the NCC tolerance, and is at least as close to the
    FP64 oracle."""
    views, imgs, truth = wall_scene()
    W, H = 160, 120
    rng = np.random.default_rng(8)
    planes = np.zeros((H, W, 4))
    n = rng.normal(size=(H, W, 3)) * 0.2 + np.array([0, 0, -1.0])
    planes[..., :3] = n / np.linalg.norm(n, axis=-1, keepdims=True)
    planes[..., 3] = rng.uniform(1.3, 1.7, size=(H, W))
    p32 = planes.astype(np.float32)
    kw = dict(min_depth=0.5, max_depth=5.0)
    plain, _ = oracle.Stereo(W, H, views, imgs, 32).plane_cost(2, [0, 1, 3, 4], p32, **kw)
    comp, _ = oracle.Stereo(W, H, views, imgs, 32, compensated=True).plane_cost(2, [0, 1, 3, 4], p32, **kw)
    c64, _ = oracle.Stereo(W, H, views, imgs, 64).plane_cost(2, [0, 1, 3, 4], p32.astype(np.float64), **kw)
    valid = (c64 < 1.5) & (plain < 1.5) & (comp < 1.5)
    assert valid.mean() > 0.8
    assert np.any(plain != comp)
    assert np.percentile(np.abs(plain - comp)[valid], 99.9) < 1e-4
    e_plain = np.abs(plain[valid] - c64[valid])
    e_comp = np.abs(comp[valid] - c64[valid])
    assert e_comp.mean() <= e_plain.mean()


def test_threads_do_not_change_results():
    """Red/black phases read only the other colour, so the parallel oracle is deterministic."""
    views, imgs, truth = wall_scene()
    W, H = 160, 120
    a = oracle.Stereo(W, H, views, imgs, 32, threads=1)
    b = oracle.Stereo(W, H, views, imgs, 32, threads=8)
    for o in (a, b):
        o.solve(2, [0, 1, 3, 4], min_depth=0.5, max_depth=5.0, iterations=2)
    assert np.array_equal(a.hyp, b.hyp) and np.array_equal(a.cost, b.cost)
    assert np.array_equal(a.depths, b.depths)


def test_consistency_filter_keeps_agreeing_wall_depths():
    views, imgs, truth = wall_scene()
    W, H = 160, 120
    o = oracle.Stereo(W, H, views, imgs, 32)
    for r in range(5):
        src = [s for s in range(5) if s != r]
        o.solve(r, src, min_depth=0.5, max_depth=5.0, iterations=4)
    f = o.filter(2, [0, 1, 3, 4], 2)
    kept = f != 0
    assert kept.mean() > 0.5
    d = packing.unpack_depth(f[kept])
    assert np.median(np.abs(d - 1.5) / 1.5) < 0.003
    # the filter keeps the normal and cost bits of the raw sample
    assert np.array_equal(f[kept] & 0xFFFF0000, o.depths[2][kept] & 0xFFFF0000)


def tsdf_hand(tsdf, w0, obs, w):
    f = np.float32
    num = _fma32(tsdf, w0, f(f(obs) * f(w)))
    return f(num / f(f(w0) + f(w))), f(min(f(w0) + f(w), f(96)))


def test_single_voxel_tsdf_update_by_hand():
    """One 8^3 brick at the origin, a camera on the -z side looking along +z; a constant packed
    depth of 1.0 facing the camera.  Voxel (3, 4, 5) is checked against the update written out by
    hand (tsdf-volume.ts:141-152)."""
    W, H = 64, 48
    voxel = 0.01
    origin = (-0.04, -0.04, 0.95)
    k = (50.0, 50.0, 32.0, 24.0)
    R = np.eye(3)
    t = np.zeros(3)
    packed = oracle.pack_sample(1.0, (0.0, 0.0, -1.0), 0.0)
    depth = np.full((H, W), packed, dtype=np.uint32)
    for q8 in (False, True):
        o = oracle.Tsdf(W, H, voxel, origin, 0.04, coords=np.array([[0, 0, 0, 0]]), weight_q8=q8)
        o.integrate(dict(k=k, R=R, t=t, max_depth=3.0), depth)
        f = np.float32
        x, y, z = 3, 4, 5
        wz = _fma32(f(z) + f(0.5), f(voxel), f(origin[2]))
        wx = _fma32(f(x) + f(0.5), f(voxel), f(origin[0]))
        wy = _fma32(f(y) + f(0.5), f(voxel), f(origin[1]))
        cam = np.array([wx, wy, wz], dtype=np.float32)
        sdf = f(f(1.0) - cam[2])
        obs = min(f(1), f(sdf / f(0.04)))
        n = oracle.unpack_normal(packed)
        il = f(1) / f(np.sqrt(f(_fma32(cam[2], cam[2], _fma32(cam[1], cam[1], f(cam[0] * cam[0]))))))
        cn = cam * il
        dot = _fma32(n[2], cn[2], _fma32(n[1], cn[1], f(n[0] * cn[0])))
        w = max(f(0.2), abs(dot))
        idx = x + 8 * y + 64 * z
        if q8:
            wi = int(np.rint(w * f(256)))
            wq = f(wi) * f(1 / 256)
            expect_t, _ = tsdf_hand(f(1), f(0), obs, wq)
            assert o.weight[idx] == wi
        else:
            expect_t, expect_w = tsdf_hand(f(1), f(0), obs, w)
            assert o.weight[idx] == expect_w
        assert o.tsdf[idx] == expect_t
        # a voxel behind the surface by more than mu is untouched
        far = 0 + 8 * 0 + 64 * 7  # z = 7 -> 1.025 m: sdf = -0.025 > -mu, updated; check z beyond
        assert o.tsdf[far] <= 1.0


def sphere_view_depth(W=96, H=72, f=80.0, dist=2.2):
    """A camera looking at the unit sphere and its rendered depth packed with the sphere normal."""
    k = Intrinsics(f, f, W / 2, H / 2)
    v = StereoView(k, look_at((0.0, 0.4, dist), (0.0, 0.0, 0.0)))
    _, truth = scenes.render_sphere([v], [(W, H)], seed=3)
    d = truth[0]
    ys, xs = np.mgrid[0:H, 0:W]
    rays = np.stack([(xs - k.cx) / k.fx, (ys - k.cy) / k.fy, np.ones_like(xs, dtype=float)], -1)
    pts_cam = rays * d[..., None]
    packed = np.zeros((H, W), dtype=np.uint32)
    for y in range(H):
        for x in range(W):
            if d[y, x] <= 0:
                continue
            pw = v.pose.R.T @ (pts_cam[y, x] - v.pose.t)
            nw = pw / np.linalg.norm(pw) if pw[1] > -0.999 else np.array([0, 1.0, 0])
            nc = v.pose.R @ nw
            packed[y, x] = oracle.pack_sample(d[y, x], nc, 0.2)
    return v, packed


def test_brick_layout_contract_pool_equals_dense():
    """The brick pool stores voxel (b, x, y, z) at b*512 + x + 8y + 64z (fusion.spec.ts:21-31);
    integrating the same map into a dense grid and into a pool holding all its bricks gives the
    same voxels."""
    v, packed = sphere_view_depth()
    W, H = packed.shape[1], packed.shape[0]
    voxel, origin = 0.05, (-1.2, -1.2, -1.2)
    dims = (48, 48, 48)
    vk = dict(k=(v.intrinsics.fx, v.intrinsics.fy, v.intrinsics.cx, v.intrinsics.cy),
              R=v.pose.R, t=v.pose.t, max_depth=5.0)
    dense = oracle.Tsdf(W, H, voxel, origin, 0.2, dense=dims)
    dense.integrate(vk, packed)
    nb = 6
    coords = np.array([[x, y, z, 0] for z in range(nb) for y in range(nb) for x in range(nb)][::-1],
                      dtype=np.int32)
    pool = oracle.Tsdf(W, H, voxel, origin, 0.2, coords=coords)
    pool.integrate(vk, packed)
    dt = dense.tsdf.reshape(dims[2], dims[1], dims[0])
    dw = dense.weight.reshape(dims[2], dims[1], dims[0])
    for b, (bx, by, bz, _) in enumerate(coords):
        blk = pool.tsdf[b * 512:(b + 1) * 512].reshape(8, 8, 8)  # [z][y][x]
        wb = pool.weight[b * 512:(b + 1) * 512].reshape(8, 8, 8)
        assert np.array_equal(blk, dt[bz * 8:bz * 8 + 8, by * 8:by * 8 + 8, bx * 8:bx * 8 + 8])
        assert np.array_equal(wb, dw[bz * 8:bz * 8 + 8, by * 8:by * 8 + 8, bx * 8:bx * 8 + 8])
    assert (dense.weight > 0).sum() > 1000
    # sign convention of fusion.spec.ts: positive in front of the surface, |tsdf| <= 1
    seen = dense.weight > 0
    assert np.all(np.abs(dense.tsdf[seen]) <= 1.0)
    assert (dense.tsdf[seen] > 0).any() and (dense.tsdf[seen] < 0).any()


def test_visible_bricks_cull_behind_and_beyond():
    """visibleBricks (tsdf-volume.ts:220-234): a camera at the centre of the grid looking along +z
    sees neither the bricks behind it nor those beyond max_depth."""
    W, H = 96, 72
    o = oracle.Tsdf(W, H, 0.05, (-1.2, -1.2, -1.2), 0.2, dense=(48, 48, 48))
    vk = dict(k=(80.0, 80.0, 48.0, 36.0), R=np.eye(3), t=np.zeros(3), max_depth=5.0)
    vis = o.visible(vk).reshape(6, 6, 6)  # [bz][by][bx]
    assert 0 < vis.sum() < vis.size
    assert vis[0].sum() == 0            # bricks centred at z = -1.0 m are behind the camera
    assert vis[5].sum() > 0
    near = o.visible(dict(vk, max_depth=0.3)).reshape(6, 6, 6)
    assert near.sum() < vis.sum() and np.all(near <= vis)
    assert near[5].sum() == 0           # z = 1.0 m is beyond 0.3 m + radius


def test_tsdf_fp32_matches_fp64_within_tolerance():
    v, packed = sphere_view_depth()
    W, H = packed.shape[1], packed.shape[0]
    vk = dict(k=(v.intrinsics.fx, v.intrinsics.fy, v.intrinsics.cx, v.intrinsics.cy),
              R=v.pose.R, t=v.pose.t, max_depth=5.0)
    a = oracle.Tsdf(W, H, 0.05, (-1.2, -1.2, -1.2), 0.2, dense=(48, 48, 48))
    b = oracle.Tsdf(W, H, 0.05, (-1.2, -1.2, -1.2), 0.2, dense=(48, 48, 48), precision=64)
    a.integrate(vk, packed)
    b.integrate(vk, packed)
    both = (a.weight > 0) & (b.weight > 0)
    assert both.sum() > 1000
    # voxels whose pixel rounds differently in FP32 and FP64 are rare
    close = np.abs(a.tsdf[both] - b.tsdf[both]) < 1e-5
    assert close.mean() > 0.99
