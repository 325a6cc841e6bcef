"""The allocation-free TSDF entry point (l3d_tsdf_integrate_noalloc).

It serves callers that cannot let the library call cudaMalloc: their device memory belongs to
another allocator (here torch's caching allocator stands in for one) or an allocation's
device-wide synchronisation would stall their pipeline.  The test owns every buffer, calls the
entry point twice in a row on the same volume and checks each result, bit for bit (the tolerance
of the other TSDF tests), against the handle-based l3d_tsdf_integrate on the same inputs.

This file is collected last so that a failure here comes after every other test has run; it also
passes on its own in a fresh process (the first call on the device does the one-time set-up).
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from luvas3d import IntegrationView, TsdfVolume, _lib, scenes
from luvas3d.camera import Intrinsics, StereoView, look_at

pytestmark = pytest.mark.gpu


def two_packed_views(W=96, H=72, f=84.0):
    """Two views of the sphere scene with packed depth maps (normals facing the camera)."""
    k = Intrinsics(f, f, W / 2, H / 2)
    views = [StereoView(k, look_at((2.2 * np.sin(a), 0.4, 2.2 * np.cos(a)), (0, -0.2, 0)))
             for a in (0.0, 0.7)]
    _, truth = scenes.render_sphere(views, [(W, H)] * 2, seed=9)
    maps = []
    for d in truth:
        m = np.zeros((H, W), dtype=np.uint32)
        for y in range(H):
            for x in range(W):
                if d[y, x] > 0:
                    m[y, x] = oracle.pack_sample(d[y, x], (0.0, 0.0, -1.0), 0.25)
        maps.append(m)
    return views, maps


def c_view(v, max_depth=6.0, confidence=1.5):
    cv = _lib.IntegrationView()
    k = v.intrinsics
    cv.intrinsics = _lib.Intrinsics(k.fx, k.fy, k.cx, k.cy)
    cv.pose.R[:] = list(np.asarray(v.pose.R, dtype=np.float64).reshape(9))
    cv.pose.t[:] = list(np.asarray(v.pose.t, dtype=np.float64).reshape(3))
    cv.max_depth = max_depth
    cv.confidence = confidence
    return cv


@pytest.mark.parametrize("layout", ["dense", "pool"])
@pytest.mark.parametrize("prior", [False, True])
@pytest.mark.parametrize("q8", [True, False])
def test_noalloc_matches_handle_integrate_twice(q8, prior, layout):
    """Dense grid or brick pool (device coordinates: the bricks of two z-rows of the grid), with
    or without a phone-depth prior filling the holes of the maps (a device buffer here, a host
    array for the handle), two calls in a row."""
    import torch

    from luvas3d import shard

    lib = _lib.load()
    views, maps = two_packed_views()
    W, H = 96, 72
    dims, voxel, origin, mu = (40, 32, 36), 0.06, (-1.2, -1.1, -1.1), 0.18
    coords = shard.slab_layout(dims, 1, 3) if layout == "pool" else None
    kw = dict(truncation=mu, weight_q8=q8)
    ref = (TsdfVolume(W, H, voxel, origin, layout=(coords,), **kw) if coords is not None
           else TsdfVolume(W, H, voxel, origin, dense=dims, **kw))
    priors = [np.where(m == 0, 1.8 + 0.1 * i, 0.0).astype(np.float32) for i, m in enumerate(maps)]

    desc = _lib.TsdfDesc()
    desc.origin[:] = list(origin)
    desc.voxel, desc.truncation, desc.max_weight, desc.prior_weight = voxel, mu, 96.0, 0.12
    desc.weight_type = _lib.WEIGHT_Q8 if q8 else _lib.WEIGHT_F32
    desc.width, desc.height = W, H
    dev = torch.device("cuda")
    if coords is None:
        desc.dense = 1
        desc.dims[:] = list(dims)
        n = int(np.prod(dims))
        coords_dev = None
    else:
        desc.dense = 0
        desc.count = int(coords.shape[0])
        n = desc.count * 512
        coords_t = torch.from_numpy(np.ascontiguousarray(coords)).to(dev)
        coords_dev = C.c_void_p(coords_t.data_ptr())
    tsdf = torch.ones(n, dtype=torch.float32, device=dev)
    weight = torch.zeros(n, dtype=torch.int16 if q8 else torch.float32, device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    for call, (v, m) in enumerate(zip(views, maps)):
        depth = torch.from_numpy(m.view(np.int32)).to(dev)
        pr = torch.from_numpy(priors[call]).to(dev) if prior else None
        cv = c_view(v)
        rc = lib.l3d_tsdf_integrate_noalloc(C.byref(desc), coords_dev, C.c_void_p(depth.data_ptr()),
                                            C.c_void_p(pr.data_ptr()) if pr is not None else None,
                                            C.byref(cv), C.c_void_p(tsdf.data_ptr()),
                                            C.c_void_p(weight.data_ptr()), C.c_void_p(stream))
        assert rc == _lib.L3D_OK, _lib.last_error()
        torch.cuda.synchronize()
        ref.integrate(IntegrationView(v.intrinsics, v.pose, 6.0, priors[call] if prior else None, 1.5),
                      depth=m)
        want_t, want_w = ref.read()
        got_t = tsdf.cpu().numpy()
        got_w = weight.cpu().numpy().view(np.uint16) if q8 else weight.cpu().numpy()
        assert np.array_equal(got_t.view(np.uint32), want_t.reshape(-1).view(np.uint32)), f"call {call}"
        assert np.array_equal(got_w, want_w.reshape(-1)), f"call {call} weights"
        assert (want_w > 0).sum() > 500
    ref.destroy()


def test_noalloc_rejects_volumes_beyond_the_limit():
    lib = _lib.load()
    desc = _lib.TsdfDesc()
    desc.voxel, desc.truncation, desc.max_weight, desc.prior_weight = 0.01, 0.04, 96.0, 0.12
    desc.dense = 1
    desc.dims[:] = [1024, 1024, 1024]  # 2^21 bricks
    desc.weight_type = _lib.WEIGHT_F32
    desc.width, desc.height = 64, 48
    cv = _lib.IntegrationView()
    cv.intrinsics = _lib.Intrinsics(50, 50, 32, 24)
    dummy = C.c_void_p(256)  # never dereferenced: the size check comes first
    rc = lib.l3d_tsdf_integrate_noalloc(C.byref(desc), None, dummy, None, C.byref(cv), dummy, dummy,
                                        None)
    assert rc == _lib.L3D_EINVAL
    assert "at most" in _lib.last_error()
    assert _lib.NOALLOC_MAX_BRICKS == 1 << 20
