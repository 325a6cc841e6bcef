"""Sparse brick TSDF of a sphere, as the reference's surface-nets test builds it
(frontend/src/app/vision/fusion/fusion.spec.ts:6-33): bricks marked around 2000 points of a
Fibonacci spiral on the sphere, tsdf = clamp(sdf / mu, -1, 1), weight 2 where sdf > -mu."""
import numpy as np

import oracle


def sphere_volume(radius=0.05, voxel=0.002):
    extent = radius * 2 + voxel * 8 * 2
    origin = np.array([-extent / 2] * 3)
    mu = voxel * 4
    a = np.arange(2000)
    z = a / 1999 * 2 - 1
    phi = a * 2.399963
    r = np.sqrt(1 - z * z)
    pts = np.stack([np.cos(phi) * r * radius, np.sin(phi) * r * radius, z * radius], -1)
    dims, coords, lookup = oracle.brick_grid(origin, voxel, [extent] * 3, pts, mu)
    local = np.arange(512)
    v = np.stack([local & 7, (local >> 3) & 7, local >> 6], -1)            # (512, 3)
    p = origin + (coords[:, None, :3] * 8 + v[None] + 0.5) * voxel          # (count, 512, 3)
    sdf = np.sqrt((p ** 2).sum(-1)) - radius
    tsdf = np.clip(sdf / mu, -1, 1).astype(np.float32).reshape(-1)
    weight = np.where(sdf > -mu, 2.0, 0.0).astype(np.float32).reshape(-1)
    return dict(origin=origin, voxel=voxel, dims=dims, lookup=lookup, coords=coords,
                tsdf=tsdf, weight=weight, radius=radius)
