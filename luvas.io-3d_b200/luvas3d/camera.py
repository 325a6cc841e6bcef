"""Pinhole cameras and poses (frontend/src/app/vision/geometry/camera.ts).

Poses map world to camera in computer-vision axes (x right, y down, z forward):
x_cam = R X + t with R row-major (camera.ts:19-26).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class Intrinsics:
    """Pinhole intrinsics in pixels of a given image size (camera.ts:12-17)."""

    fx: float
    fy: float
    cx: float
    cy: float


@dataclass
class Pose:
    """World -> camera rigid transform (camera.ts:23-26)."""

    R: np.ndarray  # (3, 3) float64
    t: np.ndarray  # (3,) float64


@dataclass
class StereoView:
    """One posed view (mvs/dense-stereo.ts:11-14)."""

    intrinsics: Intrinsics
    pose: Pose


def scale_intrinsics(k: Intrinsics, sx: float, sy: float | None = None) -> Intrinsics:
    """scaleIntrinsics (camera.ts:28-36): pixel centres stay aligned, (c + 0.5) s - 0.5."""
    sy = sx if sy is None else sy
    return Intrinsics(k.fx * sx, k.fy * sy, (k.cx + 0.5) * sx - 0.5, (k.cy + 0.5) * sy - 0.5)


def relative_pose(a: Pose, b: Pose) -> Pose:
    """relativePose (camera.ts:73-77): transform from camera a to camera b."""
    R = b.R @ a.R.T
    return Pose(R, b.t - R @ a.t)


def project(k: Intrinsics, pose: Pose, x) -> np.ndarray:
    """project (camera.ts:62-65): [u, v, depth]."""
    p = pose.R @ np.asarray(x, dtype=np.float64) + pose.t
    return np.array([k.fx * p[0] / p[2] + k.cx, k.fy * p[1] / p[2] + k.cy, p[2]])


def camera_center(pose: Pose) -> np.ndarray:
    """cameraCenter (camera.ts:42-45)."""
    return -(pose.R.T @ pose.t)


def look_at(center, target, up=(0.0, 1.0, 0.0)) -> Pose:
    """Pose of a camera at `center` looking at `target` with world `up` pointing up in the image
    (image y runs down)."""
    c = np.asarray(center, dtype=np.float64)
    f = np.asarray(target, dtype=np.float64) - c
    f /= np.linalg.norm(f)
    r = np.cross(f, np.asarray(up, dtype=np.float64))
    r /= np.linalg.norm(r)
    d = np.cross(f, r)
    R = np.stack([r, d, f])
    return Pose(R, -R @ c)


def rotation(axis, angle: float) -> np.ndarray:
    """Rodrigues rotation matrix."""
    a = np.asarray(axis, dtype=np.float64)
    n = np.linalg.norm(a)
    if n == 0 or angle == 0:
        return np.eye(3)
    a = a / n
    K = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
    return np.eye(3) + np.sin(angle) * K + (1 - np.cos(angle)) * (K @ K)


def views_array(views) -> np.ndarray:
    """(n, 16) float64 rows fx fy cx cy | R | t, the layout of the native view tables."""
    out = np.zeros((len(views), 16), dtype=np.float64)
    for i, v in enumerate(views):
        k = v.intrinsics
        out[i, :4] = (k.fx, k.fy, k.cx, k.cy)
        out[i, 4:13] = np.asarray(v.pose.R, dtype=np.float64).reshape(9)
        out[i, 13:16] = np.asarray(v.pose.t, dtype=np.float64).reshape(3)
    return out
