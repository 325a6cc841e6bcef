"""Seeded synthetic scenes and camera paths for the dense-reconstruction workloads.

Images are ray-cast on the CPU by libl3dscene.so (csrc/scene.cpp): a unit sphere resting on the
plane y = -1, both textured by a solid 3-octave value noise in [0, 1] (frequencies 24, 57 and
131 per metre, amplitudes 0.5, 0.3 and 0.2), or a 4 x 3 x 2.5 m room holding textured cuboids.
World y points up; cameras use computer-vision axes.  Every random choice derives from `seed`.

Workloads (sizes as quoted for the benchmark):
  small  8 views 320x240 on a circle of radius 1.5 m in the plane y = 0 looking at the origin,
         fx = fy = 280, cx = 160, cy = 120; 4 sources, 3 iterations, depths 0.5-3 m;
         TSDF 128^3 at 1 cm (centred at the origin), truncation 4 cm, uint16 weights.
  scan   48 views 640x480 on a helix (1 turn, radius 1.2 -> 2.0 m, elevation -10 -> 40 deg),
         fx = fy = 560, cx = 320, cy = 240; poses given to the solver carry 2 mm / 0.1 deg
         noise, pixels Gaussian noise sigma 0.01; 8 sources, 5 iterations, depths 0.15-4 m;
         TSDF 512^3 at 4 mm, truncation 2 cm, uint16 weights.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

from .camera import Intrinsics, Pose, StereoView, camera_center, look_at, rotation, views_array

_LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib", "libl3dscene.so")
_lib = None


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            raise ImportError(f"{_LIB_PATH} is missing: run `python luvas.io-3d_b200/build.py`")
        lib = C.CDLL(_LIB_PATH)
        lib.l3d_scene_sphere.restype = C.c_int
        lib.l3d_scene_sphere.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_uint32, C.c_double,
                                         C.c_void_p, C.c_void_p]
        lib.l3d_scene_room.restype = C.c_int
        lib.l3d_scene_room.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_uint32, C.c_double,
                                       C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]
        _lib = lib
    return _lib


def render_sphere(views, sizes, seed: int, sigma: float = 0.0):
    """Renders the sphere scene: lists of (H, W) float32 images and ground-truth z-depths."""
    va = views_array(views)
    sz = np.ascontiguousarray(np.asarray(sizes, dtype=np.int32).reshape(-1, 2))
    total = int((sz[:, 0].astype(np.int64) * sz[:, 1]).sum())
    img = np.empty(total, dtype=np.float32)
    dep = np.empty(total, dtype=np.float32)
    rc = _load().l3d_scene_sphere(va.ctypes.data, sz.ctypes.data, len(views), seed & 0xFFFFFFFF,
                                  float(sigma), img.ctypes.data, dep.ctypes.data)
    if rc:
        raise RuntimeError("scene rendering failed")
    return _split(img, sz), _split(dep, sz)


def render_room(views, sizes, boxes: np.ndarray, seed: int, sigma: float = 0.0):
    va = views_array(views)
    sz = np.ascontiguousarray(np.asarray(sizes, dtype=np.int32).reshape(-1, 2))
    bx = np.ascontiguousarray(boxes, dtype=np.float64).reshape(-1, 6)
    total = int((sz[:, 0].astype(np.int64) * sz[:, 1]).sum())
    img = np.empty(total, dtype=np.float32)
    dep = np.empty(total, dtype=np.float32)
    rc = _load().l3d_scene_room(va.ctypes.data, sz.ctypes.data, len(views), seed & 0xFFFFFFFF,
                                float(sigma), bx.ctypes.data, bx.shape[0], img.ctypes.data,
                                dep.ctypes.data)
    if rc:
        raise RuntimeError("scene rendering failed")
    return _split(img, sz), _split(dep, sz)


def _split(flat: np.ndarray, sizes: np.ndarray):
    out, o = [], 0
    for w, h in sizes:
        n = int(w) * int(h)
        out.append(flat[o:o + n].reshape(int(h), int(w)))
        o += n
    return out


def circle_views(n: int, width: int, height: int, radius: float, f: float) -> list[StereoView]:
    k = Intrinsics(f, f, width / 2.0, height / 2.0)
    out = []
    for i in range(n):
        a = 2 * np.pi * i / n
        c = (radius * np.sin(a), 0.0, radius * np.cos(a))
        out.append(StereoView(k, look_at(c, (0.0, 0.0, 0.0))))
    return out


def helix_views(n: int, width: int, height: int, f: float, turns: float = 2.0,
                r0: float = 1.2, r1: float = 2.0, e0: float = -10.0, e1: float = 40.0):
    k = Intrinsics(f, f, width / 2.0, height / 2.0)
    out = []
    for i in range(n):
        s = i / max(1, n - 1)
        a = 2 * np.pi * turns * i / n
        r = r0 + (r1 - r0) * s
        e = np.radians(e0 + (e1 - e0) * s)
        c = (r * np.cos(e) * np.sin(a), r * np.sin(e), r * np.cos(e) * np.cos(a))
        out.append(StereoView(k, look_at(c, (0.0, 0.0, 0.0))))
    return out


def perturb(views, seed: int, trans: float, rot_deg: float) -> list[StereoView]:
    """Moves each camera centre by `trans` metres and turns it by `rot_deg` degrees about a
    random axis (seeded)."""
    rng = np.random.default_rng(seed)
    out = []
    for v in views:
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        axis = rng.normal(size=3)
        Rn = rotation(axis, np.radians(rot_deg)) @ v.pose.R
        c = camera_center(v.pose) + trans * d
        out.append(StereoView(v.intrinsics, Pose(Rn, -Rn @ c)))
    return out


def neighbour_sources(n: int, k: int, circular: bool) -> list[list[int]]:
    """The k nearest other views by index distance (ties: the earlier view first)."""
    out = []
    for i in range(n):
        if circular:
            cand = sorted((j for j in range(n) if j != i),
                          key=lambda j: (min(abs(j - i), n - abs(j - i)), (j - i) % n > n // 2, j))
        else:
            cand = sorted((j for j in range(n) if j != i), key=lambda j: (abs(j - i), j))
        out.append(cand[:k])
    return out


@dataclass
class Workload:
    name: str
    width: int
    height: int
    views: list                      # poses handed to the solver
    true_views: list                 # poses the images were rendered with
    images: list                     # (H, W) float32
    truth: list                      # (H, W) float32 z-depth, 0 = sky
    sources: list
    ranges: list
    iterations: int
    tsdf_dims: tuple
    tsdf_voxel: float
    tsdf_origin: tuple
    tsdf_truncation: float
    needed: list = field(default_factory=list)
    window: int = 6
    dilation: int = 2
    sizes: list | None = None        # per-view (width, height) when the views differ in size
    boxes: np.ndarray | None = None

    @property
    def pixels(self) -> int:
        """Pixels per step summed over the views (width * height each when uniform)."""
        if self.sizes is not None:
            return int(sum(w * h for w, h in self.sizes))
        return self.width * self.height * len(self.views)


def small(seed: int = 1, n_views: int = 8, width: int = 320, height: int = 240) -> Workload:
    """8 views of 320x240 on a circle; 4 sources, 3 iterations; TSDF 128^3 at 1 cm."""
    f = 280.0 * width / 320.0
    views = circle_views(n_views, width, height, 1.5, f)
    imgs, truth = render_sphere(views, [(width, height)] * n_views, seed)
    src = neighbour_sources(n_views, min(4, n_views - 1), circular=True)
    dims = (128, 128, 128)
    return Workload("small", width, height, views, views, imgs, truth, src,
                    [(0.5, 3.0)] * n_views, 3, dims, 0.01, (-0.64, -0.64, -0.64), 0.04,
                    needed=[2] * n_views)


def scan(seed: int = 2, n_views: int = 48, width: int = 640, height: int = 480,
         tsdf_dim: int = 512) -> Workload:
    """48 views of 640x480 on one turn of a helix (7.5 degrees between neighbours) with pose
    and pixel noise; 8 sources, 5 iterations; TSDF 512^3 at 4 mm.  The closest views (radius
    1.2-1.4 m, 0.2-0.4 m from the sphere) see the noise texture too magnified for an 11x11
    window to match reliably; from radius 1.4 m on, median depth errors are 0.1-0.8 %."""
    f = 560.0 * width / 640.0
    true_views = helix_views(n_views, width, height, f, turns=1.0)
    imgs, truth = render_sphere(true_views, [(width, height)] * n_views, seed, sigma=0.01)
    views = perturb(true_views, seed + 1000, 0.002, 0.1)
    src = neighbour_sources(n_views, min(8, n_views - 1), circular=False)
    vox = 0.004 * 512 / tsdf_dim
    half = tsdf_dim * vox / 2
    return Workload("scan", width, height, views, true_views, imgs, truth, src,
                    [(0.15, 4.0)] * n_views, 5, (tsdf_dim,) * 3, vox, (-half, -half, -half), 0.02,
                    needed=[3] * n_views)


def polish(seed: int = 6, n_views: int = 24, width: int = 640, height: int = 480,
           trans: float = 0.005, rot_deg: float = 0.3) -> Workload:
    """The small workload's sphere scene with 24 views of 640x480 on its circle (radius 1.5 m,
    fx = fy = 560): images rendered with the true poses, poses handed to the solver perturbed by
    5 mm / 0.3 deg (seeded); 4 sources, 5 iterations, depths 0.3-3 m.  The starting point of
    gradient-based plane and pose polishing."""
    f = 280.0 * width / 320.0
    true_views = circle_views(n_views, width, height, 1.5, f)
    imgs, truth = render_sphere(true_views, [(width, height)] * n_views, seed, sigma=0.01)
    views = perturb(true_views, seed + 1000, trans, rot_deg)
    src = neighbour_sources(n_views, min(4, n_views - 1), circular=True)
    dims = (256, 256, 256)
    return Workload("polish", width, height, views, true_views, imgs, truth, src,
                    [(0.3, 3.0)] * n_views, 5, dims, 0.01, (-1.28, -1.28, -1.28), 0.04,
                    needed=[2] * n_views)


def relative_pose_errors(views, true_views, anchor: int = 0):
    """Per view, the rotation (degrees) and translation (metres) error of its pose relative to
    the anchor view's, against the same relative pose of the true views (the anchor itself
    excluded)."""
    rot, trans = [], []
    Ra, ta = np.asarray(views[anchor].pose.R), np.asarray(views[anchor].pose.t)
    Qa, qa = np.asarray(true_views[anchor].pose.R), np.asarray(true_views[anchor].pose.t)
    for i, (v, tv) in enumerate(zip(views, true_views)):
        if i == anchor:
            continue
        R = np.asarray(v.pose.R) @ Ra.T
        t = np.asarray(v.pose.t) - R @ ta
        Q = np.asarray(tv.pose.R) @ Qa.T
        q = np.asarray(tv.pose.t) - Q @ qa
        c = np.clip((np.trace(R @ Q.T) - 1) / 2, -1.0, 1.0)
        rot.append(np.degrees(np.arccos(c)))
        trans.append(float(np.linalg.norm(t - q)))
    return np.asarray(rot), np.asarray(trans)


ROOM_RESOLUTIONS = ((480, 360), (640, 480), (960, 720), (1280, 960))


def room_boxes(seed: int, n: int = 20) -> np.ndarray:
    """n axis-aligned cuboids standing on the floor of the 4 x 3 x 2.5 m room (lo.xyz, hi.xyz)."""
    rng = np.random.default_rng(seed)
    out = np.zeros((n, 6))
    for i in range(n):
        size = rng.uniform([0.2, 0.2, 0.2], [0.7, 0.9, 0.7])
        cx, cz = rng.uniform(-1.6, 1.6), rng.uniform(-1.2, 1.2)
        lo = np.array([cx - size[0] / 2, -1.25, cz - size[2] / 2])
        out[i, :3] = lo
        out[i, 3:] = lo + size
    return out


def room(seed: int = 4, n_views: int = 96, tsdf_dim: int = 768) -> Workload:
    """96 views of mixed resolutions inside a 4 x 3 x 2.5 m room with 20 textured cuboids, on an
    ellipse around the room centre looking across it; 8 sources, 5 iterations; TSDF 768^3 at
    8 mm.  The image sizes are drawn uniformly from ROOM_RESOLUTIONS."""
    rng = np.random.default_rng(seed)
    sizes = [ROOM_RESOLUTIONS[i] for i in rng.integers(0, len(ROOM_RESOLUTIONS), size=n_views)]
    views = []
    for i in range(n_views):
        a = 2 * np.pi * i / n_views
        c = np.array([1.5 * np.sin(a), 0.2 + 0.2 * np.sin(3 * a), 1.0 * np.cos(a)])
        target = np.array([-0.5 * c[0], -0.6, -0.5 * c[2]])
        W, H = sizes[i]
        k = Intrinsics(0.875 * W, 0.875 * W, W / 2.0, H / 2.0)
        views.append(StereoView(k, look_at(c, target)))
    boxes = room_boxes(seed + 1)
    imgs, truth = render_room(views, sizes, boxes, seed, sigma=0.01)
    src = neighbour_sources(n_views, min(8, n_views - 1), circular=True)
    vox = 0.008 * 768 / tsdf_dim
    half = tsdf_dim * vox / 2
    w = Workload("room", sizes[0][0], sizes[0][1], views, views, imgs, truth, src,
                 [(0.2, 6.0)] * n_views, 5, (tsdf_dim,) * 3, vox, (-half, -half, -half), 4 * vox,
                 needed=[3] * n_views)
    w.sizes = sizes
    w.boxes = boxes
    return w
