"""Benchmark of the dense-reconstruction path: PatchMatch px-iters/s and TSDF voxel-updates/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--form plain|fast]

Workload (the scan-scale configuration): 48 synthetic views of 640x480 (sphere-on-plane scene,
3-octave value noise, helical camera path, 2 mm / 0.1 deg pose noise, pixel noise 0.01), 8
sources, 5 red/black iterations, 11x11 window dilated by 2 (6 x 6 samples); consistency filter of
every view; TSDF 512^3 at 4 mm, truncation 2 cm, f32 tsdf + uint16 Q8.8 weights.

One step = the photometric PatchMatch stage over all 48 views + the consistency filter of all
views + TSDF integration of all 48 filtered maps.  `value` is the PatchMatch px-iters/s of the
step (px-iter = one pixel updated in one red/black iteration: 48 * 307200 * 5 per step) timed on
the PatchMatch stage; the TSDF stage gives voxel-updates/s (134M voxels * 48 views per step).
Inputs are resident in HBM for `value`; `e2e` repeats the step through the C ABI with the images
copied from pinned host memory every step and the filtered maps and the TSDF volume read back.
L2 is flushed (a 256 MB write) before every timed step.

Multi-GPU: the path shards by reference view with no data-path collective in the photometric
stage; each rank runs an independent replica of the workload ("scaling": "weak").
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "luvas.io-3d_b200"))

import numpy as np  # noqa: E402

METRIC = "PatchMatch px-iters/s, TSDF voxel-upd/s: chosen vs plain FP32 form, 1×B200"


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def build_workload(args):
    from luvas3d import scenes

    if args.workload == "room":
        return scenes.room(n_views=args.views or 96, tsdf_dim=args.tsdf_dim or 768)
    if args.workload == "polish":
        return scenes.polish(n_views=args.views or 24)
    return scenes.scan(n_views=args.views or 48, width=args.width, height=args.height,
                       tsdf_dim=args.tsdf_dim or 512)


def workload_name(w) -> str:
    if w.name == "room":
        return (f"room: {len(w.views)} views of mixed sizes (480x360..1280x960), 20 cuboids, "
                f"8 sources, 5 iterations, TSDF {w.tsdf_dims[0]}^3 at {w.tsdf_voxel * 1000:.0f} mm")
    return (f"scan: {len(w.views)} views {w.width}x{w.height}, 8 sources, 5 iterations, window "
            f"6x6 samples dilated by 2 (11x11 footprint), TSDF {w.tsdf_dims[0]}^3 at {w.tsdf_voxel * 1000:.0f} mm, "
            f"trunc {w.tsdf_truncation * 100:.0f} cm, Q8.8 weights")


def scene_conventions(w) -> dict:
    """Geometry, texture, camera and seed conventions of the synthetic scene (scene.cpp,
    scenes.py), recorded with every bench line."""
    if w.name == "room":
        geometry = ("inside of the box x in [-2, 2], y in [-1.25, 1.25], z in [-1.5, 1.5] m with "
                    "20 seeded axis-aligned cuboids")
    else:
        geometry = "unit sphere centred at the origin resting on the plane y = -1"
    return {"geometry": geometry,
            "texture": "3-octave value noise in [0, 1]: lattice frequencies 24, 57, 131 per m, "
                       "amplitudes 0.5, 0.3, 0.2, smoothstep interpolation, PCG-hashed lattice",
            "images": "2x2 supersampled, Gaussian pixel noise (sigma 0.01 on scan/room); "
                      "depth = camera-z of the pixel-centre ray, 0 where the ray escapes",
            "cameras": "x right, y down, z forward, x_cam = R X + t; look-at the origin with world "
                       "up +y" + ("; one helix turn, radius 1.2 -> 2.0 m, elevation -10 -> 40 deg, "
                                  "poses given to the solver perturbed by 2 mm / 0.1 deg"
                                  if w.name == "scan" else ""),
            "seeds": {"scene": {"scan": 2, "room": 4, "small": 1, "polish": 6}.get(w.name),
                      "pose_noise": "scene seed + 1000" if w.name == "scan" else None,
                      "patchmatch": "pcg(index ^ pcg(seed + 7919 iter + 104729 phase)), "
                                    "seed = (ref + 1) 0x9e3779b1 + 97 iter + 13 phase + 7 flags"}}


def cpu_baseline(w, threads: int, budget_s: float = 20.0) -> dict:
    """The FP32 oracle on the host cores: one reference view's init + 1 red/black iteration at
    full resolution with the workload's sources, and one TSDF view integration of the full
    volume.  px-iters/s and voxel-updates/s of that bounded sample."""
    import oracle

    o = oracle.Stereo(w.width, w.height, w.views, w.images, 32, threads=threads)
    h0, w0 = w.images[0].shape
    t0 = time.perf_counter()
    o.kernel(oracle.INIT, 0, w.sources[0], min_depth=w.ranges[0][0], max_depth=w.ranges[0][1])
    t_init = time.perf_counter() - t0
    t0 = time.perf_counter()
    for phase in (0, 1):
        o.kernel(oracle.PROPAGATE, 0, w.sources[0], iteration=0, phase=phase,
                 min_depth=w.ranges[0][0], max_depth=w.ranges[0][1])
    t_prop = time.perf_counter() - t0
    pm = w.images[0].size / t_prop
    # TSDF: one view into the full volume
    o.kernel(oracle.PACK, 0, w.sources[0], min_depth=w.ranges[0][0], max_depth=w.ranges[0][1])
    v = w.views[0]
    k = v.intrinsics
    ot = oracle.Tsdf(w0, h0, w.tsdf_voxel, w.tsdf_origin, w.tsdf_truncation,
                     dense=w.tsdf_dims, weight_q8=True, threads=threads)
    t0 = time.perf_counter()
    ot.integrate(dict(k=(k.fx, k.fy, k.cx, k.cy), R=v.pose.R, t=v.pose.t,
                      max_depth=w.ranges[0][1]), o.depths[0])
    t_tsdf = time.perf_counter() - t0
    vox = int(np.prod(w.tsdf_dims))
    # one thread: one colour of the same iteration (half the pixels updated)
    o1 = oracle.Stereo(w.width, w.height, w.views, w.images, 32, threads=1)
    o1.kernel(oracle.INIT, 0, w.sources[0], min_depth=w.ranges[0][0], max_depth=w.ranges[0][1])
    t0 = time.perf_counter()
    o1.kernel(oracle.PROPAGATE, 0, w.sources[0], iteration=0, phase=0,
              min_depth=w.ranges[0][0], max_depth=w.ranges[0][1])
    t_one = time.perf_counter() - t0
    return {"value": pm, "unit": "px-iters/s", "cores": threads, "kind": "port",
            "single_thread_px_iters_per_s": (w.images[0].size / 2) / t_one,
            "sample": (f"FP32 oracle: 1 reference view x 1 red/black iteration at "
                       f"{w0}x{h0}, {len(w.sources[0])} sources "
                       f"({t_prop:.2f} s); TSDF 1 view into {w.tsdf_dims[0]}^3 ({t_tsdf:.2f} s)"),
            "tsdf_voxel_updates_per_s": vox / t_tsdf, "seconds": t_prop + t_tsdf}


def run_reference(args, rank: int, world: int) -> None:
    """--impl reference: the CPU restatement of the path on the host cores (the reference has no
    CPU implementation of these stages; its WGSL needs WebGPU, unavailable on this box)."""
    if rank != 0:
        return
    w = build_workload(args)
    threads = os.cpu_count() or 1
    vals, tv, secs = [], [], []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        r = cpu_baseline(w, threads)
        if i >= args.warmup:
            vals.append(r["value"])
            tv.append(r["tsdf_voxel_updates_per_s"])
            secs.append(time.perf_counter() - t0)
    v = statistics.median(vals)
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "px-iters/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * w.pixels * w.iterations / v,
        "ms_per_step_basis": "one full step of the workload at the sampled rate; each timed step "
                             "runs the bounded sample only",
        "sample_seconds_per_step": statistics.median(secs), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": workload_name(w), "sample": r["sample"]},
        "scene": scene_conventions(w),
        "tsdf_voxel_updates_per_s": statistics.median(tv),
        "cpu_baseline": {"value": v, "unit": "px-iters/s", "cores": threads, "kind": "port",
                         "sample": r["sample"],
                         "single_thread_px_iters_per_s": r["single_thread_px_iters_per_s"]},
        "e2e": {"value": v, "unit": "px-iters/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_polish(args) -> None:
    """Differentiation configuration: 24 views of 640x480 of the sphere scene with poses perturbed
    by 5 mm / 0.3 deg.  PatchMatch (fast form) on the perturbed poses gives the starting planes;
    then 20 Adam steps polish every view's planes and pose increment against the summed NCC
    cost (4 sources per view, view 0 fixed).  Reports the gradient pass throughput
    (pixel-sources/s, one cost + plane + pose gradient evaluation each) and the relative pose
    errors before and after."""
    import torch

    from luvas3d import DTYPE_F16, FORM_FAST, DenseStereo, SolveOptions, StereoOptions, scenes
    from luvas3d import grad as G

    w = scenes.polish(n_views=args.views or 24)
    V = len(w.views)
    refs = list(range(V))
    opts = [SolveOptions(w.sources[r], w.ranges[r][0], w.ranges[r][1], iterations=w.iterations)
            for r in refs]
    st = DenseStereo(w.width, w.height, w.views)  # FP32 images for the exact bilinear gradient
    for i, im in enumerate(w.images):
        st.set_image(i, im)

    def starting_planes(views):
        """PatchMatch (fast form) planes of every view solved with `views`' poses, and the
        weights of the pixels it matched well (cost < 0.5)."""
        pm = DenseStereo(w.width, w.height, views, StereoOptions(storage=DTYPE_F16, form=FORM_FAST))
        for i, im in enumerate(w.images):
            pm.set_image(i, im)
        pm.solve_all(refs, opts)
        pl, wt = [], []
        for r in refs:
            hyp, cost = pm.read_hypotheses_layer(r)
            pl.append(G.planes_from_hypotheses(hyp).cuda().contiguous())
            wt.append(torch.tensor((cost < 0.5).astype(np.float32), device="cuda"))
        pm.destroy()
        return pl, wt

    planes, weights = starting_planes(w.views)
    n_src = len(w.sources[0])
    # gradient pass alone: every view's cost + plane + pose gradient, timed with CUDA events
    deltas = torch.zeros((V, 6), dtype=torch.float32, device="cuda")
    gd = torch.zeros((V, 6), dtype=torch.float64, device="cuda")

    def grad_pass():
        for r in refs:
            G.ncc_value_and_grad(st, r, w.sources[r], planes[r], deltas, weights[r], gd)

    for _ in range(max(3, args.warmup)):
        grad_pass()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    times = []
    for _ in range(max(1, args.steps)):
        flush.fill_(1)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        grad_pass()
        b.record()
        torch.cuda.synchronize()
        times.append(a.elapsed_time(b))
    grad_ms = statistics.median(times)
    units = w.pixels * n_src
    rot0, tr0 = scenes.relative_pose_errors(w.views, w.true_views)
    srcs = [w.sources[r] for r in refs]

    def run(pl, wt):
        res = G.polish(st, refs, srcs, pl, steps=20, weights=wt)
        rot1, tr1 = scenes.relative_pose_errors(G.apply_deltas(w.views, res.deltas), w.true_views)
        return {"steps": 20, "ms_per_step": res.ms_per_step,
                "loss_first": res.losses[0], "loss_last": res.losses[-1],
                "rot_err_deg_mean": [float(rot0.mean()), float(rot1.mean())],
                "trans_err_mm_mean": [float(tr0.mean() * 1e3), float(tr1.mean() * 1e3)],
                "weighted_pixels": int(sum(float(x.sum()) for x in wt))}

    # (1) planes from PatchMatch on the perturbed poses; (2) planes of the true geometry (solved
    # with the true poses, as a depth prior would give), poses still perturbed
    from_pm = run(planes, weights)
    true_planes, true_weights = starting_planes(w.true_views)
    from_geometry = run(true_planes, true_weights)
    line = {
        "metric": "NCC adjoint pixel-sources/s (cost + plane + se(3) pose gradient)",
        "value": units / (grad_ms / 1e3), "unit": "pixel-sources/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": grad_ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 images, f32 arithmetic, FP64 pose composition and pose-gradient sums",
        "data": "synthetic (seeded sphere-on-plane scene, value-noise texture)",
        "config": {"workload": (f"polish: {V} views {w.width}x{w.height}, {n_src} sources, window "
                                "6x6 dilated by 2, poses perturbed 5 mm / 0.3 deg"),
                   "l2": "flushed (256 MB write) before every timed gradient pass"},
        "polish_from_patchmatch_planes": from_pm,
        "polish_from_true_geometry_planes": from_geometry,
        "pose_errors": "relative to view 0 (held fixed), mean over the other views: [before, after]",
        "gpu_launches": 3 * V,
    }
    print(json.dumps(line), flush=True)
    st.destroy()


def run_fusion(args):
    """The rows on either side of the stereo stage, on the scan workload (48 views 640x480):
    image preparation from 1280x960 RGBA camera frames (rgbaToGray by block means and by the
    area filter, RGB thumbnails), the coarse-to-fine schedule of the High profile (6 iterations
    at 320x240, then 4 at 640x480 from the coarse planes, against 5 single-scale iterations),
    the dense point cloud (consistency filter + addDepthMap of every view with the cell budget
    of the High profile), the TSDF sweep and surface extraction (surface nets + normals, then
    removeSmallComponents(0.01, 200)).  Every stage runs on one stream and is timed with CUDA
    events there, after a warm-up run; a CPU-oracle sample of each stage runs on the host
    cores.  `value` is camera pixels per second through the whole chain."""
    import torch

    import oracle
    from luvas3d import (DTYPE_F16, FORM_FAST, DenseStereo, IntegrationView, SolveOptions,
                         StereoOptions, TsdfVolume, scenes)
    from luvas3d import image as I
    from luvas3d import mesh as M
    from luvas3d.camera import StereoView, scale_intrinsics
    from luvas3d.cloud import FusionView, fuse_depth_maps
    from luvas3d.packing import unpack_depth

    w = scenes.scan(n_views=args.views or 48, tsdf_dim=args.tsdf_dim or 512)
    V, W, H = len(w.views), w.width, w.height
    refs = list(range(V))
    stream = torch.cuda.Stream()
    sptr = stream.cuda_stream
    peaks, peak_kind = _peaks()
    hbm = peaks.get("hbm_gbs", 6650.0)

    def timed(fn, reps: int = 1):
        """Device ms of fn() on the bench stream (median of `reps` after one warm-up run)."""
        with torch.cuda.stream(stream):
            fn()
            out = []
            for _ in range(reps):
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                fn()
                b.record(stream)
                b.synchronize()
                out.append(a.elapsed_time(b))
        return statistics.median(out)

    def host_s(fn):
        t0 = time.perf_counter()
        fn()
        return time.perf_counter() - t0

    # camera frames: the scan's gray images at 2x, as RGBA with a colour tint (synthetic)
    with torch.cuda.stream(stream):
        g = torch.stack([torch.from_numpy(np.ascontiguousarray(im)) for im in w.images]).cuda()
        g = (g.clamp(0, 1) * 255).to(torch.uint8)
        g2 = g.repeat_interleave(2, dim=1).repeat_interleave(2, dim=2)
        rgba = torch.stack([g2, (g2.int() * 7 // 8).to(torch.uint8), (g2.int() * 3 // 4).to(torch.uint8),
                            torch.full_like(g2, 255)], dim=-1).contiguous()
    torch.cuda.synchronize()
    FW, FH = rgba.shape[2], rgba.shape[1]
    grays, thumbs = [None] * V, [None] * V

    def prep_block():
        for v in refs:
            grays[v] = I.rgba_to_gray(rgba[v], W, H)

    def prep_area():
        for v in refs:
            I.rgba_to_gray(rgba[v], 600, 450)

    def prep_thumbs():
        for v in refs:
            thumbs[v] = I.downsample_rgb(rgba[v], 160, 120)

    reps = max(1, args.steps)
    ms_block, ms_area, ms_thumb = timed(prep_block, reps), timed(prep_area, reps), timed(prep_thumbs, reps)
    frame_px = V * FW * FH
    image = {
        "rgba_to_gray_blocks": {"ms": ms_block, "frame_px_per_s": frame_px / (ms_block / 1e3),
                                "hbm_frac": frame_px * 4 / (ms_block / 1e3) / 1e9 / hbm},
        "rgba_to_gray_area_600x450": {"ms": ms_area, "frame_px_per_s": frame_px / (ms_area / 1e3)},
        "thumbnails_160x120": {"ms": ms_thumb, "frame_px_per_s": frame_px / (ms_thumb / 1e3)},
    }
    fr0 = rgba[0].cpu().numpy()
    cpu_img = host_s(lambda: oracle.rgba_to_gray(fr0, W, H))
    image["cpu_oracle_frame_px_per_s"] = FW * FH / cpu_img
    thumbs_host = [t.cpu().numpy() for t in thumbs]
    grays_host = [t.cpu().numpy() for t in grays]

    # stereo, single-scale (5 iterations) and the High profile's coarse-to-fine (6 + 4)
    so = StereoOptions(storage=DTYPE_F16, form=FORM_FAST, stream=sptr)
    single = DenseStereo(W, H, w.views, so)
    for v in refs:
        single.set_image(v, grays_host[v])
    single.set_graphs(True)
    o5 = [SolveOptions(w.sources[r], w.ranges[r][0], w.ranges[r][1], iterations=5) for r in refs]
    ms_single = timed(lambda: single.solve_all(refs, o5), reps)
    cw, ch = W // 2, H // 2
    cviews = [StereoView(scale_intrinsics(v.intrinsics, cw / W, ch / H), v.pose) for v in w.views]
    coarse = DenseStereo(cw, ch, cviews, StereoOptions(depth_maps=False, storage=DTYPE_F16,
                                                       form=FORM_FAST, stream=sptr))
    fine = DenseStereo(W, H, w.views, StereoOptions(coarse=coarse, storage=DTYPE_F16, form=FORM_FAST,
                                                    stream=sptr))
    for v in refs:
        coarse.set_image(v, I.downsample_gray(grays[v], cw, ch).cpu().numpy())
        fine.set_image(v, grays_host[v])
    oc = [SolveOptions(w.sources[r], w.ranges[r][0], w.ranges[r][1], iterations=6, pack=False)
          for r in refs]
    of = [SolveOptions(w.sources[r], w.ranges[r][0], w.ranges[r][1], iterations=4, from_coarse=True)
          for r in refs]

    def c2f():
        coarse.solve_all(refs, oc)
        fine.solve_all(refs, of)

    ms_c2f = timed(c2f, reps)

    def acc(st):
        errs, surf, valid = [], 0, 0
        for r in refs:
            packed = st.depth_map(r)
            t = w.truth[r]
            m = t > 0
            ok = m & (packed != 0)
            surf += int(m.sum())
            valid += int(ok.sum())
            errs.append(np.abs(unpack_depth(packed[ok]) - t[ok]) / t[ok])
        e = np.concatenate(errs)
        return {"valid_fraction": round(valid / max(1, surf), 4),
                "median_rel_err": float(np.percentile(e, 50)), "p90_rel_err": float(np.percentile(e, 90))}

    px_c2f = V * (cw * ch * 6 + W * H * 4)
    stereo = {
        "single_scale_5": {"ms": ms_single, "px_iters_per_s": V * W * H * 5 / (ms_single / 1e3),
                           "depth_accuracy": acc(single)},
        "coarse_to_fine_6_4": {"ms": ms_c2f, "px_iters_per_s": px_c2f / (ms_c2f / 1e3),
                               "depth_accuracy": acc(fine)},
    }
    # the geometric-consistency pass (1 iteration, as the Medium profile) on the coarse-to-fine
    # maps: the photometric cost plus 0.2 x the forward-backward reprojection error per source
    og = [SolveOptions(w.sources[r], w.ranges[r][0], w.ranges[r][1], iterations=1, geometric=True)
          for r in refs]
    fine.solve_all(refs, og)  # warm-up: the maps it reads are the previous pass's
    c2f()
    with torch.cuda.stream(stream):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fine.solve_all(refs, og)
        b.record(stream)
        b.synchronize()
    ms_geo = a.elapsed_time(b)
    stereo["geometric_1_after_coarse_to_fine"] = {
        "ms": ms_geo, "px_iters_per_s": V * W * H / (ms_geo / 1e3), "depth_accuracy": acc(fine)}

    # dense cloud: filter + addDepthMap per view (fuseDepthMaps), on the single-scale maps
    fviews = [FusionView(w.views[r], w.sources[r], w.needed[r], thumbs_host[r]) for r in refs]
    cell, budget = w.tsdf_voxel, 600_000
    cloud_out = {}

    def fuse():
        pc, final_cell = fuse_depth_maps(single, fviews, cell, budget)
        cloud_out["points"], cloud_out["cell"] = int(pc.positions.shape[0]), final_cell

    ms_cloud = timed(fuse, reps)
    f0 = single.filtered_map(0, w.sources[0], w.needed[0])
    oc0 = oracle.Cloud(cell)
    cpu_cloud = host_s(lambda: oc0.add_map(f0, w.views[0], thumbs_host[0]))
    cloud = {"ms": ms_cloud, "px_per_s": V * W * H / (ms_cloud / 1e3), "points": cloud_out["points"],
             "final_cell_m": cloud_out["cell"],
             "cpu_oracle_px_per_s": W * H / cpu_cloud,
             "note": "GPU: consistency filter + addDepthMap of every view, with the budget check "
                     "(a host round trip) after each view; CPU oracle: addDepthMap of one "
                     "already-filtered map"}

    # TSDF sweep of the filtered maps and surface extraction
    vox = int(np.prod(w.tsdf_dims))
    tsdf = TsdfVolume(W, H, w.tsdf_voxel, w.tsdf_origin, dense=w.tsdf_dims,
                      truncation=w.tsdf_truncation, weight_q8=True, stream=sptr)
    iviews = [IntegrationView(v.intrinsics, v.pose, w.ranges[i][1]) for i, v in enumerate(w.views)]
    single.filter_all(refs, w.sources, w.needed)

    def sweep():
        tsdf.reset()
        tsdf.integrate_many(iviews, stereo=single, layers=refs)

    ms_tsdf = timed(sweep, reps)
    mesh_out = {}

    def surface():
        m = M.extract_surface_device(tsdf, 0.6)
        r = m.remove_small_components(0.01, 200)
        mesh_out["raw"], mesh_out["kept"] = m.counts, r.counts
        r.destroy()
        m.destroy()

    ms_mesh = timed(surface, reps)
    # CPU oracle sample: surface nets of a 128^3 crop at the volume's centre, brick-major
    t_all, w_all = tsdf.read()
    X0, Y0, Z0 = (np.array(w.tsdf_dims) // 2 - 64)
    crop_t = t_all[Z0:Z0 + 128, Y0:Y0 + 128, X0:X0 + 128]
    crop_w = w_all[Z0:Z0 + 128, Y0:Y0 + 128, X0:X0 + 128].astype(np.float32) / 256.0

    def bricks(a):
        b = a.reshape(16, 8, 16, 8, 16, 8).transpose(0, 2, 4, 1, 3, 5)  # bz by bx, z y x
        return np.ascontiguousarray(b).reshape(-1)

    origin = [w.tsdf_origin[0] + X0 * w.tsdf_voxel, w.tsdf_origin[1] + Y0 * w.tsdf_voxel,
              w.tsdf_origin[2] + Z0 * w.tsdf_voxel]
    lookup = np.arange(16 ** 3, dtype=np.int32)
    bt, bw = bricks(crop_t), bricks(crop_w)
    cpu_mesh = host_s(lambda: oracle.extract_surface(origin, w.tsdf_voxel, (16, 16, 16), lookup, bt, bw, 0.6))
    surface_line = {"ms": ms_mesh, "voxels_per_s": vox / (ms_mesh / 1e3),
                    "vertices_indices": [int(x) for x in mesh_out["raw"]],
                    "after_remove_small_components": [int(x) for x in mesh_out["kept"]],
                    "cpu_oracle_voxels_per_s": 128 ** 3 / cpu_mesh}

    total_ms = ms_block + ms_thumb + ms_single + ms_cloud + ms_tsdf + ms_mesh
    line = {
        "metric": "camera px/s through image prep, PatchMatch, filter, dense cloud, TSDF and surface",
        "value": V * FW * FH / (total_ms / 1e3), "unit": "frame-px/s", "n_gpus": 1,
        "steps": reps, "warmup": 1, "ms_per_step": total_ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8 frames, f16 images, f32/f64 arithmetic",
        "data": "synthetic (seeded sphere-on-plane scene, value-noise texture)",
        "config": {"workload": f"fusion: scan {V} views, frames {FW}x{FH} RGBA -> {W}x{H} gray, "
                               f"TSDF {w.tsdf_dims[0]}^3, cloud cell {cell * 1e3:.0f} mm, budget {budget}",
                   "timing": "CUDA events on the one stream every handle uses, median of the steps "
                             "after a warm-up run (the calls that read counts back include those "
                             "host round trips)"},
        "image_prep": image, "stereo": stereo, "dense_cloud": cloud,
        "tsdf_sweep": {"ms": ms_tsdf, "voxel_updates_per_s": vox * V / (ms_tsdf / 1e3)},
        "surface": surface_line, "hbm_peak_source": peak_kind,
    }
    print(json.dumps(line), flush=True)
    for h in (tsdf, fine, coarse, single):
        h.destroy()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--form", default="auto", choices=["auto", "plain", "fast"])
    ap.add_argument("--workload", default="scan", choices=["scan", "room", "polish", "fusion"])
    ap.add_argument("--views", type=int, default=0)
    ap.add_argument("--width", type=int, default=640)
    ap.add_argument("--height", type=int, default=480)
    ap.add_argument("--tsdf-dim", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--storage", default="f16", choices=["f16", "u8", "f32", "bf16"],
                    help="fast-form image storage")
    ap.add_argument("--variant", type=int, default=-1,
                    help="fast-form kernel variant; default: the autotuner's choice")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local)
    if args.workload == "polish":
        if rank == 0:
            run_polish(args)
        return
    if args.workload == "fusion":
        if rank == 0:
            run_fusion(args)
        return
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))

    from luvas3d import (DTYPE_BF16, DTYPE_F16, DTYPE_F32, DTYPE_U8, FORM_FAST, FORM_PLAIN,
                         DenseStereo, IntegrationView, SolveOptions, StereoOptions, TsdfVolume)
    from luvas3d.packing import unpack_depth

    w = build_workload(args)
    V = len(w.views)
    sizes = w.sizes or [(w.width, w.height)] * V
    stream = torch.cuda.Stream()
    sptr = stream.cuda_stream
    refs = list(range(V))
    opts = [SolveOptions(w.sources[r], w.ranges[r][0], w.ranges[r][1], iterations=w.iterations)
            for r in refs]
    iviews = [IntegrationView(v.intrinsics, v.pose, w.ranges[i][1]) for i, v in enumerate(w.views)]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    vox = int(np.prod(w.tsdf_dims))
    px_iters_step = w.pixels * w.iterations
    tsdf = TsdfVolume(max(s[0] for s in sizes), max(s[1] for s in sizes), w.tsdf_voxel,
                      w.tsdf_origin, dense=w.tsdf_dims,
                      truncation=w.tsdf_truncation, weight_q8=True, stream=sptr)
    mk = lambda n=4: [torch.cuda.Event(enable_timing=True) for _ in range(n)]

    def rec(ev):
        with torch.cuda.stream(stream):
            ev.record(stream)

    tuned = {}

    def make_stereo(form):
        storage = {"f16": DTYPE_F16, "u8": DTYPE_U8, "f32": DTYPE_F32, "bf16": DTYPE_BF16}[args.storage] \
            if form == FORM_FAST else DTYPE_F32
        st = DenseStereo(w.width, w.height, w.views,
                         StereoOptions(storage=storage, form=form, stream=sptr), sizes=sizes)
        for i, im in enumerate(w.images):
            st.set_image(i, im)
        if form == FORM_FAST:
            # kernel variant picked by timing one iteration of this batch, then graph replay
            if args.variant >= 0:
                st.variant = args.variant
                tuned["variant"], tuned["ms"] = args.variant, None
            else:
                tuned["variant"], tuned["ms"] = st.autotune(refs, opts)
            st.set_graphs(True)
        return st

    def step(st, evs):
        with torch.cuda.stream(stream):
            flush.fill_(1)
        rec(evs[0])
        st.solve_all(refs, opts)
        rec(evs[1])
        tsdf.reset()  # a fresh volume per scan (tsdf 1, weight 0), outside the timed TSDF stage
        st.filter_all(refs, w.sources, w.needed)
        rec(evs[2])
        tsdf.integrate_many(iviews, stereo=st, layers=refs)
        rec(evs[3])

    def time_form(form, steps, warmup, sample_clocks):
        st = make_stereo(form)
        for _ in range(warmup):
            step(st, mk())
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        l0 = st.launches + tsdf.launches
        clocks = ClockSampler(local) if sample_clocks else None
        if clocks:
            clocks.start()
        all_evs = []
        for _ in range(steps):
            evs = mk()
            step(st, evs)
            all_evs.append(evs)
        torch.cuda.synchronize()
        launches = st.launches + tsdf.launches - l0
        if world > 1:
            dist.barrier()
        clk = clocks.stop() if clocks else None
        ms = {k: [e[a].elapsed_time(e[b]) for e in all_evs]
              for k, (a, b) in {"patchmatch": (0, 1), "filter": (1, 2), "tsdf": (2, 3),
                                "step": (0, 3)}.items()}
        tot = torch.tensor([sum(ms["patchmatch"]), sum(ms["tsdf"]), sum(ms["step"])],
                           dtype=torch.float64, device="cuda")
        if world > 1:
            dist.all_reduce(tot, op=dist.ReduceOp.MAX)
        pm_s, ts_s, st_s = (float(x) / 1e3 for x in tot.tolist())
        # propagate launches alone: solve with 5 iterations minus solve with 0 (init + pack)
        per = {}
        for its in (0, w.iterations):
            o2 = [SolveOptions(w.sources[r], w.ranges[r][0], w.ranges[r][1], iterations=its)
                  for r in refs]
            a, b = mk(2)
            rec(a)
            for _ in range(2):
                st.solve_all(refs, o2)
            rec(b)
            torch.cuda.synchronize()
            per[its] = a.elapsed_time(b) / 2
        n_prop = 2 * w.iterations * (1 if form == FORM_FAST else V)
        prop_ms = (per[w.iterations] - per[0]) / n_prop
        return st, {"pm_s": pm_s, "ts_s": ts_s, "st_s": st_s, "ms": ms, "clk": clk,
                    "launches": launches, "prop_ms": prop_ms,
                    "px_iters_per_s": px_iters_step * steps * world / pm_s}

    def accuracy(st) -> dict:
        """Packed depth maps of the last full solve against the rendered ground truth, scored
        like the reference's stereo self-test (frontend/tools/verify/stereo-check.ts:56-73):
        surface pixels (truth > 0) with a non-zero packed entry count as valid; relative error of
        the packed half depth, median and p90, over all views of this rank."""
        errs, surf, valid = [], 0, 0
        for r in refs:
            packed = st.depth_map(r)
            t = w.truth[r]
            m = t > 0
            ok = m & (packed != 0)
            surf += int(m.sum())
            valid += int(ok.sum())
            errs.append(np.abs(unpack_depth(packed[ok]) - t[ok]) / t[ok])
        e = np.concatenate(errs)
        return {"valid_fraction": round(valid / max(1, surf), 4),
                "median_rel_err": float(np.percentile(e, 50)),
                "p90_rel_err": float(np.percentile(e, 90))}

    plain_steps = max(1, min(args.steps, 2)) if args.form == "auto" else args.steps
    res = {}
    acc = {}
    stereo = None
    forms = {"auto": [FORM_PLAIN, FORM_FAST], "plain": [FORM_PLAIN], "fast": [FORM_FAST]}[args.form]
    for form in forms:
        chosen = form == forms[-1]
        st, r = time_form(form, args.steps if chosen else plain_steps, args.warmup, chosen)
        res[form] = r
        acc["fast" if form == FORM_FAST else "plain"] = accuracy(st)
        if chosen:
            stereo = st
        else:
            st.destroy()
    chosen_form = forms[-1]
    R = res[chosen_form]
    clk = R["clk"]
    value = R["px_iters_per_s"]
    voxel_updates = vox * V * args.steps * world

    # ---- roofline of the dominant kernel (red/black propagate) ------------------------------
    peaks, peak_kind = _peaks()
    S = len(w.sources[0])
    flop_per_px_phase = 14 * S * (18 + 36 * 37 + 15) + 36 * 26
    views_per_launch = V if chosen_form == FORM_FAST else 1
    prop_flops = flop_per_px_phase * (w.pixels / V / 2) * views_per_launch
    achieved = prop_flops / (R["prop_ms"] / 1e3) / 1e12
    sm_mhz = (clk or {}).get("sm_mhz") or 1965.0
    fp32_peak = 148 * 128 * 2 * sm_mhz * 1e6 / 1e12
    roof_fp32 = {"kernel": (f"k_fast_propagate (all {V} views, one colour)"
                            if chosen_form == FORM_FAST else "k_propagate (one view, one colour)"),
                 "bound": "fp32", "achieved": achieved, "peak": fp32_peak,
                 "unit": "TFLOP/s", "frac": achieved / fp32_peak, "traffic": None,
                 "peak_source": "nominal FP32 FMA rate (148 SMs x 128 lanes x 2 flops) at "
                                "the sampled median SM clock",
                 "launch_ms": R["prop_ms"], "flop_per_launch": prop_flops,
                 "flop_model": "14 candidates x sources x (18 + 36 x 37 + 15) + 936 per "
                               "pixel of the colour"}
    # the fast propagate kernel is bound by the texture data pipe: quote its bilinear samples
    # against the rate a probe kernel with the same thread layout measures on this GPU
    roof_tex = None
    if chosen_form == FORM_FAST and args.storage != "bf16":
        import ctypes as C
        from luvas3d import _lib
        rate = C.c_double()
        dt = {"f16": DTYPE_F16, "u8": DTYPE_U8, "f32": DTYPE_F32}[args.storage]
        _lib.check(_lib.load().l3d_measure_texture_rate(dt, 1, C.byref(rate)))
        samples = 14 * S * 36 * (w.pixels / V / 2) * views_per_launch
        got = samples / (R["prop_ms"] / 1e3) / 1e9
        peak_tex = rate.value / 1e9
        # DRAM traffic of one launch: the ncu capture of the 8-view launch of this kernel (F16
        # images, variant 14: 54.13 MB read + 1.90 MB written for 8 x 153 600 pixels of one
        # colour) scaled by the pixels this launch processes; hyp, cost and images all grow
        # with the views in the launch
        traffic = None
        if args.storage == "f16":
            traffic = (54.13248e6 + 1.896704e6) / (8 * 153600) * (w.pixels / V / 2) * views_per_launch
        roof_tex = {"kernel": roof_fp32["kernel"], "bound": "texture", "achieved": got,
                    "peak": peak_tex, "unit": "Gsample/s", "frac": got / peak_tex, "traffic": traffic,
                    "traffic_unit": "DRAM bytes per launch",
                    "traffic_source": "profiles/k_fast_propagate_scan8.md (8-view capture, "
                                      "scaled by the pixels per launch)" if traffic else None,
                    "peak_source": f"measured: l3d_measure_texture_rate({args.storage}, one "
                                   "red/black colour), bilinear samples/s of a 2048x2048 texture",
                    "launch_ms": R["prop_ms"], "samples_per_launch": samples,
                    "sample_model": "14 candidates x sources x 36 bilinear samples per pixel of "
                                    "the colour (the reference's count; sources the corner test "
                                    "rejects are counted although not sampled)"}
    tsdf_ms = sum(R["ms"]["tsdf"]) / len(R["ms"]["tsdf"])
    tsdf_bytes = vox * 12
    tsdf_gbs = tsdf_bytes / (tsdf_ms / 1e3) / 1e9

    # ---- end to end through the C ABI with pinned host buffers ------------------------------
    e2e = None
    if not args.no_e2e:
        import ctypes as C
        from luvas3d import _lib
        lib = _lib.load()
        pinned = [torch.from_numpy(np.ascontiguousarray(im)).pin_memory() for im in w.images]
        out_f = torch.empty(w.pixels, dtype=torch.int32).pin_memory()
        f_off = np.concatenate([[0], np.cumsum([a * b for a, b in sizes])])
        out_t = torch.empty(vox, dtype=torch.float32).pin_memory()
        out_w = torch.empty(vox, dtype=torch.int16).pin_memory()

        def e2e_step():
            for i, im in enumerate(pinned):
                stereo.set_image_device(i, im.data_ptr(), DTYPE_F32)
            stereo.solve_all(refs, opts)
            stereo.filter_all(refs, w.sources, w.needed)
            tsdf.reset()
            for r in refs:
                _lib.check(lib.l3d_stereo_read_filtered_layer(
                    stereo._h(), r, C.c_void_p(out_f[int(f_off[r]):].data_ptr())))
            # the sweep with the volume's read-back overlapped (l3d_tsdf_integrate_many_read)
            tsdf.integrate_many_read(iviews, stereo=stereo, layers=refs, out=(out_t, out_w))

        e2e_step()
        torch.cuda.synchronize()
        ea, eb = mk(2)
        rec(ea)
        for _ in range(args.steps):
            e2e_step()
        rec(eb)
        torch.cuda.synchronize()
        e2e_s = torch.tensor([ea.elapsed_time(eb) / 1e3], dtype=torch.float64, device="cuda")
        if world > 1:
            dist.all_reduce(e2e_s, op=dist.ReduceOp.MAX)
        e2e = {"value": px_iters_step * args.steps * world / float(e2e_s.item()),
               "unit": "px-iters/s", "h2d_bytes_per_step": w.pixels * 4,
               "d2h_bytes_per_step": w.pixels * 4 + vox * 6,
               "ms_per_step": float(e2e_s.item()) * 1e3 / args.steps,
               "includes": "image upload from pinned host memory, PatchMatch, filter, "
                           "read-back of the filtered maps, TSDF sweep with the volume's "
                           "read-back overlapped (l3d_tsdf_integrate_many_read)"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(w, os.cpu_count() or 1)
        cpu.pop("seconds", None)

    def stage(r):
        return {k: sum(v) / len(v) for k, v in r["ms"].items()}

    line = {
        "metric": METRIC, "value": value, "unit": "px-iters/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": R["st_s"] * 1e3 / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": f"{args.storage} images, f32 arithmetic" if chosen_form == FORM_FAST else "f32",
        "data": ("synthetic (seeded room scene with cuboids, value-noise texture)" if w.name == "room"
                 else "synthetic (seeded sphere-on-plane scene, value-noise texture)"),
        "scene": scene_conventions(w),
        "config": {"workload": workload_name(w),
                   "form": "fast" if chosen_form == FORM_FAST else "plain",
                   "variant": tuned.get("variant"),
                   "graphs": chosen_form == FORM_FAST,
                   "l2": "flushed (256 MB write) before every step",
                   "parallelism": f"replica x{world}"},
        "tsdf_voxel_updates_per_s": voxel_updates / R["ts_s"],
        "stage_ms": stage(R),
        "depth_accuracy": acc,
        "plain": ({"px_iters_per_s": res[FORM_PLAIN]["px_iters_per_s"],
                   "stage_ms": stage(res[FORM_PLAIN]),
                   "propagate_launch_ms": res[FORM_PLAIN]["prop_ms"]}
                  if FORM_PLAIN in res else None),
        "speedup_vs_plain": (value / res[FORM_PLAIN]["px_iters_per_s"]
                             if FORM_PLAIN in res and chosen_form != FORM_PLAIN else None),
        "roofline": roof_tex or roof_fp32,
        "roofline_fp32": roof_fp32,
        "roofline_tsdf": {"kernel": f"k_integrate_many ({V} views per sweep)", "bound": "hbm",
                          "achieved": tsdf_gbs, "peak": peaks.get("hbm_gbs"), "unit": "GB/s",
                          "frac": tsdf_gbs / peaks.get("hbm_gbs", 6650.0),
                          "peak_source": peak_kind, "bytes_per_launch": tsdf_bytes,
                          # the one-view-per-pass form streams 12 B per voxel-update; the sweep's
                          # time against that form's bytes is its HBM-equivalent rate
                          "per_view_form_bytes": vox * V * 12,
                          "per_view_form_equivalent_frac":
                              vox * V * 12 / (tsdf_ms / 1e3) / 1e9 / peaks.get("hbm_gbs", 6650.0)},
        "clocks": clk,
        "gpu_launches": R["launches"],
        "e2e": e2e,
        "cpu_baseline": cpu,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    stereo.destroy()
    tsdf.destroy()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
