"""Benchmark of the dense-reconstruction path: PatchMatch px-iters/s and TSDF voxel-updates/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--form auto|plain|fast|exact] [--workload scan|room|polish|fusion]

Workload (the scan-scale configuration): 48 synthetic views of 640x480 (sphere-on-plane scene,
3-octave value noise, helical camera path, 2 mm / 0.1 deg pose noise, pixel noise 0.01), 8
sources, 5 red/black iterations, 11x11 window dilated by 2 (6 x 6 samples); consistency filter of
every view; TSDF 512^3 at 4 mm, truncation 2 cm, f32 tsdf + uint16 Q8.8 weights.

One step = the photometric PatchMatch stage over all 48 views + the consistency filter of all
views + TSDF integration of all 48 filtered maps.  `value` is the PatchMatch px-iters/s of the
step (px-iter = one pixel updated in one red/black iteration: 48 * 307200 * 5 per step) timed on
the PatchMatch stage, in the fast form (FP16 texels) unless --form says otherwise; the plain FP32
form runs beside it, and the forms at the plain form's FP64 accuracy (the fast form with FP32
texels read through gathers with exact weights, and the exact form) are timed on the PatchMatch
stage.  The TSDF stage gives voxel-updates/s (134M voxels * 48 views per step); the reference's
one-view-per-launch form is timed on the same maps.  Inputs are resident in HBM for `value`;
`e2e` repeats the step through the C ABI with the images copied from pinned host memory every
step and the filtered maps and the TSDF volume read back.  L2 is flushed (a 256 MB write) before
every timed step.  The default run also times the batching configuration (room: 96 views of
mixed sizes, TSDF 768^3) and the differentiation configuration (polish: the NCC adjoint over 24
views of 640x480), and the CPU sample of the reference algorithm.

Multi-GPU (--gpus N, or N ranks under torch.distributed.run): one scan split over the GPUs, views
dealt by pixel count, one NCCL all-gather of the packed depth maps and one of the filtered maps
per step (each rank filters its own views), TSDF z-slabs per GPU ("scaling": "strong": the scan
is the same at every N).
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


class CpuSample:
    """The bounded CPU sample of the workload: the FP32 oracle (the reference algorithm restated
    in C++) on the host cores, for one reference view (the middle one) at full resolution with
    its sources.  One sample runs init + iteration 0 (both red/black colours) from scratch and
    iteration 4 (both colours) from the planes of four iterations, so the rate covers the
    random planes of the first iteration and the converged planes of the last: 2 x W x H
    px-iters per sample.  The TSDF sample integrates that view's packed map into the full
    volume."""

    def __init__(self, w, threads: int):
        import oracle

        self.w, self.threads = w, threads
        self.ref = len(w.views) // 2
        r = self.ref
        self.kw = dict(min_depth=w.ranges[r][0], max_depth=w.ranges[r][1])
        self.o = oracle.Stereo(w.width, w.height, w.views, w.images, 32, threads=threads)
        self.o.solve(r, w.sources[r], iterations=4, **self.kw)
        self.hyp4, self.cost4 = self.o.hyp.copy(), self.o.cost.copy()
        self.px = w.images[r].size

    def stereo(self) -> float:
        """Seconds of one sample (2 x W x H px-iters)."""
        import oracle

        o, r, src = self.o, self.ref, self.w.sources[self.ref]
        t0 = time.perf_counter()
        o.kernel(oracle.INIT, r, src, **self.kw)
        for phase in (0, 1):
            o.kernel(oracle.PROPAGATE, r, src, iteration=0, phase=phase, **self.kw)
        o.hyp, o.cost = self.hyp4, self.cost4
        for phase in (0, 1):
            o.kernel(oracle.PROPAGATE, r, src, iteration=4, phase=phase, **self.kw)
        return time.perf_counter() - t0

    def tsdf(self) -> float:
        """Seconds of one view integrated into the full volume."""
        import oracle

        w, r = self.w, self.ref
        self.o.kernel(oracle.PACK, r, w.sources[r], **self.kw)
        v = w.views[r]
        k = v.intrinsics
        h0, w0 = w.images[r].shape
        ot = oracle.Tsdf(w0, h0, w.tsdf_voxel, w.tsdf_origin, w.tsdf_truncation,
                         dense=w.tsdf_dims, weight_q8=True, threads=self.threads)
        t0 = time.perf_counter()
        ot.integrate(dict(k=(k.fx, k.fy, k.cx, k.cy), R=v.pose.R, t=v.pose.t,
                          max_depth=w.ranges[r][1]), self.o.depths[r])
        return time.perf_counter() - t0

    def describe(self, stereo_s: float, tsdf_s: float) -> str:
        h0, w0 = self.w.images[self.ref].shape
        return (f"FP32 oracle, reference view {self.ref} at {w0}x{h0} with "
                f"{len(self.w.sources[self.ref])} sources: init + iteration 0 from scratch and "
                f"iteration 4 from four iterations' planes, both colours each ({stereo_s:.2f} s); "
                f"TSDF 1 view into {self.w.tsdf_dims[0]}^3 ({tsdf_s:.2f} s)")


def cpu_baseline(w, threads: int) -> dict:
    """One CPU sample (CpuSample) on `threads` host threads, and the stereo sample's iteration 0
    on one thread."""
    import oracle

    smp = CpuSample(w, threads)
    t_pm = smp.stereo()
    t_ts = smp.tsdf()
    one = oracle.Stereo(w.width, w.height, w.views, w.images, 32, threads=1)
    r = smp.ref
    one.kernel(oracle.INIT, r, w.sources[r], **smp.kw)
    t0 = time.perf_counter()
    one.kernel(oracle.PROPAGATE, r, w.sources[r], iteration=0, phase=0, **smp.kw)
    t_one = time.perf_counter() - t0
    vox = int(np.prod(w.tsdf_dims))
    return {"value": 2 * smp.px / t_pm, "unit": "px-iters/s", "cores": threads, "kind": "port",
            "single_thread_px_iters_per_s": (smp.px / 2) / t_one,
            "sample": smp.describe(t_pm, t_ts), "tsdf_voxel_updates_per_s": vox / t_ts}


def run_reference(args, rank: int, world: int) -> None:
    """--impl reference: the CPU restatement of the path on the host cores (the reference has no
    CPU implementation of these stages; its WGSL needs WebGPU, unavailable on this box).  Each
    timed step is one bounded sample (CpuSample); ms_per_step is its measured duration."""
    if rank != 0:
        return
    w = build_workload(args)
    threads = os.cpu_count() or 1
    smp = CpuSample(w, threads)
    secs, tsecs = [], []
    for i in range(args.warmup + args.steps):
        t_pm = smp.stereo()
        t_ts = smp.tsdf() if i in (0, args.warmup) else None
        if i >= args.warmup:
            secs.append(t_pm)
            if t_ts is not None:
                tsecs.append(t_ts)
    sec = statistics.median(secs)
    v = 2 * smp.px / sec
    vox = int(np.prod(w.tsdf_dims))
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "px-iters/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": sec * 1e3,
        "ms_per_step_basis": "measured: one bounded sample per timed step (median)",
        "full_step_ms_extrapolated": 1e3 * w.pixels * w.iterations / v,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": {"workload": workload_name(w), "sample": smp.describe(sec, tsecs[0])},
        "scene": scene_conventions(w),
        "tsdf_voxel_updates_per_s": vox / tsecs[0],
        "cpu_baseline": {"value": v, "unit": "px-iters/s", "cores": threads, "kind": "port",
                         "sample": smp.describe(sec, tsecs[0])},
        "e2e": {"value": v, "unit": "px-iters/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_polish(args) -> None:
    print(json.dumps(polish_measure(args.views or 24, args.steps, args.warmup)), flush=True)


def polish_measure(n_views: int, steps: int, warmup: int, geometry: bool = True) -> dict:
    """Differentiation configuration: 24 views of 640x480 of the sphere scene with poses perturbed
    by 5 mm / 0.3 deg.  PatchMatch (fast form) on the perturbed poses gives the starting planes;
    then 20 Adam steps polish every view's planes and pose increment against the summed NCC
    cost (4 sources per view, view 0 fixed).  Reports the gradient pass throughput
    (pixel-sources/s, one cost + plane + pose gradient evaluation each) and the relative pose
    errors before and after."""
    import torch

    from luvas3d import DTYPE_F16, FORM_FAST, DenseStereo, SolveOptions, StereoOptions, scenes
    from luvas3d import grad as G

    w = scenes.polish(n_views=n_views)
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

    for _ in range(max(3, warmup)):
        grad_pass()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    times = []
    for _ in range(max(1, steps)):
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
    from_geometry = None
    if geometry:
        true_planes, true_weights = starting_planes(w.true_views)
        from_geometry = run(true_planes, true_weights)
    line = {
        "metric": "NCC adjoint pixel-sources/s (cost + plane + se(3) pose gradient)",
        "value": units / (grad_ms / 1e3), "unit": "pixel-sources/s", "n_gpus": 1,
        "steps": steps, "warmup": warmup, "ms_per_step": grad_ms,
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
    st.destroy()
    return line


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


def _free_port() -> int:
    import socket

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def relaunch(n: int) -> int:
    """`--gpus N` without a launcher: one process per GPU under torch.distributed.run."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr=127.0.0.1", f"--master-port={_free_port()}", os.path.abspath(__file__),
           *sys.argv[1:]]
    return subprocess.run(cmd, timeout=3600).returncode


class Stage:
    """CUDA events on one stream around the stages of a step."""

    def __init__(self, stream, names):
        import torch

        self.stream, self.names = stream, list(names)
        self.ev = [torch.cuda.Event(enable_timing=True) for _ in range(len(names) + 1)]
        self.i = 0

    def mark(self):
        import torch

        with torch.cuda.stream(self.stream):
            self.ev[self.i].record(self.stream)
        self.i += 1

    def ms(self) -> dict:
        out = {n: self.ev[k].elapsed_time(self.ev[k + 1]) for k, n in enumerate(self.names)}
        out["step"] = self.ev[0].elapsed_time(self.ev[-1])
        return out


def make_stereo(w, form, storage, stream, refs, opts, variant=None, gather=False, compensated=False):
    """A stereo handle with every view's image; for the batched forms the kernel variant is
    `variant`, or the autotuner's pick over `refs` (with `gather`, among the variants that read
    the texture through gathers with exact weights), and batched solves replay CUDA graphs."""
    from luvas3d import FORM_PLAIN, DenseStereo, StereoOptions

    st = DenseStereo(w.width, w.height, w.views,
                     StereoOptions(storage=storage, form=form, stream=stream, compensated=compensated),
                     sizes=w.sizes or [(w.width, w.height)] * len(w.views))
    for i, im in enumerate(w.images):
        st.set_image(i, im)
    tuned = {"variant": None, "ms": None}
    if form != FORM_PLAIN:
        if variant is not None:
            st.variant = variant
            tuned["variant"] = variant
        else:
            if gather:
                st.variant = 30
            tuned["variant"], tuned["ms"] = st.autotune(refs, opts)
        st.set_graphs(True)
    return st, tuned


def depth_accuracy(st, w, refs) -> dict:
    """Packed depth maps of the last solve against the rendered ground truth, scored like the
    reference's stereo self-test (frontend/tools/verify/stereo-check.ts:56-73): surface pixels
    (truth > 0) with a non-zero packed entry count as valid; relative error of the packed half
    depth, median and p90, over the given views."""
    from luvas3d.packing import unpack_depth

    def score(views):
        errs, surf, valid = [np.zeros(0)], 0, 0
        for r in views:
            packed = st.depth_map(r)
            t = w.truth[r]
            m = t > 0
            ok = m & (packed != 0)
            surf += int(m.sum())
            valid += int(ok.sum())
            errs.append(np.abs(unpack_depth(packed[ok]) - t[ok]) / t[ok])
        e = np.concatenate(errs)
        if e.size == 0:
            return {"views": len(views), "valid_fraction": 0.0}
        return {"views": len(views), "valid_fraction": round(valid / max(1, surf), 4),
                "median_rel_err": float(np.percentile(e, 50)),
                "p90_rel_err": float(np.percentile(e, 90))}

    out = score(refs)
    out.pop("views")
    if getattr(w, "name", "") == "scan":
        # the scan's helix starts 0.2 m from the unit sphere: the views whose camera is within
        # 1.4 m of its centre see the texture too magnified for the window (every form alike)
        dist = {r: float(np.linalg.norm(-np.asarray(w.views[r].pose.R).T @ np.asarray(w.views[r].pose.t)))
                for r in refs}
        out["by_camera_distance_from_the_sphere_centre"] = {
            "under_1.4m": score([r for r in refs if dist[r] < 1.4]),
            "from_1.4m": score([r for r in refs if dist[r] >= 1.4])}
    return out


def time_solves(st, refs, opts, stream, flush, steps: int, warmup: int) -> list:
    """PatchMatch stage alone (solve_all of refs), L2 flushed before each, CUDA events."""
    import torch

    out = []
    for i in range(warmup + steps):
        with torch.cuda.stream(stream):
            flush.fill_(1)
        g = Stage(stream, ["patchmatch"])
        g.mark()
        st.solve_all(refs, opts)
        g.mark()
        torch.cuda.synchronize()
        if i >= warmup:
            out.append(g.ms()["patchmatch"])
    return out


def propagate_launch_ms(st, w, refs, stream, per_view_launches: bool) -> float:
    """One propagate launch: (solve with all iterations - solve with none) / propagate launches,
    CUDA events on the handle's stream."""
    import torch

    from luvas3d import SolveOptions

    per = {}
    for its in (0, w.iterations):
        o2 = [SolveOptions(w.sources[r], w.ranges[r][0], w.ranges[r][1], iterations=its)
              for r in refs]
        g = Stage(stream, ["solve"])
        g.mark()
        for _ in range(2):
            st.solve_all(refs, o2)
        g.mark()
        torch.cuda.synchronize()
        per[its] = g.ms()["solve"] / 2
    return (per[w.iterations] - per[0]) / (2 * w.iterations * (len(refs) if per_view_launches else 1))


def fetch_rate(dtype, mode) -> float:
    """Measured bilinear samples/s of the texture unit (l3d_measure_fetch_rate, one colour)."""
    import ctypes as C

    from luvas3d import _lib

    rate = C.c_double()
    _lib.check(_lib.load().l3d_measure_fetch_rate(dtype, 1, mode, C.byref(rate)))
    return rate.value


def run_scan(args) -> None:
    """One GPU: the scan (or room) workload through every form, with the rooflines, the end-to-end
    run through the C ABI, the batching and differentiation configurations and the CPU sample."""
    import torch

    from luvas3d import (DTYPE_BF16, DTYPE_F16, DTYPE_F32, DTYPE_U8, FETCH_FILTERED, FETCH_GATHER,
                         FORM_EXACT, FORM_FAST, FORM_PLAIN, IntegrationView, SolveOptions, TsdfVolume)

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
                      w.tsdf_origin, dense=w.tsdf_dims, truncation=w.tsdf_truncation,
                      weight_q8=True, stream=sptr)
    storage = {"f16": DTYPE_F16, "u8": DTYPE_U8, "f32": DTYPE_F32, "bf16": DTYPE_BF16}[args.storage]
    fixed = args.variant if args.variant >= 0 else None

    def step(st, g):
        with torch.cuda.stream(stream):
            flush.fill_(1)
        g.mark()
        st.solve_all(refs, opts)
        g.mark()
        tsdf.reset()  # a fresh volume per scan (tsdf 1, weight 0), outside the timed TSDF stage
        st.filter_all(refs, w.sources, w.needed)
        g.mark()
        tsdf.integrate_many(iviews, stereo=st, layers=refs)
        g.mark()

    def time_form(form, stor, steps, warmup, sample_clocks, variant):
        st, tuned = make_stereo(w, form, stor, sptr, refs, opts, variant=variant)
        for _ in range(warmup):
            step(st, Stage(stream, ["patchmatch", "filter", "tsdf"]))
        torch.cuda.synchronize()
        l0 = st.launches + tsdf.launches
        clocks = ClockSampler(torch.cuda.current_device()) if sample_clocks else None
        if clocks:
            clocks.start()
        gs = []
        for _ in range(steps):
            g = Stage(stream, ["patchmatch", "filter", "tsdf"])
            step(st, g)
            gs.append(g)
        torch.cuda.synchronize()
        clk = clocks.stop() if clocks else None
        ms = [g.ms() for g in gs]
        stage = {k: sum(m[k] for m in ms) / len(ms) for k in ms[0]}
        r = {"stage_ms": stage, "clk": clk, "launches": st.launches + tsdf.launches - l0,
             "px_iters_per_s": px_iters_step / (stage["patchmatch"] / 1e3), "tuned": tuned,
             "prop_ms": propagate_launch_ms(st, w, refs, stream, form == FORM_PLAIN),
             "accuracy": depth_accuracy(st, w, refs)}
        return st, r

    chosen = {"auto": FORM_FAST, "fast": FORM_FAST, "plain": FORM_PLAIN, "exact": FORM_EXACT}[args.form]
    chosen_storage = DTYPE_F32 if chosen in (FORM_PLAIN, FORM_EXACT) else storage
    res = {}
    if args.form == "auto":
        st, res["plain"] = time_form(FORM_PLAIN, DTYPE_F32, max(1, min(args.steps, 2)),
                                     min(args.warmup, 3), False, None)
        st.destroy()
    stereo, R = time_form(chosen, chosen_storage, args.steps, args.warmup, True, fixed)
    plain = res.get("plain")
    value = R["px_iters_per_s"]
    S = len(w.sources[0])
    pix_colour = w.pixels / V / 2
    views_launch = 1 if chosen == FORM_PLAIN else V

    # ---- rooflines of the propagate kernel ------------------------------------------------
    peaks, peak_kind = _peaks()
    samples = 14 * S * 36 * pix_colour * views_launch
    flop_per_px_phase = 14 * S * (18 + 36 * 37 + 15) + 36 * 26
    prop_flops = flop_per_px_phase * pix_colour * views_launch
    sm_mhz = (R["clk"] or {}).get("sm_mhz") or 1965.0
    fp32_peak = 148 * 128 * 2 * sm_mhz * 1e6 / 1e12
    kname = (f"k_fast_propagate (all {V} views, one colour)" if chosen != FORM_PLAIN
             else "k_propagate (one view, one colour)")
    roof_fp32 = {"kernel": kname, "bound": "fp32", "achieved": prop_flops / (R["prop_ms"] / 1e3) / 1e12,
                 "peak": fp32_peak, "unit": "TFLOP/s", "traffic": None,
                 "peak_source": "nominal FP32 FMA rate (148 SMs x 128 lanes x 2 flops) at the "
                                "sampled median SM clock",
                 "launch_ms": R["prop_ms"], "flop_per_launch": prop_flops,
                 "flop_model": "14 candidates x sources x (18 + 36 x 37 + 15) + 936 per pixel of "
                               "the colour"}
    roof_fp32["frac"] = roof_fp32["achieved"] / fp32_peak
    sample_model = ("14 candidates x sources x 36 bilinear samples per pixel of the colour (the "
                    "reference's count; sources the corner test rejects are counted although not "
                    "sampled)")

    def tex_roof(kernel, launch_ms, dtype, mode, name):
        peak = fetch_rate(dtype, mode) / 1e9
        got = samples / (launch_ms / 1e3) / 1e9
        return {"kernel": kernel, "bound": "texture", "achieved": got, "peak": peak,
                "unit": "Gsample/s", "frac": got / peak, "traffic": None,
                "peak_source": f"measured: l3d_measure_fetch_rate({name}), bilinear samples/s of a "
                               "2048x2048 texture, one red/black colour",
                "launch_ms": launch_ms, "samples_per_launch": samples, "sample_model": sample_model}

    roof_tex = None
    if chosen == FORM_FAST and args.storage != "bf16":
        roof_tex = tex_roof(kname, R["prop_ms"], chosen_storage, FETCH_FILTERED,
                            f"{args.storage}, filtered")
    elif chosen == FORM_EXACT:
        roof_tex = tex_roof(kname, R["prop_ms"], DTYPE_F32, FETCH_GATHER, "f32, gather")

    # ---- the forms at the plain form's FP64 accuracy: PatchMatch stage alone ---------------
    equal = {}
    if args.workload == "scan" and not args.no_extras:
        for name, form, gather in (("fast f32 gather", FORM_FAST, True), ("exact", FORM_EXACT, False)):
            st, tuned = make_stereo(w, form, DTYPE_F32, sptr, refs, opts, gather=gather)
            n_steps = max(2, min(args.steps, 5)) if form == FORM_FAST else 2
            t = time_solves(st, refs, opts, stream, flush, n_steps, 2)
            pms = sum(t) / len(t)
            e = {"form": name, "storage": "f32", "variant": tuned["variant"],
                 "px_iters_per_s": px_iters_step / (pms / 1e3), "patchmatch_ms": pms,
                 "accuracy": depth_accuracy(st, w, refs)}
            if plain:
                e["speedup_vs_plain"] = e["px_iters_per_s"] / plain["px_iters_per_s"]
            lm = propagate_launch_ms(st, w, refs, stream, False)
            e["roofline"] = tex_roof(kname, lm, DTYPE_F32, FETCH_GATHER, "f32, gather")
            equal[name] = e
            st.destroy()

    # ---- TSDF: the sweep of the step, and the reference's one-view-per-launch form ---------
    stereo.solve_all(refs, opts)
    stereo.filter_all(refs, w.sources, w.needed)
    visible, updates, kept = tsdf.count_updates(iviews, stereo=stereo, layers=refs)
    pv = []
    for i in range(4):
        tsdf.reset()
        g = Stage(stream, ["tsdf"])
        g.mark()
        for k, r in enumerate(refs):
            tsdf.integrate_layer(iviews[k], stereo, r)
        g.mark()
        torch.cuda.synchronize()
        if i:
            pv.append(g.ms()["tsdf"])
    per_view_ms = sum(pv) / len(pv)
    sweep_ms = R["stage_ms"]["tsdf"]
    hbm = peaks.get("hbm_gbs", 6650.0)
    roof_tsdf = {"kernel": f"k_integrate_many ({V} views per sweep)", "bound": "hbm",
                 "achieved": vox * 12 / (sweep_ms / 1e3) / 1e9, "peak": hbm, "unit": "GB/s",
                 "peak_source": peak_kind, "bytes_per_launch": vox * 12,
                 "bytes_model": "12 B per voxel per sweep (f32 tsdf and Q8.8 weight, read and written)",
                 "voxel_updates": updates, "visible_voxel_views": visible,
                 "depth_kept_voxel_views": kept, "launch_ms": sweep_ms,
                 # the one-view-per-pass form moves 12 B per voxel-update it applies; the sweep's
                 # time against those bytes is its HBM-equivalent rate
                 "per_view_form_equivalent_frac": updates * 12 / (sweep_ms / 1e3) / 1e9 / hbm}
    roof_tsdf["frac"] = roof_tsdf["achieved"] / hbm
    roof_tsdf_view = {"kernel": f"k_integrate_list ({V} launches, one view each)", "bound": "hbm",
                      "achieved": updates * 12 / (per_view_ms / 1e3) / 1e9, "peak": hbm,
                      "unit": "GB/s", "peak_source": peak_kind, "traffic": None,
                      "bytes_model": "12 B per voxel-update applied (f32 tsdf and Q8.8 weight, "
                                     "read and written), counted by l3d_tsdf_count_updates",
                      "bytes_per_step": updates * 12, "voxel_updates": updates,
                      "visible_voxel_views": visible, "depth_kept_voxel_views": kept,
                      "ms_per_step": per_view_ms,
                      "voxel_updates_per_s": vox * V / (per_view_ms / 1e3),
                      # 12 B per voxel of every brick a launch visits (the bricks visibleBricks
                      # and the depth-aware cull keep): the bytes a form that streams whole kept
                      # bricks would move
                      "kept_brick_bytes_per_step": kept * 12,
                      "kept_brick_frac": kept * 12 / (per_view_ms / 1e3) / 1e9 / hbm}
    roof_tsdf_view["frac"] = roof_tsdf_view["achieved"] / hbm

    # ---- end to end through the C ABI with pinned host buffers ------------------------------
    e2e = None
    if not args.no_e2e:
        pinned = [torch.from_numpy(np.ascontiguousarray(im)).pin_memory() for im in w.images]
        # two scans in flight: two stereo handles and two volumes on two streams, used in turn,
        # so that scan k + 1's image upload and PatchMatch start while scan k's filter, sweep
        # and read-backs finish, and scan k's 805 MB volume read-back overlaps scan k + 1
        stream2 = torch.cuda.Stream()
        sptr2 = stream2.cuda_stream
        stereo2, _ = make_stereo(w, chosen, chosen_storage, sptr2, refs, opts,
                                 variant=R["tuned"]["variant"])
        sts = [stereo, stereo2]
        vols = [tsdf, TsdfVolume(max(s[0] for s in sizes), max(s[1] for s in sizes), w.tsdf_voxel,
                                 w.tsdf_origin, dense=w.tsdf_dims, truncation=w.tsdf_truncation,
                                 weight_q8=True, stream=sptr2)]
        outs = [(torch.empty(vox, dtype=torch.float32).pin_memory(),
                 torch.empty(vox, dtype=torch.int16).pin_memory()) for _ in range(2)]
        out_f = [torch.empty(w.pixels, dtype=torch.int32).pin_memory() for _ in range(2)]

        def e2e_step(k):
            st, vol = sts[k % 2], vols[k % 2]
            for i, im in enumerate(pinned):
                st.set_image_device(i, im.data_ptr(), DTYPE_F32)
            st.solve_all(refs, opts)
            st.filter_all(refs, w.sources, w.needed)
            vol.reset()  # queued after this volume's previous read-back (on the device)
            st.read_filtered_all_async(out_f[k % 2])  # every filtered map, one copy on the stream
            # the sweep, its read-back queued behind it on the volume's copy stream
            # (l3d_tsdf_integrate_many_read_async); the host goes on to the next scan
            vol.integrate_many_read(iviews, stereo=st, layers=refs, out=outs[k % 2], wait=False)

        def drain():
            for v in vols:
                v.wait_read()
            for st in sts:
                st.synchronize()

        for k in range(2):
            e2e_step(k)
        drain()
        torch.cuda.synchronize()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        stream2.wait_event(t0)
        for k in range(args.steps):
            e2e_step(k)
        drain()  # every scan's filtered maps and volume are in host memory
        t1.record(stream)
        torch.cuda.synchronize()
        g = {"e2e": t0.elapsed_time(t1)}
        e2e_s = g["e2e"] / 1e3
        e2e = {"value": px_iters_step * args.steps / e2e_s, "unit": "px-iters/s",
               "h2d_bytes_per_step": w.pixels * 4, "d2h_bytes_per_step": w.pixels * 4 + vox * 6,
               "ms_per_step": e2e_s * 1e3 / args.steps,
               "includes": "every scan: image upload from pinned host memory, PatchMatch, filter, "
                           "read-back of the filtered maps (l3d_stereo_read_filtered_all_async), "
                           "TSDF sweep, and the volume's read-back "
                           "(l3d_tsdf_integrate_many_read_async); two scans in flight (two stereo "
                           "handles, volumes, pinned buffers and streams, used in turn); the timed "
                           "region ends after the last scan's maps and volume are in host memory"}
        vols[1].destroy()
        stereo2.destroy()
    stereo.destroy()
    tsdf.destroy()

    # ---- the batching (room) and differentiation (polish) configurations ------------------
    extras = {}
    if args.workload == "scan" and not args.no_extras:
        from luvas3d import scenes

        wr = scenes.room()
        Vr = len(wr.views)
        refs_r = list(range(Vr))
        opts_r = [SolveOptions(wr.sources[r], wr.ranges[r][0], wr.ranges[r][1],
                               iterations=wr.iterations) for r in refs_r]
        iv_r = [IntegrationView(v.intrinsics, v.pose, wr.ranges[i][1]) for i, v in enumerate(wr.views)]
        st, tuned = make_stereo(wr, FORM_FAST, storage, sptr, refs_r, opts_r)
        vol = TsdfVolume(max(s[0] for s in wr.sizes), max(s[1] for s in wr.sizes), wr.tsdf_voxel,
                         wr.tsdf_origin, dense=wr.tsdf_dims, truncation=wr.tsdf_truncation,
                         weight_q8=True, stream=sptr)
        ms = []
        for i in range(4):
            with torch.cuda.stream(stream):
                flush.fill_(1)
            g = Stage(stream, ["patchmatch", "filter", "tsdf"])
            g.mark()
            st.solve_all(refs_r, opts_r)
            g.mark()
            vol.reset()
            st.filter_all(refs_r, wr.sources, wr.needed)
            g.mark()
            vol.integrate_many(iv_r, stereo=st, layers=refs_r)
            g.mark()
            torch.cuda.synchronize()
            if i >= 2:
                ms.append(g.ms())
        stage = {k: sum(m[k] for m in ms) / len(ms) for k in ms[0]}
        vox_r = int(np.prod(wr.tsdf_dims))
        extras["room"] = {
            "workload": workload_name(wr), "form": "fast", "storage": args.storage,
            "variant": tuned["variant"], "graphs": True, "steps": len(ms), "warmup": 2,
            "px_iters_per_s": wr.pixels * wr.iterations / (stage["patchmatch"] / 1e3),
            "tsdf_voxel_updates_per_s": vox_r * Vr / (stage["tsdf"] / 1e3),
            "stage_ms": stage, "depth_accuracy": depth_accuracy(st, wr, refs_r)}
        st.destroy()
        vol.destroy()
        p = polish_measure(24, 5, 3, geometry=False)
        extras["polish"] = {
            "workload": p["config"]["workload"], "grad_pass_ms": p["ms_per_step"],
            "pixel_sources_per_s": p["value"],
            "polish_ms_per_adam_step": p["polish_from_patchmatch_planes"]["ms_per_step"],
            "polish_from_patchmatch_planes": p["polish_from_patchmatch_planes"]}

    cpu = None if args.no_cpu_baseline else cpu_baseline(w, os.cpu_count() or 1)
    eq = equal.get("fast f32 gather")
    line = {
        "metric": METRIC, "value": value, "unit": "px-iters/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": R["stage_ms"]["step"], "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None,
        "dtype": (f"{args.storage} images, f32 arithmetic" if chosen == FORM_FAST else "f32"),
        "data": ("synthetic (seeded room scene with cuboids, value-noise texture)" if w.name == "room"
                 else "synthetic (seeded sphere-on-plane scene, value-noise texture)"),
        "scene": scene_conventions(w),
        "config": {"workload": workload_name(w),
                   "form": {FORM_FAST: "fast", FORM_PLAIN: "plain", FORM_EXACT: "exact"}[chosen],
                   "variant": R["tuned"]["variant"], "graphs": chosen != FORM_PLAIN,
                   "l2": "flushed (256 MB write) before every step", "parallelism": "1 GPU"},
        "tsdf_voxel_updates_per_s": vox * V / (R["stage_ms"]["tsdf"] / 1e3),
        "stage_ms": R["stage_ms"],
        "depth_accuracy": {"plain": plain["accuracy"] if plain else None, "chosen": R["accuracy"]},
        "plain": ({"px_iters_per_s": plain["px_iters_per_s"], "stage_ms": plain["stage_ms"],
                   "propagate_launch_ms": plain["prop_ms"]} if plain else None),
        "speedup_vs_plain": value / plain["px_iters_per_s"] if plain else None,
        "equal_fp64_accuracy_forms": equal or None,
        "speedup_vs_plain_at_equal_fp64_accuracy": eq.get("speedup_vs_plain") if eq else None,
        "fp64_accuracy_basis": ("depth within 1e-3 relative of the FP64 oracle's solve and plane "
                                "costs within 1e-4 at p99, per form, on the scan subset and the "
                                "small workload: tests/test_precision_gpu.py"),
        "roofline": roof_tex or roof_fp32,
        "roofline_fp32": roof_fp32,
        "roofline_tsdf": roof_tsdf,
        "roofline_tsdf_per_view": roof_tsdf_view,
        "clocks": R["clk"],
        "gpu_launches": R["launches"],
        "e2e": e2e,
        "batching_room": extras.get("room"),
        "differentiation_polish": extras.get("polish"),
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)


def run_split(args, rank: int, world: int, local: int) -> None:
    """N GPUs, one process each: one scan split over the ranks (luvas3d.shard.ScanSplit): each
    rank solves its share of the reference views (dealt by pixel count), one NCCL all-gather
    gives every rank every view's packed depth map, every rank filters every view, and each
    rank integrates every view into its z-slab of the TSDF volume (a brick pool).  The split
    equals the one-GPU scan bit for bit (tests/test_shard.py runs the same driver on gloo ranks);
    the whole-job rate is the scan's px-iters over the slowest rank's time."""
    from datetime import timedelta

    import torch
    import torch.distributed as dist

    from luvas3d import (DTYPE_BF16, DTYPE_F16, DTYPE_F32, DTYPE_U8, FORM_FAST, IntegrationView,
                         SolveOptions, TsdfVolume, shard)

    # communicator set-up lines in the log (ranks, transport) without per-call chatter
    os.environ.setdefault("NCCL_DEBUG", "INFO")
    os.environ.setdefault("NCCL_DEBUG_SUBSYS", "INIT")
    device = torch.device("cuda", local)
    dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=device)
    w = build_workload(args)
    V = len(w.views)
    sizes = w.sizes or [(w.width, w.height)] * V
    stream = torch.cuda.Stream()
    sptr = stream.cuda_stream
    refs = list(range(V))
    opts = [SolveOptions(w.sources[r], w.ranges[r][0], w.ranges[r][1], iterations=w.iterations)
            for r in refs]
    iviews = [IntegrationView(v.intrinsics, v.pose, w.ranges[i][1]) for i, v in enumerate(w.views)]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=device)
    storage = {"f16": DTYPE_F16, "u8": DTYPE_U8, "f32": DTYPE_F32, "bf16": DTYPE_BF16}[args.storage]
    mine = shard.shard_views(sizes, world)[rank]
    st, tuned = make_stereo(w, FORM_FAST, storage, sptr, mine or refs[:1],
                            [opts[v] for v in (mine or refs[:1])],
                            variant=args.variant if args.variant >= 0 else None)
    coords = shard.slab_pool(w.tsdf_dims, rank, world)
    vol = None
    if coords is not None:
        vol = TsdfVolume(max(s[0] for s in sizes), max(s[1] for s in sizes), w.tsdf_voxel,
                         w.tsdf_origin, layout=(coords,), truncation=w.tsdf_truncation,
                         weight_q8=True, stream=sptr)
    split = shard.ScanSplit(shard.DeviceScan(st, vol, opts, w.sources, w.needed, iviews), sizes,
                            rank, world, device=device)
    names = ["patchmatch", "exchange", "filter", "exchange_filtered", "tsdf"]

    def step(g):
        with torch.cuda.stream(stream):
            flush.fill_(1)
        g.mark()
        split.solve()
        g.mark()
        split.exchange()
        g.mark()
        if vol is not None:
            vol.reset()
        split.filter()
        g.mark()
        split.exchange_filtered()
        g.mark()
        split.integrate()
        g.mark()

    for _ in range(args.warmup):
        step(Stage(stream, names))
    torch.cuda.synchronize()
    dist.barrier()
    launches0 = st.launches + (vol.launches if vol else 0)
    clocks = ClockSampler(local) if rank == 0 else None
    if clocks:
        clocks.start()
    gs = []
    for _ in range(args.steps):
        g = Stage(stream, names)
        step(g)
        gs.append(g)
    torch.cuda.synchronize()
    dist.barrier()
    clk = clocks.stop() if clocks else None
    launches = st.launches + (vol.launches if vol else 0) - launches0
    ms = [g.ms() for g in gs]
    stage = {k: sum(m[k] for m in ms) / len(ms) for k in ms[0]}
    tot = torch.tensor([sum(m["patchmatch"] for m in ms), sum(m["tsdf"] for m in ms),
                        sum(m["step"] for m in ms)], dtype=torch.float64, device=device)
    dist.all_reduce(tot, op=dist.ReduceOp.MAX)
    pm_s, ts_s, st_s = (float(x) / 1e3 for x in tot.tolist())
    px_iters_step = w.pixels * w.iterations
    vox = int(np.prod(w.tsdf_dims))

    # end to end: every rank uploads every image from pinned host memory (each holds all the
    # sources), runs the split step and reads back its views' filtered maps and its slab
    e2e = None
    if not args.no_e2e:
        import ctypes as C

        from luvas3d import _lib
        lib = _lib.load()
        pinned = [torch.from_numpy(np.ascontiguousarray(im)).pin_memory() for im in w.images]
        f_off = np.concatenate([[0], np.cumsum([a * b for a, b in sizes])])
        out_f = torch.empty(w.pixels, dtype=torch.int32).pin_memory()
        nvox = 0 if vol is None else vol.voxels
        out_t = torch.empty(max(1, nvox), dtype=torch.float32).pin_memory()
        out_w = torch.empty(max(1, nvox), dtype=torch.int16).pin_memory()

        def e2e_step():
            for i, im in enumerate(pinned):
                st.set_image_device(i, im.data_ptr(), DTYPE_F32)
            split.solve()
            split.exchange()
            if vol is not None:
                vol.reset()
            split.filter()
            split.exchange_filtered()
            for r in mine:
                _lib.check(lib.l3d_stereo_read_filtered_layer(
                    st._h(), r, C.c_void_p(out_f[int(f_off[r]):].data_ptr())))
            if vol is not None:
                vol.integrate_many_read(iviews, stereo=st, layers=refs, out=(out_t, out_w))

        e2e_step()
        torch.cuda.synchronize()
        dist.barrier()
        g = Stage(stream, ["e2e"])
        g.mark()
        for _ in range(args.steps):
            e2e_step()
        g.mark()
        torch.cuda.synchronize()
        e2e_s = shard.max_over_ranks(g.ms()["e2e"] / 1e3, device=device)
        e2e = {"value": px_iters_step * args.steps / e2e_s, "unit": "px-iters/s",
               "h2d_bytes_per_step": world * w.pixels * 4, "d2h_bytes_per_step": w.pixels * 4 + vox * 6,
               "ms_per_step": e2e_s * 1e3 / args.steps,
               "includes": "every rank: every image uploaded from pinned host memory, its views' "
                           "PatchMatch, the all-gather of packed maps, its views' filter, the "
                           "all-gather of filtered maps, the read-back of its views' filtered "
                           "maps, the sweep of its slab with the slab's read-back overlapped"}
    if rank == 0:
        line = {
            "metric": METRIC, "value": px_iters_step * args.steps / pm_s, "unit": "px-iters/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": st_s * 1e3 / args.steps, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": f"{args.storage} images, f32 arithmetic",
            "data": "synthetic (seeded sphere-on-plane scene, value-noise texture)",
            "scene": scene_conventions(w),
            "config": {"workload": workload_name(w), "form": "fast", "variant": tuned["variant"],
                       "graphs": True, "l2": "flushed (256 MB write) before every step",
                       "parallelism": (f"split over {world} GPUs: reference views dealt by pixel "
                                       "count, NCCL all-gathers of the packed depth maps and of "
                                       "the filtered maps per step (each rank filters its own "
                                       "views), TSDF z-slabs of bricks per GPU")},
            "tsdf_voxel_updates_per_s": vox * V * args.steps / ts_s,
            "stage_ms_rank0": stage,
            "views_rank0": len(mine),
            "clocks": clk,
            "gpu_launches": launches,
            "e2e": e2e,
            "cpu_baseline": None,
        }
        print(json.dumps(line), flush=True)
    st.destroy()
    if vol is not None:
        vol.destroy()
    dist.barrier()
    dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--form", default="auto", choices=["auto", "plain", "fast", "exact"])
    ap.add_argument("--workload", default="scan", choices=["scan", "room", "polish", "fusion"])
    ap.add_argument("--views", type=int, default=0)
    ap.add_argument("--width", type=int, default=640)
    ap.add_argument("--height", type=int, default=480)
    ap.add_argument("--tsdf-dim", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the equal-accuracy forms and the room / polish configurations")
    ap.add_argument("--split", action="store_true",
                    help="run the multi-GPU split path even on one GPU (a one-rank communicator)")
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
    if "WORLD_SIZE" not in os.environ and args.gpus > 1:
        sys.exit(relaunch(args.gpus))

    import torch

    torch.cuda.set_device(local)
    if args.workload == "polish":
        if rank == 0:
            run_polish(args)
        return
    if args.workload == "fusion":
        if rank == 0:
            run_fusion(args)
        return
    if world > 1 or args.split:
        if "WORLD_SIZE" not in os.environ:
            os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(_free_port()), RANK="0",
                              WORLD_SIZE="1", LOCAL_RANK="0")
        run_split(args, rank, world, local)
        return
    run_scan(args)


if __name__ == "__main__":
    main()
