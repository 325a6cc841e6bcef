"""Precision report: every output of a workload solved by each form, storage type and summation
mode, against the FP64 oracle.

Test infrastructure (it runs the oracle as the checker).  `python tests/precision_report.py
[small|scan4]` prints the report as one JSON line; tests/test_precision_gpu.py checks its bounds.

Workloads:
  small  the precision configuration: 8 views of 320x240, 4 sources, 3 iterations, every view
         solved, TSDF 128^3 at 1 cm;
  scan4  a subset of the scan-scale configuration the FP64 oracle finishes in seconds: the scan's
         48 views of 640x480 (pixel noise 0.01, pose noise 2 mm / 0.1 deg), reference views 12,
         22, 32 and 42 solved against their 8 sources with 5 iterations.
"""
from __future__ import annotations

import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
for p in (ROOT, os.path.join(ROOT, "luvas.io-3d_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

SCAN4_REFS = [12, 22, 32, 42]


def _forms():
    """(name, form, storage, compensated, variant or None for the form's default)."""
    from luvas3d import DTYPE_BF16, DTYPE_F16, DTYPE_F32, DTYPE_U8, FORM_EXACT, FORM_FAST, FORM_PLAIN
    return [
        ("plain f32", FORM_PLAIN, DTYPE_F32, False, None),
        ("exact f32", FORM_EXACT, DTYPE_F32, False, 14),
        ("exact f32 comp", FORM_EXACT, DTYPE_F32, True, 14),
        ("fast f32", FORM_FAST, DTYPE_F32, False, 14),
        ("fast f32 comp", FORM_FAST, DTYPE_F32, True, 14),
        ("fast f32 gather", FORM_FAST, DTYPE_F32, False, 30),
        ("fast f32 gather comp", FORM_FAST, DTYPE_F32, True, 30),
        ("fast f32 gather shared", FORM_FAST, DTYPE_F32, False, 62),
        ("fast f16", FORM_FAST, DTYPE_F16, False, 14),
        ("fast f16 comp", FORM_FAST, DTYPE_F16, True, 14),
        ("fast f16 gather", FORM_FAST, DTYPE_F16, False, 30),
        ("fast bf16", FORM_FAST, DTYPE_BF16, False, None),
        ("fast bf16 comp", FORM_FAST, DTYPE_BF16, True, None),
        ("fast u8", FORM_FAST, DTYPE_U8, False, 14),
    ]


def _stats(x, *within) -> dict:
    """n, median, p99, p99.9 and max of x, and the fraction of x at or below each bound."""
    x = np.asarray(x, dtype=np.float64).reshape(-1)
    if x.size == 0:
        return {"n": 0}
    out = {"n": int(x.size), "median": float(np.median(x)), "p99": float(np.percentile(x, 99)),
           "p99.9": float(np.percentile(x, 99.9)), "max": float(x.max())}
    for b in within:
        out[f"within_{b:g}"] = float(np.mean(x <= b))
    return out


def _angle_deg(a, b):
    c = np.clip((a * b).sum(-1) / (np.linalg.norm(a, axis=-1) * np.linalg.norm(b, axis=-1)),
                -1.0, 1.0)
    return np.degrees(np.arccos(c))


def _workload(name):
    from luvas3d import scenes
    if name == "small":
        w = scenes.small()
        return w, list(range(len(w.views)))
    if name == "scan4":
        return scenes.scan(tsdf_dim=64), list(SCAN4_REFS)
    raise ValueError(f"unknown workload {name}")


def report(workload: str = "small", forms=None) -> dict:
    """Each form's solve and plane costs against the FP64 oracle (and, on the small workload,
    the TSDF of the FP64 oracle's packed maps):

    - solve: depth relative difference and normal angle to the FP64 oracle's own solve (pixels
      both keep with cost < 0.5; PatchMatch is chaotic, so these differences mix arithmetic and
      diverging random searches), and depth error against the rendered ground truth;
    - cost: the cost of the same planes (the FP64 oracle's solution), which isolates arithmetic
      and storage rounding from the search."""
    import oracle
    from luvas3d import (FORM_PLAIN, DenseStereo, IntegrationView, SolveOptions, StereoOptions,
                         TsdfVolume)

    w, refs = _workload(workload)
    W, H = w.width, w.height
    opts = {r: SolveOptions(w.sources[r], w.ranges[r][0], w.ranges[r][1], iterations=w.iterations)
            for r in refs}
    t0 = time.perf_counter()
    o64 = oracle.Stereo(W, H, w.views, w.images, 64)
    hyp64, cost64 = {}, {}
    for r in refs:
        o64.solve(r, w.sources[r], min_depth=w.ranges[r][0], max_depth=w.ranges[r][1],
                  iterations=w.iterations)
        hyp64[r] = o64.hyp.copy()
        cost64[r] = o64.cost.copy()
    depths64 = o64.depths.copy()
    oracle_s = time.perf_counter() - t0
    plane_cost64 = {}
    for r in refs:
        c, _ = o64.plane_cost(r, w.sources[r], hyp64[r].astype(np.float32).astype(np.float64),
                              min_depth=w.ranges[r][0], max_depth=w.ranges[r][1])
        plane_cost64[r] = c

    out = {}
    for name, form, storage, comp, variant in (forms or _forms()):
        st = DenseStereo(W, H, w.views, StereoOptions(storage=storage, form=form, compensated=comp))
        for i, im in enumerate(w.images):
            st.set_image(i, im)
        if form != FORM_PLAIN:
            if variant is not None:
                st.variant = variant
            st.solve_all(refs, [opts[r] for r in refs])
        dr, na, gt, ce = [], [], [], []
        for r in refs:
            if form != FORM_PLAIN:
                hyp, cost = st.read_hypotheses_layer(r)
            else:
                st.solve(r, opts[r])
                hyp, cost = st.read_hypotheses()
            both = (cost < 0.5) & (cost64[r] < 0.5)
            d64 = hyp64[r][..., 3]
            dr.append((np.abs(hyp[..., 3] - d64) / d64)[both])
            na.append(_angle_deg(hyp[..., :3], hyp64[r][..., :3])[both])
            truth = w.truth[r]
            m = (truth > 0) & (cost < 0.5)
            gt.append(np.abs(hyp[..., 3][m] - truth[m]) / truth[m])
            pc = st.plane_cost(r, opts[r], hyp64[r].astype(np.float32))
            ok = plane_cost64[r] < 2.0
            ce.append(np.abs(pc - plane_cost64[r])[ok])
        dr, na, gt, ce = (np.concatenate(x) for x in (dr, na, gt, ce))
        out[name] = {
            "compensated": comp, "variant": st.variant if form != FORM_PLAIN else None,
            "depth_rel_vs_fp64_solve": _stats(dr, 1e-3),
            "normal_deg_vs_fp64_solve": _stats(na, 1.0),
            "depth_rel_vs_truth": _stats(gt, 0.01),
            "plane_cost_abs_vs_fp64": _stats(ce, 1e-4, 1e-3),
        }
        st.destroy()

    tsdf_report = None
    if workload == "small":
        tsdf_report = {}
        t64 = oracle.Tsdf(W, H, w.tsdf_voxel, w.tsdf_origin, w.tsdf_truncation, dense=w.tsdf_dims,
                          precision=64)
        for r, v in enumerate(w.views):
            k = v.intrinsics
            t64.integrate(dict(k=(k.fx, k.fy, k.cx, k.cy), R=v.pose.R, t=v.pose.t,
                               max_depth=w.ranges[r][1]), depths64[r])
        for q8 in (False, True):
            vol = TsdfVolume(W, H, w.tsdf_voxel, w.tsdf_origin, dense=w.tsdf_dims,
                             truncation=w.tsdf_truncation, weight_q8=q8)
            for r, v in enumerate(w.views):
                vol.integrate(IntegrationView(v.intrinsics, v.pose, w.ranges[r][1]), depth=depths64[r])
            tt, ww = vol.read()
            seen = t64.weight > 0
            wt = ww.reshape(-1).astype(np.float64) / (256.0 if q8 else 1.0)
            key = "q8.8 weights (FP64 reference has f32 weights)" if q8 else "f32 weights"
            tsdf_report[key] = {
                "tsdf_abs_vs_fp64": _stats(np.abs(tt.reshape(-1)[seen] - t64.tsdf[seen]), 1e-5, 1e-3),
                "weight_rel_vs_fp64": _stats(np.abs(wt[seen] - t64.weight[seen]) / t64.weight[seen],
                                             1e-6, 1e-2),
                "voxels_updated_differently": int(np.sum((wt > 0) != seen)),
            }
            vol.destroy()
    S = len(w.sources[refs[0]])
    desc = {"small": f"small: {len(w.views)} views {W}x{H}, {S} sources, {w.iterations} iterations, "
                     f"TSDF {w.tsdf_dims[0]}^3 at {w.tsdf_voxel * 1000:.0f} mm",
            "scan4": f"scan subset: reference views {refs} of the scan's {len(w.views)} views "
                     f"{W}x{H}, {S} sources, {w.iterations} iterations"}[workload]
    return {
        "metric": "error of each output against the FP64 oracle", "n_gpus": 1,
        "config": {"workload": desc, "oracle_seconds": oracle_s},
        "data": "synthetic (seeded sphere-on-plane scene, value-noise texture)",
        "forms": out, "tsdf": tsdf_report,
    }


if __name__ == "__main__":
    print(json.dumps(report(sys.argv[1] if len(sys.argv) > 1 else "small")), flush=True)
