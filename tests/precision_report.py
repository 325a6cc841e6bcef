"""Precision report: every output of the small workload (8 views of 320x240, 4 sources, 3
iterations, TSDF 128^3 at 1 cm) solved by each form and storage type, against the FP64 oracle.

Test infrastructure (it runs the oracle as the checker).  `python tests/precision_report.py`
prints the report as one JSON line; tests/test_precision_gpu.py checks its bounds.
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


def report() -> dict:
    """Precision configuration: the small workload (8 views of 320x240, 4 sources, 3 iterations,
    TSDF 128^3 at 1 cm) solved by every form and storage type, each output against the FP64
    oracle run on the host.

    - solve: depth relative difference and normal angle to the FP64 oracle's own solve (pixels
      both keep with cost < 0.5; PatchMatch is chaotic, so these differences mix arithmetic and
      diverging random searches), and depth error against the rendered ground truth;
    - cost: the cost of the same planes (the FP64 oracle's solution), which isolates arithmetic
      and storage rounding from the search;
    - TSDF: the FP64 oracle's packed maps integrated by the GPU (f32 and Q8.8 weights) against
      the FP64 integrate oracle."""
    import oracle
    from luvas3d import (DTYPE_BF16, DTYPE_F16, DTYPE_F32, DTYPE_U8, FORM_FAST, FORM_PLAIN,
                         DenseStereo, IntegrationView, SolveOptions, StereoOptions, TsdfVolume,
                         scenes)

    w = scenes.small()
    V, W, H = len(w.views), w.width, w.height
    refs = list(range(V))
    opts = [SolveOptions(w.sources[r], w.ranges[r][0], w.ranges[r][1], iterations=w.iterations)
            for r in refs]
    t0 = time.perf_counter()
    o64 = oracle.Stereo(W, H, w.views, w.images, 64)
    hyp64, cost64 = [], []
    for r in refs:
        o64.solve(r, w.sources[r], min_depth=w.ranges[r][0], max_depth=w.ranges[r][1],
                  iterations=w.iterations)
        hyp64.append(o64.hyp.copy())
        cost64.append(o64.cost.copy())
    depths64 = o64.depths.copy()
    oracle_s = time.perf_counter() - t0
    plane_cost64 = []
    for r in refs:
        c, _ = o64.plane_cost(r, w.sources[r], hyp64[r].astype(np.float32).astype(np.float64),
                              min_depth=w.ranges[r][0], max_depth=w.ranges[r][1])
        plane_cost64.append(c)

    def angle_deg(a, b):
        c = np.clip((a * b).sum(-1) / (np.linalg.norm(a, axis=-1) * np.linalg.norm(b, axis=-1)),
                    -1.0, 1.0)
        return np.degrees(np.arccos(c))

    forms = [("plain f32", FORM_PLAIN, DTYPE_F32), ("fast f32", FORM_FAST, DTYPE_F32),
             ("fast f16", FORM_FAST, DTYPE_F16), ("fast bf16", FORM_FAST, DTYPE_BF16),
             ("fast u8", FORM_FAST, DTYPE_U8)]
    report = {}
    for name, form, storage in forms:
        st = DenseStereo(W, H, w.views, StereoOptions(storage=storage, form=form))
        for i, im in enumerate(w.images):
            st.set_image(i, im)
        if form == FORM_FAST:
            st.solve_all(refs, opts)
        dr, na, gt, ce = [], [], [], []
        for r in refs:
            if form == FORM_FAST:
                hyp, cost = st.read_hypotheses_layer(r)
            else:
                st.solve(r, opts[r])
                hyp, cost = st.read_hypotheses()
            both = (cost < 0.5) & (cost64[r] < 0.5)
            d64 = hyp64[r][..., 3]
            dr.append((np.abs(hyp[..., 3] - d64) / d64)[both])
            na.append(angle_deg(hyp[..., :3], hyp64[r][..., :3])[both])
            truth = w.truth[r]
            m = (truth > 0) & (cost < 0.5)
            gt.append(np.abs(hyp[..., 3][m] - truth[m]) / truth[m])
            pc = st.plane_cost(r, opts[r], hyp64[r].astype(np.float32))
            ok = plane_cost64[r] < 2.0
            ce.append(np.abs(pc - plane_cost64[r])[ok])
        dr, na, gt, ce = (np.concatenate(x) for x in (dr, na, gt, ce))
        report[name] = {
            "depth_rel_vs_fp64_solve": _stats(dr, 1e-3),
            "normal_deg_vs_fp64_solve": _stats(na, 1.0),
            "depth_rel_vs_truth": _stats(gt, 0.01),
            "plane_cost_abs_vs_fp64": _stats(ce, 1e-4, 1e-3),
        }
        st.destroy()

    # TSDF of the FP64 oracle's packed maps
    k0 = w.views[0].intrinsics
    t64 = oracle.Tsdf(W, H, w.tsdf_voxel, w.tsdf_origin, w.tsdf_truncation, dense=w.tsdf_dims,
                      precision=64)
    for r, v in enumerate(w.views):
        k = v.intrinsics
        t64.integrate(dict(k=(k.fx, k.fy, k.cx, k.cy), R=v.pose.R, t=v.pose.t,
                           max_depth=w.ranges[r][1]), depths64[r])
    tsdf_report = {}
    for q8 in (False, True):
        vol = TsdfVolume(W, H, w.tsdf_voxel, w.tsdf_origin, dense=w.tsdf_dims,
                         truncation=w.tsdf_truncation, weight_q8=q8)
        for r, v in enumerate(w.views):
            vol.integrate(IntegrationView(v.intrinsics, v.pose, w.ranges[r][1]), depth=depths64[r])
        tt, ww = vol.read()
        seen = t64.weight > 0
        wt = ww.reshape(-1).astype(np.float64) / (256.0 if q8 else 1.0)
        tsdf_report["q8.8 weights (FP64 reference has f32 weights)" if q8 else "f32 weights"] = {
            "tsdf_abs_vs_fp64": _stats(np.abs(tt.reshape(-1)[seen] - t64.tsdf[seen]), 1e-5, 1e-3),
            "weight_rel_vs_fp64": _stats(np.abs(wt[seen] - t64.weight[seen]) / t64.weight[seen],
                                         1e-6, 1e-2),
            "voxels_updated_differently": int(np.sum((wt > 0) != seen)),
        }
        vol.destroy()
    line = {
        "metric": "error of each output against the FP64 oracle", "n_gpus": 1,
        "config": {"workload": (f"small: {V} views {W}x{H}, 4 sources, {w.iterations} iterations, "
                                f"TSDF {w.tsdf_dims[0]}^3 at {w.tsdf_voxel * 1000:.0f} mm"),
                   "oracle_seconds": oracle_s},
        "data": "synthetic (seeded sphere-on-plane scene, value-noise texture)",
        "forms": report, "tsdf": tsdf_report,
    }
    return line


if __name__ == "__main__":
    print(json.dumps(report()), flush=True)
