"""Precision configuration: each form, storage type and summation mode against the FP64 oracle,
on the small workload and on a subset of the scan-scale workload (tests/precision_report.py
prints the full tables of these figures).

Bounds (depth within 1e-3 relative of the FP64 oracle's own solve, on the pixels both keep; plane
cost of the FP64 oracle's planes at p99):
  - the plain FP32 form (the FP32 oracle's arithmetic) and the exact batched form, which equals it
    bit for bit;
  - the forms that meet the 99.5 % / 1e-4 targets on both workloads: the exact form with
    compensated sums and the fast form with FP32 texels read as texture gathers with exact
    bilinear weights (with and without compensation);
  - the fast form's storage types, which degrade in order FP32 texture (8-bit filter weights),
    FP16, BF16 / U8 (8-bit mantissa or 8-bit values), each with a stated floor.
TSDF values of the same packed maps agree within 1e-5 except for the rare voxels whose pixel
rounds to a different texel in FP32 and FP64.
"""
import pytest

from precision_report import report

pytestmark = pytest.mark.gpu

# form: workload -> (depth within 1e-3 of the FP64 solve, plane-cost p99 bound)
FLOORS = {
    "plain f32": {"small": (0.995, 2e-4), "scan4": (0.99, 2e-4)},
    "exact f32 comp": {"small": (0.998, 1e-4), "scan4": (0.995, 1e-4)},
    "fast f32 gather": {"small": (0.998, 1e-4), "scan4": (0.995, 1e-4)},
    "fast f32 gather comp": {"small": (0.998, 1e-4), "scan4": (0.995, 1e-4)},
    "fast f32 gather shared": {"small": (0.998, 1e-4), "scan4": (0.995, 1e-4)},
    "fast f32": {"small": (0.98, 5e-4), "scan4": (0.97, 5e-4)},
    "fast f16": {"small": (0.94, 3e-3), "scan4": (0.92, 3e-3)},
    "fast f16 comp": {"small": (0.94, 3e-3), "scan4": (0.92, 3e-3)},
    "fast bf16": {"small": (0.70, 2e-2), "scan4": (0.75, 2e-2)},
    "fast u8": {"small": (0.70, 2e-2), "scan4": (0.75, 2e-2)},
}


@pytest.fixture(scope="module", params=["small", "scan4"])
def rep(request):
    return request.param, report(request.param)


@pytest.mark.parametrize("form", list(FLOORS))
def test_form_against_fp64_oracle(rep, form):
    workload, r = rep
    r = r["forms"][form]
    depth_floor, cost_p99 = FLOORS[form][workload]
    assert r["depth_rel_vs_fp64_solve"]["within_0.001"] >= depth_floor, r["depth_rel_vs_fp64_solve"]
    assert r["plane_cost_abs_vs_fp64"]["p99"] <= cost_p99, r["plane_cost_abs_vs_fp64"]


def test_shared_window_equals_register_window(rep):
    """+32 moves the window to shared memory without changing any arithmetic."""
    workload, r = rep
    a, b = dict(r["forms"]["fast f32 gather shared"]), dict(r["forms"]["fast f32 gather"])
    a.pop("variant"), b.pop("variant")
    assert a == b


def test_exact_form_equals_plain_form(rep):
    """Bit-exact twins: every statistic of the exact batched form equals the plain form's."""
    workload, r = rep
    a, b = dict(r["forms"]["exact f32"]), dict(r["forms"]["plain f32"])
    for k in ("compensated", "variant"):
        a.pop(k), b.pop(k)
    assert a == b


def test_storage_types_degrade_in_order(rep):
    workload, r = rep
    p99 = {k: v["plane_cost_abs_vs_fp64"]["p99"] for k, v in r["forms"].items()}
    assert p99["fast f32 gather"] <= p99["plain f32"] <= p99["fast f16"] <= p99["fast bf16"]
    assert p99["fast f32"] <= p99["fast f16"]
    # the compensated sums do not lose accuracy anywhere
    assert p99["exact f32 comp"] <= p99["exact f32"]


def test_tsdf_against_fp64_oracle(rep):
    workload, r = rep
    if r["tsdf"] is None:
        pytest.skip("TSDF is reported on the small workload")
    t = r["tsdf"]["f32 weights"]
    assert t["tsdf_abs_vs_fp64"]["within_1e-05"] >= 0.999, t
    assert t["voxels_updated_differently"] <= 1e-3 * t["tsdf_abs_vs_fp64"]["n"], t
