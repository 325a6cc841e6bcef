"""Precision configuration: each form and storage type against the FP64 oracle on the small
workload (tests/precision_report.py prints the full table of these figures).

Bounds: the plain FP32 form follows the FP64 oracle's search on >= 99 % of the kept pixels
(depth within 1e-3 relative) and the costs of fixed planes to 5e-4 at p99; the fast form's
storage types degrade in order FP32 texture, FP16, BF16 / U8 (8-bit mantissa or 8-bit values),
each with a stated floor.  TSDF values of the same packed maps agree within 1e-5 except for the
rare voxels whose pixel rounds to a different texel in FP32 and FP64.
"""
import pytest

from precision_report import report

pytestmark = pytest.mark.gpu

FLOORS = {  # form: (depth within 1e-3 of the FP64 solve, plane-cost p99 bound)
    "plain f32": (0.99, 5e-4),
    "fast f32": (0.98, 1e-3),
    "fast f16": (0.93, 5e-3),
    "fast bf16": (0.70, 2e-2),
    "fast u8": (0.70, 2e-2),
}


@pytest.fixture(scope="module")
def rep():
    return report()


@pytest.mark.parametrize("form", list(FLOORS))
def test_form_against_fp64_oracle(rep, form):
    r = rep["forms"][form]
    depth_floor, cost_p99 = FLOORS[form]
    assert r["depth_rel_vs_fp64_solve"]["within_0.001"] >= depth_floor, r["depth_rel_vs_fp64_solve"]
    assert r["plane_cost_abs_vs_fp64"]["p99"] <= cost_p99, r["plane_cost_abs_vs_fp64"]


def test_storage_types_degrade_in_order(rep):
    p99 = {k: v["plane_cost_abs_vs_fp64"]["p99"] for k, v in rep["forms"].items()}
    assert p99["plain f32"] <= p99["fast f16"] <= p99["fast bf16"]
    assert p99["fast f32"] <= p99["fast f16"]


def test_tsdf_against_fp64_oracle(rep):
    r = rep["tsdf"]["f32 weights"]
    assert r["tsdf_abs_vs_fp64"]["within_1e-05"] >= 0.999, r
    assert r["voxels_updated_differently"] <= 1e-3 * r["tsdf_abs_vs_fp64"]["n"], r
