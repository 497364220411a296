"""The FP32 precision form against the FP64 path (the FP64 path itself is
pinned to the CPU oracle by test_gpu_parity.py).

Targets: max depth error <= 1e-3 m, relative volume error <= 1e-6, and the
FP64 volume accounts closing the FP32 run's mass balance to <= 1e-6."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_fp32_watershed_against_fp64():
    from triton_b200 import precision, scenarios
    sc = scenarios.watershed(n=192, dx=10.0, seed=3, duration=1800.0, nsrc=2, peak_flow=20.0)
    r = precision.compare(sc)
    assert r["steps_fp32"] > 50
    assert r["max_depth_error_m"] <= 1e-3, r
    assert r["volume_rel_error"] <= 1e-6, r
    assert abs(r["mass_balance_residual"]) <= 1e-6, r
    assert r["arrival_cells"] > 0


def test_fp32_thacker_against_fp64_and_analytic():
    from triton_b200 import precision, scenarios
    sc = scenarios.thacker(n=256, dx=32.0, periods=0.25)
    r = precision.compare(sc)
    assert r["max_depth_error_m"] <= 1e-3, r
    assert r["volume_rel_error"] <= 1e-6, r


def test_fp32_domain_roundtrip_of_bed():
    """The FP32 form keeps the bed as FP64 tile bases plus FP32 offsets; the
    bed read back is within FP32 rounding of the offset, not of the level."""
    from triton_b200 import scenarios
    sc = scenarios.watershed(n=100, dx=10.0, seed=5, duration=60.0, nsrc=1)
    sc.z[1:-1, 1:-1] += 2500.0  # a high plateau: FP32 of the level alone would lose 1e-4 m
    d = sc.to_domain("fp32")
    try:
        z = d.download("z")
    finally:
        d.close()
    inner = sc.z[1:-1, 1:-1]
    assert np.abs(z[1:-1, 1:-1] - inner).max() < 2e-5
