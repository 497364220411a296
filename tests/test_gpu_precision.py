"""The FP32 precision form against the FP64 path (the FP64 path itself is
pinned to the CPU oracle by test_gpu_parity.py).

Targets of the FP32 form: max depth error <= 1e-3 m and relative volume
error <= 1e-6 against FP64.  The small watersheds below meet them and are
held to them.  The watershed recipe over 6 h (the 8192^2 precision workload
at 1024^2) does not meet the max-depth target: a few hundred cells at wet/dry
fronts on steep slopes part by millimetres (the FP64 run moved by up to 1 cm
under a 1e-6 m bed perturbation there, and FP32 rounding is larger); it is
held to its measured regression bounds, with the target kept visible as an
expected failure.  Each bound states the value measured on a B200 (both runs
are deterministic)."""
import functools

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_fp32_rain_watershed_against_fp64():
    """Rain on a fractal watershed with an open outflow edge, 30 min: at the
    targets (measured max 2.3e-5 m, volume 9.5e-7)."""
    from triton_b200 import precision, scenarios
    sc = scenarios.watershed(n=192, dx=10.0, seed=3, duration=1800.0, nsrc=0)
    r = precision.compare(sc)
    assert r["steps_fp32"] > 50
    assert r["max_depth_error_m"] <= 1e-3, r          # target
    assert r["rms_depth_error_m"] <= 2e-6, r          # measured 4.4e-7 m
    assert r["volume_rel_error"] <= 1e-6, r           # target
    assert abs(r["mass_balance_residual"]) <= 1e-6, r  # FP64 accounts close the FP32 run
    assert r["arrival_cells"] > 0


def test_fp32_source_watershed_against_fp64():
    """Two point sources (20 m3/s peaks) and rain, 30 min, CFL dt in each
    form: at the targets (measured max 2.3e-5 m, volume 1.8e-7)."""
    from triton_b200 import precision, scenarios
    sc = scenarios.watershed(n=192, dx=10.0, seed=3, duration=1800.0, nsrc=2, peak_flow=20.0)
    r = precision.compare(sc)
    assert r["max_depth_error_m"] <= 1e-3, r          # target
    assert r["rms_depth_error_m"] <= 2e-6, r          # measured 4.7e-7 m
    assert r["volume_rel_error"] <= 1e-6, r           # target
    assert abs(r["mass_balance_residual"]) <= 1e-6, r


@functools.lru_cache(maxsize=1)
def _watershed_6h():  # run once, checked by both tests below
    from triton_b200 import precision, scenarios
    sc = scenarios.watershed(n=1024, dx=10.0, seed=1234, gpu_noise=True)  # 6 h, 3 sources, rain, open edge
    return precision.compare(sc)


def test_fp32_watershed_6h_regression():
    """The precision workload's recipe at 1024^2 over 6 h (80 756 steps).
    Measured: max 7.5e-3 m, RMS 6.3e-5 m, 99.9th percentile 5.8e-4 m, 296
    cells (0.03 %) over 1 mm, volume 2.2e-6."""
    r = _watershed_6h()
    assert r["max_depth_error_m"] <= 1.5e-2, r
    assert r["rms_depth_error_m"] <= 1.5e-4, r
    assert r["p999_depth_error_m"] <= 1.5e-3, r
    assert r["cells_over_1mm"] <= 600, r
    assert r["volume_rel_error"] <= 5e-6, r
    assert abs(r["mass_balance_residual"]) <= 1e-6, r


@pytest.mark.xfail(strict=False, reason="the FP32 form's targets (1e-3 m max depth error, 1e-6 relative volume "
                                        "error) are not met on the 6 h watershed recipe at 1024^2 (measured "
                                        "7.5e-3 m, 2.2e-6); at 8192^2 the volume target is met (4e-8), the max "
                                        "is 1.9e-2 m")
def test_fp32_watershed_6h_at_target_bounds():
    r = _watershed_6h()
    assert r["max_depth_error_m"] <= 1e-3, r
    assert r["volume_rel_error"] <= 1e-6, r


def test_fp32_fixed_dt_thacker_against_fp64():
    """Thacker bowl on the same time levels in both forms (fixed dt below the
    CFL limit): the difference is the FP32 form's arithmetic alone.  Away from
    the moving shoreline the two forms agree to micrometres after 20 steps
    (99.9th percentile 1.7e-6 m); at the shoreline a cell that dries or wets
    one step apart differs by up to the depth of one cell's bank step (about
    5 cm on this 32 m grid).  Measured after 673 steps: RMS 1.1e-3 m, 99.9th
    percentile 1.3e-2 m, volume 4e-9, mass-balance residual 3e-9."""
    from triton_b200 import precision, scenarios
    sc = scenarios.thacker(n=256, dx=32.0, periods=0.25)
    r = precision.compare(sc, fixed_dt=0.5)
    assert r["steps_fp32"] == r["steps_fp64"]
    assert r["rms_depth_error_m"] <= 3e-3, r
    assert r["p999_depth_error_m"] <= 4e-2, r
    assert r["volume_rel_error"] <= 1e-6, r
    assert abs(r["mass_balance_residual"]) <= 1e-6, r
    short = precision.compare(sc, duration=10.0, fixed_dt=0.5)
    assert short["p999_depth_error_m"] <= 1e-5, short
    assert short["rms_depth_error_m"] <= 1e-4, short


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
