"""End-to-end tests of the drop-in executable (triton_b200/lib/triton_b200)
on the GPU, against the reference's own golden outputs and against the
reference executable itself (oracle/_ref, built from the reference sources).

* Golden cases (test/reference/{circular,paraboloid,allatoona} of the
  reference, copied next to its build in oracle/_ref/cases): the ASCII outputs
  must match the golden files as the reference's own comparison does
  (compare_runs_simple.py: |a-b| < 1e-15 on the 6-decimal values, i.e. the
  same text).
* A synthetic case with every forcing type, run by both executables: binary
  FP64 outputs within 1e-9 of each field's scale, identical wet/dry masks,
  identical observation series text and restart cfg.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "triton_b200", "lib", "triton_b200")
REF = os.path.join(ROOT, "oracle", "_ref", "triton_ref")
CASES = os.path.join(ROOT, "oracle", "_ref", "cases")


def _run(exe, workdir, cfg, timeout=900):
    env = dict(os.environ, LD_LIBRARY_PATH=os.path.join(ROOT, "triton_b200", "lib"))
    p = subprocess.run([exe, cfg], cwd=workdir, capture_output=True, text=True, timeout=timeout, env=env)
    assert p.returncode == 0, p.stderr[-3000:]
    return p


def _layout(tmp_path, exe):
    """The reference's test layout: <run>/triton.exe, <run>/input, cwd <run>/test,
    so the project directory (executable path up two levels) is <run>/test."""
    run = tmp_path / "run"
    (run / "test").mkdir(parents=True)
    os.symlink(exe, run / "triton.exe")
    os.symlink(os.path.join(CASES, "input"), run / "input")
    return run


@pytest.mark.parametrize("case,cfg,out", [("circular", "circular_dambreak.cfg", "output_circular_dambreak"),
                                          ("paraboloid", "paraboloid.cfg", "output_paraboloid"),
                                          ("allatoona", "allatoona.cfg", "output_allatoona")])
def test_reference_golden_case(tmp_path, case, cfg, out):
    if not os.path.isdir(CASES):
        pytest.skip("reference example cases were not copied next to the reference build")
    run = _layout(tmp_path, EXE)
    shutil.copy(os.path.join(CASES, "test", cfg), run / "test" / cfg)
    _run("../triton.exe", run / "test", "./" + cfg)
    gold = os.path.join(CASES, "golden", case)
    for f in sorted(os.listdir(gold)):
        got = (run / "test" / out / "asc" / f).read_text()
        ref = open(os.path.join(gold, f)).read()
        if got != ref:
            a = np.array(got.split(), dtype=float)
            b = np.array(ref.split(), dtype=float)
            bad = np.abs(a - b) >= 1e-15
            raise AssertionError(f"{case}/{f}: {bad.sum()} of {a.size} values differ, max {np.abs(a - b).max():.2e}")


def _read_bin(path):
    v = np.fromfile(path, dtype=np.float64)
    r, c = int(v[0]), int(v[1])
    return v[2:].reshape(r, c)


@pytest.mark.parametrize("fmt,partitions", [("BIN", 0), ("ASC", 1)])
def test_synthetic_case_matches_reference_executable(tmp_path, fmt, partitions):
    """partitions 1: the rasters as partitioned input (input_option=PAR, a
    header file and one file per field), which the reference reads on one
    rank as it would on many."""
    if not os.path.exists(REF):
        pytest.skip("reference executable not built")
    from triton_b200 import scenarios
    sc = scenarios.mixed(rows=45, cols=71, seed=17, open_boundaries=0, friction=True, duration=12.0)
    outs = {}
    cfg = scenarios.write_case(sc, str(tmp_path / "input"), fmt=fmt, output_format="ASC", max_value_print="h",
                               partitions=partitions)
    for name, exe in (("ours", EXE), ("ref", REF)):
        base = tmp_path / name
        (base / "bin").mkdir(parents=True)
        os.symlink(exe, base / "bin" / "triton.exe")
        _run(str(base / "bin" / "triton.exe"), base, cfg)
        outs[name] = base / "output"
    for f in sorted(os.listdir(outs["ref"] / "bin")):
        a, b = _read_bin(outs["ours"] / "bin" / f), _read_bin(outs["ref"] / "bin" / f)
        scale = max(np.abs(b).max(), 1e-300)
        assert np.abs(a - b).max() <= 1e-9 * scale, f"{f}: {np.abs(a - b).max() / scale:.2e}"
        if f.startswith("H_"):
            assert np.array_equal(a > sc.hextra, b > sc.hextra), f"{f}: wet mask differs"
    for f in ("H_at_Xsec.txt", "QX_at_Xsec.txt", "QY_at_Xsec.txt"):
        ta = (outs["ours"] / "series" / f).read_text().splitlines()
        tb = (outs["ref"] / "series" / f).read_text().splitlines()
        assert len(ta) == len(tb) and ta[0] == tb[0]
        for la, lb in zip(ta[1:], tb[1:]):
            va, vb = np.array(la.split(","), float), np.array(lb.split(","), float)
            assert np.allclose(va, vb, rtol=0, atol=2e-6), (f, la, lb)
    for f in sorted(os.listdir(outs["ref"] / "cfg")):
        ca = (outs["ours"] / "cfg" / f).read_text().splitlines()
        cb = (outs["ref"] / "cfg" / f).read_text().splitlines()
        for la, lb in zip(ca, cb):
            if la.startswith(("sim_start_time=", "time_step=")):
                assert abs(float(la.split("=")[1]) - float(lb.split("=")[1])) <= 1e-9 * max(1.0, abs(float(lb.split("=")[1])))
            else:
                assert la == lb, (f, la, lb)


def test_checkpoint_resume_matches_reference_executable(tmp_path):
    """Resume from a checkpoint (triton_init.h:24-27,98-101,303-353): each
    executable runs a case with three prints, then resumes it from print 1
    (command line <cfg> <threads> 1) after the restart cfg it wrote there
    (output.h:754-811) is placed where the reference looks for it
    (<project>//cfg/config_1.cfg: the folder name is still empty when that
    path is formed).  The resumed runs must agree with each other (binary
    outputs within 1e-9 of each field's scale, identical wet/dry masks,
    the same series text and restart cfgs) and each with its own
    uninterrupted run (the checkpoint holds the state exactly)."""
    if not os.path.exists(REF):
        pytest.skip("reference executable not built")
    from triton_b200 import scenarios
    sc = scenarios.mixed(rows=45, cols=71, seed=23, open_boundaries=0, friction=True, duration=12.0)
    cfg = scenarios.write_case(sc, str(tmp_path / "input"), fmt="BIN", output_format="BIN", max_value_print="h")
    runs = {}
    for name, exe in (("ours", EXE), ("ref", REF)):
        base = tmp_path / name
        (base / "bin").mkdir(parents=True)
        os.symlink(exe, base / "bin" / "triton.exe")
        _run(str(base / "bin" / "triton.exe"), base, cfg)
        full = {f: _read_bin(base / "output" / "bin" / f) for f in os.listdir(base / "output" / "bin")}
        (base / "cfg").mkdir()
        shutil.copy(base / "output" / "cfg" / "config_1.cfg", base / "cfg" / "config_1.cfg")
        env = dict(os.environ, LD_LIBRARY_PATH=os.path.join(ROOT, "triton_b200", "lib"))
        p = subprocess.run([str(base / "bin" / "triton.exe"), cfg, "1", "1"], cwd=base, capture_output=True,
                           text=True, timeout=900, env=env)
        assert p.returncode == 0, p.stderr[-3000:]
        resumed = {f: _read_bin(base / "output" / "bin" / f) for f in os.listdir(base / "output" / "bin")}
        assert sorted(full) == sorted(resumed) and len(full) == 12  # H/QX/QY/MH at prints 1-3
        for f in full:
            assert np.array_equal(full[f], resumed[f]), f"{name}: resumed {f} differs from the uninterrupted run"
        runs[name] = (base, resumed)
    (ba, ra), (bb, rb) = runs["ours"], runs["ref"]
    for f in sorted(rb):
        a, b = ra[f], rb[f]
        scale = max(np.abs(b).max(), 1e-300)
        assert np.abs(a - b).max() <= 1e-9 * scale, f"{f}: {np.abs(a - b).max() / scale:.2e}"
        if f.startswith("H_"):
            assert np.array_equal(a > sc.hextra, b > sc.hextra), f"{f}: wet mask differs"
    for f in ("H_at_Xsec.txt", "QX_at_Xsec.txt", "QY_at_Xsec.txt"):
        ta = (ba / "output" / "series" / f).read_text().splitlines()
        tb = (bb / "output" / "series" / f).read_text().splitlines()
        assert len(ta) == len(tb) and ta[0] == tb[0], f
        for la, lb in zip(ta[1:], tb[1:]):
            va, vb = np.array(la.split(","), float), np.array(lb.split(","), float)
            assert va.shape == vb.shape and np.allclose(va, vb, rtol=0, atol=2e-6), (f, la, lb)
    _compare_restart_cfgs(ba / "output" / "cfg", bb / "output" / "cfg")


def _compare_restart_cfgs(da, db):
    """Restart cfgs equal line for line; the simtime and mean dt they carry
    within 1e-9 (the state, hence dt, may differ in the last bits where cube
    roots are taken)."""
    names = sorted(os.listdir(db))
    assert names and sorted(os.listdir(da)) == names
    for f in names:
        ca, cb = (da / f).read_text().splitlines(), (db / f).read_text().splitlines()
        assert len(ca) == len(cb), f
        for la, lb in zip(ca, cb):
            if la.startswith(("sim_start_time=", "time_step=")):
                va, vb = float(la.split("=")[1]), float(lb.split("=")[1])
                assert abs(va - vb) <= 1e-9 * max(1.0, abs(vb)), (f, la, lb)
            else:
                assert la == lb, (f, la, lb)
