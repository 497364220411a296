"""Pins the CPU oracles to the reference (CPU only, no GPU).

Two links of the parity chain that the GPU tests build on:

* the reference built here from its own sources (oracle/_ref/triton_ref_mt:
  OpenMP, no FMA contraction; the same bits as the serial build where no two
  point sources share a cell) reproduces
  the reference's golden outputs of its three example cases as text
  (test/reference/{circular,paraboloid,allatoona}; the reference's own check,
  compare_runs_simple.py, accepts |a-b| < 1e-15 on those 6-decimal values);
* the C restatement (oracle/tri_oracle.c), which the lockstep GPU tests
  compare against, equals that reference build bit for bit at every print of
  the example cases and of synthetic cases with every forcing type (point
  sources sharing a cell, zoned runoff, external boundaries of types 0-3,
  friction, open boundaries), read from the same case files.

Skipped where the reference build is absent."""
from __future__ import annotations

import os

import numpy as np
import pytest

from tests import _cases

pytestmark = pytest.mark.skipif(not os.path.exists(_cases.REF_MT) or not os.path.isdir(_cases.CASES),
                                reason="reference build or its example cases absent")

GOLDEN = [("circular", "circular_dambreak.cfg", "output_circular_dambreak", None),
          ("paraboloid", "paraboloid.cfg", "output_paraboloid", None),
          ("allatoona", "allatoona.cfg", "output_allatoona", None)]


@pytest.mark.parametrize("case,cfg,out,_", GOLDEN)
def test_reference_build_reproduces_golden_outputs(tmp_path, case, cfg, out, _):
    run, text = _cases.golden_layout(str(tmp_path), _cases.REF_MT, cfg)
    with open(os.path.join(run, "test", cfg), "w") as f:
        f.write(text)
    _cases.run_exe("../triton.exe", os.path.join(run, "test"), ["./" + cfg])
    gold = os.path.join(_cases.CASES, "golden", case)
    for name in sorted(os.listdir(gold)):
        got = open(os.path.join(run, "test", out, "asc", name)).read()
        ref = open(os.path.join(gold, name)).read()
        if got != ref:
            a, b = np.array(got.split(), float), np.array(ref.split(), float)
            raise AssertionError(f"{case}/{name}: {(np.abs(a - b) >= 1e-15).sum()} values differ")


def _compare_prints(o, outdir, what):
    n = 0
    for pid, fields in _cases.oracle_prints(o):
        for name, got in zip(("H", "QX", "QY"), fields):
            ref = _cases.read_bin(os.path.join(outdir, "bin", f"{name}_{pid:02d}_00.out"))
            bad = got != ref
            if bad.any():
                i = tuple(np.argwhere(bad)[0])
                raise AssertionError(f"{what} print {pid} {name}: {bad.sum()} cells differ, first at {i}: "
                                     f"oracle {got[i]!r} reference {ref[i]!r}")
        n += 1
    assert n >= 1
    return n


# allatoona runs its first print only (2 416 of its 4 833 steps) to keep the
# CPU suite short; the golden test above runs it whole
@pytest.mark.parametrize("case,cfg,out,duration", [g[:3] + (7200.0 if g[0] == "allatoona" else None,)
                                                   for g in GOLDEN])
def test_oracle_matches_reference_on_example_cases(tmp_path, case, cfg, out, duration):
    run, text = _cases.golden_layout(str(tmp_path), _cases.REF_MT, cfg)
    if duration is not None:
        text = text.replace("sim_duration=14400", f"sim_duration={duration:g}")
    with open(os.path.join(run, "test", cfg), "w") as f:
        f.write(text)
    cwd = os.path.join(run, "test")
    _cases.run_exe("../triton.exe", cwd, ["./" + cfg])
    # the same case as the drop-in's host reads it (its parity with the
    # reference's preprocessing is tested on its own)
    os.symlink(_cases.EXE, os.path.join(run, "drop_in"))
    info, rd = _cases.dump("../drop_in", cwd, "./" + cfg, str(tmp_path / "dump"))
    o = _cases.oracle_of_dump(info, rd)
    _compare_prints(o, os.path.join(cwd, out), case)


@pytest.mark.parametrize("seed,open_b,fmt", [(3, 0, "BIN"), (4, 1, "ASC")])
def test_oracle_matches_reference_on_mixed_cases(tmp_path, seed, open_b, fmt):
    from tests._harness import oracle_from_scenario
    from triton_b200 import scenarios
    sc = scenarios.mixed(rows=41, cols=59, seed=seed, open_boundaries=open_b, friction=True, duration=12.0,
                         with_extbc=not open_b)
    cfg = scenarios.write_case(sc, str(tmp_path / "input"), fmt=fmt, output_format="BIN")
    base = str(tmp_path / "ref")
    # the serial build: two sources share a cell here, and the reference's
    # parallel loop over sources adds them in whatever order its threads run
    _cases.run_exe(_cases.project(base, _cases.REF), base, [cfg])
    n = _compare_prints(oracle_from_scenario(sc), os.path.join(base, "output"), f"mixed seed {seed}")
    assert n == 3
