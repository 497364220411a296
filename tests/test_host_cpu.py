"""CPU tests of the drop-in host and the C ABI library (no GPU needed).

* The C++ host (triton_b200/lib/triton_b200) reads a reference-format case
  (cfg, ASCII or binary rasters, whole or partitioned, hydrograph, runoff,
  extbc and observation files) and preprocesses it as triton_init.h does; its
  arrays must equal the scenario the case was written from, value for value.
* libtriton_b200.so loads and exports every symbol include/triton_b200.h
  declares.
* The ASCII raster formatter gives printf's "%.6f" text for every double:
  exact ties, negatives that round to zero, subnormals, values past its
  integer range, infinities.
"""
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "triton_b200", "lib", "triton_b200")
HDR = os.path.join(ROOT, "include", "triton_b200.h")


def _dump(tmp_path, cfg):
    out = tmp_path / "dump"
    out.mkdir()
    p = subprocess.run([EXE, "--dump-problem", str(out), cfg], capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stderr
    info = dict(l.split() for l in (out / "info.txt").read_text().splitlines())
    rd = lambda n, dt: np.fromfile(out / n, dtype=dt)
    return info, rd


@pytest.mark.parametrize("fmt", ["ASC", "BIN"])
@pytest.mark.parametrize("open_b", [0, 1])
@pytest.mark.parametrize("partitions", [0, 1, 3])
def test_host_preprocessing_matches_scenario(tmp_path, fmt, open_b, partitions):
    """partitions 0: one file per raster (input_option=SEQ); 1 or 3: a header
    file and one file per partition (input_option=PAR), 3 being rows split as
    for three ranks and stacked again by the host."""
    from triton_b200 import scenarios
    sc = scenarios.mixed(rows=23, cols=37, seed=9 + open_b, open_boundaries=open_b, duration=5.0)
    cfg = scenarios.write_case(sc, str(tmp_path / "case"), fmt=fmt, partitions=partitions)
    info, rd = _dump(tmp_path, cfg)
    R, C = int(info["rows"]), int(info["cols"])
    assert (R, C) == (sc.rows, sc.cols)
    for name in ("h", "qx", "qy", "z", "n2"):
        got = rd(f"{name}.f64", np.float64).reshape(R, C)
        ref = getattr(sc, name)
        assert np.array_equal(got, ref), f"{fmt} {name}: max diff {np.abs(got - ref).max()}"
    # max depth starts from h before the boundary ghosts are filled (triton_init.h:1239-1248 runs before
    # :1250-1289); ghost values of maxh are never read or written out
    assert np.array_equal(rd("maxh.f64", np.float64).reshape(R, C)[1:-1, 1:-1], sc.h[1:-1, 1:-1])
    assert np.array_equal(rd("src_cells.i32", np.int32), sc.sources["cells"])
    assert np.array_equal(rd("hyg_t.f64", np.float64), sc.sources["times"])
    assert np.array_equal(rd("hyg_v.f64", np.float64), sc.sources["flows"])
    zone = rd("zone.i32", np.int32).reshape(R, C)
    assert np.array_equal(zone[1:-1, 1:-1], sc.runoff["zone"][1:-1, 1:-1])
    assert np.array_equal(rd("roff_t.f64", np.float64), sc.runoff["times"])
    assert np.array_equal(rd("roff_v.f64", np.float64), sc.runoff["rates"])
    for k in ("cells", "types", "start", "nrows"):
        assert np.array_equal(rd(f"bc_{k}.i32", np.int32), sc.extbc[k]), k
    assert np.array_equal(rd("bc_v1.f64", np.float64), sc.extbc["var1"])
    assert np.array_equal(rd("bc_v2.f64", np.float64), sc.extbc["var2"])
    assert np.array_equal(rd("obs_cells.i32", np.int32), sc.obs_cells)
    assert float(info["init_dt"]) == sc.init_dt()


@pytest.mark.parametrize("partitions,output_option", [(0, "SEQ"), (0, "PAR"), (1, "SEQ"), (3, "SEQ"), (3, "PAR")])
def test_host_reads_checkpoint_rasters(tmp_path, partitions, output_option):
    """A restart cfg (checkpoint_id > 0) replaces the initial depth,
    discharges and max depth with the checkpoint's binary rasters
    <output_folder>/bin/<H|QX|QY|MH>_<id>_<rank>.out.  Sequential input reads
    rank 00's file holding the whole domain, and only when output_option is
    SEQ (triton_init.h:303-353; otherwise the initial fields stand);
    partitioned input reads one file per rank with that rank's rows
    (triton_init.h:577-626), here written as 1 or 3 ranks would write them
    and stacked in rank order."""
    from triton_b200 import scenarios
    sc = scenarios.mixed(rows=23, cols=37, seed=11, open_boundaries=0, duration=5.0)
    cfg = scenarios.write_case(sc, str(tmp_path / "case"), fmt="BIN", partitions=partitions)
    text = open(cfg).read().replace("checkpoint_id=0", "checkpoint_id=1").replace(
        "output_option=SEQ", f"output_option={output_option}") + "max_value_print_option=h\n"
    open(cfg, "w").write(text)
    base = tmp_path / "proj"
    (base / "bin").mkdir(parents=True)
    os.symlink(EXE, base / "bin" / "triton.exe")
    (base / "output" / "bin").mkdir(parents=True)
    rng = np.random.default_rng(1)
    R, C = sc.rows - 2, sc.cols - 2
    hot = {k: rng.random((R, C)) for k in ("H", "QX", "QY", "MH")}
    for k, a in hot.items():
        if partitions == 0:
            scenarios._write_raster(str(base / "output" / "bin" / f"{k}_01_00.out"), a, "BIN")
        else:  # per-rank slabs as create_local_dims splits rows (mpi_utils.h:73-89)
            scenarios._write_parts(str(base / "output" / "bin" / f"{k}_01"), ".out", a, "BIN", partitions)
    out = tmp_path / "dump"
    out.mkdir()
    p = subprocess.run([str(base / "bin" / "triton.exe"), "--dump-problem", str(out), cfg], capture_output=True,
                       text=True, timeout=120)
    assert p.returncode == 0, p.stderr
    rd = lambda n: np.fromfile(out / n, dtype=np.float64).reshape(sc.rows, sc.cols)[1:-1, 1:-1]
    read = partitions > 0 or output_option == "SEQ"
    for k, name in (("H", "h"), ("QX", "qx"), ("QY", "qy"), ("MH", "maxh")):
        want = hot[k] if read else (sc.h if k == "MH" else getattr(sc, name))[1:-1, 1:-1]
        assert np.array_equal(rd(f"{name}.f64"), want), (k, partitions, output_option)


def test_host_rejects_bad_inputs(tmp_path):
    from triton_b200 import scenarios
    sc = scenarios.mixed(rows=11, cols=13, seed=2, duration=2.0)
    cfg = scenarios.write_case(sc, str(tmp_path / "case"), fmt="ASC")
    # a source outside the grid: the reference exits with "Source 1 is out of bounds"
    src = tmp_path / "case" / "mixed.src"
    src.write_text("%X,Y\n-50.0,12.5\n7.5,7.5\n7.5,7.5\n")
    p = subprocess.run([EXE, "--dump-problem", str(tmp_path), cfg], capture_output=True, text=True, timeout=60)
    assert p.returncode != 0 and "Source 1 is out of bounds" in p.stderr
    # a raster with the wrong size
    sc2 = scenarios.mixed(rows=11, cols=13, seed=2, duration=2.0)
    cfg2 = scenarios.write_case(sc2, str(tmp_path / "case2"), fmt="ASC")
    hfile = tmp_path / "case2" / "mixed.h.asc"
    hfile.write_text("\n".join(hfile.read_text().splitlines()[:-1]) + "\n")
    p = subprocess.run([EXE, "--dump-problem", str(tmp_path), cfg2], capture_output=True, text=True, timeout=60)
    assert p.returncode != 0 and "Invalid dimension" in p.stderr
    # a missing file
    p = subprocess.run([EXE, "--dump-problem", str(tmp_path), str(tmp_path / "nope.cfg")], capture_output=True,
                       text=True, timeout=60)
    assert p.returncode != 0 and "Error reading file" in p.stderr
    # partitioned input without its first partition, and an unknown input option
    cfg3 = scenarios.write_case(sc2, str(tmp_path / "case3"), fmt="BIN", partitions=2)
    os.remove(tmp_path / "case3" / "mixed_dem_00.dem")
    p = subprocess.run([EXE, "--dump-problem", str(tmp_path), cfg3], capture_output=True, text=True, timeout=60)
    assert p.returncode != 0 and "mixed_dem_00.dem" in p.stderr
    cfg4 = tmp_path / "case3" / "other.cfg"
    cfg4.write_text(open(cfg3).read().replace("input_option=PAR", "input_option=XYZ"))
    p = subprocess.run([EXE, "--dump-problem", str(tmp_path), str(cfg4)], capture_output=True, text=True, timeout=60)
    assert p.returncode != 0 and "input_option=XYZ is not supported" in p.stderr


def test_cfg_parser_rules(tmp_path):
    """The reference's cfg rules (config_utils.h:195-238): the first
    occurrence of a key wins, surrounding quotes are stripped, '#' is removed
    as a single character unless it follows a quote."""
    from triton_b200 import scenarios
    sc = scenarios.dambreak(n=8, dx=1.0, radius=2.0, depth=1.0, duration=1.0)
    cfg = scenarios.write_case(sc, str(tmp_path / "case"), fmt="ASC")
    text = open(cfg).read()
    text = text.replace("courant=0.5", "courant=0.4#5\ncourant=0.9")  # '#' dropped -> 0.45; second ignored
    text = text.replace("hextra=0.001", 'hextra="0.002"')
    open(cfg, "w").write(text)
    out = tmp_path / "dump"
    out.mkdir()
    p = subprocess.run([EXE, "--dump-problem", str(out), cfg], capture_output=True, text=True, timeout=60)
    assert p.returncode == 0, p.stderr
    info = dict(l.split() for l in (out / "info.txt").read_text().splitlines())
    assert float(info["courant"]) == 0.45
    assert float(info["hextra"]) == 0.002


def test_abi_exports_every_declared_symbol():
    from triton_b200 import _abi
    L = _abi.lib()
    declared = re.findall(r"^\s*(?:int|const char\*)\s+(tri_\w+)\s*\(", open(HDR).read(), flags=re.M)
    assert len(declared) >= 30
    missing = [s for s in declared if not hasattr(L, s)]
    assert not missing, missing
    assert L.tri_abi_version() == 1
    assert set(declared) <= set(_abi.exported_symbols()) | set(declared)


def test_abi_without_gpu_fails_cleanly():
    """Creating a domain where no GPU is visible returns an error status with a
    message; it never falls back to a CPU implementation."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    from triton_b200 import Domain, TriError
    with pytest.raises(TriError):
        Domain(10, 10, 1.0)


def test_footprint():
    from triton_b200 import Domain
    assert Domain.footprint(8194, 8194, "fp64") > 8194 * 8194 * 72
    assert Domain.footprint(8194, 8194, "fp32") < Domain.footprint(8194, 8194, "fp64")


def test_ascii_formatter_matches_printf(tmp_path):
    rng = np.random.default_rng(5)
    mag = 10.0 ** rng.uniform(-12, 15, 200000)
    vals = [mag * rng.choice([-1.0, 1.0], mag.size),
            (2 * rng.integers(0, 5 * 10 ** 5, 20000) + 1) / 128.0,  # exact decimal ties at the 6th digit
            -(2 * rng.integers(0, 5 * 10 ** 5, 2000) + 1) / 128.0,
            rng.integers(-10 ** 9, 10 ** 9, 20000) / 10.0 ** rng.integers(0, 9, 20000),
            np.array([0.0, -0.0, 5e-7, -5e-7, 4.9999999e-7, -1e-9, 2.0 ** -1074, -(2.0 ** -1074), 2.0 ** -1022,
                      0.0078125, 0.0234375, 1.0000005, 123456.0000005, 9.9999995, 18446744073709.55,
                      18446744073709.553, 1.8446744073709552e13, 2.0 ** 64, 1e20, -1e20, 1e300, -1.7976931348623157e308,
                      np.inf, -np.inf])]
    v = np.concatenate(vals)
    src = tmp_path / "v.f64"
    v.astype("<f8").tofile(src)
    out = tmp_path / "v.txt"
    p = subprocess.run([EXE, "--format-fixed6", str(src), str(out)], capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stderr
    got = out.read_text().splitlines()
    assert len(got) == v.size
    want = ["%.6f" % x for x in v]  # Python's formatting is correctly rounded, ties to even, like glibc's
    bad = [(float(x), g, w) for x, g, w in zip(v, got, want) if g != w]
    assert not bad, bad[:10]
