"""Helpers for tests that run reference-format cases (a .cfg with its input
files) through an executable with the reference's command line: the drop-in
(triton_b200/lib/triton_b200) or the reference itself built from its sources
(oracle/_ref/triton_ref, triton_ref_mt).

The reference finds its project directory two levels above the executable's
path (config_utils.h:542-580) and writes output/ there, so every run gets its
own directory holding a link to the executable."""
from __future__ import annotations

import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "triton_b200", "lib", "triton_b200")
REF_DIR = os.path.join(ROOT, "oracle", "_ref")
REF = os.path.join(REF_DIR, "triton_ref")
REF_MT = os.path.join(REF_DIR, "triton_ref_mt")
CASES = os.path.join(REF_DIR, "cases")


def run_exe(exe, cwd, args, timeout=1800, threads=None):
    env = dict(os.environ, LD_LIBRARY_PATH=os.path.join(ROOT, "triton_b200", "lib"))
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
    p = subprocess.run([exe] + [str(a) for a in args], cwd=cwd, capture_output=True, text=True, timeout=timeout,
                       env=env)
    assert p.returncode == 0, f"{exe} {args}: {p.stderr[-3000:]}"
    return p


def project(base, exe):
    """<base>/bin/triton.exe -> exe: the project directory is <base>."""
    os.makedirs(os.path.join(base, "bin"), exist_ok=True)
    link = os.path.join(base, "bin", "triton.exe")
    if not os.path.lexists(link):
        os.symlink(exe, link)
    return link


def golden_layout(tmp, exe, cfg_name):
    """The reference's own test layout: <run>/triton.exe, <run>/input (the
    example inputs), cfg in <run>/test, run from <run>/test with
    ../triton.exe, so the project directory is <run>/test."""
    run = os.path.join(tmp, "run")
    os.makedirs(os.path.join(run, "test"), exist_ok=True)
    os.symlink(exe, os.path.join(run, "triton.exe"))
    os.symlink(os.path.join(CASES, "input"), os.path.join(run, "input"))
    with open(os.path.join(CASES, "test", cfg_name)) as f:
        text = f.read()
    return run, text


def read_bin(path):
    """A binary raster as the reference writes it (output_binary.h:71-80):
    rows and cols as doubles, then the interior values row by row."""
    v = np.fromfile(path, dtype=np.float64)
    r, c = int(v[0]), int(v[1])
    return v[2:].reshape(r, c)


def dump(exe_link, cwd, cfg, out):
    """The drop-in's --dump-problem: the padded arrays and tables a run would
    upload, and its loop parameters (info)."""
    os.makedirs(out, exist_ok=True)
    run_exe(exe_link, cwd, ["--dump-problem", out, cfg], timeout=600)
    info = {}
    for line in open(os.path.join(out, "info.txt")).read().splitlines():
        k, v = line.split()
        info[k] = float(v)
    rd = lambda n, dt: np.fromfile(os.path.join(out, n), dtype=dt)
    return info, rd


def oracle_of_dump(info, rd):
    """An OracleSim (the C restatement) holding the case a dump describes."""
    from oracle.tri_oracle import OracleSim
    R, C = int(info["rows"]), int(info["cols"])
    f = lambda n: rd(n, np.float64).reshape(R, C)
    runoff = sources = extbc = None
    if int(info["nzones"]) > 0:
        runoff = dict(zone=rd("zone.i32", np.int32).reshape(R, C), times=rd("roff_t.f64", np.float64),
                      rates=rd("roff_v.f64", np.float64), nzones=int(info["nzones"]), row=int(info["runoff_row"]))
    cells = rd("src_cells.i32", np.int32)
    if cells.size:
        sources = dict(cells=cells, times=rd("hyg_t.f64", np.float64), flows=rd("hyg_v.f64", np.float64))
    bcc = rd("bc_cells.i32", np.int32)
    if bcc.size:
        extbc = dict(cells=bcc, types=rd("bc_types.i32", np.int32), start=rd("bc_start.i32", np.int32),
                     nrows=rd("bc_nrows.i32", np.int32), var1=rd("bc_v1.f64", np.float64),
                     var2=rd("bc_v2.f64", np.float64))
    simtime = info["simtime"]
    clock = dict(simtime=simtime, sim_duration=info["sim_duration"], print_interval=info["print_interval"],
                 print_observation=info["print_observation"] if info["time_series"] else info["print_interval"],
                 last_obs_time=simtime, init_dt=info["init_dt"], time_step=info["time_step"],
                 print_id=int(info["checkpoint_id"]), it_count=int(info["it_count"]), it_print=int(info["it_print"]),
                 time_series=int(info["time_series"]), time_increment_fixed=int(info["time_increment_fixed"]))
    return OracleSim(R, C, info["dx"], info["courant"], info["hextra"], f("h.f64"), f("qx.f64"), f("qy.f64"),
                     f("z.f64"), f("n2.f64"), maxh=f("maxh.f64"), open_boundaries=int(info["open_boundaries"]),
                     runoff=runoff, sources=sources, extbc=extbc, clock=clock)


def oracle_prints(o):
    """Runs an OracleSim to its end; yields (print id, h, qx, qy interior
    copies) at every print event, as the reference writes them."""
    from tests._harness import oracle_bookkeeping, EV_END, EV_PRINT
    while True:
        n, ev = o.advance(1 << 30)
        if ev & EV_PRINT:
            pid = o.s.print_id + 1
            yield pid, tuple(o.grid(k)[1:-1, 1:-1].copy() for k in ("h", "qx", "qy"))
        oracle_bookkeeping(o, ev)
        if ev & EV_END or n == 0:
            return
