#!/usr/bin/env python
"""Throughput of the TRITON time-stepping hot path on B200: cell-updates/s.

A step is one time step of the reference loop (triton_simulate.h:54-134) over
the whole grid: CFL dt reduction + dt policy, face fluxes, conserved update,
wet/dry masks and max depth, all on the GPU.  Workload at N=1: the FP64
Thacker planar oscillation in a paraboloid bowl, 2048 x 2048 cells, dx 4 m,
closed walls, CFL 0.5 (seeded-free analytic initial state, synthetic).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times the reference's own CPU implementation (the
unmodified TRITON sources compiled with OpenMP into oracle/_ref) on the same
workload with every host thread.  With N > 1 each rank runs an independent
replica (the path is not sharded: one domain per GPU), value is the total over
ranks divided by the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import re
import shutil
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-updates/s"
ALG_BYTES_STEP = {"fp64": 80, "fp32": 40}      # per interior cell and step (whole step)
ALG_BYTES_FLUX = {"fp64": 64, "fp32": 32}      # flux/update kernel: h,qx,qy,z,n2 read + h,qx,qy written
REF_EXE = os.path.join(ROOT, "oracle", "_ref", "triton_ref_omp")


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _traffic_per_cell(kernel, precision):
    """Per-cell DRAM bytes of a kernel from the committed ncu summary
    (profiles/*.txt line 'traffic_bytes_per_cell <kernel> <precision> <B>')."""
    pat = re.compile(r"traffic_bytes_per_cell\s+(\S+)\s+(\S+)\s+([0-9.eE+-]+)")
    pdir = os.path.join(ROOT, "profiles")
    if not os.path.isdir(pdir):
        return None
    for fn in sorted(os.listdir(pdir)):
        if not fn.endswith((".txt", ".md")):
            continue
        with open(os.path.join(pdir, fn)) as f:
            for line in f:
                m = pat.search(line)
                if m and m.group(1) == kernel and m.group(2) == precision:
                    return float(m.group(3))
    return None


def _profile_metric(fname, metric):
    """A metric's value from a committed ncu summary (profiles/<fname>)."""
    path = os.path.join(ROOT, "profiles", fname)
    if not os.path.exists(path):
        return None
    with open(path) as f:
        for line in f:
            parts = line.split()
            if len(parts) >= 2 and parts[0] == metric:
                try:
                    return float(parts[1].replace(",", ""))
                except ValueError:
                    return None
    return None


def _issue_bound(precision):
    """The flux kernel's second ceiling, instruction issue (FP64 pipe busy
    fraction and issue-slot fraction), from its committed ncu summary."""
    fname = f"k_flux_update_thacker2048_{precision}.txt"
    pct = lambda m: (lambda v: None if v is None else v / 100.0)(_profile_metric(fname, m))  # noqa: E731
    return {"fp64_pipe_active_frac": pct("sm__pipe_fp64_cycles_active.avg.pct_of_peak_sustained_active"),
            "issue_active_frac": pct("smsp__issue_active.avg.pct_of_peak_sustained_active"),
            "source": f"profiles/{fname} (ncu, one launch in the timed steps)"}


def _fp64_pipe(precision, launch_s, sm_mhz):
    """The flux kernel against the FP64 pipe: its FP64 warp instructions per
    launch (committed ncu summary of the same workload and launch shape) over
    the launch time measured here, against the pipe's peak of 148 SMs x 4
    schedulers x 1/2 warp instruction per cycle (16 FP64 lanes per scheduler)
    at the SM clock sampled during the run."""
    fname = f"k_flux_update_thacker2048_{precision}.txt"
    n = _profile_metric(fname, "smsp__inst_executed_pipe_fp64.sum")
    if n is None or not launch_s or not sm_mhz:
        return None
    achieved = n / launch_s / 1e9
    peak = 148 * 4 * 0.5 * sm_mhz * 1e6 / 1e9
    return {"bound": "fp64_pipe", "unit": "G warp-instructions/s", "achieved": achieved, "peak": peak,
            "frac": achieved / peak, "fp64_warp_instructions_per_launch": n,
            "source": f"profiles/{fname} (instruction count), launch time and SM clock of this run"}


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap,utilization.gpu")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        if not shutil.which("nvidia-smi"):
            return
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        self.f = open(self.path, "w")
        self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                     stderr=subprocess.DEVNULL)

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = max(float(r[2]) for r in rows if r[2].replace(".", "").isdigit())
        load = [s for s in sm if s > 0.5 * smax] or sm
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        util = [float(r[9]) for r in rows if len(r) > 9 and r[9].replace(".", "").isdigit()]
        return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": smax, "reasons": reasons,
                "samples": len(rows), "util_mean": statistics.mean(util) / 100.0 if util else None}


# ---------------------------------------------------------------------------
def workload(name, n):
    from triton_b200 import scenarios
    if name == "thacker":
        sc = scenarios.thacker(n=n or 2048, dx=4.0)
        desc = (f"Thacker planar oscillation in a paraboloid bowl, {sc.rows - 2}x{sc.cols - 2} cells, dx 4 m, "
                f"h0 10 m, a 3000 m, rim amplitude 0.5 m, closed walls, frictionless, CFL 0.5")
    elif name == "dambreak":
        sc = scenarios.dambreak(n=n or 512)
        desc = f"circular dam break {sc.rows - 2}x{sc.cols - 2}, dx 1 m, 10 m inside r=50 m, closed, CFL 0.5"
    else:
        raise SystemExit(f"unknown workload {name}")
    return sc, desc


def cfl_dt0(sc):
    import numpy as np
    h, qx, qy = sc.h, sc.qx, sc.qy
    wet = h > sc.hextra
    with np.errstate(divide="ignore"):
        u = np.where(wet, np.maximum(abs(qx), abs(qy)) / np.where(wet, h, 1), 0)
        dt = np.where(wet, sc.courant * sc.dx / (u + 3.132091953 * np.sqrt(np.where(wet, h, 0))), np.inf)
    return float(dt.min())


def run_reference(sc, steps, threads):
    """Runs the reference OpenMP build on `sc` for about `steps` time steps;
    returns (cell-updates/s, iterations, compute seconds)."""
    from triton_b200 import scenarios
    if not os.path.exists(REF_EXE):
        return None
    tmp = tempfile.mkdtemp(prefix="tri_ref_")
    try:
        sc = scenarios.Scenario(**{k: getattr(sc, k) for k in sc.__dataclass_fields__})
        sc.sim_duration = cfl_dt0(sc) * steps
        sc.print_interval = sc.sim_duration
        sc.time_series = 0
        sc.it_print = 1 << 30
        cfg = scenarios.write_case(sc, os.path.join(tmp, "input"), fmt="BIN", output_format="BIN")
        os.makedirs(os.path.join(tmp, "bin"))
        exe = os.path.join(tmp, "bin", "triton.exe")
        os.symlink(REF_EXE, exe)
        env = dict(os.environ, OMP_NUM_THREADS=str(threads), OMP_PROC_BIND="close", OMP_PLACES="cores")
        p = subprocess.run([exe, cfg], cwd=tmp, env=env, capture_output=True, text=True, timeout=1800)
        if p.returncode != 0:
            raise RuntimeError(f"reference run failed: {p.stderr[-2000:]}")
        its = int(re.findall(r"it:\s*(\d+)", p.stderr)[-1])
        with open(os.path.join(tmp, "output", "performance.txt")) as f:
            line = [l for l in f if l.startswith("0,")][0]
        compute = float(line.split(",")[1])
        return sc.interior_cells * its / compute, its, compute
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


def host_cores():
    """(physical cores, logical CPUs) this process may run on: distinct
    (package, core) pairs of /proc/cpuinfo among the CPUs of its affinity."""
    cpus = sorted(os.sched_getaffinity(0))
    pairs, cur, phys = {}, None, "0"
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                k, _, v = line.partition(":")
                k, v = k.strip(), v.strip()
                if k == "processor":
                    cur = int(v)
                elif k == "physical id":
                    phys = v
                elif k == "core id" and cur is not None:
                    pairs[cur] = (phys, v)
    except OSError:
        pass
    cores = len({pairs[c] for c in cpus if c in pairs}) or len(cpus)
    return cores, len(cpus)


def workload_config(sc, desc, precision, world):
    return {"workload": desc, "grid": [sc.rows - 2, sc.cols - 2], "interior_cells": sc.interior_cells,
            "precision": precision, "parallelism": f"replicas x{world}" if world > 1 else "single"}


def reference_arm(args, sc, desc):
    cores, logical = host_cores()
    if args.warmup > 0 and os.path.exists(REF_EXE):
        run_reference(sc, args.warmup, cores)  # untimed: warms the host caches and the page cache
    r = run_reference(sc, args.steps, cores)
    if r is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/triton_ref_omp was not built"}))
        return
    val, its, secs = r
    cfg = workload_config(sc, desc, args.precision, 1)
    cfg["engine"] = (f"reference TRITON sources, OpenMP build, {cores} threads (one per physical core of "
                     f"{logical} logical CPUs)")
    line = {"metric": METRIC, "value": val, "unit": "cell-updates/s", "n_gpus": args.gpus, "steps": its,
            "warmup": args.warmup, "ms_per_step": 1000.0 * secs / its, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference", "config": cfg,
            "cpu_baseline": {"value": val, "unit": "cell-updates/s", "cores": cores, "kind": "reference",
                             "sample": f"{its} time steps of the workload ({secs:.2f} s compute) after an "
                                       f"untimed run of {args.warmup}, {cores} OpenMP threads on {cores} "
                                       f"physical cores"},
            "e2e": {"value": val, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# -- ranks: one process per GPU, replicas of the workload ---------------------
def ranks():
    """(rank, world size, local rank) from the torchrun environment."""
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def init_ranks(world, backend="nccl"):
    """Joins the process group when there is more than one rank (a short
    timeout, so ranks that wait for a missing one end with an error)."""
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world, device):
    """The largest x over all ranks (every rank gets it)."""
    import torch
    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    if world > 1:
        import torch.distributed as dist
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def close_ranks(world):
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def _timed(stream, fn):
    """Runs fn() between two CUDA events on `stream`; returns (result, ms)."""
    import torch
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    out = fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return out, e0.elapsed_time(e1)


def _form(out, name, fn):
    """Runs one form; a failure is recorded in its entry instead of ending
    the run (the headline line is printed either way)."""
    t0 = time.perf_counter()
    try:
        out[name] = fn()
    except Exception as e:  # noqa: BLE001
        out[name] = {"error": f"{type(e).__name__}: {e}"[:500]}
    out[name]["wall_s"] = round(time.perf_counter() - t0, 1)


def _domain_window(sc, prec, stream, spinup, steps, warmup):
    """One domain of `sc` in `prec`, launch shape autotuned: `spinup` +
    `warmup` untimed steps, `steps` timed with CUDA events at the two ends,
    then the same number again with an event pair around every flux and
    wet-dry launch for the per-kernel figures."""
    d = sc.to_domain(prec, stream=stream.cuda_stream)
    try:
        d.set_clock(sim_duration=1e300, print_interval=1e300, print_observation=1e300, it_print=0, time_series=0)
        tune = d.autotune(trial_steps=8)
        d.advance(spinup + warmup)
        (n, _), ms = _timed(stream, lambda: d.advance(steps))
        d.set_timing(True)
        d.advance(steps)
        torch_sync()
        flux_ms, flux_n, wet_ms, wet_n = d.get_timing()
        fcells, _ = d.get_work()
        d.set_timing(False)
    finally:
        d.close()
    cells = sc.interior_cells
    peak, kind = _peaks()
    flux_s = flux_ms / max(flux_n, 1) / 1000.0
    fl_cells = fcells / max(flux_n, 1)
    step_gbs = ALG_BYTES_STEP[prec] * cells * n / (ms / 1000.0) / 1e9
    return {"value": cells * n / (ms / 1000.0), "unit": "cell-updates/s", "ms_per_step": ms / n, "steps": n,
            "flux_launch_shape": {k: tune[k] for k in ("variant", "rows_per_tile")},
            "roofline": {"bound": "hbm", "kernel": "k_flux_update", "unit": "GB/s",
                         "achieved": ALG_BYTES_FLUX[prec] * fl_cells / flux_s / 1e9, "peak": peak,
                         "frac": ALG_BYTES_FLUX[prec] * fl_cells / flux_s / 1e9 / peak,
                         "peak_source": f"MEASURED_PEAKS.json hbm_gbs ({kind})",
                         "computed_cell_frac": fl_cells / cells, "avg_launch_ms": flux_s * 1000.0,
                         "wetdry_dt_avg_launch_ms": wet_ms / max(wet_n, 1), "step_achieved_gbs": step_gbs,
                         "step_frac": step_gbs / peak}}


def torch_sync():
    import torch
    torch.cuda.synchronize()


def form_watershed(args, stream):
    """The precision form's watershed (side --ws-n, 8192 by default: 67 M
    cells, dx 10 m, fractal terrain 0-300 m with a carved valley, log-normal
    Manning, 3 point inflows, rain 50 mm/h, open outflow on the lowest edge)
    in FP64 and in FP32: a window of --ws-steps steps after 120 steps of
    spin-up.  Rain falls on every cell, so every tile is computed (a domain
    with runoff never skips dry tiles)."""
    from triton_b200 import scenarios
    sc = scenarios.watershed(n=args.ws_n, dx=10.0, seed=1234, gpu_noise=True)
    out = {"workload": f"watershed {args.ws_n}x{args.ws_n}, dx 10 m, fractal DEM 0-300 m + carved valley, "
                       "log-normal Manning (median 0.035, sigma 0.3), 3 inflows, rain 50 mm/h, open outflow "
                       f"edge; {args.ws_steps} steps after 120 of spin-up, every tile computed",
           "interior_cells": sc.interior_cells}
    for prec in ("fp64", "fp32"):
        out[prec] = _domain_window(sc, prec, stream, 120, args.ws_steps, args.warmup)
    out["fp32_vs_fp64"] = out["fp32"]["value"] / out["fp64"]["value"]
    return out


def form_ensemble(args, stream):
    """--ens-members watershed members (side log-uniform in
    256..--ens-max-side, dx 5-20 m, rain 10-100 mm/h for 1 h, Manning
    median +/-30 %, 3 h), advanced as one batch in FP32 and in FP64, and the
    same members one after another as plain FP64 domains; every figure is
    interior cells x steps over CUDA-event time on one stream.  Members are
    built one at a time straight into their domains."""
    from triton_b200 import scenarios
    from triton_b200.batch import Batch
    doms = {"fp32": [], "fp64": []}
    cells = []
    try:
        for m in scenarios.ensemble_iter(members=args.ens_members, seed=2024, side_min=256,
                                         side_max=args.ens_max_side, duration=3 * 3600.0, gpu_noise=True):
            cells.append(m.interior_cells)
            for prec, lst in doms.items():
                dm = m.to_domain(prec, stream=stream.cuda_stream)
                dm.set_clock(print_interval=1e300, print_observation=1e300, it_print=0, time_series=0)
                lst.append(dm)
        ens = {"members": len(cells), "interior_cells": sum(cells), "batched_steps": args.ens_steps,
               "workload": f"{len(cells)} rain-on-grid watersheds, side log-uniform 256..{args.ens_max_side}, "
                           "dx 5-20 m, rain 10-100 mm/h for 1 h, Manning median +/-30 %, 3 h"}
        for prec in ("fp32", "fp64"):
            b = Batch(doms[prec], stream=stream.cuda_stream)
            tune = b.autotune(3)
            b.advance(args.warmup)
            p, ms = _timed(stream, lambda: b.advance(args.ens_steps))
            ens[f"{prec}_batched"] = p.cell_updates / (ms / 1000.0)
            ens[f"{prec}_batched_ms_per_step"] = ms / args.ens_steps
            ens[f"{prec}_batched_shape"] = {k: tune[k] for k in ("variant", "rows_per_tile")}
            # the same steps in single persistent launches (per-member
            # dependencies instead of a launch per kernel type and step)
            b.set_mode(True)
            b.advance(args.warmup)
            p, ms = _timed(stream, lambda: b.advance(args.ens_steps))
            ens[f"{prec}_batched_single_launch"] = p.cell_updates / (ms / 1000.0)
            b.close()
        def solo():  # the same members as plain FP64 runs, one after another
            u = 0
            for dm, c in zip(doms["fp64"], cells):
                k, _ = dm.advance(args.ens_steps)
                u += k * c
            return u
        u, ms = _timed(stream, solo)
        ens["fp64_sequential"] = u / (ms / 1000.0)
    finally:
        for lst in doms.values():
            for dm in lst:
                dm.close()
    ens["fp32_batched_vs_fp64_batched"] = ens["fp32_batched"] / ens["fp64_batched"]
    ens["fp32_batched_vs_fp64_sequential"] = ens["fp32_batched"] / ens["fp64_sequential"]
    return ens


def form_serving(args):
    """A short serving window below capacity: Poisson arrivals at
    --form-serve-rate per s for --form-serve-seconds (the serving workload's
    scenarios: side log-uniform 512..4096, 0.5-6 h simulated, 20 % FP64),
    stopped after --form-serve-max-wall s; p50/p99 solve latency of the
    completed requests, scenarios/hour, cell-updates/s and the GPU's busy
    fraction (nvidia-smi utilization.gpu) over the window."""
    from triton_b200.serving import Server, poisson_requests, summary
    reqs = poisson_requests(rate=args.form_serve_rate, seconds=args.form_serve_seconds, seed=11)
    srv = Server(hbm_budget=150e9, chunk_steps=32)
    sampler = ClockSampler(os.environ.get("CUDA_VISIBLE_DEVICES", "0").split(",")[0])
    sampler.start()
    t0 = time.perf_counter()
    srv.run(reqs, deadline=args.form_serve_max_wall)
    wall = time.perf_counter() - t0
    clocks = sampler.stop()
    s = summary(reqs, wall)
    return dict(s, workload=f"Poisson arrivals {args.form_serve_rate}/s for {args.form_serve_seconds:.0f} s, side "
                            "log-uniform 512..4096, 0.5-6 h simulated, 20% FP64 / 80% FP32, 150 GB budget",
                wall_limit_s=args.form_serve_max_wall, unfinished=sum(r.finished is None for r in reqs),
                peak_hbm_used_bytes=srv.peak_used, cell_updates_per_s_all_work=srv.cell_updates / wall,
                gpu_utilisation=(clocks or {}).get("util_mean"), clocks=clocks)


def measure_forms(args, sc, stream, value64):
    """The other forms on one GPU, after the headline measurement: the same
    Thacker workload in FP32, the watershed window in both precisions, the
    batched ensemble, and a short serving window."""
    out = {}

    def fp32():
        d = sc.to_domain("fp32", stream=stream.cuda_stream)
        try:
            d.set_clock(sim_duration=1e300, print_interval=1e300, print_observation=1e300, it_print=0,
                        time_series=0)
            tune32 = d.autotune(trial_steps=8)
            d.advance(args.warmup)
            (n, _), ms = _timed(stream, lambda: d.advance(args.steps))
        finally:
            d.close()
        v32 = sc.interior_cells * n / (ms / 1000.0)
        return {"value": v32, "unit": "cell-updates/s", "ms_per_step": ms / n, "vs_fp64": v32 / value64,
                "flux_launch_shape": {k: tune32[k] for k in ("variant", "rows_per_tile")}}
    _form(out, "fp32", fp32)
    if args.ws_n > 0:
        _form(out, "watershed", lambda: form_watershed(args, stream))
    if args.ens_members > 0:
        _form(out, "ensemble", lambda: form_ensemble(args, stream))
    if args.form_serve_seconds > 0:
        _form(out, "serving", lambda: form_serving(args))
    return out


def serve_arm(args):
    """Serving workload: Poisson arrivals of flood scenarios (side
    log-uniform 512..4096, 0.5-6 h simulated, terrain/roughness/rain as the
    ensemble workload, 20 % FP64 / 80 % FP32) admitted under a 150 GB HBM
    budget.  Reports scenarios/hour, cell-updates/s and p50/p99 solve latency
    (arrival to result) of the requests completed before the wall limit."""
    import torch
    from triton_b200.serving import Server, poisson_requests, summary
    torch.cuda.set_device(0)
    reqs = poisson_requests(rate=args.serve_rate, seconds=args.serve_seconds, seed=7)
    limit = args.serve_max_wall or 2.0 * args.serve_seconds
    srv = Server(hbm_budget=150e9, chunk_steps=32)
    sampler = ClockSampler(os.environ.get("CUDA_VISIBLE_DEVICES", "0").split(",")[0])
    sampler.start()
    t0 = time.perf_counter()
    srv.run(reqs, deadline=limit)
    wall = time.perf_counter() - t0
    clocks = sampler.stop()
    s = summary(reqs, wall)
    line = {"metric": "scenarios/hour", "value": s["scenarios_per_hour"], "unit": "scenarios/hour", "n_gpus": 1,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic", "impl": "ours",
            "config": {"workload": f"Poisson arrivals {args.serve_rate}/s for {args.serve_seconds:.0f} s, side "
                                   "log-uniform 512..4096, 0.5-6 h simulated, 20% FP64 / 80% FP32, "
                                   "150 GB HBM admission budget", "wall_limit_s": limit},
            "serving": dict(s, peak_hbm_used_bytes=srv.peak_used, chunks=srv.chunks,
                            unfinished=sum(r.finished is None for r in reqs),
                            cell_updates_per_s_all_work=srv.cell_updates / wall),
            "clocks": clocks}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="thacker")
    ap.add_argument("--n", type=int, default=0, help="grid side (default: the workload's full size)")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--shape", default="", help="flux kernel launch shape 'variant:rows_per_tile' (skips autotune)")
    ap.add_argument("--no-forms", action="store_true",
                    help="skip the other forms (FP32, watershed window, ensemble, serving window)")
    ap.add_argument("--ws-n", type=int, default=8192, help="forms: watershed side (0: skip)")
    ap.add_argument("--ws-steps", type=int, default=200, help="forms: watershed window steps")
    ap.add_argument("--ens-members", type=int, default=256, help="forms: ensemble members (0: skip)")
    ap.add_argument("--ens-max-side", type=int, default=2048)
    ap.add_argument("--ens-steps", type=int, default=100)
    ap.add_argument("--form-serve-rate", type=float, default=0.15, help="forms: serving window arrival rate (1/s)")
    ap.add_argument("--form-serve-seconds", type=float, default=60.0, help="forms: serving window (s; 0: skip)")
    ap.add_argument("--form-serve-max-wall", type=float, default=150.0, help="forms: serving window wall limit (s)")
    ap.add_argument("--serve-seconds", type=float, default=600.0, help="serve: arrival window (s)")
    ap.add_argument("--serve-rate", type=float, default=2.0, help="serve: Poisson arrival rate (1/s)")
    ap.add_argument("--serve-max-wall", type=float, default=0.0, help="serve: stop after this many s (0: window x 2)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank, world, local = ranks()
    if args.workload == "serve":
        if rank == 0:
            serve_arm(args)
        return
    sc, desc = workload(args.workload, args.n)

    if args.impl == "reference":
        if rank == 0:
            reference_arm(args, sc, desc)
        return

    import torch

    from triton_b200 import Domain  # noqa: F401  (fails loudly if the library is missing)

    torch.cuda.set_device(local)
    init_ranks(world, "nccl")

    stream = torch.cuda.current_stream()
    d = sc.to_domain(args.precision, stream=stream.cuda_stream)
    # no events inside the measured steps: the loop never stops to print
    d.set_clock(sim_duration=1e300, print_interval=1e300, print_observation=1e300, it_print=0, time_series=0)
    if args.shape:
        v, rb = (int(x) for x in args.shape.split(":"))
        d.set_shape(v, rb)
        tuning = {"variant": v, "rows_per_tile": rb, "source": "--shape"}
    else:
        tuning = d.autotune(trial_steps=8)
    n, _ = d.advance(args.warmup)
    assert n == args.warmup
    barrier(world)
    torch.cuda.synchronize()
    sampler = ClockSampler(local if "CUDA_VISIBLE_DEVICES" not in os.environ
                           else os.environ["CUDA_VISIBLE_DEVICES"].split(",")[local])
    sampler.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    n, ev = d.advance(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    assert n == args.steps, (n, ev)
    ms = e0.elapsed_time(e1)
    # per-launch durations for the roofline: the same number of steps again
    # with a CUDA event pair around every flux and wet-dry launch.  An event
    # between two kernels costs a few microseconds of step time, so the
    # timed region above carries events only at its two ends.
    d.set_timing(True)
    n_r, ev = d.advance(args.steps)
    torch.cuda.synchronize()
    barrier(world)
    clocks = sampler.stop()
    assert n_r == args.steps, (n_r, ev)
    flux_ms, flux_n, wet_ms, wet_n = d.get_timing()
    flux_cells, wet_cells = d.get_work()  # interior cells the launches computed (dry tiles skipped)
    d.set_timing(False)
    ms_max = max_over_ranks(ms, world, "cuda")
    cells = sc.interior_cells
    value = cells * args.steps * world / (ms_max / 1000.0)

    # end to end through the public API from pinned host buffers: upload the
    # initial fields, run the same number of steps, read the result back
    import numpy as np
    host = {k: torch.from_numpy(np.ascontiguousarray(getattr(sc, k), dtype=np.float64)).pin_memory()
            for k in ("h", "qx", "qy", "z", "n2")}
    outs = {k: torch.empty(sc.rows * sc.cols, dtype=torch.float64).pin_memory() for k in ("h", "qx", "qy", "maxh")}
    d2 = sc.to_domain(args.precision, stream=stream.cuda_stream)
    quiet = dict(sim_duration=1e300, print_interval=1e300, print_observation=1e300, it_print=0, time_series=0)
    d2.set_clock(**quiet)
    d2.set_shape(tuning["variant"], tuning["rows_per_tile"])  # the launch shape the device-timed run used
    d2.advance(args.warmup)  # a domain that has stepped before (its step graph exists), as a served one has
    import ctypes as C

    from triton_b200 import _abi
    L = _abi.lib()
    fid = {"h": 0, "qx": 1, "qy": 2, "n2": 3, "z": 4, "maxh": 5}
    barrier(world)
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    # a new job: terrain, roughness and initial state from host memory, max
    # depth started from the initial depth on the device, the clock reset
    for k in ("z", "n2", "h", "qx", "qy"):
        _abi.check(L.tri_domain_upload(d2._h, fid[k], C.cast(host[k].data_ptr(), _abi._dp), sc.rows * sc.cols))
    _abi.check(L.tri_domain_init_max_depth(d2._h))
    d2.set_clock(**dict(sc.clock(), **quiet))
    n2_, _ = d2.advance(args.steps)
    for k in ("h", "qx", "qy", "maxh"):
        _abi.check(L.tri_domain_download(d2._h, fid[k], C.cast(outs[k].data_ptr(), _abi._dp), sc.rows * sc.cols))
    f1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    ems = f0.elapsed_time(f1)
    e2e_val = cells * n2_ * world / (max_over_ranks(ems, world, "cuda") / 1000.0)
    h2d = 5 * sc.rows * sc.cols * 8
    d2h = 4 * sc.rows * sc.cols * 8
    d2.close()

    peak, peak_kind = _peaks()
    flux_avg_s = (flux_ms / max(flux_n, 1)) / 1000.0
    # algorithmic bytes of the cells one launch computed (a skipped dry tile
    # moves nothing), and the same over every interior cell for comparison
    flux_cells_launch = flux_cells / max(flux_n, 1)
    achieved = ALG_BYTES_FLUX[args.precision] * flux_cells_launch / flux_avg_s / 1e9
    achieved_all = ALG_BYTES_FLUX[args.precision] * cells / flux_avg_s / 1e9
    tpc = _traffic_per_cell("flux_update", args.precision)
    step_gbs = ALG_BYTES_STEP[args.precision] * cells * args.steps / (ms / 1000.0) / 1e9

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cores, logical = host_cores()
        r = run_reference(sc, 60, cores)
        if r is not None:
            cpu = {"value": r[0], "unit": "cell-updates/s", "cores": cores, "kind": "reference",
                   "sample": f"{r[1]} time steps of the same workload, reference OpenMP build ({r[2]:.2f} s "
                             f"compute), {cores} threads on {cores} physical cores ({logical} logical CPUs)"}

    forms = None
    if rank == 0 and world == 1 and not args.no_forms and args.precision == "fp64":
        forms = measure_forms(args, sc, stream, value)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32",
            "data": "synthetic",
            "config": dict(workload_config(sc, desc, args.precision, world),
                           l2="inputs larger than L2 (state ~%d MB per GPU)" % (
                               sc.rows * sc.cols * (72 if args.precision == "fp64" else 36) // 2 ** 20),
                           flux_launch_shape=tuning),
            "roofline": {"bound": "hbm", "kernel": "k_flux_update", "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak,
                         "traffic": (tpc * cells) if tpc is not None else None,
                         "algorithmic_bytes_per_launch": ALG_BYTES_FLUX[args.precision] * flux_cells_launch,
                         "computed_cell_frac": flux_cells_launch / cells,
                         "achieved_all_cells": achieved_all,
                         "wetdry_computed_cell_frac": wet_cells / max(wet_n, 1) / cells,
                         "avg_launch_ms": flux_avg_s * 1000.0, "peak_source": f"MEASURED_PEAKS.json hbm_gbs "
                                                                               f"({peak_kind})",
                         "step_achieved_gbs": step_gbs, "step_frac": step_gbs / peak,
                         "wetdry_dt_avg_launch_ms": wet_ms / max(wet_n, 1),
                         "issue_bound": _issue_bound(args.precision),
                         "fp64_pipe": _fp64_pipe(args.precision, flux_avg_s, (clocks or {}).get("sm_mhz")),
                         "launch_timing": f"CUDA event pair around each of {flux_n} flux launches, in a "
                                          f"second pass of the same {args.steps} steps right after the "
                                          f"timed region"},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_val, "unit": "cell-updates/s", "h2d_bytes_per_step": h2d / max(n2_, 1),
                    "d2h_bytes_per_step": d2h / max(n2_, 1)},
            "gpu_launches": 3 * args.steps,
            "clocks": clocks,
        }
        if forms is not None:
            line["forms"] = forms
        print(json.dumps(line))
    d.close()
    close_ranks(world)


if __name__ == "__main__":
    main()
