"""Accuracy report of the FP32 precision form against the FP64 path.

The FP64 GPU path is the reference here: it matches the reference CPU build
bit for bit (or within 1e-9 where CUDA's cube root differs), so it stands in
for the FP64 oracle at sizes the CPU cannot run.  Both forms run the same
scenario for the same simulated time; the report gives

  max / RMS depth error over interior cells (m),
  arrival-time error: first time h exceeds 0.1 m, cells reached in both runs
      (max and RMS, s) plus cells reached in one run only,
  volume error: |V32 - V64| / V64 of the interior volume at the end,
  mass-balance residual of the FP32 run: (V_end - V_0 - sum of the FP64
      accounts) / V_end, the accounts being inflow through boundary faces,
      sources, runoff, external-boundary resets and negative-depth clipping.
"""
from __future__ import annotations

import time

import numpy as np


def run_form(sc, precision, duration=None, arrival_depth=0.1, autotune=False, progress=False, fixed_dt=None):
    d = sc.to_domain(precision)
    try:
        if duration is not None:
            d.set_clock(sim_duration=duration)
        if fixed_dt is not None:  # the same time levels in both forms
            d.set_clock(time_increment_fixed=1, time_step=float(fixed_dt))
        d.set_clock(print_interval=1e300, print_observation=1e300, time_series=0, it_print=0)
        if autotune:
            d.autotune(4)
        d.track_arrival(arrival_depth)
        v0 = d.volume()
        steps = 0
        chunk = 2000 if progress else 1 << 30
        t0 = time.perf_counter()
        while True:
            n, ev = d.advance(chunk)
            steps += n
            if progress:
                print(f"  {precision}: {steps} steps, simtime {d.get_clock().simtime:.1f} s", flush=True)
            if ev & 1 or n == 0:
                break
        wall = time.perf_counter() - t0  # the stepping loop only
        out = dict(h=d.download("h"), arrival=d.arrival(), volume=d.volume(), v0=v0, steps=steps, wall_s=wall,
                   simtime=d.get_clock().simtime, balance=d.mass_balance())
    finally:
        d.close()
    return out


def fp32_bed(sc):
    """A copy of the scenario whose bed is the one the FP32 form computes
    with: per 32x32 tile the lowest interior cell as FP64 base, plus each
    cell's offset from it rounded to FP32.  Running the FP64 path on it
    separates the effect of the bed representation from FP32 arithmetic."""
    import copy
    z = np.asarray(sc.z, dtype=np.float64)
    R, C = z.shape
    tr, tc = (R + 31) // 32, (C + 31) // 32
    base = np.zeros((tr, tc))
    for i in range(tr):
        for j in range(tc):
            r0, r1 = max(32 * i, 1), min(32 * i + 32, R - 1)
            c0, c1 = max(32 * j, 1), min(32 * j + 32, C - 1)
            if r1 > r0 and c1 > c0:
                base[i, j] = z[r0:r1, c0:c1].min()
    b = np.repeat(np.repeat(base, 32, 0), 32, 1)[:R, :C]
    out = copy.copy(sc)
    out.z = b + (z - b).astype(np.float32).astype(np.float64)
    return out


def compare(sc, duration=None, arrival_depth=0.1, fixed_dt=None):
    a = run_form(sc, "fp64", duration, arrival_depth, fixed_dt=fixed_dt)
    b = run_form(sc, "fp32", duration, arrival_depth, fixed_dt=fixed_dt)
    ha, hb = a["h"][1:-1, 1:-1], b["h"][1:-1, 1:-1]
    err = np.abs(hb - ha)
    worst = np.unravel_index(int(np.argmax(err)), err.shape)
    ta, tb = a["arrival"][1:-1, 1:-1], b["arrival"][1:-1, 1:-1]
    both = (ta >= 0) & (tb >= 0)
    terr = np.abs(tb[both] - ta[both])
    bal = b["balance"]
    terms = ("boundary", "sources", "runoff", "extbc", "clipping")
    accounts = sum(bal[k] for k in terms)
    resid = (b["volume"] - b["v0"] - accounts) / max(abs(b["volume"]), 1e-300)
    resid64 = (a["volume"] - a["v0"] - sum(a["balance"][k] for k in terms)) / max(abs(a["volume"]), 1e-300)
    # where the volumes part: each account of the FP32 run minus the FP64 run's
    # (forcing totals differ with the time levels: runoff and sources apply
    # over whole steps, so the step that crosses a table time decides them)
    dacc = {k: b["balance"][k] - a["balance"][k] for k in terms}
    return dict(
        steps_fp64=a["steps"], steps_fp32=b["steps"], simtime=a["simtime"],
        wall_fp64_s=a["wall_s"], wall_fp32_s=b["wall_s"],
        max_depth_error_m=float(err.max()), rms_depth_error_m=float(np.sqrt(np.mean(err ** 2))),
        p999_depth_error_m=float(np.quantile(err, 0.999)),
        cells_over_1mm=int((err > 1e-3).sum()), worst_cell=tuple(int(i) + 1 for i in worst),
        worst_h_fp64=float(ha[worst]), worst_h_fp32=float(hb[worst]),
        arrival_max_error_s=float(terr.max()) if terr.size else 0.0,
        arrival_rms_error_s=float(np.sqrt(np.mean(terr ** 2))) if terr.size else 0.0,
        arrival_cells=int(both.sum()), arrival_mismatch_cells=int(((ta >= 0) != (tb >= 0)).sum()),
        volume_fp64=a["volume"], volume_fp32=b["volume"],
        volume_rel_error=abs(b["volume"] - a["volume"]) / max(abs(a["volume"]), 1e-300),
        mass_balance_residual=float(resid), mass_balance_residual_fp64=float(resid64),
        accounts_fp32=bal, accounts_fp64=a["balance"],
        account_differences=dacc,
    )
