"""Shared helpers for the parity tests: run a Scenario on the CPU oracle and
on the GPU domain path side by side, event by event."""
from __future__ import annotations

import numpy as np

EV_END, EV_PRINT, EV_OBS, EV_LOG = 1, 2, 4, 8

# Plain-form parity bound: values within 1e-9 of the field's scale, wet/dry
# masks equal.  Cases without cube roots (no friction, no type-2 boundary)
# must match bit for bit.
REL_TOL = 1e-9


def oracle_from_scenario(sc):
    from oracle.tri_oracle import OracleSim
    return OracleSim(sc.rows, sc.cols, sc.dx, sc.courant, sc.hextra, sc.h, sc.qx, sc.qy, sc.z, sc.n2,
                     open_boundaries=sc.open_boundaries, runoff=sc.runoff, sources=sc.sources, extbc=sc.extbc,
                     clock=sc.clock())


def oracle_bookkeeping(o, ev):
    s = o.s
    if ev & EV_LOG:
        s.it_count_average = 0
        s.average_dt = 0.0
    if ev & EV_OBS:
        s.last_obs_time += s.print_observation
    if ev & EV_PRINT:
        s.print_id += 1


def domain_bookkeeping(d, ev):
    c = d.get_clock()
    kw = {}
    if ev & EV_LOG:
        kw["average_dt"] = 0.0
    if ev & EV_OBS:
        kw["last_obs_time"] = c.last_obs_time + c.print_observation
    if ev & EV_PRINT:
        kw["print_id"] = c.print_id + 1
    if kw:
        d.set_clock(**kw)


def compare_fields(o, d, exact, hextra, where=""):
    out = {}
    for name in ("h", "qx", "qy", "maxh"):
        a = d.download(name)
        b = o.grid(name)
        if exact:
            bad = ~((a == b) | (np.isnan(a) & np.isnan(b)))
            if bad.any():
                i = np.argwhere(bad)[0]
                raise AssertionError(f"{where}{name} differs at {tuple(i)}: gpu {a[tuple(i)]!r} oracle "
                                     f"{b[tuple(i)]!r} ({bad.sum()} cells)")
        else:
            scale = max(np.abs(b).max(), 1e-300)
            err = np.abs(a - b).max() / scale
            out[name] = err
            assert err <= REL_TOL, f"{where}{name}: max |gpu-oracle|/max|oracle| = {err:.3e} > {REL_TOL}"
    ha, hb = d.download("h"), o.grid("h")
    assert np.array_equal(ha > hextra, hb > hextra), f"{where}wet mask (h > hextra) differs"
    return out


def run_lockstep(sc, precision="fp64", exact=True, max_events=10 ** 6, chunk=10 ** 6, check_every_event=True):
    """Run both engines to sim_duration, comparing at every event.  Returns
    (steps, number of events)."""
    o = oracle_from_scenario(sc)
    d = sc.to_domain(precision)
    steps, nev = 0, 0
    try:
        while nev < max_events:
            n1, e1 = o.advance(chunk)
            n2, e2 = d.advance(chunk)
            assert (n1, e1) == (n2, e2), f"oracle ran {n1} steps (events {e1}), gpu {n2} (events {e2})"
            c = d.get_clock()
            assert c.it_count == o.s.it_count
            if exact:
                assert c.simtime == o.s.simtime, f"simtime gpu {c.simtime!r} oracle {o.s.simtime!r}"
                assert c.average_dt == o.s.average_dt
            else:  # dt follows the state, which may differ in the last bits (cbrt)
                assert abs(c.simtime - o.s.simtime) <= REL_TOL * max(abs(o.s.simtime), 1.0)
                assert abs(c.average_dt - o.s.average_dt) <= REL_TOL * max(abs(o.s.average_dt), 1e-3)
            steps += n1
            nev += 1
            if check_every_event or e1 & EV_END:
                compare_fields(o, d, exact, sc.hextra, where=f"after {steps} steps: ")
            if sc.obs_cells is not None and e1 & EV_OBS:
                hh, qq, vv = d.observe()
                cells = np.asarray(sc.obs_cells)
                for got, name in ((hh, "h"), (qq, "qx"), (vv, "qy")):
                    ref = getattr(o, name)[cells]
                    if exact:
                        assert np.array_equal(got, ref)
                    else:
                        assert np.allclose(got, ref, rtol=REL_TOL, atol=1e-12)
            oracle_bookkeeping(o, e1)
            domain_bookkeeping(d, e2)
            if e1 & EV_END or n1 == 0:
                break
    finally:
        d.close()
    return steps, nev
