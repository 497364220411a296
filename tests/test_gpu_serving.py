"""The request loop (continuous batching under an HBM budget): every result
equals the same scenario solved alone, bit for bit (tolerance 0), whatever
else shared its batches while it ran."""
from __future__ import annotations

import numpy as np
import pytest

from triton_b200 import scenarios
from triton_b200.domain import Domain
from triton_b200.serving import Request, Server, poisson_requests, summary


def _spec(i):
    rng = np.random.default_rng(100 + i)
    return dict(n=int(rng.integers(40, 110)), dx=float(rng.uniform(5, 20)), seed=int(rng.integers(1 << 30)),
                duration=float(rng.uniform(300, 900)), rain_mm_h=float(rng.uniform(30, 150)), rain_hours=0.1,
                manning_median=0.035 * (1 + float(rng.uniform(-0.3, 0.3))), nsrc=0)


def _solo(kw, prec):
    sc = scenarios.watershed(**kw)
    d = sc.to_domain(prec)
    try:
        d.set_clock(print_interval=sc.sim_duration, print_observation=sc.sim_duration, time_series=0,
                    it_print=1 << 30)
        d.run()
        return {f: d.download(f) for f in ("h", "qx", "qy", "maxh")}, d.get_clock().it_count
    finally:
        d.close()


@pytest.mark.gpu
def test_served_results_equal_solo_runs():
    specs = [_spec(i) for i in range(8)]
    precs = ["fp32", "fp64", "fp32", "fp32", "fp64", "fp32", "fp32", "fp64"]
    reqs = [Request(rid=i, arrival=0.02 * i, precision=p, build=(lambda kw=kw: scenarios.watershed(**kw)),
                    keep=("h", "qx", "qy", "maxh")) for i, (kw, p) in enumerate(zip(specs, precs))]
    # a budget of about three scenarios: later requests wait for memory
    fp = sorted(Domain.footprint(kw["n"] + 2, kw["n"] + 2, p) for kw, p in zip(specs, precs))
    srv = Server(hbm_budget=fp[-1] + fp[-2] + fp[-3], chunk_steps=16)
    srv.run(reqs)
    assert all(r.finished is not None for r in reqs)
    assert srv.peak_used <= srv.budget
    # the loop really mixed them: some request was admitted while others ran
    assert any(r.admitted > min(q.admitted for q in reqs) for r in reqs)
    for r, kw, p in zip(reqs, specs, precs):
        fields, it = _solo(kw, p)
        assert r.steps == it, f"request {r.rid}: {r.steps} steps served, {it} alone"
        for f, ref in fields.items():
            assert np.array_equal(r.result[f], ref), f"request {r.rid} ({p}): {f} differs from the solo run"
    s = summary(reqs, 1.0)
    assert s["completed"] == len(reqs) and s["fp64"] == 3


def test_poisson_requests_shape():
    reqs = poisson_requests(rate=2.0, seconds=300.0, seed=3, gpu_noise=False)
    assert 450 < len(reqs) < 750
    arr = np.array([r.arrival for r in reqs])
    assert np.all(np.diff(arr) > 0) and arr[-1] <= 300.0
    sides = np.array([r.rows - 2 for r in reqs])
    assert sides.min() >= 512 and sides.max() <= 4096
    share = np.mean([r.precision == "fp64" for r in reqs])
    assert 0.12 < share < 0.28
