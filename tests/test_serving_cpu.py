"""The serving loop's control logic on CPU: stand-ins replace the GPU domains
and batches (a stand-in batch advances each member's clock by its dt per
step), so admission by footprint under the HBM budget, arrival order,
retirement at the end time, freeing of memory and the deadline are checked
without a GPU.  The GPU test checks the numbers the real batches compute."""
from __future__ import annotations

import types

import pytest

from triton_b200 import serving


class _Clock:
    def __init__(self, duration):
        self.simtime, self.sim_duration, self.it_count = 0.0, duration, 0


class _Domain:
    live = 0
    peak = 0

    def __init__(self, n, duration, dt):
        self.rows = self.cols = n + 2
        self.c, self.dt, self.closed = _Clock(duration), dt, False
        _Domain.live += 1
        _Domain.peak = max(_Domain.peak, _Domain.live)

    def set_clock(self, **kw):
        pass

    def get_clock(self):
        return self.c

    def volume(self):
        return 1.0

    def download(self, name):
        return name

    def close(self):
        if not self.closed:
            self.closed = True
            _Domain.live -= 1


class _Scenario:
    def __init__(self, n, duration, dt):
        self.n, self.duration, self.dt = n, duration, dt
        self.rows = self.cols = n + 2
        self.sim_duration = duration

    def to_domain(self, precision):
        return _Domain(self.n, self.duration, self.dt)


class _Batch:
    def __init__(self, members):
        self.members, self.steps = list(members), 0

    def set_shape(self, variant, rows_per_tile):
        pass

    def set_members(self, members):
        self.members = list(members)

    def launch(self, steps):
        self.steps = steps

    def wait(self):
        updates = 0
        for d in self.members:
            for _ in range(self.steps):
                if d.c.simtime >= d.c.sim_duration:
                    break
                d.c.simtime += d.dt
                d.c.it_count += 1
                updates += (d.rows - 2) * (d.cols - 2)
        self.steps = 0
        return types.SimpleNamespace(cell_updates=updates)

    def close(self):
        pass


@pytest.fixture
def stand_ins(monkeypatch):
    monkeypatch.setattr(serving, "Batch", _Batch)
    monkeypatch.setattr(serving.Domain, "footprint", staticmethod(lambda r, c, p: r * c * (72 if p == "fp64" else 36)))
    _Domain.live = _Domain.peak = 0
    yield


def _requests(k, n=100, duration=40.0, dt=1.0, gap=0.001, precision="fp32"):
    return [serving.Request(rid=i, arrival=i * gap, precision=precision,
                            build=(lambda: _Scenario(n, duration, dt)), rows=n + 2, cols=n + 2) for i in range(k)]


def test_admission_respects_budget_and_order(stand_ins):
    reqs = _requests(7)
    one = 102 * 102 * 36
    srv = serving.Server(hbm_budget=2.5 * one, chunk_steps=8, prefetch=2, build_threads=2)
    done = srv.run(reqs)
    assert all(r.finished is not None for r in done)
    assert _Domain.peak == 2 and _Domain.live == 0          # two fit the budget; all freed
    assert srv.peak_used <= srv.budget and srv.used == 0
    adm = [r.admitted for r in sorted(done, key=lambda r: r.arrival)]
    assert adm == sorted(adm)                                # first come, first admitted
    for r in done:
        assert r.steps == 40 and r.simtime == 40.0 and r.cell_updates == 40 * 100 * 100
        assert r.latency >= 0.0


def test_request_larger_than_budget_is_refused(stand_ins):
    srv = serving.Server(hbm_budget=1000.0)
    with pytest.raises(ValueError, match="exceeds the budget"):
        srv.run(_requests(1))
    assert _Domain.live == 0


def test_deadline_leaves_requests_unfinished_and_frees_them(stand_ins):
    reqs = _requests(3, duration=1e12, dt=1.0)             # never reach their end time
    srv = serving.Server(hbm_budget=1e12, chunk_steps=4, prefetch=0)
    done = srv.run(reqs, deadline=0.05)
    assert all(r.finished is None for r in done)
    assert _Domain.live == 0 and srv.batches == {}
