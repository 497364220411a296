"""Request loop for flood scenarios on one GPU: continuous batching under an
HBM budget.

The reference solves one scenario per run (triton_simulate.h); this loop
keeps many scenarios resident and steps them together.  Requests arrive over
time; each is admitted, in arrival order, as soon as its device footprint
(tri_domain_footprint) fits the HBM budget and its batch has a free slot.
Admitted scenarios of one precision form one tri_batch: every batched step
moves each of them by one of its own time steps, so a request that arrives
while others run joins the next chunk of steps and its work overlaps theirs
on the device.  FP64 and FP32 batches are launched back to back on their own
streams and run concurrently; the host builds and uploads newly arrived
scenarios while the GPU steps (tri_batch_launch / tri_batch_wait).  A
scenario leaves the batch when it reaches its end time; its memory is freed
and the next waiting request can take it.

A member's result does not depend on what else is in its batch: the batched
kernels compute each member exactly as the single-domain path does, so every
result is bit-for-bit the one the scenario gets alone.
"""
from __future__ import annotations

import collections
import concurrent.futures
import time
from dataclasses import dataclass, field
from typing import Callable

import numpy as np

from .batch import Batch
from .domain import Domain

# Default launch shapes of the batched flux kernel (variant, rows per tile).
SHAPES = {"fp64": (1, 16), "fp32": (1, 16)}


@dataclass
class Request:
    rid: int
    arrival: float            # seconds after the loop starts
    precision: str            # "fp64" or "fp32"
    build: Callable           # () -> Scenario (host arrays)
    rows: int = 0             # padded grid, for the footprint (0: from build())
    cols: int = 0
    keep: tuple = ()          # fields to download at the end ("h", "qx", "qy", "maxh")
    # filled by the server
    footprint: int = 0
    admitted: float | None = None
    finished: float | None = None
    steps: int = 0
    simtime: float = 0.0
    cell_updates: int = 0
    volume: float = 0.0
    result: dict = field(default_factory=dict)

    @property
    def latency(self):
        return None if self.finished is None else self.finished - self.arrival


class Server:
    """`prefetch` requests at the head of the waiting queue have their inputs
    built on host threads while the GPU steps (a request carries a builder,
    not arrays; building is the client's work and runs off the loop)."""

    def __init__(self, hbm_budget=150e9, chunk_steps=32, max_members=512, shapes=None, prefetch=6,
                 build_threads=4):
        self.prefetch = int(prefetch)
        self.build_threads = int(build_threads)
        self.budget = float(hbm_budget)
        self.chunk = int(chunk_steps)
        self.max_members = int(max_members)
        self.shapes = dict(SHAPES, **(shapes or {}))
        self.used = 0
        self.peak_used = 0
        self.batches: dict[str, Batch] = {}
        self.live: dict[str, list] = {"fp64": [], "fp32": []}
        self.chunks = 0
        self.cell_updates = 0

    # -- admission ---------------------------------------------------------------
    @staticmethod
    def _ready(r):
        fut = getattr(r, "_future", None)
        return fut is None or fut.done()

    def _fits(self, r):
        if not r.footprint:
            if not r.rows:
                fut = getattr(r, "_future", None)
                sc = fut.result() if fut is not None else r.build()
                r.rows, r.cols = sc.rows, sc.cols
                r._sc, r._future = sc, None
            r.footprint = Domain.footprint(r.rows, r.cols, r.precision)
        if r.footprint > self.budget:
            raise ValueError(f"request {r.rid}: footprint {r.footprint} B exceeds the budget {self.budget:.0f} B")
        return self.used + r.footprint <= self.budget and len(self.live[r.precision]) < self.max_members

    def _admit(self, r, now):
        fut = getattr(r, "_future", None)
        sc = getattr(r, "_sc", None) or (fut.result() if fut is not None else r.build())
        r._sc = None
        r._future = None
        d = sc.to_domain(r.precision)
        # no intermediate outputs: the request wants its final state
        d.set_clock(print_interval=sc.sim_duration, print_observation=sc.sim_duration, time_series=0,
                    it_print=1 << 30)
        self.used += r.footprint
        self.peak_used = max(self.peak_used, self.used)
        r.admitted = now
        r._interior = (sc.rows - 2) * (sc.cols - 2)
        self.live[r.precision].append((r, d))

    def _retire(self, prec, now):
        keep = []
        for r, d in self.live[prec]:
            c = d.get_clock()
            if c.simtime < c.sim_duration:
                keep.append((r, d))
                continue
            r.steps, r.simtime = c.it_count, c.simtime
            r.cell_updates = r.steps * r._interior
            r.volume = d.volume()
            r.result = {f: d.download(f) for f in r.keep}
            d.close()
            self.used -= r.footprint
            r.finished = now
        changed = len(keep) != len(self.live[prec])
        self.live[prec] = keep
        return changed

    def _sync_batch(self, prec):
        doms = [d for _, d in self.live[prec]]
        b = self.batches.get(prec)
        if b is None:
            if not doms:
                return
            b = self.batches[prec] = Batch(doms)
            b.set_shape(*self.shapes[prec])
        else:
            b.set_members(doms)

    # -- loop ------------------------------------------------------------------
    def run(self, requests, clock=time.perf_counter, idle_sleep=0.002, deadline=None):
        """Serves `requests` (arrival times relative to the start) until all
        are done, or until `deadline` seconds after the start (requests not
        finished by then keep finished=None); returns them with admission and
        finish times filled in."""
        pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
        waiting = collections.deque()
        pool = concurrent.futures.ThreadPoolExecutor(max_workers=self.build_threads) if self.prefetch > 0 else None
        t0 = clock()
        now = lambda: clock() - t0  # noqa: E731
        dirty = set()
        try:
            while pending or waiting or any(self.live.values()):
                t = now()
                if deadline is not None and t > deadline:
                    break
                while pending and pending[0].arrival <= t:
                    waiting.append(pending.popleft())
                running = [p for p in ("fp64", "fp32") if self.live[p]]
                for p in running:
                    self.batches[p].launch(self.chunk)
                # inputs of the next waiting requests are built on host threads
                if pool is not None:
                    for r in list(waiting)[:self.prefetch]:
                        if getattr(r, "_future", None) is None and getattr(r, "_sc", None) is None:
                            r._future = pool.submit(r.build)
                # admit while the GPU steps (arrival order, head of line first;
                # a head whose inputs are still being built waits for them)
                while waiting and self._ready(waiting[0]) and self._fits(waiting[0]):
                    r = waiting.popleft()
                    self._admit(r, now())
                    dirty.add(r.precision)
                for p in running:
                    prog = self.batches[p].wait()
                    self.cell_updates += prog.cell_updates
                if running:
                    self.chunks += 1
                for p in running:
                    if self._retire(p, now()):
                        dirty.add(p)
                for p in dirty:
                    self._sync_batch(p)
                dirty.clear()
                if not running and not waiting and pending:
                    time.sleep(min(idle_sleep, max(pending[0].arrival - now(), 0.0)))
                elif not running and waiting:  # inputs still being built
                    time.sleep(idle_sleep)
        finally:
            if pool is not None:
                pool.shutdown(wait=True, cancel_futures=True)
            for p, b in self.batches.items():
                b.close()
            self.batches.clear()
            for p in self.live:
                for _, d in self.live[p]:
                    d.close()
                self.live[p] = []
        return requests


def summary(requests, wall_s):
    done = [r for r in requests if r.finished is not None]
    lat = np.array([r.latency for r in done]) if done else np.zeros(1)
    upd = sum(r.cell_updates for r in done)
    return dict(
        requests=len(requests), completed=len(done),
        p50_latency_s=float(np.percentile(lat, 50)), p99_latency_s=float(np.percentile(lat, 99)),
        mean_latency_s=float(lat.mean()), scenarios_per_hour=len(done) / wall_s * 3600.0,
        cell_updates=int(upd), cell_updates_per_s=upd / wall_s, wall_s=wall_s,
        fp64=sum(r.precision == "fp64" for r in done), fp32=sum(r.precision == "fp32" for r in done))


def poisson_requests(rate=2.0, seconds=600.0, seed=7, side=(512, 4096), hours=(0.5, 6.0), fp64_share=0.2,
                     dx=(5.0, 20.0), rain=(10.0, 100.0), manning_spread=0.3, gpu_noise=True, keep=()):
    """Poisson arrivals of flood scenarios: grid side log-uniform in `side`,
    simulated duration uniform in `hours`, terrain, roughness and rain drawn
    as in the ensemble workload (scenarios.ensemble), `fp64_share` of them in
    FP64 and the rest in FP32."""
    from . import scenarios
    rng = np.random.default_rng(seed)
    t, out, i = 0.0, [], 0
    while True:
        t += rng.exponential(1.0 / rate)
        if t > seconds:
            break
        n = int(np.exp(rng.uniform(np.log(side[0]), np.log(side[1]))))
        kw = dict(n=n, dx=float(rng.uniform(*dx)), seed=int(rng.integers(1 << 31)),
                  duration=float(rng.uniform(*hours)) * 3600.0, rain_mm_h=float(rng.uniform(*rain)),
                  rain_hours=1.0, manning_median=0.035 * (1.0 + float(rng.uniform(-manning_spread, manning_spread))),
                  nsrc=0, gpu_noise=gpu_noise)
        prec = "fp64" if rng.random() < fp64_share else "fp32"
        out.append(Request(rid=i, arrival=t, precision=prec, build=(lambda kw=kw: scenarios.watershed(**kw)),
                           rows=n + 2, cols=n + 2, keep=keep))
        i += 1
    return out
