"""Ensembles of member domains advanced together on one GPU (tri_batch_*).

The reference runs ensemble members as separate groups of MPI ranks
(src/Ensify.h:43-72).  Here the members are ``Domain`` objects sharing one
GPU; ``Batch.advance`` moves every member by its own time steps with one
launch per kernel type for all members.
"""
from __future__ import annotations

import ctypes as C

from . import _abi
from ._abi import check, lib


class Batch:
    def __init__(self, members, stream=None):
        self.members = list(members)
        arr = (C.c_void_p * len(self.members))(*[m._h for m in self.members])
        h = C.c_void_p()
        check(lib().tri_batch_create(len(self.members), arr, stream, C.byref(h)))
        self._h = h

    def close(self):
        if self._h:
            lib().tri_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_members(self, members):
        self.members = list(members)
        arr = (C.c_void_p * max(len(self.members), 1))(*[m._h for m in self.members])
        check(lib().tri_batch_set_members(self._h, len(self.members), arr))

    def advance(self, max_steps):
        """Runs until every member has raised an event or max_steps batched
        steps have run; returns a BatchProgress."""
        p = _abi.BatchProgress()
        check(lib().tri_batch_advance(self._h, int(max_steps), C.byref(p)))
        return p

    def launch(self, steps):
        """Queues `steps` batched steps and returns at once (see wait)."""
        check(lib().tri_batch_launch(self._h, int(steps)))

    def wait(self):
        p = _abi.BatchProgress()
        check(lib().tri_batch_wait(self._h, C.byref(p)))
        return p

    def autotune(self, trial_steps=10):
        t = _abi.Tuning()
        check(lib().tri_batch_autotune(self._h, int(trial_steps), C.byref(t)))
        return dict(variant=t.variant, rows_per_tile=t.rows_per_tile, candidates=t.candidates,
                    flux_blocks=t.flux_blocks, ms_per_step=t.ms_per_step)

    def set_shape(self, variant, rows_per_tile):
        check(lib().tri_batch_set_tuning(self._h, int(variant), int(rows_per_tile)))

    def set_mode(self, single_launch):
        """True: batched steps run in single persistent launches (members
        advance without grid-wide barriers); False: one launch per kernel
        type and step, captured as CUDA graphs (the default)."""
        check(lib().tri_batch_set_mode(self._h, _abi.BATCH_SINGLE_LAUNCH if single_launch else _abi.BATCH_GRAPHS))

    def set_wait_test(self, polls):
        """Single-launch mode test hook: the next advances' first clock item
        waits for a count that is never reached and gives up after `polls`
        polls (TRI_E_TIMEOUT); 0 turns it off."""
        check(lib().tri_batch_set_wait_test(self._h, int(polls)))

    def run(self, on_event=None, max_chunk=1 << 30):
        """Runs every member to its sim_duration.  After each batched advance,
        every member that raised an event gets ``on_event(member, events)``
        and then the same clock bookkeeping as ``Domain.run`` (observation
        time, print id, dt average).  Returns (batched steps, cell updates)."""
        steps = updates = 0
        while True:
            p = self.advance(max_chunk)
            steps += p.steps
            updates += p.cell_updates
            for m in self.members:
                c = m.get_clock()
                ev = c.last_events
                if not ev:
                    continue
                if on_event is not None:
                    on_event(m, ev)
                if ev & _abi.EV_LOG:
                    c.average_dt = 0.0
                if ev & _abi.EV_OBS:
                    c.last_obs_time += c.print_observation
                if ev & _abi.EV_PRINT:
                    c.print_id += 1
                check(lib().tri_domain_set_clock(m._h, C.byref(c)))
            if p.members_ended == len(self.members) or (p.steps == 0 and p.members_with_events == 0):
                return steps, updates
