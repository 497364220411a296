"""Python handle on one simulation domain of the C ABI (tri_domain_*).

A ``Domain`` owns the device state of one TRITON simulation: the padded
rows x cols fields (ghost ring included, row 0 = north, Manning squared, the
reference's layout from triton_init.h:1452-1591), the forcing tables and the
loop clock of ``triton<T>::simulate`` (triton_simulate.h:41-52).  ``advance``
runs time steps on the GPU until the next event; ``run`` mirrors the
reference loop and reacts to the events as it does (triton_simulate.h:54-134).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from ._abi import check, lib

FIELDS = {"h": _abi.FIELD_H, "qx": _abi.FIELD_QX, "qy": _abi.FIELD_QY, "n2": _abi.FIELD_NMAN2,
          "z": _abi.FIELD_DEM, "maxh": _abi.FIELD_MAXH}


def _f64(a, n):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1))
    if a.size != n:
        raise ValueError(f"field has {a.size} values, grid has {n}")
    return a


class Domain:
    def __init__(self, rows, cols, dx, courant=0.5, hextra=0.001, open_boundaries=0, precision="fp64",
                 stream=None):
        self.rows, self.cols = int(rows), int(cols)
        self.n = self.rows * self.cols
        self.dx = float(dx)
        prec = {"fp64": _abi.TRI_FP64, "fp32": _abi.TRI_FP32}[precision]
        self.precision = precision
        self.desc = _abi.GridDesc(self.rows, self.cols, self.dx, float(courant), float(hextra),
                                  int(open_boundaries), prec)
        h = C.c_void_p()
        check(lib().tri_domain_create(C.byref(self.desc), C.c_void_p(stream) if stream else None, C.byref(h)))
        self._h = h
        self._keep = []

    # -- lifetime -------------------------------------------------------------
    def close(self):
        if self._h:
            lib().tri_domain_destroy(self._h)
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

    @staticmethod
    def footprint(rows, cols, precision="fp64"):
        d = _abi.GridDesc(int(rows), int(cols), 1.0, 0.5, 0.001, 0,
                          {"fp64": _abi.TRI_FP64, "fp32": _abi.TRI_FP32}[precision])
        b = C.c_int64()
        check(lib().tri_domain_footprint(C.byref(d), C.byref(b)))
        return b.value

    # -- fields ---------------------------------------------------------------
    def upload(self, name, values):
        a = _f64(values, self.n)
        check(lib().tri_domain_upload(self._h, FIELDS[name], a.ctypes.data_as(_abi._dp), self.n))

    def download(self, name):
        a = np.empty(self.n, dtype=np.float64)
        check(lib().tri_domain_download(self._h, FIELDS[name], a.ctypes.data_as(_abi._dp), self.n))
        return a.reshape(self.rows, self.cols)

    def set_state(self, h, qx, qy, z, n2, maxh=None):
        self.upload("z", z)
        self.upload("n2", n2)
        self.upload("h", h)
        self.upload("qx", qx)
        self.upload("qy", qy)
        self.upload("maxh", h if maxh is None else maxh)

    # -- forcing --------------------------------------------------------------
    def set_runoff(self, zone, times, rates, nzones):
        zone = np.ascontiguousarray(np.asarray(zone, dtype=np.int32).reshape(-1))
        t = np.ascontiguousarray(times, dtype=np.float64)
        r = np.ascontiguousarray(rates, dtype=np.float64).reshape(-1)
        self._keep = [zone, t, r]
        check(lib().tri_domain_set_runoff(self._h, int(nzones), t.size, t.ctypes.data_as(_abi._dp),
                                          r.ctypes.data_as(_abi._dp), zone.ctypes.data_as(_abi._ip), zone.size))

    def set_sources(self, cells, times, flows):
        cells = np.ascontiguousarray(cells, dtype=np.int32)
        t = np.ascontiguousarray(times, dtype=np.float64)
        f = np.ascontiguousarray(flows, dtype=np.float64).reshape(-1)
        check(lib().tri_domain_set_sources(self._h, cells.size, cells.ctypes.data_as(_abi._ip), t.size,
                                           t.ctypes.data_as(_abi._dp), f.ctypes.data_as(_abi._dp)))

    def set_extbc(self, cells, types, start, nrows, var1, var2):
        a = [np.ascontiguousarray(x, dtype=np.int32) for x in (cells, types, start, nrows)]
        v1 = np.ascontiguousarray(var1, dtype=np.float64)
        v2 = np.ascontiguousarray(var2, dtype=np.float64)
        check(lib().tri_domain_set_extbc(self._h, a[0].size, *[x.ctypes.data_as(_abi._ip) for x in a], v1.size,
                                         v1.ctypes.data_as(_abi._dp), v2.ctypes.data_as(_abi._dp)))

    def set_observations(self, cells):
        cells = np.ascontiguousarray(cells, dtype=np.int32)
        self.nobs = cells.size
        check(lib().tri_domain_set_observations(self._h, cells.size, cells.ctypes.data_as(_abi._ip)))

    # -- clock and stepping ---------------------------------------------------
    def set_clock(self, **kw):
        c = self.get_clock()
        for k, v in kw.items():
            setattr(c, k, v)
        check(lib().tri_domain_set_clock(self._h, C.byref(c)))

    def get_clock(self):
        c = _abi.Clock()
        check(lib().tri_domain_get_clock(self._h, C.byref(c)))
        return c

    def advance(self, max_steps):
        p = _abi.Progress()
        check(lib().tri_domain_advance(self._h, int(max_steps), C.byref(p)))
        return p.steps, p.events

    def compute_dt(self):
        v = C.c_double()
        check(lib().tri_domain_compute_dt(self._h, C.byref(v)))
        return v.value

    def observe(self):
        n = getattr(self, "nobs", 0)
        h, qx, qy = (np.empty(n) for _ in range(3))
        if n:
            check(lib().tri_domain_observe(self._h, h.ctypes.data_as(_abi._dp), qx.ctypes.data_as(_abi._dp),
                                           qy.ctypes.data_as(_abi._dp)))
        return h, qx, qy

    def volume(self):
        v = C.c_double()
        check(lib().tri_domain_volume(self._h, C.byref(v)))
        return v.value

    def mass_balance(self):
        """(volume, inflow_boundary, sources, runoff, extbc, clipping) in m^3."""
        out = np.zeros(6)
        check(lib().tri_domain_mass_balance(self._h, out.ctypes.data_as(_abi._dp)))
        return dict(zip(("volume", "boundary", "sources", "runoff", "extbc", "clipping"), out.tolist()))

    def track_arrival(self, depth=0.1):
        check(lib().tri_domain_track_arrival(self._h, float(depth)))

    def arrival(self):
        a = np.empty(self.n)
        check(lib().tri_domain_download_arrival(self._h, a.ctypes.data_as(_abi._dp), self.n))
        return a.reshape(self.rows, self.cols)

    def synchronize(self):
        check(lib().tri_domain_synchronize(self._h))

    def set_timing(self, on):
        check(lib().tri_domain_set_timing(self._h, int(bool(on))))

    def get_timing(self):
        a, b = C.c_double(), C.c_double()
        na, nb = C.c_int32(), C.c_int32()
        check(lib().tri_domain_get_timing(self._h, C.byref(a), C.byref(na), C.byref(b), C.byref(nb)))
        return a.value, na.value, b.value, nb.value

    def get_work(self):
        """(flux cells, wet-dry cells) computed since set_timing: interior
        cells of the tiles that were not skipped as dry."""
        a, b = C.c_int64(), C.c_int64()
        check(lib().tri_domain_get_work(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def autotune(self, trial_steps=10):
        """Times every flux-kernel launch shape on this domain's own state and
        keeps the fastest; the state and clock are restored afterwards."""
        t = _abi.Tuning()
        check(lib().tri_domain_autotune(self._h, int(trial_steps), C.byref(t)))
        return dict(variant=t.variant, rows_per_tile=t.rows_per_tile, candidates=t.candidates,
                    flux_blocks=t.flux_blocks, ms_per_step=t.ms_per_step)

    def set_shape(self, variant, rows_per_tile):
        check(lib().tri_domain_set_tuning(self._h, int(variant), int(rows_per_tile)))

    def run(self, on_event=None, max_chunk=1 << 30):
        """Run to sim_duration reacting to events like triton_simulate.h:54-134.

        ``on_event(domain, events)`` is called after every event, before the
        clock bookkeeping (observation time, print id, dt average reset) is
        applied, which is where the reference writes its outputs.  Returns the
        number of steps run."""
        total = 0
        while True:
            n, ev = self.advance(max_chunk)
            total += n
            if ev and on_event is not None:
                on_event(self, ev)
            c = self.get_clock()
            if ev & _abi.EV_LOG:
                c.average_dt = 0.0
            if ev & _abi.EV_OBS:
                c.last_obs_time += c.print_observation
            if ev & _abi.EV_PRINT:
                c.print_id += 1
            check(lib().tri_domain_set_clock(self._h, C.byref(c)))
            if ev & _abi.EV_END or (n == 0 and ev == 0):
                return total
