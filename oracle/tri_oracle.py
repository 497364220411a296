"""ctypes wrapper of the CPU oracle (oracle/tri_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
``bench.py``'s cpu_baseline leg as the checker.  The product never imports it.

``OracleSim`` owns numpy copies of a padded grid (rows x cols including the
ghost ring, row 0 = north, as the reference's device arrays,
triton_init.h:1452-1591) and drives ``tor_advance``, the restatement of
``triton<T>::simulate`` (triton_simulate.h:12-346).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libtri_oracle.so")

EV_END, EV_PRINT, EV_OBS, EV_LOG = 1, 2, 4, 8

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


class _TorSim(C.Structure):
    _fields_ = [
        ("rows", C.c_int32), ("cols", C.c_int32),
        ("dx", C.c_double), ("courant", C.c_double), ("hextra", C.c_double),
        ("open_boundaries", C.c_int32),
        ("h", _dp), ("qx", _dp), ("qy", _dp), ("z", _dp), ("n2", _dp), ("maxh", _dp),
        ("sqrth", _dp), ("dtv", _dp), ("rhsh0", _dp), ("rhsh1", _dp), ("rhsqx0", _dp),
        ("rhsqx1", _dp), ("rhsqy0", _dp), ("rhsqy1", _dp),
        ("nroff", C.c_int32), ("roff_rows", C.c_int32), ("runoff_id", _ip),
        ("roff_t", _dp), ("roff_v", _dp),
        ("nsrc", C.c_int32), ("hyg_rows", C.c_int32), ("src_idx", _ip),
        ("hyg_t", _dp), ("hyg_v", _dp),
        ("nbc", C.c_int32), ("bc_idx", _ip), ("bc_type", _ip), ("bc_start", _ip),
        ("bc_nrows", _ip), ("bc_v1", _dp), ("bc_v2", _dp),
        ("simtime", C.c_double), ("sim_duration", C.c_double), ("print_interval", C.c_double),
        ("print_observation", C.c_double), ("last_obs_time", C.c_double),
        ("init_dt", C.c_double), ("time_step", C.c_double), ("global_dt", C.c_double),
        ("average_dt", C.c_double),
        ("print_id", C.c_int32), ("it_count", C.c_int32), ("it_count_average", C.c_int32),
        ("it_print", C.c_int32), ("time_series", C.c_int32), ("time_increment_fixed", C.c_int32),
        ("runoff_row", C.c_int32), ("src_idx_low", C.c_int32),
    ]


_lib = None


def build():
    """Compile the oracle library (gcc, no FMA contraction)."""
    subprocess.run(["make", "-s", "-C", _HERE, "oracle"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = C.CDLL(_LIB_PATH)
        _lib.tor_advance.argtypes = [C.POINTER(_TorSim), C.c_int, C.POINTER(C.c_int32)]
        _lib.tor_advance.restype = C.c_int
        _lib.tor_step.argtypes = [C.POINTER(_TorSim)]
        _lib.tor_find_min_dt.restype = C.c_double
        _lib.tor_find_min_dt.argtypes = [C.c_int, _dp]
    return _lib


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


class OracleSim:
    """One single-rank simulation on the CPU oracle.

    ``fields`` holds padded float64 arrays h, qx, qy, z, n2 (Manning squared)
    and maxh; optional forcing tables mirror the flattened host tables the
    reference builds in triton_init.h (sources :723-816, runoff :1299-1357,
    external boundaries :913-1055).
    """

    def __init__(self, rows, cols, dx, courant, hextra, h, qx, qy, z, n2, maxh=None,
                 open_boundaries=0, runoff=None, sources=None, extbc=None, clock=None):
        self.rows, self.cols = int(rows), int(cols)
        n = self.rows * self.cols
        c = lambda a, dt=np.float64: np.ascontiguousarray(np.asarray(a, dtype=dt).reshape(-1)).copy()
        self.h, self.qx, self.qy, self.z, self.n2 = c(h), c(qx), c(qy), c(z), c(n2)
        self.maxh = c(h if maxh is None else maxh)
        for a in (self.h, self.qx, self.qy, self.z, self.n2, self.maxh):
            assert a.size == n
        self._scratch = [np.zeros(n) for _ in range(8)]
        s = _TorSim()
        s.rows, s.cols, s.dx, s.courant, s.hextra = self.rows, self.cols, dx, courant, hextra
        s.open_boundaries = int(open_boundaries)
        s.h, s.qx, s.qy, s.z, s.n2, s.maxh = map(_d, (self.h, self.qx, self.qy, self.z, self.n2, self.maxh))
        (s.sqrth, s.dtv, s.rhsh0, s.rhsh1, s.rhsqx0, s.rhsqx1, s.rhsqy0, s.rhsqy1) = map(_d, self._scratch)
        self._keep = []
        if runoff is not None:
            rid = c(runoff["zone"], np.int32)
            rt, rv = c(runoff["times"]), c(runoff["rates"])
            self._keep += [rid, rt, rv]
            s.nroff, s.roff_rows = int(runoff["nzones"]), rt.size
            s.runoff_id, s.roff_t, s.roff_v = _i(rid), _d(rt), _d(rv)
            s.runoff_row = int(runoff.get("row", 0))
        if sources is not None and len(sources["cells"]) > 0:
            si, ht, hv = c(sources["cells"], np.int32), c(sources["times"]), c(sources["flows"])
            self._keep += [si, ht, hv]
            s.nsrc, s.hyg_rows = si.size, ht.size
            s.src_idx, s.hyg_t, s.hyg_v = _i(si), _d(ht), _d(hv)
        if extbc is not None and len(extbc["cells"]) > 0:
            arrs = [c(extbc[k], np.int32) for k in ("cells", "types", "start", "nrows")]
            v1, v2 = c(extbc["var1"]), c(extbc["var2"])
            self._keep += arrs + [v1, v2]
            s.nbc = arrs[0].size
            s.bc_idx, s.bc_type, s.bc_start, s.bc_nrows = map(_i, arrs)
            s.bc_v1, s.bc_v2 = _d(v1), _d(v2)
        clock = dict(clock or {})
        s.simtime = clock.get("simtime", 0.0)
        s.sim_duration = clock.get("sim_duration", 1e300)
        s.print_interval = clock.get("print_interval", 1e300)
        s.print_observation = clock.get("print_observation", 1e300)
        s.last_obs_time = clock.get("last_obs_time", s.simtime)
        s.init_dt = clock.get("init_dt", 0.01)
        s.time_step = clock.get("time_step", 0.01)
        s.global_dt = clock.get("time_step", 0.01)
        s.average_dt = 0.0
        s.print_id = clock.get("print_id", 0)
        s.it_count = clock.get("it_count", 0)
        s.it_print = clock.get("it_print", 0)
        s.time_series = clock.get("time_series", 0)
        s.time_increment_fixed = clock.get("time_increment_fixed", 0)
        self.s = s

    def advance(self, max_steps):
        ev = C.c_int32(0)
        n = lib().tor_advance(C.byref(self.s), int(max_steps), C.byref(ev))
        return n, ev.value

    def step(self):
        lib().tor_step(C.byref(self.s))

    def grid(self, name):
        return getattr(self, name).reshape(self.rows, self.cols)
