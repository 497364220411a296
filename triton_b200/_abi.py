"""ctypes declarations of the C ABI in include/triton_b200.h.

The shared library is built in-tree (triton_b200/lib/libtriton_b200.so).  If
it is missing, loading fails loudly: there is no fallback implementation.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libtriton_b200.so")

NOALLOC_EXTBC_MAX_CELLS = 65536  # TRI_NOALLOC_EXTBC_MAX_CELLS
TRI_OK, TRI_E_INVALID, TRI_E_CUDA, TRI_E_NOMEM, TRI_E_STATE, TRI_E_IO, TRI_E_TIMEOUT = range(7)
TRI_FP64, TRI_FP32 = 0, 1
FIELD_H, FIELD_QX, FIELD_QY, FIELD_NMAN2, FIELD_DEM, FIELD_MAXH = range(6)
EV_END, EV_PRINT, EV_OBS, EV_LOG = 1, 2, 4, 8
BATCH_GRAPHS, BATCH_SINGLE_LAUNCH = 0, 1

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
_vp = C.c_void_p


class GridDesc(C.Structure):
    _fields_ = [("rows", C.c_int32), ("cols", C.c_int32), ("cell_size", C.c_double), ("courant", C.c_double),
                ("hextra", C.c_double), ("open_boundaries", C.c_int32), ("precision", C.c_int32)]


class Clock(C.Structure):
    _fields_ = [("simtime", C.c_double), ("sim_duration", C.c_double), ("print_interval", C.c_double),
                ("print_observation", C.c_double), ("last_obs_time", C.c_double), ("init_dt", C.c_double),
                ("time_step", C.c_double), ("average_dt", C.c_double), ("global_dt", C.c_double),
                ("print_id", C.c_int32), ("it_count", C.c_int32), ("it_print", C.c_int32),
                ("time_series", C.c_int32), ("time_increment_fixed", C.c_int32), ("runoff_row", C.c_int32),
                ("src_idx_low", C.c_int32), ("last_events", C.c_int32)]


class Progress(C.Structure):
    _fields_ = [("steps", C.c_int32), ("events", C.c_int32)]


class Tuning(C.Structure):
    _fields_ = [("variant", C.c_int32), ("rows_per_tile", C.c_int32), ("candidates", C.c_int32),
                ("flux_blocks", C.c_int32), ("ms_per_step", C.c_double)]


class BatchProgress(C.Structure):
    _fields_ = [("steps", C.c_int32), ("members_with_events", C.c_int32), ("members_ended", C.c_int32),
                ("reserved", C.c_int32), ("cell_updates", C.c_int64)]


class TriError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"triton_b200 error {code}: {msg}")
        self.code = code


# name -> (restype, argtypes)
_SIGS = {
    "tri_abi_version": (C.c_int, []),
    "tri_last_error": (C.c_char_p, []),
    "tri_domain_footprint": (C.c_int, [C.POINTER(GridDesc), C.POINTER(C.c_int64)]),
    "tri_domain_create": (C.c_int, [C.POINTER(GridDesc), _vp, C.POINTER(_vp)]),
    "tri_domain_destroy": (C.c_int, [_vp]),
    "tri_domain_upload": (C.c_int, [_vp, C.c_int32, _dp, C.c_int64]),
    "tri_domain_download": (C.c_int, [_vp, C.c_int32, _dp, C.c_int64]),
    "tri_domain_init_max_depth": (C.c_int, [_vp]),
    "tri_domain_set_runoff": (C.c_int, [_vp, C.c_int32, C.c_int32, _dp, _dp, _ip, C.c_int64]),
    "tri_domain_set_sources": (C.c_int, [_vp, C.c_int32, _ip, C.c_int32, _dp, _dp]),
    "tri_domain_set_extbc": (C.c_int, [_vp, C.c_int32, _ip, _ip, _ip, _ip, C.c_int32, _dp, _dp]),
    "tri_domain_set_observations": (C.c_int, [_vp, C.c_int32, _ip]),
    "tri_domain_set_clock": (C.c_int, [_vp, C.POINTER(Clock)]),
    "tri_domain_get_clock": (C.c_int, [_vp, C.POINTER(Clock)]),
    "tri_domain_advance": (C.c_int, [_vp, C.c_int32, C.POINTER(Progress)]),
    "tri_domain_compute_dt": (C.c_int, [_vp, _dp]),
    "tri_domain_observe": (C.c_int, [_vp, _dp, _dp, _dp]),
    "tri_domain_volume": (C.c_int, [_vp, _dp]),
    "tri_domain_synchronize": (C.c_int, [_vp]),
    "tri_domain_mass_balance": (C.c_int, [_vp, _dp]),
    "tri_domain_track_arrival": (C.c_int, [_vp, C.c_double]),
    "tri_domain_download_arrival": (C.c_int, [_vp, _dp, C.c_int64]),
    "tri_domain_set_timing": (C.c_int, [_vp, C.c_int32]),
    "tri_domain_get_timing": (C.c_int, [_vp, _dp, _ip, _dp, _ip]),
    "tri_domain_get_work": (C.c_int, [_vp, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "tri_domain_set_wait_test": (C.c_int, [_vp, C.c_uint32]),
    "tri_domain_autotune": (C.c_int, [_vp, C.c_int32, C.POINTER(Tuning)]),
    "tri_domain_get_tuning": (C.c_int, [_vp, C.POINTER(Tuning)]),
    "tri_domain_set_tuning": (C.c_int, [_vp, C.c_int32, C.c_int32]),
    "tri_batch_create": (C.c_int, [C.c_int32, C.POINTER(_vp), _vp, C.POINTER(_vp)]),
    "tri_batch_destroy": (C.c_int, [_vp]),
    "tri_batch_set_members": (C.c_int, [_vp, C.c_int32, C.POINTER(_vp)]),
    "tri_batch_advance": (C.c_int, [_vp, C.c_int32, C.POINTER(BatchProgress)]),
    "tri_batch_launch": (C.c_int, [_vp, C.c_int32]),
    "tri_batch_wait": (C.c_int, [_vp, C.POINTER(BatchProgress)]),
    "tri_batch_autotune": (C.c_int, [_vp, C.c_int32, C.POINTER(Tuning)]),
    "tri_batch_set_tuning": (C.c_int, [_vp, C.c_int32, C.c_int32]),
    "tri_batch_set_mode": (C.c_int, [_vp, C.c_int32]),
    "tri_batch_set_wait_test": (C.c_int, [_vp, C.c_uint32]),
    "tri_selftest_division": (C.c_int, [C.c_int64, C.c_uint64, C.POINTER(C.c_int64)]),
    "tri_kernel_compute_dt_and_sqrt_f64": (C.c_int, [C.c_int, C.c_double, _vp, _vp, _vp, _vp, _vp, C.c_double,
                                                     C.c_double, _vp]),
    "tri_kernel_find_min_dt_f64": (C.c_int, [C.c_int, _vp, _vp, _vp]),
    "tri_kernel_flux_x_f64": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double] + [_vp] * 11 +
                              [C.c_double, _vp]),
    "tri_kernel_flux_y_f64": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double] + [_vp] * 11 +
                              [C.c_double, _vp]),
    "tri_kernel_update_cells_f64": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_double] + [_vp] * 11 +
                                    [C.c_double, _vp]),
    "tri_kernel_update_runoff_f64": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_double, _vp, C.c_int, C.c_int, _vp,
                                               _vp, _vp, _vp, C.c_double, _vp]),
    "tri_kernel_compute_flow_f64": (C.c_int, [C.c_int, _vp, _vp, C.c_double, C.c_double, C.c_double, C.c_int,
                                              C.c_int, _vp, _vp, _vp]),
    "tri_kernel_copy_info_to_exterior_boundaries_west_east_f64": (C.c_int, [C.c_int, C.c_int, C.c_int, _vp, _vp,
                                                                            _vp, _vp]),
    "tri_kernel_copy_info_to_exterior_boundaries_north_south_f64": (C.c_int, [C.c_int, C.c_int, C.c_int, _vp, _vp,
                                                                              _vp, C.c_int, C.c_int, _vp]),
    "tri_kernel_compute_extbc_values_f64": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_double] + [_vp] * 11 +
                                            [C.c_double, C.c_int, C.c_int, _vp]),
    "tri_kernel_compute_extbc_values_noalloc_f64": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_double] + [_vp] * 11 +
                                                    [C.c_double, C.c_int, C.c_int, _vp]),
    "tri_kernel_wet_dry_f64": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_double, _vp, _vp, _vp, _vp, _vp, C.c_double,
                                         C.c_int, _vp]),
    "tri_kernel_copy_observation_points_f64": (C.c_int, [C.c_int, _vp, _vp, _vp, _vp]),
}

_lib = None


def lib():
    """Load the library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m triton_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def exported_symbols():
    return list(_SIGS)


def check(rc):
    if rc != TRI_OK:
        msg = lib().tri_last_error()
        raise TriError(rc, msg.decode() if msg else "")
    return rc
