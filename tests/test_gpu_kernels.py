"""The per-kernel entry points (tri_kernel_*_f64, one per reference device
kernel) against the oracle's restatement of the same kernel, on the same
seeded state, through the C ABI with device buffers."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


def _state():
    from triton_b200 import scenarios
    sc = scenarios.mixed(rows=37, cols=51, seed=13, open_boundaries=0, friction=True, duration=5.0)
    return sc


def _dev(torch, a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a)).cuda()
    return t


def _p(t):
    return C.c_void_p(t.data_ptr())


def _np(a):
    return np.ascontiguousarray(a, dtype=np.float64).reshape(-1)


def test_kernel_entry_points_match_oracle(oracle):
    import torch
    from triton_b200 import _abi
    L = _abi.lib()
    O = oracle.lib()
    for f in ("tor_compute_dt_and_sqrt", "tor_flux_x", "tor_flux_y", "tor_update_cells", "tor_update_runoff",
              "tor_compute_flow", "tor_open_boundaries", "tor_compute_extbc_values", "tor_wet_dry",
              "tor_copy_observation_points"):
        getattr(O, f).restype = None
    sc = _state()
    R, Cc = sc.rows, sc.cols
    N = R * Cc
    h, qx, qy, z, n2 = (_np(getattr(sc, k)) for k in ("h", "qx", "qy", "z", "n2"))
    cn, hx, dx = sc.courant, sc.hextra, sc.dx
    # --- compute_dt_and_sqrt + find_min_dt
    sq_o, dt_o = np.zeros(N), np.zeros(N)
    O.tor_compute_dt_and_sqrt(N, C.c_double(dx), qx.ctypes.data_as(_dp), qy.ctypes.data_as(_dp),
                              h.ctypes.data_as(_dp), sq_o.ctypes.data_as(_dp), dt_o.ctypes.data_as(_dp),
                              C.c_double(cn), C.c_double(hx))
    dh, dqx, dqy, dz, dn2 = (_dev(torch, a) for a in (h, qx, qy, z, n2))
    dsq, ddt = torch.zeros(N, dtype=torch.float64, device="cuda"), torch.zeros(N, dtype=torch.float64, device="cuda")
    _abi.check(L.tri_kernel_compute_dt_and_sqrt_f64(N, dx, _p(dqx), _p(dqy), _p(dh), _p(dsq), _p(ddt), cn, hx, None))
    torch.cuda.synchronize()
    assert np.array_equal(dsq.cpu().numpy(), sq_o)
    assert np.array_equal(ddt.cpu().numpy(), dt_o)
    dmin = torch.zeros(1, dtype=torch.float64, device="cuda")
    _abi.check(L.tri_kernel_find_min_dt_f64(N, _p(ddt), _p(dmin), None))
    torch.cuda.synchronize()
    m = O.tor_find_min_dt(N, dt_o.ctypes.data_as(_dp))
    assert dmin.item() == m
    dt = m
    # --- flux_x, flux_y (rhs arrays start from random garbage, as in the reference nothing clears them)
    rng = np.random.default_rng(0)
    rhs_o = [rng.standard_normal(N) for _ in range(6)]
    rhs_d = [_dev(torch, a.copy()) for a in rhs_o]
    args_o = [a.ctypes.data_as(_dp) for a in rhs_o]
    O.tor_flux_x(R, Cc, C.c_double(dx), C.c_double(dt), h.ctypes.data_as(_dp), qx.ctypes.data_as(_dp),
                 qy.ctypes.data_as(_dp), z.ctypes.data_as(_dp), sq_o.ctypes.data_as(_dp), *args_o, C.c_double(hx))
    O.tor_flux_y(R, Cc, C.c_double(dx), C.c_double(dt), h.ctypes.data_as(_dp), qx.ctypes.data_as(_dp),
                 qy.ctypes.data_as(_dp), z.ctypes.data_as(_dp), sq_o.ctypes.data_as(_dp), *args_o, C.c_double(hx))
    _abi.check(L.tri_kernel_flux_x_f64(N, R, Cc, dx, dt, _p(dh), _p(dqx), _p(dqy), _p(dz), _p(dsq),
                                       *[_p(t) for t in rhs_d], hx, None))
    _abi.check(L.tri_kernel_flux_y_f64(N, R, Cc, dx, dt, _p(dh), _p(dqx), _p(dqy), _p(dz), _p(dsq),
                                       *[_p(t) for t in rhs_d], hx, None))
    torch.cuda.synchronize()
    for a, t in zip(rhs_o, rhs_d):
        assert np.array_equal(t.cpu().numpy(), a)
    # --- update_cells (friction: cube root, tolerance)
    O.tor_update_cells(R, Cc, C.c_double(dt), h.ctypes.data_as(_dp), qx.ctypes.data_as(_dp), qy.ctypes.data_as(_dp),
                       n2.ctypes.data_as(_dp), *args_o, C.c_double(hx))
    _abi.check(L.tri_kernel_update_cells_f64(N, R, Cc, dt, _p(dh), _p(dqx), _p(dqy), _p(dz), _p(dn2),
                                             *[_p(t) for t in rhs_d], hx, None))
    torch.cuda.synchronize()
    for a, t in ((h, dh), (qx, dqx), (qy, dqy)):
        g = t.cpu().numpy()
        assert np.abs(g - a).max() <= 1e-12 * max(np.abs(a).max(), 1.0)
    # continue from identical states
    for a, t in ((h, dh), (qx, dqx), (qy, dqy)):
        t.copy_(torch.from_numpy(a))
    # --- runoff
    ro = sc.runoff
    zone = np.ascontiguousarray(ro["zone"].reshape(-1), dtype=np.int32)
    rates = _np(ro["rates"])
    nrows = ro["times"].size
    O.tor_update_runoff(R, Cc, C.c_double(dt), zone.ctypes.data_as(_ip), 2, nrows, rates.ctypes.data_as(_dp),
                        h.ctypes.data_as(_dp), qx.ctypes.data_as(_dp), qy.ctypes.data_as(_dp), C.c_double(hx))
    dzone, drates = _dev(torch, zone), _dev(torch, rates)
    _abi.check(L.tri_kernel_update_runoff_f64(N, R, Cc, dt, _p(dzone), 2, nrows, _p(drates), _p(dh), _p(dqx), _p(dqy),
                                              hx, None))
    # --- point sources (two share a cell)
    so = sc.sources
    cells = np.ascontiguousarray(so["cells"], dtype=np.int32)
    ht, hv = _np(so["times"]), _np(so["flows"])
    O.tor_compute_flow(cells.size, ht.ctypes.data_as(_dp), hv.ctypes.data_as(_dp), C.c_double(dx), C.c_double(dt),
                       C.c_double(3.0), 0, 1, h.ctypes.data_as(_dp), cells.ctypes.data_as(_ip))
    dcells, dht, dhv = _dev(torch, cells), _dev(torch, ht), _dev(torch, hv)
    _abi.check(L.tri_kernel_compute_flow_f64(cells.size, _p(dht), _p(dhv), dx, dt, 3.0, 0, 1, _p(dh), _p(dcells),
                                             None))
    # --- open boundaries (west/east then north/south)
    O.tor_open_boundaries(R, Cc, h.ctypes.data_as(_dp), qx.ctypes.data_as(_dp), qy.ctypes.data_as(_dp))
    _abi.check(L.tri_kernel_copy_info_to_exterior_boundaries_west_east_f64(2 * R, R, Cc, _p(dh), _p(dqx), _p(dqy),
                                                                           None))
    _abi.check(L.tri_kernel_copy_info_to_exterior_boundaries_north_south_f64(Cc, R, Cc, _p(dh), _p(dqx), _p(dqy), 0,
                                                                             1, None))
    torch.cuda.synchronize()
    for a, t in ((h, dh), (qx, dqx), (qy, dqy)):
        assert np.array_equal(t.cpu().numpy(), a)
    # --- external boundaries
    e = sc.extbc
    arrs = [np.ascontiguousarray(e[k], dtype=np.int32) for k in ("cells", "types", "start", "nrows")]
    v1, v2 = _np(e["var1"]), _np(e["var2"])
    O.tor_compute_extbc_values(arrs[0].size, R, Cc, C.c_double(dt), h.ctypes.data_as(_dp), qx.ctypes.data_as(_dp),
                               qy.ctypes.data_as(_dp), z.ctypes.data_as(_dp), n2.ctypes.data_as(_dp),
                               *[a.ctypes.data_as(_ip) for a in arrs], v1.ctypes.data_as(_dp),
                               v2.ctypes.data_as(_dp), C.c_double(7.0))
    darrs = [_dev(torch, a) for a in arrs]
    dv1, dv2 = _dev(torch, v1), _dev(torch, v2)
    _abi.check(L.tri_kernel_compute_extbc_values_f64(arrs[0].size, R, Cc, dt, _p(dh), _p(dqx), _p(dqy), _p(dz),
                                                     _p(dn2), *[_p(t) for t in darrs], _p(dv1), _p(dv2), 7.0, 0, 1,
                                                     None))
    torch.cuda.synchronize()
    for a, t in ((h, dh), (qx, dqx), (qy, dqy)):
        g = t.cpu().numpy()
        assert np.abs(g - a).max() <= 1e-12 * max(np.abs(a).max(), 1.0)
        t.copy_(torch.from_numpy(a))
    # --- wet_dry + max depth
    maxh = h.copy() * 0.5
    dmaxh = _dev(torch, maxh.copy())
    O.tor_wet_dry(R, Cc, h.ctypes.data_as(_dp), qx.ctypes.data_as(_dp), qy.ctypes.data_as(_dp), z.ctypes.data_as(_dp),
                  maxh.ctypes.data_as(_dp), C.c_double(hx))
    _abi.check(L.tri_kernel_wet_dry_f64(N, R, Cc, dt, _p(dh), _p(dqx), _p(dqy), _p(dz), _p(dmaxh), hx, 1, None))
    torch.cuda.synchronize()
    for a, t in ((qx, dqx), (qy, dqy), (maxh, dmaxh)):
        assert np.array_equal(t.cpu().numpy(), a)
    # --- observation gather
    obs = np.ascontiguousarray(sc.obs_cells, dtype=np.int32)
    out_o = np.zeros(obs.size)
    O.tor_copy_observation_points(obs.size, h.ctypes.data_as(_dp), out_o.ctypes.data_as(_dp), obs.ctypes.data_as(_ip))
    dobs, dout = _dev(torch, obs), torch.zeros(obs.size, dtype=torch.float64, device="cuda")
    _abi.check(L.tri_kernel_copy_observation_points_f64(obs.size, _p(dh), _p(dout), _p(dobs), None))
    torch.cuda.synchronize()
    assert np.array_equal(dout.cpu().numpy(), out_o)
