"""tri_kernel_compute_extbc_values_noalloc_f64 (external-boundary cells with
the application order in a fixed device array instead of allocated scratch)
against tri_kernel_compute_extbc_values_f64 on the same device state.

The file is named to be collected last, so the no-alloc entry's first call on
the device (the address lookup of its fixed array) also runs after every
other test has used the library; the test passes alone and after the rest."""
import ctypes as C

import numpy as np
import pytest

from triton_b200 import _abi


def _p(t):
    return C.c_void_p(t.data_ptr())


def test_noalloc_rejects_lists_over_its_limit():
    # host-side check, before any CUDA call
    L = _abi.lib()
    n = _abi.NOALLOC_EXTBC_MAX_CELLS + 1
    rc = L.tri_kernel_compute_extbc_values_noalloc_f64(n, 10, 10, 0.1, *([None] * 11), 0.0, 0, 1, None)
    assert rc == _abi.TRI_E_INVALID
    assert b"fixed limit of 65536" in L.tri_last_error()


@pytest.mark.gpu
def test_noalloc_extbc_matches_allocating_entry():
    import torch
    from triton_b200 import scenarios
    L = _abi.lib()
    sc = scenarios.mixed(rows=37, cols=51, seed=13, open_boundaries=0, friction=True, duration=5.0)
    R, Cc = sc.rows, sc.cols
    dev = lambda a, dt=torch.float64: torch.as_tensor(np.ascontiguousarray(a), dtype=dt).reshape(-1).cuda()
    e = sc.extbc
    lists = [dev(e[k], torch.int32) for k in ("cells", "types", "start", "nrows")]
    dv1, dv2 = dev(e["var1"]), dev(e["var2"])
    dz, dn2 = dev(sc.z), dev(sc.n2)
    state = {}
    for arm in ("alloc", "noalloc"):
        state[arm] = [dev(getattr(sc, k)) for k in ("h", "qx", "qy")]
    entries = {"alloc": L.tri_kernel_compute_extbc_values_f64,
               "noalloc": L.tri_kernel_compute_extbc_values_noalloc_f64}

    def call(arm, cells, dt, simtime):
        n = cells[0].numel()
        h, qx, qy = state[arm]
        _abi.check(entries[arm](n, R, Cc, dt, _p(h), _p(qx), _p(qy), _p(dz), _p(dn2), *[_p(t) for t in cells],
                                _p(dv1), _p(dv2), simtime, 0, 1, None))

    def same(where):
        torch.cuda.synchronize()
        for name, a, b in zip(("h", "qx", "qy"), state["alloc"], state["noalloc"]):
            assert torch.equal(a, b), f"{where}: {name} differs in {int((a != b).sum())} cells"

    # two calls in a row with the same cell list
    for k, (dt, t) in enumerate(((0.05, 7.0), (0.04, 7.05))):
        for arm in ("alloc", "noalloc"):
            call(arm, lists, dt, t)
        same(f"call {k + 1}")
    # then another cell list (every second cell, reversed): the order is rebuilt
    sub = [t[::2].flip(0).contiguous() for t in lists]
    for arm in ("alloc", "noalloc"):
        call(arm, sub, 0.03, 7.09)
    same("call 3, other list")
    # and the first list again
    for arm in ("alloc", "noalloc"):
        call(arm, lists, 0.05, 7.12)
    same("call 4, first list again")
