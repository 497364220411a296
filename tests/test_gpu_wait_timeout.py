"""A bounded device wait that runs out: the kernel gives up, records a status,
and the host returns TRI_E_TIMEOUT; the context stays usable and the domain
computes on as if nothing had happened.

The wait that runs out is the test hook's (tri_domain_set_wait_test): one
thread of each step's wet-dry launch waits on a barrier that expects bytes no
copy ever delivers, with a short poll limit.  No copy is issued on that
barrier, so nothing is left in flight when the wait gives up; the staged
copies of the real bands are untouched."""
from __future__ import annotations

import numpy as np
import pytest

from triton_b200 import _abi, scenarios

pytestmark = pytest.mark.gpu


def _fields(d):
    return [d.download(n) for n in ("h", "qx", "qy", "maxh")]


def test_wait_that_runs_out_returns_timeout_and_context_stays_usable():
    sc = scenarios.dambreak(n=96, dx=1.0, radius=20.0, depth=4.0, duration=10.0)
    sc.print_interval = 10.0
    ref = sc.to_domain()
    hooked = sc.to_domain()
    try:
        ref.advance(40)
        _abi.check(_abi.lib().tri_domain_set_wait_test(hooked._h, 64))
        with pytest.raises(_abi.TriError) as e:
            hooked.advance(20)
        assert e.value.code == _abi.TRI_E_TIMEOUT
        assert "gave up" in str(e.value)
        c = hooked.get_clock()
        assert c.it_count == 20  # the steps ran; only the hook's wait gave up
        # hook off: the same domain advances normally and ends where the
        # domain that never waited ends, bit for bit
        _abi.check(_abi.lib().tri_domain_set_wait_test(hooked._h, 0))
        steps, _ = hooked.advance(20)
        assert steps == 20
        for a, b in zip(_fields(hooked), _fields(ref)):
            assert np.array_equal(a, b)
        assert hooked.get_clock().simtime == ref.get_clock().simtime
    finally:
        ref.close()
        hooked.close()


def test_single_launch_batch_wait_that_runs_out_returns_timeout():
    """The persistent batch kernel's dependency waits are bounded too: with
    the batch's test hook the first clock item waits for a count no item ever
    reaches; it gives up, every other wait then gives up at once, the launch
    ends and the advance returns TRI_E_TIMEOUT.  The context stays usable: a
    new batch over fresh members steps normally afterwards."""
    from triton_b200.batch import Batch

    scs = []
    for i in range(3):
        sc = scenarios.dambreak(n=64 + 16 * i, dx=1.0, radius=12.0, depth=4.0, duration=10.0)
        sc.print_interval = 10.0
        scs.append(sc)
    doms = [sc.to_domain() for sc in scs]
    try:
        with Batch(doms) as b:
            b.set_mode(True)
            b.set_wait_test(1000)
            with pytest.raises(_abi.TriError) as e:
                b.advance(8)
            assert e.value.code == _abi.TRI_E_TIMEOUT
            assert "single-launch" in str(e.value)
    finally:
        for d in doms:
            d.close()
    fresh = [sc.to_domain() for sc in scs]
    solo = [sc.to_domain() for sc in scs]
    try:
        with Batch(fresh) as b:
            b.set_mode(True)
            p = b.advance(8)
            assert p.steps == 8
        for d in solo:
            steps, _ = d.advance(8)
            assert steps == 8
        for f, s in zip(fresh, solo):
            for a, c in zip(_fields(f), _fields(s)):
                assert np.array_equal(a, c)
    finally:
        for d in fresh + solo:
            d.close()
