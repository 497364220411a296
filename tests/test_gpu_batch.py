"""Batched ensembles: every member of a tri_batch must end exactly where the
same domain run alone ends (same fields bit for bit, same step count and
simulated time), whatever the mix of member sizes and forcing.  The solo
path is itself checked against the oracle by the parity tests."""
from __future__ import annotations

import numpy as np
import pytest

from triton_b200 import scenarios
from triton_b200.batch import Batch

pytestmark = pytest.mark.gpu


def _members():
    ms = scenarios.ensemble(members=6, seed=11, side_min=40, side_max=160, duration=600.0, rain_range=(50, 200))
    for i, sc in enumerate(ms):
        sc.print_interval = 150.0 + 50.0 * i  # uneven print events
        sc.it_print = 37 + i
    mx = scenarios.mixed(rows=37, cols=53, seed=5)
    mx.name = "mixed"
    # open edges (zero-gradient ghosts, kernels.h:437-512) with sources and runoff
    op = scenarios.mixed(rows=29, cols=44, seed=8, open_boundaries=1, with_extbc=False)
    op.name = "open"
    return ms + [mx, op]


def _solo(sc, precision):
    d = sc.to_domain(precision)
    try:
        d.run()
        c = d.get_clock()
        return {f: d.download(f) for f in ("h", "qx", "qy", "maxh")}, c.it_count, c.simtime
    finally:
        d.close()


@pytest.mark.parametrize("single_launch", [False, True], ids=["graphs", "single_launch"])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_batch_members_equal_solo_runs(precision, single_launch):
    """Both launch modes: one launch per kernel type and step (CUDA graphs),
    and one persistent launch per chunk of steps whose blocks take work items
    with per-member dependencies."""
    scs = _members()
    solo = [_solo(sc, precision) for sc in scs]
    doms = [sc.to_domain(precision) for sc in scs]
    try:
        with Batch(doms) as b:
            b.set_mode(single_launch)
            steps, updates = b.run()
        assert steps > 0 and updates > 0
        for sc, d, (fields, it, t) in zip(scs, doms, solo):
            c = d.get_clock()
            assert c.it_count == it, f"{sc.name}: {c.it_count} steps batched, {it} alone"
            assert c.simtime == t, f"{sc.name}: simtime {c.simtime!r} batched, {t!r} alone"
            for f, ref in fields.items():
                got = d.download(f)
                bad = got != ref
                assert not bad.any(), f"{sc.name}: {f} differs in {int(bad.sum())} cells"
    finally:
        for d in doms:
            d.close()


def test_batch_autotune_keeps_members():
    scs = _members()[:4]
    doms = [sc.to_domain("fp64") for sc in scs]
    try:
        before = [(d.download("h"), d.get_clock().simtime) for d in doms]
        with Batch(doms) as b:
            t = b.autotune(3)
            assert t["candidates"] >= 1 and t["ms_per_step"] > 0
            for d, (h, st) in zip(doms, before):
                assert np.array_equal(d.download("h"), h)
                assert d.get_clock().simtime == st
            b.run()
        solo = [_solo(sc, "fp64") for sc in scs]
        for d, (fields, it, _) in zip(doms, solo):
            assert d.get_clock().it_count == it
            assert np.array_equal(d.download("h"), fields["h"])
    finally:
        for d in doms:
            d.close()


def test_batch_rejects_bad_members():
    from triton_b200 import TriError
    sc = scenarios.dambreak(n=32, duration=0.5)
    a = sc.to_domain("fp64")
    b = sc.to_domain("fp32")
    try:
        with pytest.raises(TriError):
            Batch([a, b])
        with pytest.raises(TriError):
            Batch([a, a])
    finally:
        a.close()
        b.close()
