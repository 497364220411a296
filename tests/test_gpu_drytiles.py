"""Dry-tile skipping of the single-domain flux kernel: a tile whose cells and
neighbour tiles hold only +0 is not computed.  Skipping must be exact, so a
domain stepped alone (tiles skipped) must end bit for bit where the same
domain ends when stepped as a one-member batch (the batched kernels compute
every tile; batch members are checked against solo runs elsewhere), or, for
open boundaries (which batches do not take), where it ends with a runoff
table of zero rates (a domain with runoff computes every tile; a zero rate
changes no value).  The cases are mostly dry and add each kind of forcing
that writes into cells after the flux kernel (point source, external
boundary cells, open boundaries), a negative max depth and arrival tracking
(what the wet-dry kernel records in cells that stay dry), and the solo run
changes its state and tile shape midway (both must reset what is known to
be dry)."""
from __future__ import annotations

import numpy as np
import pytest

from triton_b200 import scenarios
from triton_b200.batch import Batch

pytestmark = pytest.mark.gpu


def _case(kind, n=150):
    X, Y = np.meshgrid(np.arange(n) + 0.5, np.arange(n) + 0.5)
    h = np.where((X - 40.0) ** 2 + (Y - 40.0) ** 2 <= 15.0 ** 2, 2.0, 0.0)
    dem = 0.002 * X  # gentle slope down to the west
    ob = 1 if kind == "open" else 0
    z = scenarios._walls(dem, ob)
    hp = scenarios._pad(h)
    zero = np.zeros_like(hp)
    if ob:
        hp = scenarios._copy_ghosts(hp)
    sc = scenarios.Scenario(kind, 1.0, z, hp, zero.copy(), zero.copy(), np.full_like(hp, 0.03 ** 2),
                            courant=0.5, hextra=0.001, open_boundaries=ob, sim_duration=1e300,
                            print_interval=1e300, print_observation=1e300)
    if kind == "source":
        scenarios.sources_table(sc, [(n - 20, n - 30)], [0.0, 1.0], [[3.0], [3.0]])
    if kind == "extbc":
        scenarios.extbc_segments(sc, [(1, (0, n - 1), (n - 1, n - 1), [(0.0, 0.6), (1.0, 0.6)])])
    return sc


def _quiet(d):
    d.set_clock(sim_duration=1e300, print_interval=1e300, print_observation=1e300, it_print=0, time_series=0)


def _fields(d):
    return {f: d.download(f) for f in ("h", "qx", "qy", "maxh")}


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("kind", ["walls", "source", "extbc", "open", "negmaxh", "arrival"])
def test_dry_tiles_skipped_exactly(kind, precision):
    sc = _case(kind)
    steps = (37, 60, 43)
    solo = sc.to_domain(precision)
    if kind == "open":
        scenarios.runoff_table(sc, np.zeros((sc.rows - 2, sc.cols - 2), np.int32), [0.0, 1.0], [[0.0], [0.0]])
    ref = sc.to_domain(precision)
    try:
        _quiet(solo)
        _quiet(ref)
        for d in (solo, ref):
            if kind == "negmaxh":  # a negative max depth: dry bands must still record 0
                d.upload("maxh", np.full((sc.rows, sc.cols), -1.0))
            if kind == "arrival":
                d.track_arrival(0.05)
        solo.set_shape(0, 8)
        total = 0
        for i, n in enumerate(steps):
            k, _ = solo.advance(n)
            assert k == n
            total += k
            if i == 0:  # the same state uploaded again: flags reset
                for f in ("h", "qx", "qy"):
                    solo.upload(f, solo.download(f))
            if i == 1:  # another tile shape: flags reset
                solo.set_shape(1, 16)
        if kind == "open":
            k, _ = ref.advance(total)
            assert k == total
        else:
            with Batch([ref]) as b:
                done = 0
                while done < total:
                    p = b.advance(total - done)
                    assert p.steps > 0
                    done += p.steps
        assert solo.get_clock().it_count == ref.get_clock().it_count
        a, r = _fields(solo), _fields(ref)
        if kind == "arrival":
            a["arrival"], r["arrival"] = solo.arrival(), ref.arrival()
            assert (a["arrival"] >= 0).any()
        for f in a:
            bad = a[f] != r[f]
            assert not bad.any(), f"{kind}/{precision}: {f} differs in {int(bad.sum())} cells"
        # the case really is mostly dry, and water has reached new cells
        wet = a["h"][1:-1, 1:-1] > 0
        assert 0.02 < wet.mean() < 0.6
    finally:
        solo.close()
        ref.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_dry_tiles_are_skipped_and_counted(precision):
    """The mostly dry case computes well under all of its cells (the skip is
    on), and a domain with runoff computes every cell (the skip is off)."""
    sc = _case("walls")
    interior = (sc.rows - 2) * (sc.cols - 2)
    d = sc.to_domain(precision)
    try:
        _quiet(d)
        d.advance(10)  # flags known after two steps
        d.set_timing(True)
        k, _ = d.advance(20)
        flux_cells, wet_cells = d.get_work()
        d.set_timing(False)
        assert k == 20
        assert 0 < flux_cells < 0.6 * 20 * interior, flux_cells / (20 * interior)
        assert 0 < wet_cells < 0.8 * 20 * interior, wet_cells / (20 * interior)
    finally:
        d.close()
    scenarios.runoff_table(sc, np.zeros((sc.rows - 2, sc.cols - 2), np.int32), [0.0, 1.0], [[0.0], [0.0]])
    d = sc.to_domain(precision)
    try:
        _quiet(d)
        d.advance(10)
        d.set_timing(True)
        k, _ = d.advance(20)
        flux_cells, wet_cells = d.get_work()
        d.set_timing(False)
        assert flux_cells == wet_cells == 20 * interior
    finally:
        d.close()
