"""Per-launch timing (tri_domain_set_timing / tri_domain_get_timing): CUDA
events around every flux and wet-dry launch, recorded inside the step graphs
as event-record nodes.  Timing must not change a result, must count one
flux and one wet-dry launch per step, and the timed launches must fit inside
the elapsed time of the steps."""
from __future__ import annotations

import pytest

from triton_b200 import scenarios

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_timing_keeps_results_and_counts_every_launch(precision):
    import torch

    sc = scenarios.mixed(rows=67, cols=91, seed=3)
    plain, timed = sc.to_domain(precision), sc.to_domain(precision)
    try:
        for d in (plain, timed):
            d.set_clock(sim_duration=1e300, print_interval=1e300, print_observation=1e300, it_print=0,
                        time_series=0)
        # 29 + 16 + 3 steps: whole graphs, a remainder, and a short call
        timed.set_timing(True)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        total = 0
        for n in (29, 16, 3):
            k, _ = timed.advance(n)
            total += k
        e1.record()
        torch.cuda.synchronize()
        flux_ms, flux_n, wet_ms, wet_n = timed.get_timing()
        timed.set_timing(False)
        assert total == 48
        assert flux_n == wet_n == 48
        assert flux_ms > 0 and wet_ms > 0
        assert flux_ms + wet_ms <= e0.elapsed_time(e1) * 1.01 + 0.01
        for n in (29, 16, 3):
            plain.advance(n)
        for f in ("h", "qx", "qy", "maxh"):
            a, b = plain.download(f), timed.download(f)
            assert (a == b).all(), f"{f} differs in {int((a != b).sum())} cells with timing on"
        # timing off again: graphs without events, same results
        plain.advance(16)
        timed.advance(16)
        for f in ("h", "qx", "qy"):
            assert (plain.download(f) == timed.download(f)).all()
    finally:
        plain.close()
        timed.close()
