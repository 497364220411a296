"""CPU checks of the precision-report helpers."""
import numpy as np

from triton_b200 import precision, scenarios


def test_fp32_bed_rounds_offsets_only():
    sc = scenarios.mixed(rows=70, cols=90, seed=3)
    s2 = precision.fp32_bed(sc)
    assert s2 is not sc and s2.z.shape == sc.z.shape
    z, z2 = sc.z[1:-1, 1:-1], s2.z[1:-1, 1:-1]
    # each interior level moves by at most half an FP32 ulp of its offset from
    # the tile base (the offsets here are below 16 m)
    assert np.all(np.abs(z2 - z) <= 2.0 ** -20)
    assert (z2 != z).any()
    # the tile bases themselves are exact: the lowest interior cell of each tile
    for tr in range(0, 70, 32):
        for tc in range(0, 90, 32):
            r0, r1 = max(tr, 1), min(tr + 32, sc.rows - 1)
            c0, c1 = max(tc, 1), min(tc + 32, sc.cols - 1)
            blk, blk2 = sc.z[r0:r1, c0:c1], s2.z[r0:r1, c0:c1]
            assert blk2.min() == blk.min()
