"""Bench helpers that need no GPU."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_roofline_traffic_comes_from_the_committed_capture():
    """The level-5 bench line reports the DRAM bytes per launch of the sweep
    kernel: the level-3 ncu capture scaled by cells (traffic per cell does not
    depend on the level to first order)."""
    cells3, cells5 = 548 * 4096, 4692 * 4096
    t3, src3 = bench.profile_traffic(3, cells3)
    t5, src5 = bench.profile_traffic(5, cells5)
    assert t3 is not None and t5 is not None, (src3, src5)
    assert abs(t5 - t3 * cells5 / cells3) < 1.0
    # within a few per cent of the algorithmic 80 B per cell of one fused pass
    assert 1.0 <= t5 / (80.0 * cells5) < 1.1
