"""Bench helpers that need no GPU."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_roofline_traffic_comes_from_the_committed_capture():
    """The level-5 bench line reports the DRAM bytes per launch of the sweep
    kernel: the level-3 ncu capture scaled by the bytes of the pool's format
    (uniform blocks at 24 B per cell, the others at 80), since the share of
    uniform blocks differs between levels."""
    cells3, cells5 = 548 * 4096, 4692 * 4096
    fmt3 = 4096 * ((548 - 376) * 80 + 376 * 24)
    fmt5 = 4096 * ((4692 - 4256) * 80 + 4256 * 24)
    t3, src3 = bench.profile_traffic(3, cells3, fmt3)
    t5, src5 = bench.profile_traffic(5, cells5, fmt5)
    assert t3 is not None and t5 is not None, (src3, src5)
    assert "format bytes" in src5
    assert abs(t5 - t3 * fmt5 / fmt3) < 1.0
    # traffic within a few per cent of the format's bytes, well under the
    # algorithmic 80 B per cell of one fused pass
    assert 0.9 <= t3 / fmt3 <= 1.1
    assert t5 < 0.5 * 80.0 * cells5
