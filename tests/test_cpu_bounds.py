"""CPU check of the device exchange's index arithmetic (no GPU needed):
tests/native/guide_bounds_check.cpp compiles the kernels' guide-value code
for the host with a bounds-checking load and evaluates every guide cell of
real grids against the neighbour table the pool derives."""
import os
import subprocess

import numpy as np
import pytest

import ffvgpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "native", "guide_bounds_check.cpp")


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("bounds") / "guide_bounds_check")
    subprocess.run(["g++", "-O1", "-std=c++17", "-o", exe, SRC], check=True)
    return exe


def table_text(g):
    kind, ids = g.neighbors()
    rows = [str(g.nb)]
    for b in range(g.nb):
        for f in range(6):
            ax = f // 2
            ta, tb = (1, 2) if ax == 0 else ((0, 2) if ax == 1 else (0, 1))
            so_u = so_v = 0
            if kind[b, f] == ffvgpu.NB_COARSE:
                so_u, so_v = g.index[b, ta] & 1, g.index[b, tb] & 1
            rows.append(" ".join(map(str, [kind[b, f], *ids[b, f], so_u, so_v])))
    return "\n".join(rows) + "\n"


@pytest.mark.parametrize("level,kw", [(0, {}), (2, {}), (3, {}), (4, {}),
                                      (3, dict(center=(2.3, -1.1, 0.7), radius=0.8)),
                                      (5, dict(center=(1.0, 0.5, -0.25), radius=0.3))])
def test_guide_gathers_in_bounds(checker, level, kw):
    g = ffvgpu.SphereGrid(level, **kw)
    out = subprocess.run([checker], input=table_text(g), capture_output=True, text=True)
    evals, bad, wrong = map(int, out.stdout.split())
    assert evals == g.nb * 6 * 2 * 256
    assert bad == 0, "out-of-range load in guide_value"
    assert wrong == 0, "constant field not reproduced across an inner face"
