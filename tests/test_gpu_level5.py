"""Parity on the level-5 sphere grid, the configuration the benchmark times.

4692 leaf blocks of 16^3 (19,218,432 cells), refined in six levels around the
sphere, with every 2:1 transition of the benchmark grid, several blocks per
CTA and cross-block sums over 4692 partials.  Against the oracle in its
canonical-sum mode the bar is bit equality: the FP64 RBGS solve (pressure,
both guide layers, residual history), the FP64 BiCGSTAB solve (the reference's
default solver, FFVILS.h:793-974) and the mixed-precision solve against the
oracle's restatement of it.  The iteration counts are bounded so that the
oracle, on all host cores, finishes in about a minute.
"""
import os

import numpy as np
import pytest

import ffv_oracle as fo
from helpers import VC, assert_bitwise, device_problem, interior, problem

pytestmark = pytest.mark.gpu
THREADS = os.cpu_count() or 8


@pytest.fixture(scope="module")
def level5():
    g, inp, O = problem(5, threads=THREADS)
    assert g.nb == 4692
    P = device_problem(g, inp)
    del inp
    yield g, O, P
    P.close()
    O.close()


def zero_x(g):
    return np.zeros((g.nb, 16 + 2 * VC, 16 + 2 * VC, 16 + 2 * VC))


def test_level5_assembly_matches_oracle(level5):
    g, O, P = level5
    for name in ("AP", "AW", "AE", "AS", "AN", "AB", "AT", "B"):
        assert_bitwise(interior(P.download(name, VC)), interior(O.field(name)), name)


def test_level5_rbgs_bitwise(level5):
    g, O, P = level5
    O.field("X")[...] = 0.0
    P.upload("X", zero_x(g), VC)
    ro = O.solve_rbgs(1.5, 20, 0.0)
    rg = P.solve_rbgs(1.5, 20, 0.0)
    assert rg["count"] == ro["count"] == 21
    assert_bitwise(rg["history"], ro["history"], "residual history")
    got = P.download("X", VC)
    assert_bitwise(interior(got), interior(O.field("X")), "pressure")
    gg, rg2 = fo.face_guides(got, VC, 2), fo.face_guides(O.field("X"), VC, 2)
    for f in range(6):
        assert_bitwise(gg[f], rg2[f], f"guides face {f}")


def test_level5_bicgstab_bitwise(level5):
    g, O, P = level5
    O.field("X")[...] = 0.0
    P.upload("X", zero_x(g), VC)
    ro = O.solve_bicgstab(1.0, 2, 5, 1e-10)
    rg = P.solve_bicgstab(1.0, 2, 5, 1e-10)
    assert rg["count"] == ro["count"] == 6
    assert_bitwise(rg["history"], ro["history"], "residual history")
    assert_bitwise(interior(P.download("X", VC)), interior(O.field("X")), "pressure")


def test_level5_mixed_bitwise(level5):
    g, O, P = level5
    O.field("X")[...] = 0.0
    P.fill("X", 0.0)
    ro = O.solve_mixed(1.5, 8, 4, 3, 0.0)
    rg = P.solve_mixed(1.5, 8, 4, 3, 0.0)
    assert rg["count"] == ro["count"] == 4
    assert_bitwise(rg["history"], ro["history"], "residual history")
    assert_bitwise(interior(P.download("X", VC)), interior(O.field("X")), "pressure")


def test_level5_bicgstab_restarts_bitwise(level5):
    """160 iterations with restarts on a thousandfold residual drop: past the
    first restart (where the residual jumps), so the A*x kernel's sums feed
    a long, sensitive recurrence; one wrong block sum changes the history."""
    g, O, P = level5
    O.field("X")[...] = 0.0
    P.upload("X", zero_x(g), VC)
    ro = O.solve_bicgstab(1.0, 2, 160, 0.0, restart_drop=1e-3)
    rg = P.solve_bicgstab(1.0, 2, 160, 0.0, restart_drop=1e-3)
    assert rg["count"] == ro["count"] == 161
    h = np.asarray(ro["history"])
    assert np.any(h[1:] > 10.0 * h[:-1]), "no restart within the run"
    assert_bitwise(rg["history"], ro["history"], "residual history")
    assert_bitwise(interior(P.download("X", VC)), interior(O.field("X")), "pressure")


def test_level5_solves_repeat_bitwise(level5):
    """The same solve three times gives the same history bit for bit: the
    persistent kernels' per-block and cross-block sums do not depend on
    timing (FP64 BiCGSTAB with restarts to 1e-8, the mixed solve to 1e-8)."""
    g, O, P = level5

    def bicg():
        P.fill("X", 0.0)
        return P.solve_bicgstab(1.0, 2, 50000, 1e-8, restart_drop=1e-3)

    def mixed():
        P.fill("X", 0.0)
        return P.solve_mixed(1.5, 8, 4, 5000, 1e-8)

    for solve in (bicg, mixed):
        runs = [solve() for _ in range(3)]
        for r in runs[1:]:
            assert r["count"] == runs[0]["count"]
            assert_bitwise(r["history"], runs[0]["history"], "repeated residual history")
