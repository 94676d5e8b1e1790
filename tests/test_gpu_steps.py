"""The pressure part of the fractional time step on the GPU against the oracle.

Solver::UpdateP and Solver::UpdateU (src/FFV/Solver.cpp:5294-5771) run on the
device through ffvgpu_update_p / ffvgpu_update_u, with u* regenerated every
step from a per-step seed (sigma 0.05, the at-scale workload's noise) by the
device generator, and on the oracle through the same sequence with the host
generator's u*.  The pressure of every step (which enters the next step's
bcut_remove_p and is its solve's starting iterate), the corrected velocity
and the solve's residual history are compared bit for bit.
"""
import numpy as np
import pytest

import ffvgpu
import ffv_oracle as fo
from helpers import VC, assert_bitwise, device_problem, interior, problem

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("level,steps,solver", [
    (2, 3, ffvgpu.SOLVER_BICGSTAB),
    (1, 3, ffvgpu.SOLVER_RBGS),
])
def test_time_steps_bitwise(level, steps, solver):
    g, inp, O = problem(level, sigma=0.05)
    P = device_problem(g, inp)
    P.fill("X", 0.0)
    O.field("X")[...] = 0.0
    for n in range(steps):
        seed = 100 + n
        P.generate_sphere(ffvgpu.sphere_problem(level, seed=seed, sigma=0.05))
        u_star = g.fill(seed=seed, sigma=0.05, vc=VC)
        if solver == ffvgpu.SOLVER_BICGSTAB:
            rg = P.update_p(solver, omega=1.0, pre_count=2, count_max=4, epsilon=0.0)
            ro = fo.time_step(O, u_star, lambda o: o.solve_bicgstab(1.0, 2, 4, 0.0))
        else:
            rg = P.update_p(solver, omega=1.0, count_max=6, epsilon=0.0)
            ro = fo.time_step(O, u_star, lambda o: o.solve_rbgs(1.0, 6, 0.0))
        P.update_u()
        assert rg["count"] == ro["count"], (n, rg, ro["count"])
        assert rg["residual"] == ro["residual"], (n, rg["residual"], ro["residual"])
        assert_bitwise(interior(P.download("X", VC)), interior(O.field("X")), f"p, step {n}")
        for u in ("UX", "UY", "UZ"):
            assert_bitwise(interior(P.download(u, VC)), interior(O.field(u)), f"{u}, step {n}")
    P.close()
