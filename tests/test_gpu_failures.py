"""Failure handling on the GPU, without faulting it.

* A bounded device wait that runs out.  The wait limit is a pool setting;
  set to 0, the sweep kernel's waits on work of its other roles give up (the
  copies they wait for take microseconds), and a test hook makes the mixed
  sweep wait for a copy it never issues; the solve must end with
  FFVGPU_TIMEOUT --
  the kernel's roles leave their loops, copies in flight are waited for, the
  state reports the roles that gave up -- and, with the limit restored, the
  same pool must solve again bit for bit as the oracle does.
* A zero diagonal (a cell whose Ap is 0): the reference divides by it and
  its IsConverged exits on the NaN/Inf residual (src/FFV/FFVILS.h:36-43);
  here the solve reports FFVGPU_NAN_DETECTED and the pool stays usable.
* Cancellation of a running solve and of serve requests, while waiting and
  while solving; the other solves' results are unchanged.
"""
import numpy as np
import pytest

import ffvgpu
from helpers import VC, assert_bitwise, device_problem, interior, problem

pytestmark = pytest.mark.gpu


def zero_x(g):
    return np.zeros((g.nb, 16 + 2 * VC, 16 + 2 * VC, 16 + 2 * VC))


def test_rbgs_wait_limit_runs_out_and_pool_stays_usable():
    g, inp, O = problem(2)
    P = device_problem(g, inp)
    P.upload("X", zero_x(g), VC)
    P.set_wait_limit(0.0)
    with pytest.raises(ffvgpu.FFVGPUError) as e:
        P.solve_rbgs(1.5, 30, 0.0)
    assert e.value.status == ffvgpu.TIMEOUT
    assert "bounded device wait" in str(e.value) and "drain" not in str(e.value)
    with pytest.raises(ffvgpu.FFVGPUError) as e:
        P.calc_r2()
    assert e.value.status == ffvgpu.TIMEOUT
    P.set_wait_limit(4.0)
    P.upload("X", zero_x(g), VC)
    O.field("X")[...] = 0.0
    ro = O.solve_rbgs(1.5, 30, 0.0)
    rg = P.solve_rbgs(1.5, 30, 0.0)
    assert_bitwise(rg["history"], ro["history"], "history after the timeout")
    assert_bitwise(interior(P.download("X", VC)), interior(O.field("X")), "x after the timeout")
    P.close()
    O.close()


def test_mixed_wait_limit_runs_out_and_pool_stays_usable():
    """The mixed sweep's one wait is for the block copy it issued itself, which
    lands within the wait instruction's own suspend time even with a zero
    limit; the test hook makes the sweep wait for a copy it never issues."""
    g, inp, O = problem(2)
    P = device_problem(g, inp)
    P.fill("X", 0.0)
    P.set_wait_limit(0.05)
    P.stall_next_solve()
    with pytest.raises(ffvgpu.FFVGPUError) as e:
        P.solve_mixed(1.5, 8, 4, 6, 0.0)
    assert e.value.status == ffvgpu.TIMEOUT
    assert "sweep" in str(e.value) and "drain" not in str(e.value)
    P.set_wait_limit(4.0)  # the captured graph is rebuilt with the new limit
    P.fill("X", 0.0)
    O.field("X")[...] = 0.0
    ro = O.solve_mixed(1.5, 8, 4, 6, 0.0)
    rg = P.solve_mixed(1.5, 8, 4, 6, 0.0)
    assert_bitwise(rg["history"], ro["history"], "history after the timeout")
    assert_bitwise(interior(P.download("X", VC)), interior(O.field("X")), "x after the timeout")
    P.close()
    O.close()


def test_matvec_wait_limit_runs_out_and_pool_stays_usable():
    """The pipelined A*x's consumers wait for ring slots its producer issues;
    the test hook makes the producer issue none, so the first wait runs out:
    TIMEOUT naming the A*x, no copy left in flight, and the pool then solves
    bit for bit as before."""
    g, inp, O = problem(2)
    P = device_problem(g, inp)
    P.fill("X", 0.0)
    P.set_wait_limit(0.05)
    P.stall_next_matvec()
    with pytest.raises(ffvgpu.FFVGPUError) as e:
        P.solve_mixed(1.5, 8, 4, 6, 0.0)
    assert e.value.status == ffvgpu.TIMEOUT
    assert "A*x" in str(e.value) and "drain" not in str(e.value)
    P.set_wait_limit(4.0)
    P.fill("X", 0.0)
    O.field("X")[...] = 0.0
    ro = O.solve_mixed(1.5, 8, 4, 6, 0.0)
    rg = P.solve_mixed(1.5, 8, 4, 6, 0.0)
    assert_bitwise(rg["history"], ro["history"], "history after the timeout")
    assert_bitwise(interior(P.download("X", VC)), interior(O.field("X")), "x after the timeout")
    P.close()
    O.close()


def test_zero_diagonal_is_reported_as_nan_and_pool_stays_usable():
    g, inp, O = problem(1)
    P = device_problem(g, inp)
    ap = P.download("AP", VC)
    bad = ap.copy()
    bad[3, 9, 9, 9] = 0.0
    P.upload("AP", bad, VC)
    P.upload("X", zero_x(g), VC)
    r = P.solve_rbgs(1.0, 10, 0.0)
    assert r["status"] == ffvgpu.NAN_DETECTED
    P.fill("X", 0.0)
    r = P.solve_bicgstab(1.0, 2, 10, 1e-10)
    assert r["status"] == ffvgpu.NAN_DETECTED
    P.fill("X", 0.0)
    r = P.solve_mixed(1.5, 8, 4, 10, 1e-8)
    assert r["status"] == ffvgpu.NAN_DETECTED
    # the good diagonal back: the solve is the oracle's again
    P.upload("AP", ap, VC)
    P.upload("X", zero_x(g), VC)
    O.field("X")[...] = 0.0
    ro = O.solve_rbgs(1.0, 10, 0.0)
    rg = P.solve_rbgs(1.0, 10, 0.0)
    assert_bitwise(rg["history"], ro["history"], "history")
    P.close()
    O.close()


def sphere(level, seed, **kw):
    return ffvgpu.sphere_problem(level, seed=seed, **kw)


def test_cancel_a_running_instance_leaves_the_others_unchanged():
    def run(cancel):
        B = ffvgpu.Batch(2000, 4)
        a = B.admit_sphere(sphere(2, 5))
        b = B.admit_sphere(sphere(2, 6, center=(2.0, 0.5, 0.0)))
        B.begin(a, count_max=300)
        B.begin(b, count_max=300)
        B.advance(3)
        if cancel:
            B.cancel(b)
        done = set(B.poll())
        while a not in done or (not cancel and b not in done):
            B.advance(4)
            done |= set(B.poll())
        ra, xa = B.result(a, count_max=300), interior(B.download(a, "X", VC)).copy()
        rb = B.result(b, count_max=300)
        if cancel:
            # b can be solved again from scratch after its cancellation
            B.fill(b, "X", 0.0)
            B.begin(b, count_max=300)
            while b not in B.poll():
                B.advance(4)
            rb = (rb, B.result(b, count_max=300))
        free = B.free_blocks()[0]
        B.close()
        return ra, xa, rb, free

    ra0, xa0, rb0, _ = run(False)
    ra1, xa1, (rb_cancelled, rb_again), _ = run(True)
    assert ra1["count"] == ra0["count"] and ra1["residual"] == ra0["residual"]
    assert_bitwise(xa1, xa0, "x of the instance that was not cancelled")
    assert rb_cancelled["status"] == ffvgpu.CANCELLED and rb_cancelled["count"] == 3
    assert_bitwise(rb_cancelled["history"], rb0["history"][:3], "history before the cancel")
    assert rb_again["count"] == rb0["count"] and rb_again["residual"] == rb0["residual"]


def test_serve_cancels_waiting_and_running_requests():
    big = sphere(3, 21)                    # 548 blocks, ~190 iterations
    other = sphere(3, 22, center=(0.5, 0.0, 0.0))
    B = ffvgpu.Batch(600, 4)               # room for one of them at a time
    alone = B.serve([0.0], [big], iterations_per_step=8, count_max=2000)[0]
    assert alone["status"] == ffvgpu.OK
    # 'other' arrives with 'big' but cannot be admitted while 'big' runs; it is
    # withdrawn after 5 ms, long before 'big' ends
    out = B.serve([0.0, 0.0], [big, other], iterations_per_step=8, count_max=2000,
                  cancels=[0.0, 0.005])
    assert out[0]["status"] == ffvgpu.OK
    assert out[0]["count"] == alone["count"] and out[0]["residual"] == alone["residual"]
    assert out[1]["status"] == ffvgpu.CANCELLED and out[1]["count"] == 0
    assert out[1]["admit_s"] == 0.0 and out[1]["blocks"] == 0
    # a request withdrawn while it solves: stopped, its blocks released
    out = B.serve([0.0], [big], iterations_per_step=8, count_max=2000, cancels=[0.01])
    assert out[0]["status"] == ffvgpu.CANCELLED
    assert 0 < out[0]["count"] < alone["count"]
    assert B.free_blocks()[0] == 600
    B.close()
