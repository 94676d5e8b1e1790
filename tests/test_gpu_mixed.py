"""Mixed-precision form, batches and the device generator, on the GPU.

The mixed solve (FP64 BiCGSTAB recurrence, red-black SOR preconditioner on
32-bit coefficients with FP64 arithmetic) is checked bit for bit against the
oracle's restatement (orc_mixed) for several sweep groupings, on grids with
fewer blocks than CTAs and with several blocks per CTA; its converged pressure is compared
with the FP64 solve of the same system (tolerance stated in the test).  A
batch's instances are checked to give the same bits alone and in a mix,
admitted together or while others run, and the device generator + assembly
of an instance is checked against the host generator + oracle assembly.
"""
import numpy as np
import pytest

import ffvgpu
from helpers import VC, assert_bitwise, device_problem, interior, problem

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("level,omega,sweeps,per,count", [
    (1, 1.5, 8, 4, 12),
    (1, 1.0, 4, 4, 10),
    (2, 1.5, 8, 4, 8),
    (2, 1.2, 6, 2, 6),
    (1, 1.5, 3, 1, 6),
    (3, 1.5, 8, 4, 3),   # 548 blocks: several blocks per CTA (coefficient copy pipeline)
    (3, 1.2, 6, 2, 2),
])
def test_mixed_solve_bitwise_against_oracle(level, omega, sweeps, per, count):
    g, inp, O = problem(level)
    P = device_problem(g, inp)
    P.fill("X", 0.0)
    O.field("X")[...] = 0.0
    ro = O.solve_mixed(omega, sweeps, per, count, 0.0)
    rg = P.solve_mixed(omega, sweeps, per, count, 0.0)
    assert rg["count"] == ro["count"] == count + 1
    assert_bitwise(rg["history"], ro["history"], "residual history")
    assert_bitwise(interior(P.download("X", VC)), interior(O.field("X")), "pressure")
    P.close()


@pytest.mark.parametrize("level,omega,sweeps,per,count", [
    (1, 1.5, 8, 4, 8),
    (2, 1.2, 6, 2, 5),
    (3, 1.5, 8, 4, 2),   # several blocks per CTA, uniform and non-uniform blocks
])
def test_fp64_data_variant_bitwise_against_oracle(level, omega, sweeps, per, count):
    """The same preconditioner on FP64 data (coefficients unrounded, FP64
    iterate between exchanges): bit for bit the oracle's restatement."""
    g, inp, O = problem(level)
    P = device_problem(g, inp)
    P.fill("X", 0.0)
    O.field("X")[...] = 0.0
    ro = O.solve_mixed(omega, sweeps, per, count, 0.0, fp64_data=True)
    rg = P.solve_mixed(omega, sweeps, per, count, 0.0, fp64_data=True)
    assert rg["count"] == ro["count"] == count + 1
    assert_bitwise(rg["history"], ro["history"], "residual history")
    assert_bitwise(interior(P.download("X", VC)), interior(O.field("X")), "pressure")
    # and it is a different computation from the 32-bit data form
    P.fill("X", 0.0)
    r32 = P.solve_mixed(omega, sweeps, per, count, 0.0)
    assert not np.array_equal(r32["history"], rg["history"])
    P.close()


@pytest.mark.parametrize("threads,depth,sweep_threads,form,extra", [
    (128, 1, 512, 1, {}), (512, 3, 512, 1, {}), (256, 2, 256, 0, {}), (128, 3, 256, 1, {}),
    (256, 1, 512, 1, {"fp64_data": True}), (256, 1, 512, 1, {"flux_correction": True})])
def test_launch_settings_do_not_change_results(threads, depth, sweep_threads, form, extra):
    """CTA sizes of the A*x, update and sweep kernels, the sweep kernel's
    staging depth and the A*x kernel's form (pipelined or a block per CTA)
    are tuning knobs only: the same bits as the defaults (the 512-lane block
    tree and the 256-lane cross-block tree do not depend on them, and the
    sweep keeps each cell's order of terms)."""
    g, inp, O = problem(3)
    P = device_problem(g, inp)
    P.fill("X", 0.0)
    ref = P.solve_mixed(1.5, 8, 4, 4, 0.0, **extra)
    xr = interior(P.download("X", VC)).copy()
    P.fill("X", 0.0)
    r = P.solve_mixed(1.5, 8, 4, 4, 0.0, threads_per_block=threads, stage_depth=depth,
                      sweep_threads=sweep_threads, matvec_form=form, **extra)
    assert_bitwise(r["history"], ref["history"], "residual history")
    assert_bitwise(interior(P.download("X", VC)), xr, "pressure")
    P.close()


def test_mixed_converges_and_matches_fp64_solution():
    g, inp, O = problem(2)
    P = device_problem(g, inp)
    P.fill("X", 0.0)
    rm = P.solve_mixed(1.5, 8, 4, 500, 1e-8)
    assert rm["status"] == ffvgpu.OK and rm["residual"] <= 1e-8, rm
    # blocks whose seven coefficients are bitwise the same in every cell are
    # read once per block by the mixed kernels: the count matches the oracle's A
    A = np.stack([interior(O.field(f)).reshape(g.nb, -1)
                  for f in ("AP", "AW", "AE", "AS", "AN", "AB", "AT")]).view(np.int64)
    n_uniform = int(np.all(A == A[:, :, :1], axis=(0, 2)).sum())
    assert 0 < n_uniform < g.nb and rm["uniform_blocks"] == n_uniform, (rm["uniform_blocks"], n_uniform)
    pm = interior(P.download("X", VC)).copy()
    # the oracle's converged mixed solve: same iteration count, same bits
    O.field("X")[...] = 0.0
    ro = O.solve_mixed(1.5, 8, 4, 500, 1e-8)
    assert ro["count"] == rm["count"]
    assert_bitwise(pm, interior(O.field("X")), "converged pressure")
    # FP64 reference solution of the same system, far below the mixed tolerance
    P.fill("X", 0.0)
    rf = P.solve_bicgstab(1.0, 2, 3000, 1e-12)
    assert rf["status"] == ffvgpu.OK
    pf = interior(P.download("X", VC))
    err = np.linalg.norm(pm - pf) / np.linalg.norm(pf)
    # both solve A p = b; a 1e-8 relative residual bounds the relative error of
    # p by the condition number times 1e-8 -- here it must stay below 1e-5
    assert err < 1e-5, err
    P.close()


def test_mixed_edge_cases():
    g, inp, O = problem(1)
    P = device_problem(g, inp)
    P.fill("X", 0.0)
    r = P.solve_mixed(1.5, 8, 4, 0, 1e-8)          # countMax 0: no iteration
    assert r["count"] == 1
    with pytest.raises(ffvgpu.FFVGPUError):
        P.solve_mixed(1.5, 6, 4, 10, 1e-8)          # sweeps not a multiple
    with pytest.raises(ffvgpu.FFVGPUError):
        P.solve_mixed(2.5, 8, 4, 10, 1e-8)          # omega outside (0, 2)
    P.fill("B", 0.0)                                # b = 0: count 0, residual 0
    r = P.solve_mixed(1.5, 8, 4, 10, 1e-8)
    assert r["count"] == 0 and r["residual"] == 0.0
    P.close()


def sphere(level, seed, **kw):
    return ffvgpu.sphere_problem(level, seed=seed, **kw)


@pytest.mark.parametrize("form", [0, 1])
def test_capped_grids_and_list_chunks_give_the_same_bits(form):
    """One CTA per persistent grid: a level-4 pool (1164 blocks) then spans two
    chunks of the sweep kernel's live-block list (1024 entries per CTA) and of
    the pipelined A*x's (800), and every block of a CTA's list goes through
    one pipeline; three CTAs leave one chunk each.  Same bits as the full
    grids: the block and cross-block trees do not depend on the grid."""
    g = ffvgpu.SphereGrid(4)
    P = ffvgpu.Pool(g.desc())
    P.assemble_sphere(sphere(4, 11))
    P.fill("X", 0.0)
    ref = P.solve_mixed(1.5, 8, 4, 3, 0.0, matvec_form=form)
    xr = interior(P.download("X", VC)).copy()
    for ctas in (1, 3):
        P.cap_grids(ctas)
        P.fill("X", 0.0)
        r = P.solve_mixed(1.5, 8, 4, 3, 0.0, matvec_form=form)
        assert r["count"] == ref["count"] == 4
        assert_bitwise(r["history"], ref["history"], f"residual history, {ctas} CTAs")
        assert_bitwise(interior(P.download("X", VC)), xr, f"pressure, {ctas} CTAs")
    P.cap_grids(0)
    P.close()


def test_capped_grid_batch_instance_runs_across_chunks():
    """Three instances (1644 blocks) on one CTA per grid: the pipelined A*x
    advances an instance's ticket once per run of its blocks in a chunk of
    800, so runs are cut by chunk ends; every instance keeps its bits."""
    B = ffvgpu.Batch(2000, 4)
    ids = [B.admit_sphere(sphere(3, s)) for s in (5, 6, 7)]
    for i in ids:
        B.fill(i, "X", 0.0)
    B.solve_mixed(1.5, 8, 4, 3, 0.0)
    ref = [(B.result(i, 8), interior(B.download(i, "X", VC)).copy()) for i in ids]
    B.cap_grids(1)
    for i in ids:
        B.fill(i, "X", 0.0)
    B.solve_mixed(1.5, 8, 4, 3, 0.0)
    for i, (rr, xr) in zip(ids, ref):
        r = B.result(i, 8)
        assert r["count"] == rr["count"] >= 3
        assert_bitwise(r["history"], rr["history"], f"instance {i} residual history")
        assert_bitwise(interior(B.download(i, "X", VC)), xr, f"instance {i} pressure")
    B.close()


def test_device_generator_and_assembly_match_host_and_oracle():
    B = ffvgpu.Batch(2000, 8)
    kw = dict(center=(1.0, 0.5, -0.25), radius=0.4)
    i = B.admit_sphere(sphere(2, 77, **kw))
    g, inp, O = problem(2, seed=77, **kw)
    assert B.blocks(i) == g.nb
    for f in ("AP", "AW", "AE", "AS", "AN", "AB", "AT", "B"):
        assert_bitwise(interior(B.download(i, f, VC)), interior(O.field(f)), f)
    for u in ("UX", "UY", "UZ"):
        assert_bitwise(interior(B.download(i, u, VC)), interior(inp[u]), u)
    B.close()


def solve_alone(level, seed, count, eps, kw):
    B = ffvgpu.Batch(4000, 4)
    i = B.admit_sphere(sphere(level, seed, **kw))
    B.begin(i, count_max=count, epsilon=eps)
    for _ in range(count):
        B.advance(4)
        if i in B.poll():
            break
    r = B.result(i, count_max=count)
    x = interior(B.download(i, "X", VC)).copy()
    B.close()
    return r, x


CASES = [(2, 5, dict()), (1, 9, dict(center=(2.0, 0.0, 0.0), radius=0.7)),
         (2, 13, dict(center=(-1.0, 1.0, 0.5), radius=0.3))]


def test_batch_instances_bitwise_alone_and_in_a_mix():
    alone = [solve_alone(L, s, 40, 1e-8, kw) for (L, s, kw) in CASES]
    B = ffvgpu.Batch(8000, 8)
    ids = [B.admit_sphere(sphere(L, s, **kw)) for (L, s, kw) in CASES]
    for i in ids:
        B.begin(i, count_max=40, epsilon=1e-8)
    left = set(ids)
    for _ in range(100):
        if not left:
            break
        B.advance(3)
        left -= set(B.poll())
    assert not left
    for i, (ra, xa) in zip(ids, alone):
        r = B.result(i, count_max=40)
        assert r["count"] == ra["count"]
        assert_bitwise(r["history"], ra["history"], "history in the mix")
        assert_bitwise(interior(B.download(i, "X", VC)), xa, "pressure in the mix")
    B.close()


def test_batch_admission_while_others_run_and_release():
    alone = [solve_alone(L, s, 40, 1e-8, kw) for (L, s, kw) in CASES]
    B = ffvgpu.Batch(6000, 4)
    name = {}  # instance slot -> case; a released slot is reused by the next admission
    a = B.admit_sphere(sphere(*CASES[0][:2], **CASES[0][2]))
    name[a] = 0
    B.begin(a, count_max=40, epsilon=1e-8)
    B.advance(5)
    b = B.admit_sphere(sphere(*CASES[1][:2], **CASES[1][2]))   # joins mid-solve
    name[b] = 1
    B.begin(b, count_max=40, epsilon=1e-8)
    done = {}
    admitted_third = False
    for _ in range(200):
        if len(done) == 3:
            break
        B.advance(2)
        for i in B.poll():
            done[name.pop(i)] = (B.result(i, count_max=40),
                                 interior(B.download(i, "X", VC)).copy())
            B.release(i)
            if not admitted_third:
                admitted_third = True
                c = B.admit_sphere(sphere(*CASES[2][:2], **CASES[2][2]))
                name[c] = 2
                B.begin(c, count_max=40, epsilon=1e-8)
    assert len(done) == 3
    for k, (ra, xa) in enumerate(alone):
        r, x = done[k]
        assert r["count"] == ra["count"]
        assert_bitwise(r["history"], ra["history"], "history, staggered")
        assert_bitwise(x, xa, "pressure, staggered")
    assert B.free_blocks()[0] == 6000
    B.close()


def test_batch_instance_matches_one_grid_pool():
    g, inp, O = problem(2, seed=21)
    P = device_problem(g, inp)
    P.fill("X", 0.0)
    rp = P.solve_mixed(1.5, 8, 4, 30, 1e-8)
    xp = interior(P.download("X", VC)).copy()
    P.close()
    B = ffvgpu.Batch(1000, 2)
    i = B.admit_sphere(sphere(2, 21))
    B.begin(i, count_max=30, epsilon=1e-8)
    for _ in range(30):
        if i in B.poll():
            break
        B.advance(4)
    r = B.result(i, count_max=30)
    assert r["count"] == rp["count"]
    assert_bitwise(r["history"], rp["history"], "history")
    assert_bitwise(interior(B.download(i, "X", VC)), xp, "pressure")
    B.close()


def test_batch_refuses_pool_wide_calls_and_full_capacity():
    B = ffvgpu.Batch(190, 2)
    i = B.admit_sphere(sphere(1, 3))                 # 72 blocks
    assert B.admit_sphere(sphere(2, 4)) is None      # 128 blocks do not fit in the other 118
    with pytest.raises(ffvgpu.FFVGPUError):
        ffvgpu._check(ffvgpu.lib().ffvgpu_fold_bc(B._h), "fold_bc")
    B.release(i)
    assert B.admit_sphere(sphere(2, 4)) is not None
    B.close()


def test_serve_continuous_batching_results_equal_alone():
    """ffvgpu_serve: requests arriving while others run are admitted as blocks
    free up; each result equals the same request solved alone."""
    cases = CASES + [(1, 17, dict(center=(5.0, -1.0, 1.0), radius=0.6))]
    alone = [solve_alone(L, s, 60, 1e-8, kw)[0] for (L, s, kw) in cases]
    B = ffvgpu.Batch(300, 4)            # room for two of these requests at a time
    arrivals = [0.0, 0.0, 0.002, 0.004]
    probs = [sphere(L, s, **kw) for (L, s, kw) in cases]
    out = B.serve(arrivals, probs, iterations_per_step=4, count_max=60)
    for o, ra in zip(out, alone):
        assert o["finish_s"] >= o["admit_s"] >= o["arrival_s"] - 1e-9
        assert o["count"] == ra["count"]
        assert o["residual"] == ra["residual"]
    assert B.free_blocks()[0] == 300
    B.close()


def test_autotuner_times_candidates_and_leaves_x_zero():
    B = ffvgpu.Batch(600, 4)
    ids = [B.admit_sphere(sphere(1, 3)), B.admit_sphere(sphere(1, 4, center=(3.0, 1.0, 0.0)))]
    space = [(1.5, 8, 4, 8), (1.2, 4, 4, 4), (1.5, 8, 8, 16)]
    recs, best = B.autotune(ids, space=space, count_max=400)
    # stage 1: the three numerical settings; stage 2 (when one converged): the
    # fastest of them at the 35 other launch settings
    assert len(recs) in (3, 38) and all(r["ms"] > 0 and r["max_count"] >= 1 for r in recs)
    if len(recs) == 38:
        assert {(r["threads_per_block"], r["stage_depth"], r["sweep_threads"], r["matvec_form"])
                for r in recs[3:]} == {(nt, dp, st, mv) for nt in (128, 256, 512)
                                       for dp in (1, 2, 3) for st in (512, 256)
                                       for mv in (0, 1)} - {(256, 1, 256, 0)}
    assert best == -1 or recs[best]["converged"]
    if best >= 0:
        assert recs[best]["ms"] == min(r["ms"] for r in recs if r["converged"])
    for i in ids:
        assert not np.any(interior(B.download(i, "X", VC)))
    # the tuned setting reproduces the solve it timed
    if best >= 0:
        r = recs[best]
        B.begin(ids[0], omega=r["omega"], sweeps=r["sweeps"],
                sweeps_per_exchange=r["sweeps_per_exchange"], count_max=400,
                threads_per_block=r["threads_per_block"], stage_depth=r["stage_depth"],
                sweep_threads=r["sweep_threads"])
        for _ in range(400):
            B.advance(r["iterations_per_replay"])
            if ids[0] in B.poll():
                break
        assert B.result(ids[0])["count"] <= r["max_count"]
    B.close()
