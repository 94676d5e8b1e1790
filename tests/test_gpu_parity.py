"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Every FP64 kernel of the path rounds exactly as the reference's Fortran does
and every sum uses the same fixed tree in both, so the bar is bit equality:
interior values, guide layers, residual histories and Krylov scalars.  The
reference's own block-sum order (serial per block, blocks in id order) is
checked separately to a stated relative tolerance.
"""
import os

import numpy as np
import pytest

import ffvgpu
import ffv_oracle as fo
from helpers import VC, assert_bitwise, device_problem, interior, problem, rel_err

pytestmark = pytest.mark.gpu
THREADS = os.cpu_count() or 8
# Relative tolerance of the FP64 path against the reference-order oracle
# (sums in a different order): residual histories agree to 1e-12.
TOL_REFERENCE_ORDER = 1e-12


@pytest.fixture(scope="module")
def l2():
    g, inp, O = problem(2, threads=THREADS)
    P = device_problem(g, inp)
    yield g, inp, O, P
    P.close()
    O.close()


def random_field(g, seed):
    rng = np.random.default_rng(seed)
    w = 16 + 2 * VC
    return rng.standard_normal((g.nb, w, w, w))


def test_upload_download_interior_roundtrip(l2):
    g, inp, O, P = l2
    for name in ("UX", "C3", "AP", "AT", "B", "VN"):
        got = P.download(name, VC)
        assert_bitwise(interior(got), interior(O.field(name)), name)
    for name in ("CID0", "CID5", "PID"):
        got = P.download(name, VC)
        assert_bitwise(interior(got), interior(O.field(name)), name)


@pytest.mark.parametrize("bc", [
    (ffvgpu.P_BC_TYPE, ffvgpu.P_BC_VALUE),
    ((0, 1, 1, 0, 0, 1), (0.25, -0.5, 1.5, -2.0, 0.125, 3.0)),
])
def test_exchange_two_layers_match_oracle(bc):
    g, inp, O = problem(2, threads=THREADS)
    P = ffvgpu.Pool(g.desc(*bc))
    x = random_field(g, 7)
    O.set_bc(*bc)
    O.field("X")[...] = x
    O.exchange("X", *bc)
    P.upload("X", x, VC)
    P.exchange("X")
    got = P.download("X", VC)
    ref = O.field("X")
    assert_bitwise(interior(got), interior(ref), "interior")
    gg = fo.face_guides(got, VC, 2)
    rg = fo.face_guides(ref, VC, 2)
    for f in range(6):
        assert_bitwise(gg[f], rg[f], f"face {f}")
    P.close()


def test_assembly_and_bc_folding_match_oracle(l2):
    g, inp, O, P = l2
    for name in ("AP", "AW", "AE", "AS", "AN", "AB", "AT", "B", "VW", "VE", "VS", "VN", "VB", "VT"):
        assert_bitwise(interior(P.download(name, VC)), interior(O.field(name)), name)


def test_single_sweep_and_residual_match_oracle():
    g, inp, O = problem(2, threads=THREADS)
    P = device_problem(g, inp)
    x = random_field(g, 11)
    O.field("X")[...] = x
    O.exchange("X", ffvgpu.P_BC_TYPE, ffvgpu.P_BC_VALUE)
    P.upload("X", O.field("X").copy(), VC)
    # stale (uploaded) guides are what the first sweep must read
    assert P.calc_r2() == O.calc_r2()
    O.rbgs_sweep(1.5)
    P.rbgs_sweep(1.5)
    got = P.download("X", VC)
    assert_bitwise(interior(got), interior(O.field("X")), "x after sweep")
    gg, rg = fo.face_guides(got, VC, 2), fo.face_guides(O.field("X"), VC, 2)
    for f in range(6):
        assert_bitwise(gg[f], rg[f], f"guides face {f}")
    assert P.calc_r2() == O.calc_r2()
    assert P.dot("B", "B") == O.dot("B", "B")
    assert P.dot("X", "B") == O.dot("X", "B")
    P.close()


def test_first_sweep_reads_stored_guides():
    """RBGS_Smoother reads whatever x holds in its guide cells: upload
    deliberately inconsistent guides and check the sweep follows them."""
    g, inp, O = problem(1, threads=THREADS)
    P = device_problem(g, inp)
    x = random_field(g, 5)  # guide cells random, not an exchange result
    O.field("X")[...] = x
    P.upload("X", x, VC)
    O.rbgs_sweep(1.2)
    P.rbgs_sweep(1.2)
    assert_bitwise(interior(P.download("X", VC)), interior(O.field("X")), "x")
    P.close()


@pytest.mark.parametrize("level,omega,sweeps", [(2, 1.5, 60), (3, 1.5, 200), (2, 1.0, 40)])
def test_rbgs_solve_bitwise(level, omega, sweeps):
    g, inp, O = problem(level, threads=THREADS)
    P = device_problem(g, inp)
    x0 = np.zeros((g.nb, 20, 20, 20))
    O.field("X")[...] = x0
    P.upload("X", x0, VC)
    ro = O.solve_rbgs(omega, sweeps, 0.0)
    rg = P.solve_rbgs(omega, sweeps, 0.0)
    assert rg["count"] == ro["count"] == sweeps + 1
    assert_bitwise(rg["history"], ro["history"], "residual history")
    assert rg["residual"] == ro["residual"]
    got = P.download("X", VC)
    assert_bitwise(interior(got), interior(O.field("X")), "pressure")
    gg, rgd = fo.face_guides(got, VC, 2), fo.face_guides(O.field("X"), VC, 2)
    for f in range(6):
        assert_bitwise(gg[f], rgd[f], f"guides face {f}")
    # blocks whose seven coefficients are bitwise the same in every cell stream
    # b only (their coefficients come from one record): the count the solve
    # reports is the oracle's A's
    A = np.stack([interior(O.field(f)).reshape(g.nb, -1)
                  for f in ("AP", "AW", "AE", "AS", "AN", "AB", "AT")]).view(np.int64)
    n_uniform = int(np.all(A == A[:, :, :1], axis=(0, 2)).sum())
    assert 0 < n_uniform < g.nb and rg["uniform_blocks"] == n_uniform
    P.close()


def test_rbgs_history_vs_reference_sum_order():
    g, inp, O = problem(2, threads=THREADS, reduction=fo.RED_REFERENCE)
    P = device_problem(g, inp)
    x0 = np.zeros((g.nb, 20, 20, 20))
    O.field("X")[...] = x0
    P.upload("X", x0, VC)
    ro = O.solve_rbgs(1.5, 50, 0.0)
    rg = P.solve_rbgs(1.5, 50, 0.0)
    assert rel_err(rg["history"], ro["history"]) <= TOL_REFERENCE_ORDER
    np.testing.assert_allclose(rg["history"], ro["history"], rtol=TOL_REFERENCE_ORDER, atol=0)
    # x never depends on the sums: still bit equal
    assert_bitwise(interior(P.download("X", VC)), interior(O.field("X")), "pressure")
    P.close()


def test_rbgs_converges_early_and_keeps_that_iterate():
    g, inp, O = problem(0, threads=THREADS, radius=0.0)
    P = device_problem(g, inp)
    x0 = np.zeros((g.nb, 20, 20, 20))
    O.field("X")[...] = x0
    P.upload("X", x0, VC)
    ro = O.solve_rbgs(1.0, 500, 2e-2)
    rg = P.solve_rbgs(1.0, 500, 2e-2, check_every=7)
    assert 1 < ro["count"] < 500
    assert rg["count"] == ro["count"]
    assert rg["residual"] == ro["residual"]
    assert_bitwise(interior(P.download("X", VC)), interior(O.field("X")), "pressure")
    P.close()


@pytest.mark.parametrize("level,radius,count,eps", [(0, 0.0, 400, 1e-10), (0, 0.5, 400, 1e-10),
                                                    (2, 0.5, 40, 1e-10)])
def test_cg_solve_bitwise(level, radius, count, eps):
    g, inp, O = problem(level, threads=THREADS, radius=radius)
    P = device_problem(g, inp)
    x0 = np.zeros((g.nb, 20, 20, 20))
    O.field("X")[...] = x0
    P.upload("X", x0, VC)
    ro = O.solve_cg(1.0, 2, count, eps)
    rg = P.solve_cg(1.0, 2, count, eps)
    assert rg["count"] == ro["count"], (rg["count"], ro["count"])
    assert_bitwise(rg["history"], ro["history"], "residual history")
    assert_bitwise(interior(P.download("X", VC)), interior(O.field("X")), "pressure")
    if level == 0:
        assert ro["residual"] <= eps  # symmetric problem: CG converges
    P.close()


def test_config1_rbsor_then_cg_bitwise():
    """Level-3 sphere grid (548 blocks): RBSOR w=1.5 x 200 then CG."""
    g, inp, O = problem(3, threads=THREADS)
    assert g.nb == 548
    P = device_problem(g, inp)
    x0 = np.zeros((g.nb, 20, 20, 20))
    O.field("X")[...] = x0
    P.upload("X", x0, VC)
    ro = O.solve_rbgs(1.5, 200, 0.0)
    rg = P.solve_rbgs(1.5, 200, 0.0)
    assert_bitwise(rg["history"], ro["history"], "rbgs history")
    co = O.solve_cg(1.0, 2, 30, 1e-10)
    cg = P.solve_cg(1.0, 2, 30, 1e-10)
    assert cg["count"] == co["count"]
    assert_bitwise(cg["history"], co["history"], "cg history")
    assert_bitwise(interior(P.download("X", VC)), interior(O.field("X")), "pressure")
    P.close()


def test_cg_edge_cases():
    g, inp, O = problem(1, threads=THREADS)
    P = device_problem(g, inp)
    zero = np.zeros((g.nb, 20, 20, 20))
    P.upload("X", zero, VC)
    # PreCount = 0: z stays zero, r.z = 0 -> count 0 (FFVILS.h:720-724)
    r = P.solve_cg(1.0, 0, 50, 1e-10)
    assert r["count"] == 0 and r["residual"] == 0.0
    # countMax = 0 -> the loop variable ends at 1
    r = P.solve_rbgs(1.5, 0, 0.0)
    assert r["count"] == 1
    # b = 0 -> |bb| < FLT_MIN -> count 0, residual 0 (FFVILS.h:686-690)
    P.upload("B", zero, VC)
    r = P.solve_cg(1.0, 2, 50, 1e-10)
    assert r["count"] == 0 and r["residual"] == 0.0
    P.close()


def test_nan_rhs_is_reported_not_fatal():
    g, inp, O = problem(1, threads=THREADS)
    P = device_problem(g, inp)
    b = P.download("B", VC)
    b[3, 5, 6, 7] = np.nan
    P.upload("B", b, VC)
    P.upload("X", np.zeros_like(b), VC)
    r = P.solve_rbgs(1.5, 20, 1e-6)
    assert r["status"] == ffvgpu.NAN_DETECTED
    assert r["count"] == 1
    # the pool is still usable afterwards
    b[3, 5, 6, 7] = 0.0
    P.upload("B", b, VC)
    P.upload("X", np.zeros_like(b), VC)
    r = P.solve_rbgs(1.5, 5, 0.0)
    assert r["status"] == ffvgpu.OK
    P.close()


@pytest.mark.parametrize("level,radius,count,eps", [(0, 0.5, 300, 1e-10), (2, 0.5, 60, 1e-10),
                                                    (2, 0.5, 400, 1e-6)])
def test_bicgstab_solve_bitwise(level, radius, count, eps):
    """FFVILS::BiCGSTAB, the reference's default pressure solver."""
    g, inp, O = problem(level, threads=THREADS, radius=radius)
    P = device_problem(g, inp)
    x0 = np.zeros((g.nb, 20, 20, 20))
    O.field("X")[...] = x0
    P.upload("X", x0, VC)
    ro = O.solve_bicgstab(1.0, 2, count, eps)
    rg = P.solve_bicgstab(1.0, 2, count, eps)
    assert rg["count"] == ro["count"], (rg["count"], ro["count"])
    assert_bitwise(rg["history"], ro["history"], "residual history")
    assert_bitwise(interior(P.download("X", VC)), interior(O.field("X")), "pressure")
    if eps >= 1e-6:
        assert ro["residual"] <= eps  # converges on the refined, non-symmetric grid
    P.close()


@pytest.mark.parametrize("solver", ["cg", "bicgstab"])
def test_krylov_pre_count3_bitwise(solver):
    """Three Jacobi passes per application: the later passes read the stored
    iterate (CG's last one also forms r.z), on a 2:1 grid against the oracle."""
    g, inp, O = problem(2, threads=THREADS, radius=0.5)
    P = device_problem(g, inp)
    x0 = np.zeros((g.nb, 20, 20, 20))
    O.field("X")[...] = x0
    P.upload("X", x0, VC)
    ro = getattr(O, "solve_" + solver)(1.0, 3, 30, 0.0)
    rg = getattr(P, "solve_" + solver)(1.0, 3, 30, 0.0)
    assert rg["count"] == ro["count"] == 31
    assert_bitwise(rg["history"], ro["history"], "residual history")
    assert_bitwise(interior(P.download("X", VC)), interior(O.field("X")), "pressure")
    P.close()


def test_krylov_capped_grids_bitwise():
    """The FP64 solvers' persistent A*x and Jacobi kernels on one and three
    CTAs: the 1164-block level-4 list spans two chunks of 800; same bits as
    the full grid."""
    g, inp, _ = problem(4, threads=THREADS)
    P = device_problem(g, inp)
    x0 = np.zeros((g.nb, 20, 20, 20))

    def run(solver):
        P.upload("X", x0, VC)
        r = getattr(P, "solve_" + solver)(1.0, 3, 8, 0.0)
        return r, interior(P.download("X", VC)).copy()

    for solver in ("cg", "bicgstab"):
        ref, xr = run(solver)
        for ctas in (1, 3):
            P.cap_grids(ctas)
            r, x = run(solver)
            P.cap_grids(0)
            assert r["count"] == ref["count"] == 9
            assert_bitwise(r["history"], ref["history"], f"{solver} history, {ctas} CTAs")
            assert_bitwise(x, xr, f"{solver} pressure, {ctas} CTAs")
    P.close()


@pytest.mark.parametrize("level,drop,count,eps", [(2, 1e-3, 300, 1e-10), (3, 1e-2, 40, 0.0)])
def test_bicgstab_with_restarts_bitwise(level, drop, count, eps):
    """The FP64 BiCGSTAB's restart option (no counterpart in the reference):
    the same restarts, iterations and bits as the oracle's."""
    g, inp, O = problem(level, threads=THREADS)
    P = device_problem(g, inp)
    P.fill("X", 0.0)
    O.field("X")[...] = 0.0
    ro = O.solve_bicgstab(1.0, 2, count, eps, restart_drop=drop)
    rg = P.solve_bicgstab(1.0, 2, count, eps, restart_drop=drop)
    assert rg["count"] == ro["count"], (rg["count"], ro["count"])
    assert_bitwise(rg["history"], ro["history"], "residual history")
    assert_bitwise(interior(P.download("X", VC)), interior(O.field("X")), "pressure")
    P.close()


def test_bicgstab_after_rbsor_and_edge_cases():
    g, inp, O = problem(1, threads=THREADS)
    P = device_problem(g, inp)
    x0 = np.zeros((g.nb, 20, 20, 20))
    O.field("X")[...] = x0
    P.upload("X", x0, VC)
    O.solve_rbgs(1.2, 10, 0.0)
    P.solve_rbgs(1.2, 10, 0.0)
    ro = O.solve_bicgstab(1.0, 3, 25, 1e-12)
    rg = P.solve_bicgstab(1.0, 3, 25, 1e-12)
    assert rg["count"] == ro["count"]
    assert_bitwise(rg["history"], ro["history"], "history after RBSOR")
    assert_bitwise(interior(P.download("X", VC)), interior(O.field("X")), "pressure")
    # PreCount = 0: p_ = 0, alpha = rr1 / 0 -> NaN residual (the reference exits)
    r = P.solve_bicgstab(1.0, 0, 5, 1e-10)
    assert r["status"] == ffvgpu.NAN_DETECTED and r["count"] == 1
    P.close()


ALL_NEUMANN = ((ffvgpu.BC_NEUMANN,) * 6, (0.0,) * 6)


@pytest.mark.parametrize("level,omega,count,eps", [(1, 1.0, 40, 0.0), (2, 1.2, 60, 0.0),
                                                   (0, 1.0, 400, 2e-2)])
def test_rbgs_fixed_average_bitwise(level, omega, count, eps):
    """FFVILS::RBGS_WithFixedAverage on an all-Neumann problem: every
    iteration's residual, the pressure and its guide layers bit-equal."""
    g, inp, O = problem(level, threads=THREADS, bc_type=ALL_NEUMANN[0], bc_value=ALL_NEUMANN[1])
    P = device_problem(g, inp, bc_type=ALL_NEUMANN[0], bc_value=ALL_NEUMANN[1])
    x0 = np.zeros((g.nb, 20, 20, 20))
    O.field("X")[...] = x0
    P.upload("X", x0, VC)
    ro = O.solve_rbgs_fixed_average(omega, None, count, eps)
    rg = P.solve_rbgs_fixed_average(omega, None, count, eps, check_every=7)
    assert rg["count"] == ro["count"], (rg["count"], ro["count"])
    assert_bitwise(rg["history"], ro["history"], "residual history")
    got = P.download("X", VC)
    assert_bitwise(interior(got), interior(O.field("X")), "pressure")
    gg, rgd = fo.face_guides(got, VC, 1), fo.face_guides(O.field("X"), VC, 1)
    for f in range(6):
        assert_bitwise(gg[f], rgd[f], f"guides face {f}")
    if eps > 0:
        assert 1 < ro["count"] <= count
    # the shifted pressure has zero mean up to rounding
    assert abs(interior(got).mean()) < 1e-12 * (np.abs(interior(got)).max() + 1.0)
    P.close()


def test_dump2_load2_roundtrip_and_half_resolution(tmp_path):
    """LocalScalar3D::Dump2 / Load2: the file layout, a round trip through
    another pool, and a half-resolution file spread 2x2x2 (sf3d_copy_x2)."""
    g, inp, O = problem(1, threads=THREADS)
    P = device_problem(g, inp)
    x = random_field(g, 31)
    P.upload("X", x, VC)
    fn = str(tmp_path / ffvgpu.restart_filename(".", "ffv_", "p", 0, 7).lstrip("./"))
    P.dump2("X", fn, VC)
    raw = np.fromfile(fn, dtype=np.int32, count=6)
    assert list(raw) == [16, 16, 16, VC, 1, g.nb]
    body = np.fromfile(fn, dtype=np.float64, offset=24).reshape(g.nb, 20, 20, 20)
    P.exchange("X")
    assert_bitwise(body, P.download("X", VC), "file body = exchanged field")
    Q = ffvgpu.Pool(g.desc())
    Q.load2("X", fn, VC)
    assert_bitwise(interior(Q.download("X", VC)), interior(body), "loaded interior")
    # a file of 8^3 blocks
    rng = np.random.default_rng(3)
    coarse = rng.standard_normal((g.nb, 12, 12, 12))
    fc = str(tmp_path / "coarse.bin")
    with open(fc, "wb") as f:
        np.array([8, 8, 8, VC, 1, g.nb], np.int32).tofile(f)
        coarse.tofile(f)
    Q.load2("X", fc, VC)
    want = np.repeat(np.repeat(np.repeat(coarse[:, 2:10, 2:10, 2:10], 2, 1), 2, 2), 2, 3)
    assert_bitwise(interior(Q.download("X", VC)), want, "x2 spread interior")
    bad_file = str(tmp_path / "bad.bin")
    with open(bad_file, "wb") as f:
        np.array([16, 16, 16, VC, 1, g.nb + 1], np.int32).tofile(f)
    with pytest.raises(ffvgpu.FFVGPUError):
        Q.load2("X", bad_file, VC)
    P.close()
    Q.close()


def test_projection_remove_p_and_corr_u_bitwise():
    """bcut_remove_p and bcut_corr_u around the solve: u, the face velocities
    and the Laplacian of p bit-equal to the oracle on a cut-cell grid."""
    g, inp, O = problem(2, threads=THREADS)
    P = device_problem(g, inp)
    x = random_field(g, 41) * 1e-3
    O.field("X")[...] = x
    O.exchange("X", ffvgpu.P_BC_TYPE, ffvgpu.P_BC_VALUE)
    P.upload("X", O.field("X").copy(), VC)
    O.remove_p(1.0, 0.002)
    P.remove_p(1.0, 0.002)
    for u in ("UX", "UY", "UZ"):
        assert_bitwise(interior(P.download(u, VC)), interior(O.field(u)), f"remove_p {u}")
    O.corr_u(1.0, 0.002)
    P.corr_u(1.0, 0.002)
    for f in ("UX", "UY", "UZ", "VW", "VE", "VS", "VN", "VB", "VT", "LAPP"):
        assert_bitwise(interior(P.download(f, VC)), interior(O.field(f)), f"corr_u {f}")
    assert np.abs(interior(O.field("LAPP"))).max() > 0
    P.close()
