"""CPU tests of the oracle's coarse-fine flux restatement (no GPU).

The flux correction has no counterpart in the reference; its per-cell
quantities are checked here against facts that do not depend on how they
are coded: for a linear pressure field and the uncut-cell coefficients
1/dx^2, the reference's 2:1 prolongation and restriction are exact
(src/CGMfuncs/sup.f90:54-179 interpolate and extrapolate linearly), so the
fine-side flux F through each coarse-fine face equals the exact flux
gradient / dx_coarse and the mismatch delta vanishes to rounding; for a
quadratic field it does not.
"""
import numpy as np

import ffvgpu
import ffv_oracle as fo

VC = 2
NB_FINE = 3  # FFVGPU_NB_FINE: the face's neighbours are four finer blocks


def linear_oracle(level=2, grad=(0.7, -0.3, 0.2), quad=0.0):
    g = ffvgpu.SphereGrid(level)
    O = fo.Oracle.from_grid(g, vc=VC, bc_type=ffvgpu.P_BC_TYPE, bc_value=ffvgpu.P_BC_VALUE)
    p = g.params
    w = 16 + 2 * VC
    h = p["root_length"] / np.exp2(g.level.astype(np.float64))  # block edge
    dx = h / 16.0
    org = np.asarray(p["domain_origin"])[None, :] + g.index * h[:, None]
    ii = (np.arange(w) - VC + 0.5)
    X = org[:, 0, None, None, None] + dx[:, None, None, None] * ii[None, None, None, :]
    Y = org[:, 1, None, None, None] + dx[:, None, None, None] * ii[None, None, :, None]
    Z = org[:, 2, None, None, None] + dx[:, None, None, None] * ii[None, :, None, None]
    field = grad[0] * X + grad[1] * Y + grad[2] * Z + quad * X * X
    O.field("X")[...] = field
    # interior values stand; the exchange refills every guide cell (2:1 rules)
    O.exchange("X", (fo.BC_NEUMANN,) * 6, (0.0,) * 6)
    inv = (1.0 / (dx * dx))[:, None, None, None] * np.ones((1, w, w, w))
    for f in ("AW", "AE", "AS", "AN", "AB", "AT"):
        O.field(f)[...] = inv
    O.field("AP")[...] = -6.0 * inv
    return g, O, dx


def test_linear_field_has_no_coarse_fine_mismatch():
    grad = (0.7, -0.3, 0.2)
    g, O, dx = linear_oracle(grad=grad)
    cells = O.cf_cells("X")
    assert len(cells) > 0 and len(cells) % 256 == 0
    d, F = cells[:, 0], cells[:, 1]
    # |F| = |gradient component| / dx_coarse: at least min|g_i| / max dx
    scale = np.abs(F).max()
    assert scale > 0
    assert np.abs(d).max() <= 1e-10 * scale, (np.abs(d).max(), scale)
    # F is the exact flux: +-grad[axis] / dx of the coarse block, per face
    k = 0
    for b in range(g.nb):
        for f in range(6):
            kind, _, _ = O.neighbor(b, f)
            if kind != NB_FINE:
                continue
            want = (1.0 if f & 1 else -1.0) * grad[f >> 1] / dx[b]
            np.testing.assert_allclose(F[k:k + 256], want, rtol=1e-10, atol=0)
            k += 256
    assert k == len(cells)


def test_quadratic_field_shows_a_mismatch():
    g, O, dx = linear_oracle(grad=(0.0, 0.0, 0.0), quad=1.0)
    cells = O.cf_cells("X")
    assert np.abs(cells[:, 0]).max() > 1e-3 * np.abs(cells[:, 1]).max()


def test_flux_correction_conserves_across_coarse_fine_faces():
    """With uncut coefficients 1/dx^2 and Neumann outer faces folded into A
    (so no flux leaves the domain), sum over cells of V (A x) is a sum of
    face-flux mismatches: same-level faces cancel pairwise, coarse-fine faces
    do not under the interpolating exchange, and do under the correction.
    So for any x, sum V (A x) vanishes to rounding only with the correction."""
    g = ffvgpu.SphereGrid(2)
    neumann = (fo.BC_NEUMANN,) * 6
    O = fo.Oracle.from_grid(g, vc=VC, bc_type=neumann, bc_value=(0.0,) * 6)
    w = 16 + 2 * VC
    dx = 4.0 / np.exp2(g.level.astype(np.float64)) / 16.0
    inv = (1.0 / (dx * dx))[:, None, None, None] * np.ones((1, w, w, w))
    for f in ("AW", "AE", "AS", "AN", "AB", "AT"):
        O.field(f)[...] = inv
    O.field("AP")[...] = -6.0 * inv
    O.fold_bc()
    rng = np.random.default_rng(3)
    O.field("X")[...] = rng.standard_normal((g.nb, w, w, w))
    O.exchange("X", neumann, (0.0,) * 6)
    vol = (dx ** 3)[:, None, None, None]
    out = {}
    for corr in (False, True):
        O.calc_ax("Q", "X", flux_correction=corr)
        vy = vol * fo.interior(O.field("Q"), VC)
        out[corr] = abs(vy.sum()) / np.abs(vy).sum()
    assert out[False] > 1e-6, out
    assert out[True] < 1e-13, out
