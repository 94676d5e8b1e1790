"""Shared set-up for the parity tests: one synthetic sphere problem built
identically in the CPU oracle and in the device pool."""
import numpy as np

import ffvgpu
import ffv_oracle as fo

VC = 2


def problem(max_level, seed=1, sigma=0.01, dt=0.002, rhof=1.0, threads=8,
            reduction=fo.RED_CANONICAL, bc_type=ffvgpu.P_BC_TYPE, bc_value=ffvgpu.P_BC_VALUE,
            **grid_kw):
    """Grid + inputs + oracle with A, b assembled and BCs folded (UpdateP P02-P05)."""
    g = ffvgpu.SphereGrid(max_level, **grid_kw)
    inp = g.fill(seed=seed, sigma=sigma, vc=VC)
    O = fo.Oracle.from_grid(g, vc=VC, bc_type=bc_type, bc_value=bc_value, threads=threads,
                            reduction=reduction)
    for k, v in inp.items():
        O.field(k)[...] = v
    for u in ("UX", "UY", "UZ"):
        O.exchange(u, ffvgpu.U_BC_TYPE, ffvgpu.U_BC_VALUE[u])
    O.assemble_p(rhof, dt)
    O.fold_bc()
    return g, inp, O


def device_problem(g, inp, dt=0.002, rhof=1.0, bc_type=ffvgpu.P_BC_TYPE,
                   bc_value=ffvgpu.P_BC_VALUE):
    """The same problem on the device: upload inputs, exchange u, assemble, fold."""
    P = ffvgpu.Pool(g.desc(bc_type, bc_value))
    for k, v in inp.items():
        P.upload(k, v, VC)
    for u in ("UX", "UY", "UZ"):
        P.exchange(u, ffvgpu.U_BC_TYPE, ffvgpu.U_BC_VALUE[u])
    P.assemble_p(rhof, dt)
    P.fold_bc()
    return P


def interior(a):
    return fo.interior(a, VC)


def assert_bitwise(a, b, what=""):
    a = np.asarray(a)
    b = np.asarray(b)
    assert a.shape == b.shape, (what, a.shape, b.shape)
    bad = ~((a == b) | (np.isnan(a) & np.isnan(b)))
    n = int(bad.sum())
    if n:
        idx = np.argwhere(bad)[0]
        raise AssertionError(f"{what}: {n} values differ, first at {tuple(idx)}: "
                             f"{a[tuple(idx)]!r} vs {b[tuple(idx)]!r}")


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    d = np.abs(a - b).max() if a.size else 0.0
    s = np.abs(b).max() if b.size else 0.0
    return d / s if s > 0 else d
