"""ctypes binding of the CPU oracle (oracle/libffvoracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU baseline / reference legs, never by the product.  The oracle
restates FFV-HC's pressure path in C++ (ffv_oracle.cpp); parity is unpinned
by reference tests because the reference ships none and cannot be compiled
here (see the header of ffv_oracle.cpp).
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libffvoracle.so")

F = dict(X=0, AP=1, AW=2, AE=3, AS=4, AN=5, AB=6, AT=7, B=8, UX=9, UY=10, UZ=11,
         C0=12, C1=13, C2=14, C3=15, C4=16, C5=17, VW=18, VE=19, VS=20, VN=21, VB=22, VT=23,
         R=24, P=25, Q=26, Z=27, X0=28, R0=29, P_=30, Q_=31, S=32, S_=33, T_=34, LAPP=35)
FI = dict(CID0=0, CID1=1, CID2=2, CID3=3, CID4=4, CID5=5, PID=6)
RED_REFERENCE, RED_CANONICAL = 0, 1

_lib = None


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        vp, i32, dbl = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        L.orc_create.restype = vp
        L.orc_create.argtypes = [i32, i32, i32, vp, vp, vp, dbl, vp]
        L.orc_destroy.argtypes = [vp]
        L.orc_field.restype = ctypes.POINTER(ctypes.c_double)
        L.orc_field.argtypes = [vp, i32]
        L.orc_ifield.restype = ctypes.POINTER(ctypes.c_int)
        L.orc_ifield.argtypes = [vp, i32]
        L.orc_cells_per_block.restype = ctypes.c_long
        L.orc_cells_per_block.argtypes = [vp]
        L.orc_set_threads.argtypes = [vp, i32]
        L.orc_set_reduction.argtypes = [vp, i32]
        L.orc_neighbor.argtypes = [vp, i32, i32, vp, vp, vp]
        L.orc_block_dx.restype = dbl
        L.orc_block_dx.argtypes = [vp, i32]
        L.orc_set_bc.argtypes = [vp, vp, vp]
        L.orc_exchange.argtypes = [vp, i32, vp, vp]
        L.orc_assemble_p.argtypes = [vp, dbl, dbl]
        L.orc_fold_bc.argtypes = [vp]
        L.orc_rbgs_sweep.argtypes = [vp, dbl]
        L.orc_calc_r2.restype = dbl
        L.orc_calc_r2.argtypes = [vp]
        L.orc_dot.restype = dbl
        L.orc_dot.argtypes = [vp, i32, i32]
        L.orc_calc_ax.argtypes = [vp, i32, i32]
        L.orc_calc_r.argtypes = [vp, i32, i32, i32]
        L.orc_jacobi_smoother.argtypes = [vp, i32, i32, i32, dbl]
        L.orc_slot.argtypes = [vp, i32]
        for fn in (L.orc_rbgs,):
            fn.argtypes = [vp, dbl, i32, dbl, vp, vp, vp]
        for fn in (L.orc_cg, L.orc_bicgstab):
            fn.argtypes = [vp, dbl, i32, i32, dbl, vp, vp, vp]
        L.orc_projection.argtypes = [vp, i32, dbl, dbl]
        L.orc_projection.restype = None
        L.orc_rbgs_fixed_average.argtypes = [vp, dbl, ctypes.c_long, i32, dbl, vp, vp, vp]
        L.orc_bicgstab_restart.argtypes = [vp, dbl, i32, i32, dbl, dbl, vp, vp, vp]
        L.orc_mixed.argtypes = [vp, dbl, i32, i32, i32, dbl, dbl, dbl, i32, i32, i32, vp, vp, vp]
        L.orc_mixed_dc.argtypes = [vp, dbl, i32, i32, i32, dbl, i32, vp, vp, vp]
        L.orc_cf_apply.argtypes = [vp, i32, i32, i32]
        L.orc_cf_apply.restype = None
        L.orc_cf_cells.restype = ctypes.c_long
        L.orc_cf_cells.argtypes = [vp, i32, vp, ctypes.c_long]
        # the host sphere-grid generator compiled into this library
        L.ffvgpu_sphere_grid_create.argtypes = [ctypes.POINTER(_SphereParams),
                                                ctypes.POINTER(vp)]
        L.ffvgpu_sphere_grid_destroy.argtypes = [vp]
        L.ffvgpu_sphere_grid_destroy.restype = None
        L.ffvgpu_sphere_grid_num_blocks.argtypes = [vp]
        L.ffvgpu_sphere_grid_blocks.argtypes = [vp, vp, vp]
        L.ffvgpu_sphere_grid_blocks.restype = None
        L.ffvgpu_sphere_grid_fill.argtypes = [vp, ctypes.c_uint64, dbl, i32, vp, vp, vp, vp, vp,
                                              vp]
        _lib = L
    return _lib


# ---------------------------------------------------------------------------
# Inputs of the sphere-flow workload, built with the generator compiled into
# this library (the same source as the device library's host generator), so
# that CPU-only runs never load the device library.
# ---------------------------------------------------------------------------
BC_DIRICHLET, BC_NEUMANN = 0, 1
# Pressure BCs of the sphere example (examples/FlowPastASphere/sphere.tpp):
# Neumann 0 at the inlet (X_M) and side walls, Dirichlet 0 at the outlet (X_P).
P_BC_TYPE = (BC_NEUMANN, BC_DIRICHLET, BC_NEUMANN, BC_NEUMANN, BC_NEUMANN, BC_NEUMANN)
P_BC_VALUE = (0.0,) * 6
# Velocity BCs: inlet Dirichlet (1,0,0); outlet and walls Neumann 0.
U_BC_TYPE = (BC_DIRICHLET, BC_NEUMANN, BC_NEUMANN, BC_NEUMANN, BC_NEUMANN, BC_NEUMANN)
U_BC_VALUE = {"UX": (1.0, 0, 0, 0, 0, 0), "UY": (0.0,) * 6, "UZ": (0.0,) * 6}
FLOW_PAST_SPHERE = dict(domain_origin=(-4.0, -4.0, -4.0), root_grid=(4, 2, 2), root_length=4.0,
                        center=(0.0, 0.0, 0.0), radius=0.5, margin=0.5)


class _SphereParams(ctypes.Structure):
    _fields_ = [
        ("domain_origin", ctypes.c_double * 3), ("root_grid", ctypes.c_int32 * 3),
        ("root_length", ctypes.c_double), ("max_level", ctypes.c_int32),
        ("center", ctypes.c_double * 3), ("radius", ctypes.c_double),
        ("margin", ctypes.c_double),
    ]


class SphereGrid:
    """2:1-balanced octree of 16^3 leaf blocks refined around a sphere, and its
    per-cell inputs in the reference layout (the device library's SphereGrid,
    from this library's copy of the generator)."""

    def __init__(self, max_level, **kw):
        p = dict(FLOW_PAST_SPHERE)
        p.update(kw)
        self.params = p
        self.max_level = max_level
        sp = _SphereParams(p["domain_origin"], p["root_grid"], p["root_length"], max_level,
                           p["center"], p["radius"], p["margin"])
        self._h = ctypes.c_void_p()
        if lib().ffvgpu_sphere_grid_create(ctypes.byref(sp), ctypes.byref(self._h)) != 0:
            raise ValueError("sphere grid parameters rejected")
        self.nb = lib().ffvgpu_sphere_grid_num_blocks(self._h)
        self.level = np.zeros(self.nb, np.int32)
        self.index = np.zeros((self.nb, 3), np.int32)
        lib().ffvgpu_sphere_grid_blocks(self._h, self.level.ctypes.data, self.index.ctypes.data)

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.ffvgpu_sphere_grid_destroy(self._h)
            self._h = None

    @property
    def cells(self):
        return self.nb * 4096

    def fill_u(self, seed=0, sigma=0.01, vc=2):
        """Only u* = (1,0,0) + N(0, sigma^2) in the reference layout (guides 0)."""
        w = 16 + 2 * vc
        shape = (self.nb, w, w, w)
        out = {k: np.zeros(shape, np.float64) for k in ("UX", "UY", "UZ")}
        st = lib().ffvgpu_sphere_grid_fill(self._h, seed, sigma, vc, out["UX"].ctypes.data,
                                           out["UY"].ctypes.data, out["UZ"].ctypes.data,
                                           None, None, None)
        if st != 0:
            raise ValueError("sphere_grid_fill failed")
        return out

    def fill(self, seed=0, sigma=0.01, vc=2):
        """Per-cell inputs in the reference layout: dict of numpy arrays."""
        w = 16 + 2 * vc
        shape = (self.nb, w, w, w)
        out = {k: np.zeros(shape, np.float64) for k in ("UX", "UY", "UZ")}
        for f in range(6):
            out[f"C{f}"] = np.zeros(shape, np.float64)
            out[f"CID{f}"] = np.zeros(shape, np.int32)
        out["PID"] = np.zeros(shape, np.int32)
        c6 = (ctypes.c_void_p * 6)(*[out[f"C{f}"].ctypes.data for f in range(6)])
        i6 = (ctypes.c_void_p * 6)(*[out[f"CID{f}"].ctypes.data for f in range(6)])
        st = lib().ffvgpu_sphere_grid_fill(self._h, seed, sigma, vc, out["UX"].ctypes.data,
                                           out["UY"].ctypes.data, out["UZ"].ctypes.data,
                                           ctypes.cast(c6, ctypes.c_void_p),
                                           ctypes.cast(i6, ctypes.c_void_p),
                                           out["PID"].ctypes.data)
        if st != 0:
            raise ValueError("sphere_grid_fill failed")
        return out


def sphere_problem(max_level, seed=1, sigma=0.01, rhof=1.0, dt=0.002, threads=1,
                   reduction=RED_REFERENCE, **grid_kw):
    """The sphere-flow pressure problem on the CPU: grid, inputs, oracle with
    u exchanged, A and b assembled and the BCs folded (UpdateP P02-P05)."""
    g = SphereGrid(max_level, **grid_kw)
    inp = g.fill(seed=seed, sigma=sigma, vc=2)
    O = Oracle.from_grid(g, vc=2, bc_type=P_BC_TYPE, bc_value=P_BC_VALUE, threads=threads,
                         reduction=reduction)
    for k, v in inp.items():
        O.field(k)[...] = v
    del inp
    for u in ("UX", "UY", "UZ"):
        O.exchange(u, U_BC_TYPE, U_BC_VALUE[u])
    O.assemble_p(rhof, dt)
    O.fold_bc()
    return g, O


class Oracle:
    """Block pool in the reference layout (vc guide layers) + FFVILS drivers."""

    def __init__(self, level, index, domain_origin, root_length, root_grid, vc=2,
                 bc_type=None, bc_value=None, threads=1, reduction=RED_CANONICAL):
        L = lib()
        self.nb = len(level)
        self.vc = vc
        self.w = 16 + 2 * vc
        lev = np.ascontiguousarray(level, np.int32)
        idx = np.ascontiguousarray(np.asarray(index).reshape(-1), np.int64)
        org = np.ascontiguousarray(domain_origin, np.float64)
        rg = np.ascontiguousarray(root_grid, np.int32)
        self._h = L.orc_create(self.nb, 16, vc, lev.ctypes.data, idx.ctypes.data, org.ctypes.data,
                               float(root_length), rg.ctypes.data)
        if not self._h:
            raise ValueError("oracle: grid is not 2:1 face balanced")
        self.set_threads(threads)
        self.set_reduction(reduction)
        if bc_type is not None:
            self.set_bc(bc_type, bc_value)

    @classmethod
    def from_grid(cls, grid, **kw):
        p = grid.params
        return cls(grid.level, grid.index, p["domain_origin"], p["root_length"], p["root_grid"],
                   **kw)

    def close(self):
        if getattr(self, "_h", None):
            lib().orc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_threads(self, n):
        lib().orc_set_threads(self._h, int(n))

    def set_reduction(self, mode):
        lib().orc_set_reduction(self._h, int(mode))

    def set_bc(self, bc_type, bc_value):
        t = np.ascontiguousarray(bc_type, np.int32)
        v = np.ascontiguousarray(bc_value, np.float64)
        lib().orc_set_bc(self._h, t.ctypes.data, v.ctypes.data)

    def field(self, name):
        """Live numpy view [block][k][j][i] of a field (follows LSSwap slots)."""
        n = self.nb * self.w ** 3
        if name in FI:
            p = lib().orc_ifield(self._h, FI[name])
            return np.ctypeslib.as_array(p, shape=(n,)).reshape(self.nb, self.w, self.w, self.w)
        p = lib().orc_field(self._h, F[name])
        return np.ctypeslib.as_array(p, shape=(n,)).reshape(self.nb, self.w, self.w, self.w)

    def set_field(self, name, arr):
        self.field(name)[...] = arr

    def neighbor(self, b, face):
        kind = ctypes.c_int()
        nbr = np.zeros(4, np.int32)
        so = np.zeros(2, np.int32)
        lib().orc_neighbor(self._h, b, face, ctypes.byref(kind), nbr.ctypes.data, so.ctypes.data)
        return kind.value, nbr, so

    def exchange(self, name, bc_type, bc_value):
        t = np.ascontiguousarray(bc_type, np.int32)
        v = np.ascontiguousarray(bc_value, np.float64)
        lib().orc_exchange(self._h, F[name], t.ctypes.data, v.ctypes.data)

    def assemble_p(self, rhof=1.0, dt=0.002):
        lib().orc_assemble_p(self._h, rhof, dt)

    def fold_bc(self):
        lib().orc_fold_bc(self._h)

    def remove_p(self, rhof=1.0, dt=0.002):
        lib().orc_projection(self._h, 0, rhof, dt)

    def corr_u(self, rhof=1.0, dt=0.002):
        lib().orc_projection(self._h, 1, rhof, dt)

    def rbgs_sweep(self, omega):
        lib().orc_rbgs_sweep(self._h, omega)

    def calc_r2(self):
        return lib().orc_calc_r2(self._h)

    def dot(self, a, b):
        return lib().orc_dot(self._h, F[a], F[b])

    def _solve(self, fn, args, count_max):
        count = ctypes.c_int()
        res = ctypes.c_double()
        hist = np.zeros(max(count_max, 1), np.float64)
        st = fn(self._h, *args, ctypes.byref(count), ctypes.byref(res), hist.ctypes.data)
        n = count.value if 1 <= count.value <= count_max else (count_max if count.value > 0 else 0)
        return dict(status=st, count=count.value, residual=res.value, history=hist[:n].copy())

    def solve_rbgs(self, omega=1.5, count_max=200, epsilon=0.0):
        return self._solve(lib().orc_rbgs, (float(omega), int(count_max), float(epsilon)), count_max)

    def solve_rbgs_fixed_average(self, omega=1.0, ncells=None, count_max=200, epsilon=0.0):
        n = self.nb * 4096 if ncells is None else ncells
        return self._solve(lib().orc_rbgs_fixed_average, (float(omega), int(n), int(count_max),
                                                          float(epsilon)), count_max)

    def solve_cg(self, omega=1.0, pre_count=2, count_max=10000, epsilon=1e-10):
        return self._solve(lib().orc_cg, (float(omega), int(pre_count), int(count_max),
                                          float(epsilon)), count_max)

    def solve_mixed(self, omega=1.5, sweeps=8, sweeps_per_exchange=4, count_max=1000,
                    epsilon=1e-8, restart_drop=1e-3, restart_growth=100.0, restart_every=0,
                    flux_correction=False, fp64_data=False):
        """Mixed-precision form: BiCGSTAB with RB-SOR preconditioning on 32-bit data;
        flux_correction: the FP64 residual and A*x use the coarse-fine
        flux-conserving operator; fp64_data: the same preconditioner on FP64 data."""
        return self._solve(lib().orc_mixed, (float(omega), int(sweeps), int(sweeps_per_exchange),
                                             int(count_max), float(epsilon), float(restart_drop),
                                             float(restart_growth), int(restart_every),
                                             int(bool(flux_correction)), int(bool(fp64_data))),
                           count_max)

    def solve_mixed_dc(self, omega=1.5, sweeps=8, sweeps_per_exchange=4, count_max=1000,
                       epsilon=1e-8, fp64_data=False):
        """The precision form as a defect correction: r = b - A x in FP64, e the
        RB-SOR preconditioner of solve_mixed applied to r, x += e."""
        return self._solve(lib().orc_mixed_dc, (float(omega), int(sweeps),
                                                int(sweeps_per_exchange), int(count_max),
                                                float(epsilon), int(bool(fp64_data))), count_max)

    def calc_ax(self, out, x, flux_correction=False):
        """out = A x (CalcAx, FFVILS.h:164-202), with flux_correction the
        coarse-fine flux-conserving operator; x's guide cells as held."""
        lib().orc_calc_ax(self._h, F[out], F[x])
        if flux_correction:
            lib().orc_cf_apply(self._h, F[out], F[x], 1)

    def cf_cells(self, name="X"):
        """Per coarse cell at a face with finer neighbours, in (block, face,
        position) order: array [n][2] of (delta, F) of the field as it is held
        (guide cells included)."""
        n = lib().orc_cf_cells(self._h, F[name], None, 0)
        out = np.zeros((max(n, 1), 2), np.float64)
        lib().orc_cf_cells(self._h, F[name], out.ctypes.data, n)
        return out[:n]

    def solve_bicgstab(self, omega=1.0, pre_count=2, count_max=1000, epsilon=1e-10,
                       restart_drop=0.0):
        if restart_drop > 0.0:
            return self._solve(lib().orc_bicgstab_restart,
                               (float(omega), int(pre_count), int(count_max), float(epsilon),
                                float(restart_drop)), count_max)
        return self._solve_plain_bicgstab(omega, pre_count, count_max, epsilon)

    def _solve_plain_bicgstab(self, omega, pre_count, count_max, epsilon):
        return self._solve(lib().orc_bicgstab, (float(omega), int(pre_count), int(count_max),
                                                float(epsilon)), count_max)


def time_step(O, u_star, solve, rhof=1.0, dt=0.002):
    """The pressure part of one fractional step on the oracle, in
    Solver::UpdateP / UpdateU's order (src/FFV/Solver.cpp:5294-5771): u* set
    from u_star (dict UX, UY, UZ in the reference layout), P01 bcut_remove_p
    with the previous pressure, P02 exchange of u, P03 bcut_calc_ab_p, P05 BC
    folding, P06 solve(O) (x from the previous pressure), P07 exchange of p,
    U01 bcut_corr_u, U02 exchange of u, U03 exchange of p.  Returns solve's
    result."""
    for k in ("UX", "UY", "UZ"):
        O.field(k)[...] = u_star[k]
    O.remove_p(rhof, dt)
    for k in ("UX", "UY", "UZ"):
        O.exchange(k, U_BC_TYPE, U_BC_VALUE[k])
    O.assemble_p(rhof, dt)
    O.fold_bc()
    r = solve(O)
    O.exchange("X", P_BC_TYPE, P_BC_VALUE)
    O.corr_u(rhof, dt)
    for k in ("UX", "UY", "UZ"):
        O.exchange(k, U_BC_TYPE, U_BC_VALUE[k])
    O.exchange("X", P_BC_TYPE, P_BC_VALUE)
    return r


def interior(a, vc=2):
    """Interior cells [block][k][j][i] of a reference-layout array."""
    return a[:, vc:vc + 16, vc:vc + 16, vc:vc + 16]


def face_guides(a, vc=2, layers=1):
    """Face guide slabs (layers nearest the interior first) of a reference-layout array,
    as a dict face -> array [block][layer][v][u]."""
    s = slice(vc, vc + 16)
    out = {}
    for L in range(1, layers + 1):
        lo, hi = vc - L, vc + 15 + L
        out.setdefault(0, []).append(a[:, s, s, lo])
        out.setdefault(1, []).append(a[:, s, s, hi])
        out.setdefault(2, []).append(a[:, s, lo, s])
        out.setdefault(3, []).append(a[:, s, hi, s])
        out.setdefault(4, []).append(a[:, lo, s, s])
        out.setdefault(5, []).append(a[:, hi, s, s])
    return {f: np.stack(v, axis=1) for f, v in out.items()}
