"""ctypes binding of libffvhc_b200.so (include/ffvgpu.h).

Thin plumbing for tests and benchmarks: every call goes through the C ABI;
nothing here computes.  Loading fails loudly when the library is missing:
there is no CPU fallback.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libffvhc_b200.so")

OK, NOT_CONVERGED, NAN_DETECTED, TIMEOUT, OOM, BAD_ARG, CUDA_ERROR, NO_DEVICE, CANCELLED = range(9)
BC_DIRICHLET, BC_NEUMANN = 0, 1
NB_OUTER, NB_SAME, NB_COARSE, NB_FINE = range(4)

FIELD = {
    "X": 0, "AP": 1, "AW": 2, "AE": 3, "AS": 4, "AN": 5, "AB": 6, "AT": 7, "B": 8,
    "UX": 9, "UY": 10, "UZ": 11,
    "C0": 12, "C1": 13, "C2": 14, "C3": 15, "C4": 16, "C5": 17,
    "VW": 18, "VE": 19, "VS": 20, "VN": 21, "VB": 22, "VT": 23, "LAPP": 24,
    "CID0": 100, "CID1": 101, "CID2": 102, "CID3": 103, "CID4": 104, "CID5": 105,
    "PID": 106,
}

# Declared entry points of include/ffvgpu.h (checked by the CPU tests).
EXPORTS = [
    "ffvgpu_pool_create", "ffvgpu_pool_destroy", "ffvgpu_pool_num_blocks",
    "ffvgpu_pool_set_stream", "ffvgpu_fill", "ffvgpu_grid_neighbors",
    "ffvgpu_pool_neighbors", "ffvgpu_pool_device_bytes", "ffvgpu_pool_upload",
    "ffvgpu_pool_download", "ffvgpu_exchange", "ffvgpu_assemble_p", "ffvgpu_fold_bc",
    "ffvgpu_solve_rbgs", "ffvgpu_solve_cg", "ffvgpu_solve_bicgstab", "ffvgpu_rbgs_sweep", "ffvgpu_calc_r2",
    "ffvgpu_dot", "ffvgpu_version", "ffvgpu_last_error", "ffvgpu_sphere_grid_create",
    "ffvgpu_sphere_grid_destroy", "ffvgpu_sphere_grid_num_blocks",
    "ffvgpu_sphere_grid_blocks", "ffvgpu_sphere_grid_fill", "ffvgpu_dot_noalloc",
    "ffvgpu_solve_mixed", "ffvgpu_cf_flux_mismatch", "ffvgpu_update_p", "ffvgpu_update_u",
    "ffvgpu_generate_sphere", "ffvgpu_shard_create", "ffvgpu_shard_destroy", "ffvgpu_shard_info",
    "ffvgpu_shard_local_blocks", "ffvgpu_shard_zorder", "ffvgpu_shard_local_desc",
    "ffvgpu_shard_peer", "ffvgpu_rbgs_pass", "ffvgpu_block_dots", "ffvgpu_pool_field_device",
    "ffvgpu_canonical_sum", "ffvgpu_batch_create", "ffvgpu_instance_admit",
    "ffvgpu_instance_admit_sphere", "ffvgpu_instance_upload", "ffvgpu_instance_download",
    "ffvgpu_instance_release", "ffvgpu_instance_blocks", "ffvgpu_pool_free_blocks",
    "ffvgpu_mixed_begin", "ffvgpu_mixed_advance", "ffvgpu_mixed_poll", "ffvgpu_instance_result",
    "ffvgpu_assemble_sphere", "ffvgpu_instance_fill", "ffvgpu_serve",
    "ffvgpu_solve_rbgs_fixed_average", "ffvgpu_dump2", "ffvgpu_load2",
    "ffvgpu_restart_filename", "ffvgpu_remove_p", "ffvgpu_corr_u", "ffvgpu_mixed_autotune",
    "ffvgpu_pool_set_wait_limit", "ffvgpu_mixed_cancel", "ffvgpu_pool_stall_next_solve",
    "ffvgpu_pool_cap_grids", "ffvgpu_pool_stall_next_matvec",
]


class GridDesc(ctypes.Structure):
    _fields_ = [
        ("num_blocks", ctypes.c_int32), ("cells", ctypes.c_int32),
        ("level", ctypes.c_void_p), ("block_index", ctypes.c_void_p),
        ("domain_origin", ctypes.c_double * 3), ("root_length", ctypes.c_double),
        ("root_grid", ctypes.c_int32 * 3),
        ("neighbor_kind", ctypes.c_void_p), ("neighbor_ids", ctypes.c_void_p),
        ("bc_type", ctypes.c_int32 * 6), ("bc_value", ctypes.c_double * 6),
    ]


class IterParams(ctypes.Structure):
    _fields_ = [
        ("omega", ctypes.c_double), ("count_max", ctypes.c_int32),
        ("epsilon", ctypes.c_double), ("pre_count", ctypes.c_int32),
        ("check_every", ctypes.c_int32), ("history", ctypes.c_void_p),
        ("restart_drop", ctypes.c_double),
    ]


class StepParams(ctypes.Structure):
    _fields_ = [
        ("rhof", ctypes.c_double), ("dt", ctypes.c_double),
        ("u_bc_type", (ctypes.c_int32 * 6) * 3), ("u_bc_value", (ctypes.c_double * 6) * 3),
        ("solver", ctypes.c_int32), ("iter", IterParams),
    ]


SOLVER_RBGS, SOLVER_BICGSTAB, SOLVER_MIXED = 0, 1, 2


class Result(ctypes.Structure):
    _fields_ = [
        ("count", ctypes.c_int32), ("residual", ctypes.c_double),
        ("elapsed_ms", ctypes.c_double), ("sweep_ms", ctypes.c_double),
        ("sweep_launches", ctypes.c_int32), ("bytes_moved", ctypes.c_int64),
        ("kernel_launches", ctypes.c_int32), ("uniform_blocks", ctypes.c_int32),
    ]


class SphereParams(ctypes.Structure):
    _fields_ = [
        ("domain_origin", ctypes.c_double * 3), ("root_grid", ctypes.c_int32 * 3),
        ("root_length", ctypes.c_double), ("max_level", ctypes.c_int32),
        ("center", ctypes.c_double * 3), ("radius", ctypes.c_double),
        ("margin", ctypes.c_double),
    ]


class MixedParams(ctypes.Structure):
    _fields_ = [
        ("omega", ctypes.c_double), ("sweeps", ctypes.c_int32),
        ("sweeps_per_exchange", ctypes.c_int32), ("count_max", ctypes.c_int32),
        ("epsilon", ctypes.c_double), ("check_every", ctypes.c_int32),
        ("history", ctypes.c_void_p), ("restart_drop", ctypes.c_double),
        ("restart_growth", ctypes.c_double), ("restart_every", ctypes.c_int32),
        ("flux_correction", ctypes.c_int32), ("fp64_data", ctypes.c_int32),
        ("threads_per_block", ctypes.c_int32), ("stage_depth", ctypes.c_int32),
        ("sweep_threads", ctypes.c_int32), ("matvec_form", ctypes.c_int32),
    ]


# Restart settings of the mixed form used by default (see ffvgpu_mixed_params).
RESTART = dict(restart_drop=1e-3, restart_growth=100.0, restart_every=0)


class BatchDesc(ctypes.Structure):
    _fields_ = [
        ("capacity_blocks", ctypes.c_int32), ("max_instances", ctypes.c_int32),
        ("bc_type", ctypes.c_int32 * 6), ("bc_value", ctypes.c_double * 6),
    ]


class SphereProblem(ctypes.Structure):
    _fields_ = [
        ("grid", SphereParams), ("seed", ctypes.c_uint64), ("sigma", ctypes.c_double),
        ("rhof", ctypes.c_double), ("dt", ctypes.c_double),
        ("u_bc_type", (ctypes.c_int32 * 6) * 3), ("u_bc_value", (ctypes.c_double * 6) * 3),
    ]


class TuneRecord(ctypes.Structure):
    _fields_ = [
        ("omega", ctypes.c_double), ("sweeps", ctypes.c_int32),
        ("sweeps_per_exchange", ctypes.c_int32), ("iterations_per_replay", ctypes.c_int32),
        ("ms", ctypes.c_double), ("max_count", ctypes.c_int32), ("converged", ctypes.c_int32),
        ("threads_per_block", ctypes.c_int32), ("stage_depth", ctypes.c_int32),
        ("sweep_threads", ctypes.c_int32), ("matvec_form", ctypes.c_int32),
    ]


# Candidate settings the batch autotuner sweeps: sweeps per exchange 1, 2, 4,
# 8 (8 sweeps per application, and 4), omega 1.2 and 1.5, 4 / 8 / 16 graph
# iterations per replay.
TUNE_SPACE = [(om, sw, per, it) for om in (1.5, 1.2) for (sw, per) in
              ((8, 4), (8, 8), (8, 2), (8, 1), (4, 4), (4, 2)) for it in (4, 8, 16)]
# Then, for the fastest of those: threads per block of the update kernel
# (and of the A*x kernel in form 1) 128 / 256 / 512, the sweep kernel's
# staging depth 1 / 2 / 3 and its threads per block 512 / 256, and the A*x
# kernel's form (0 pipelined, 1 a block per CTA).
TUNE_LAUNCH = [(nt, dp, st, mv) for nt in (128, 256, 512) for dp in (1, 2, 3)
               for st in (512, 256) for mv in (0, 1)]
TUNE_LAUNCH_DEFAULT = (256, 1, 256, 0)


class Request(ctypes.Structure):
    _fields_ = [("arrival_s", ctypes.c_double), ("cancel_s", ctypes.c_double),
                ("problem", SphereProblem)]


class RequestResult(ctypes.Structure):
    _fields_ = [
        ("admit_s", ctypes.c_double), ("finish_s", ctypes.c_double),
        ("count", ctypes.c_int32), ("residual", ctypes.c_double),
        ("status", ctypes.c_int32), ("blocks", ctypes.c_int32),
    ]


_lib = None


def lib():
    """Loads the library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run `make -C ffv-hc_b200` (or "
                               "__graft_entry__.build()); there is no CPU fallback")
        L = ctypes.CDLL(LIB_PATH)
        vp, i32, dbl = ctypes.c_void_p, ctypes.c_int32, ctypes.c_double
        L.ffvgpu_last_error.restype = ctypes.c_char_p
        L.ffvgpu_pool_create.argtypes = [ctypes.POINTER(GridDesc), ctypes.POINTER(vp)]
        L.ffvgpu_pool_destroy.argtypes = [vp]
        L.ffvgpu_pool_destroy.restype = None
        L.ffvgpu_pool_num_blocks.argtypes = [vp]
        L.ffvgpu_pool_device_bytes.argtypes = [vp]
        L.ffvgpu_pool_device_bytes.restype = ctypes.c_int64
        L.ffvgpu_pool_neighbors.argtypes = [vp, i32, vp, vp]
        L.ffvgpu_pool_set_stream.argtypes = [vp, vp]
        L.ffvgpu_pool_set_wait_limit.argtypes = [vp, dbl]
        L.ffvgpu_pool_stall_next_solve.argtypes = [vp]
        L.ffvgpu_pool_cap_grids.argtypes = [vp, i32]
        L.ffvgpu_pool_stall_next_matvec.argtypes = [vp]
        L.ffvgpu_fill.argtypes = [vp, i32, dbl]
        L.ffvgpu_grid_neighbors.argtypes = [ctypes.POINTER(GridDesc), vp, vp]
        L.ffvgpu_pool_upload.argtypes = [vp, i32, vp, i32]
        L.ffvgpu_pool_download.argtypes = [vp, i32, vp, i32]
        L.ffvgpu_exchange.argtypes = [vp, i32, vp, vp]
        L.ffvgpu_assemble_p.argtypes = [vp, dbl, dbl]
        L.ffvgpu_fold_bc.argtypes = [vp]
        L.ffvgpu_solve_rbgs.argtypes = [vp, ctypes.POINTER(IterParams), ctypes.POINTER(Result)]
        L.ffvgpu_solve_cg.argtypes = [vp, ctypes.POINTER(IterParams), ctypes.POINTER(Result)]
        L.ffvgpu_solve_bicgstab.argtypes = [vp, ctypes.POINTER(IterParams), ctypes.POINTER(Result)]
        L.ffvgpu_remove_p.argtypes = [vp, dbl, dbl]
        L.ffvgpu_corr_u.argtypes = [vp, dbl, dbl]
        L.ffvgpu_dump2.argtypes = [vp, i32, i32, ctypes.c_char_p]
        L.ffvgpu_load2.argtypes = [vp, i32, i32, ctypes.c_char_p]
        L.ffvgpu_restart_filename.argtypes = [ctypes.c_char_p, i32, ctypes.c_char_p,
                                              ctypes.c_char_p, ctypes.c_char_p, i32, i32]
        L.ffvgpu_solve_rbgs_fixed_average.argtypes = [vp, ctypes.POINTER(IterParams),
                                                      ctypes.c_int64, ctypes.POINTER(Result)]
        L.ffvgpu_rbgs_sweep.argtypes = [vp, dbl]
        L.ffvgpu_calc_r2.argtypes = [vp, ctypes.POINTER(dbl)]
        L.ffvgpu_dot.argtypes = [vp, i32, i32, ctypes.POINTER(dbl)]
        L.ffvgpu_sphere_grid_create.argtypes = [ctypes.POINTER(SphereParams), ctypes.POINTER(vp)]
        L.ffvgpu_sphere_grid_destroy.argtypes = [vp]
        L.ffvgpu_sphere_grid_destroy.restype = None
        L.ffvgpu_sphere_grid_num_blocks.argtypes = [vp]
        L.ffvgpu_sphere_grid_blocks.argtypes = [vp, vp, vp]
        L.ffvgpu_sphere_grid_blocks.restype = None
        L.ffvgpu_sphere_grid_fill.argtypes = [vp, ctypes.c_uint64, dbl, i32, vp, vp, vp, vp, vp, vp]
        L.ffvgpu_dot_noalloc.argtypes = [vp, vp, i32, vp, vp]
        MP, R = ctypes.POINTER(MixedParams), ctypes.POINTER(Result)
        L.ffvgpu_solve_mixed.argtypes = [vp, MP, R]
        L.ffvgpu_cf_flux_mismatch.argtypes = [vp, vp, vp, vp, vp, i32]
        L.ffvgpu_update_p.argtypes = [vp, ctypes.POINTER(StepParams), vp, R]
        L.ffvgpu_shard_create.argtypes = [ctypes.POINTER(GridDesc), i32, i32, ctypes.POINTER(vp)]
        L.ffvgpu_shard_destroy.argtypes = [vp]
        L.ffvgpu_shard_destroy.restype = None
        L.ffvgpu_shard_info.argtypes = [vp, vp, vp]
        L.ffvgpu_shard_local_blocks.argtypes = [vp, vp]
        L.ffvgpu_shard_zorder.argtypes = [vp, vp, vp]
        L.ffvgpu_shard_local_desc.argtypes = [vp]
        L.ffvgpu_shard_local_desc.restype = ctypes.POINTER(GridDesc)
        L.ffvgpu_shard_peer.argtypes = [vp, i32, vp, vp, vp, vp]
        L.ffvgpu_rbgs_pass.argtypes = [vp, i32, i32, i32, i32, dbl, vp]
        L.ffvgpu_block_dots.argtypes = [vp, i32, i32, i32, vp]
        L.ffvgpu_pool_field_device.argtypes = [vp, i32, ctypes.POINTER(vp)]
        L.ffvgpu_canonical_sum.argtypes = [vp, i32, vp]
        L.ffvgpu_update_u.argtypes = [vp, ctypes.POINTER(StepParams)]
        L.ffvgpu_generate_sphere.argtypes = [vp, ctypes.POINTER(SphereProblem)]
        L.ffvgpu_batch_create.argtypes = [ctypes.POINTER(BatchDesc), ctypes.POINTER(vp)]
        L.ffvgpu_instance_admit.argtypes = [vp, ctypes.POINTER(GridDesc), vp]
        L.ffvgpu_instance_admit_sphere.argtypes = [vp, ctypes.POINTER(SphereProblem), vp]
        L.ffvgpu_assemble_sphere.argtypes = [vp, ctypes.POINTER(SphereProblem)]
        L.ffvgpu_instance_upload.argtypes = [vp, i32, i32, vp, i32]
        L.ffvgpu_instance_download.argtypes = [vp, i32, i32, vp, i32]
        L.ffvgpu_instance_release.argtypes = [vp, i32]
        L.ffvgpu_instance_fill.argtypes = [vp, i32, i32, dbl]
        L.ffvgpu_mixed_autotune.argtypes = [vp, vp, i32, MP, ctypes.POINTER(TuneRecord), i32,
                                             vp]
        L.ffvgpu_serve.argtypes = [vp, MP, i32, ctypes.POINTER(Request), i32,
                                   ctypes.POINTER(RequestResult)]
        L.ffvgpu_instance_blocks.argtypes = [vp, i32]
        L.ffvgpu_pool_free_blocks.argtypes = [vp, vp, vp]
        L.ffvgpu_mixed_begin.argtypes = [vp, i32, MP]
        L.ffvgpu_mixed_advance.argtypes = [vp, i32]
        L.ffvgpu_mixed_poll.argtypes = [vp, vp, i32, vp]
        L.ffvgpu_mixed_cancel.argtypes = [vp, i32]
        L.ffvgpu_instance_result.argtypes = [vp, i32, R, vp]
        _lib = L
    return _lib


def restart_filename(path, prefix, label, rank, step):
    """The reference's Dump2/Load2 file name (ffvgpu_restart_filename)."""
    buf = ctypes.create_string_buffer(4096)
    n = lib().ffvgpu_restart_filename(buf, 4096, path.encode(), prefix.encode(), label.encode(),
                                      rank, step)
    if n < 0:
        raise ValueError("file name too long")
    return buf.value.decode()


class FFVGPUError(RuntimeError):
    def __init__(self, status, what):
        msg = lib().ffvgpu_last_error().decode(errors="replace")
        super().__init__(f"{what} failed with status {status}: {msg}")
        self.status = status


def _check(status, what, allow=(OK,)):
    if status not in allow:
        raise FFVGPUError(status, what)
    return status


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


# ---------------------------------------------------------------------------
# Synthetic sphere grids (host only)
# ---------------------------------------------------------------------------
FLOW_PAST_SPHERE = dict(domain_origin=(-4.0, -4.0, -4.0), root_grid=(4, 2, 2), root_length=4.0,
                        center=(0.0, 0.0, 0.0), radius=0.5, margin=0.5)

# Pressure BCs of the sphere example (examples/FlowPastASphere/sphere.tpp):
# Neumann 0 at the inlet (X_M) and side walls, Dirichlet 0 at the outlet (X_P).
P_BC_TYPE = (BC_NEUMANN, BC_DIRICHLET, BC_NEUMANN, BC_NEUMANN, BC_NEUMANN, BC_NEUMANN)
P_BC_VALUE = (0.0,) * 6
# Velocity BCs: inlet Dirichlet (1,0,0); outlet and walls Neumann 0.
U_BC_TYPE = (BC_DIRICHLET, BC_NEUMANN, BC_NEUMANN, BC_NEUMANN, BC_NEUMANN, BC_NEUMANN)
U_BC_VALUE = {"UX": (1.0, 0, 0, 0, 0, 0), "UY": (0.0,) * 6, "UZ": (0.0,) * 6}


class SphereGrid:
    """2:1-balanced octree of 16^3 leaf blocks refined around a sphere."""

    def __init__(self, max_level, **kw):
        p = dict(FLOW_PAST_SPHERE)
        p.update(kw)
        self.params = p
        self.max_level = max_level
        sp = SphereParams(p["domain_origin"], p["root_grid"], p["root_length"], max_level,
                          p["center"], p["radius"], p["margin"])
        self._h = ctypes.c_void_p()
        _check(lib().ffvgpu_sphere_grid_create(ctypes.byref(sp), ctypes.byref(self._h)),
               "sphere_grid_create")
        self.nb = lib().ffvgpu_sphere_grid_num_blocks(self._h)
        self.level = np.zeros(self.nb, np.int32)
        self.index = np.zeros((self.nb, 3), np.int32)
        lib().ffvgpu_sphere_grid_blocks(self._h, _ptr(self.level), _ptr(self.index))

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.ffvgpu_sphere_grid_destroy(self._h)
            self._h = None

    @property
    def cells(self):
        return self.nb * 4096

    def fill(self, seed=0, sigma=0.01, vc=2):
        """Per-cell inputs in the reference layout: dict of numpy arrays."""
        w = 16 + 2 * vc
        shape = (self.nb, w, w, w)  # [block][k][j][i]
        out = {k: np.zeros(shape, np.float64) for k in ("UX", "UY", "UZ")}
        for f in range(6):
            out[f"C{f}"] = np.zeros(shape, np.float64)
            out[f"CID{f}"] = np.zeros(shape, np.int32)
        out["PID"] = np.zeros(shape, np.int32)
        c6 = (ctypes.c_void_p * 6)(*[out[f"C{f}"].ctypes.data for f in range(6)])
        i6 = (ctypes.c_void_p * 6)(*[out[f"CID{f}"].ctypes.data for f in range(6)])
        _check(lib().ffvgpu_sphere_grid_fill(self._h, seed, sigma, vc, _ptr(out["UX"]),
                                             _ptr(out["UY"]), _ptr(out["UZ"]),
                                             ctypes.cast(c6, ctypes.c_void_p),
                                             ctypes.cast(i6, ctypes.c_void_p), _ptr(out["PID"])),
               "sphere_grid_fill")
        return out

    def neighbors(self):
        """Host-only derived neighbour table: (kind [nb][6], ids [nb][6][4])."""
        d = self.desc()
        kind = np.zeros((self.nb, 6), np.int32)
        ids = np.zeros((self.nb, 6, 4), np.int32)
        _check(lib().ffvgpu_grid_neighbors(ctypes.byref(d), _ptr(kind), _ptr(ids)),
               "grid_neighbors")
        return kind, ids

    def desc(self, bc_type=P_BC_TYPE, bc_value=P_BC_VALUE):
        p = self.params
        d = GridDesc()
        d.num_blocks = self.nb
        d.cells = 16
        self._lev_keep = np.ascontiguousarray(self.level)
        self._idx_keep = np.ascontiguousarray(self.index.reshape(-1))
        d.level = self._lev_keep.ctypes.data
        d.block_index = self._idx_keep.ctypes.data
        d.domain_origin = tuple(p["domain_origin"])
        d.root_length = p["root_length"]
        d.root_grid = tuple(p["root_grid"])
        d.neighbor_kind = None
        d.neighbor_ids = None
        d.bc_type = tuple(bc_type)
        d.bc_value = tuple(bc_value)
        return d


# ---------------------------------------------------------------------------
# Device pool
# ---------------------------------------------------------------------------
class Pool:
    """A device-resident leaf-block pool (ffvgpu_pool)."""

    def __init__(self, desc):
        self._desc = desc
        self._h = ctypes.c_void_p()
        _check(lib().ffvgpu_pool_create(ctypes.byref(desc), ctypes.byref(self._h)), "pool_create")
        self.nb = lib().ffvgpu_pool_num_blocks(self._h)

    def close(self):
        # the handle is cleared in place: at interpreter exit __del__ may run
        # after module globals such as ctypes are gone
        h = getattr(self, "_h", None)
        if h is not None and h.value and _lib is not None:
            _lib.ffvgpu_pool_destroy(h)
            h.value = None

    def __del__(self):
        self.close()

    @property
    def device_bytes(self):
        return lib().ffvgpu_pool_device_bytes(self._h)

    def neighbors(self, b):
        kind = np.zeros(6, np.int32)
        ids = np.zeros(24, np.int32)
        _check(lib().ffvgpu_pool_neighbors(self._h, b, _ptr(kind), _ptr(ids)), "pool_neighbors")
        return kind, ids.reshape(6, 4)

    def upload(self, field, arr, vc=2):
        fid = FIELD[field]
        dt = np.int32 if fid >= 100 else np.float64
        a = np.ascontiguousarray(arr, dtype=dt)
        assert a.size == self.nb * (16 + 2 * vc) ** 3, (a.shape, vc)
        _check(lib().ffvgpu_pool_upload(self._h, fid, _ptr(a), vc), f"upload {field}")

    def upload_ptr(self, field, host_ptr, vc=2):
        """Upload from a raw host pointer (e.g. pinned memory)."""
        _check(lib().ffvgpu_pool_upload(self._h, FIELD[field], ctypes.c_void_p(host_ptr), vc),
               f"upload {field}")

    def download(self, field, vc=2):
        fid = FIELD[field]
        w = 16 + 2 * vc
        a = np.zeros((self.nb, w, w, w), np.int32 if fid >= 100 else np.float64)
        _check(lib().ffvgpu_pool_download(self._h, fid, _ptr(a), vc), f"download {field}")
        return a

    def download_ptr(self, field, host_ptr, vc=2):
        _check(lib().ffvgpu_pool_download(self._h, FIELD[field], ctypes.c_void_p(host_ptr), vc),
               f"download {field}")

    def exchange(self, field, bc_type=None, bc_value=None):
        if bc_type is None:
            _check(lib().ffvgpu_exchange(self._h, FIELD[field], None, None), f"exchange {field}")
            return
        t = np.asarray(bc_type, np.int32)
        v = np.asarray(bc_value, np.float64)
        _check(lib().ffvgpu_exchange(self._h, FIELD[field], _ptr(t), _ptr(v)), f"exchange {field}")

    def assemble_p(self, rhof=1.0, dt=0.002):
        _check(lib().ffvgpu_assemble_p(self._h, rhof, dt), "assemble_p")

    def fold_bc(self):
        _check(lib().ffvgpu_fold_bc(self._h), "fold_bc")

    def _solve(self, fn, what, omega, count_max, epsilon, pre_count, history, check_every,
               restart_drop=0.0):
        hist = np.zeros(max(count_max, 1), np.float64) if history else None
        prm = IterParams(omega, count_max, epsilon, pre_count, check_every,
                         hist.ctypes.data if history else None, restart_drop)
        res = Result()
        st = fn(self._h, ctypes.byref(prm), ctypes.byref(res))
        _check(st, what, allow=(OK, NOT_CONVERGED, NAN_DETECTED))
        out = dict(status=st, count=res.count, residual=res.residual, elapsed_ms=res.elapsed_ms,
                   sweep_ms=res.sweep_ms, sweep_launches=res.sweep_launches,
                   bytes_moved=res.bytes_moved, kernel_launches=res.kernel_launches,
                   uniform_blocks=res.uniform_blocks)
        if history:
            if res.count == 0:  # early exit: the residuals written before it
                n = int(np.argmax(hist == 0)) if (hist == 0).any() else len(hist)
            else:
                n = res.count if 1 <= res.count <= count_max else count_max
            out["history"] = hist[:n].copy()
        return out

    def solve_rbgs(self, omega=1.5, count_max=200, epsilon=0.0, history=True, check_every=0):
        return self._solve(lib().ffvgpu_solve_rbgs, "solve_rbgs", omega, count_max, epsilon, 0,
                           history, check_every)

    def solve_rbgs_fixed_average(self, omega=1.0, ncells=None, count_max=200, epsilon=0.0,
                                 history=True, check_every=0):
        n = self.nb * 4096 if ncells is None else ncells
        hist = np.zeros(max(count_max, 1), np.float64) if history else None
        prm = IterParams(omega, count_max, epsilon, 0, check_every,
                         hist.ctypes.data if history else None, 0.0)
        res = Result()
        st = lib().ffvgpu_solve_rbgs_fixed_average(self._h, ctypes.byref(prm), n,
                                                   ctypes.byref(res))
        _check(st, "solve_rbgs_fixed_average", allow=(OK, NOT_CONVERGED, NAN_DETECTED))
        out = dict(status=st, count=res.count, residual=res.residual, elapsed_ms=res.elapsed_ms)
        if history:
            nh = res.count if 1 <= res.count <= count_max else count_max
            out["history"] = hist[:nh].copy()
        return out

    def solve_cg(self, omega=1.0, pre_count=2, count_max=10000, epsilon=1e-10, history=True,
                 check_every=0):
        return self._solve(lib().ffvgpu_solve_cg, "solve_cg", omega, count_max, epsilon,
                           pre_count, history, check_every)

    def solve_bicgstab(self, omega=1.0, pre_count=2, count_max=1000, epsilon=1e-10,
                       history=True, check_every=0, restart_drop=0.0):
        return self._solve(lib().ffvgpu_solve_bicgstab, "solve_bicgstab", omega, count_max,
                           epsilon, pre_count, history, check_every, restart_drop)

    def remove_p(self, rhof=1.0, dt=0.002):
        _check(lib().ffvgpu_remove_p(self._h, rhof, dt), "remove_p")

    @staticmethod
    def _step_params(rhof, dt, solver, omega, pre_count, count_max, epsilon, restart_drop):
        sp = StepParams()
        sp.rhof, sp.dt, sp.solver = rhof, dt, solver
        for c, u in enumerate(("UX", "UY", "UZ")):
            for f in range(6):
                sp.u_bc_type[c][f] = U_BC_TYPE[f]
                sp.u_bc_value[c][f] = U_BC_VALUE[u][f]
        sp.iter = IterParams(omega, count_max, epsilon, pre_count, 0, None, restart_drop)
        return sp

    def update_p(self, solver=SOLVER_BICGSTAB, omega=1.0, pre_count=2, count_max=1000,
                 epsilon=1e-8, restart_drop=0.0, rhof=1.0, dt=0.002, mixed=None):
        """Solver::UpdateP's pressure sequence (ffvgpu_update_p) with the sphere
        example's velocity BCs; mixed: dict of solve_mixed settings for SOLVER_MIXED."""
        sp = self._step_params(rhof, dt, solver, omega, pre_count, count_max, epsilon,
                               restart_drop)
        mp = None
        if solver == SOLVER_MIXED:
            m = dict(omega=1.5, sweeps=8, sweeps_per_exchange=4, flux_correction=False)
            m.update(mixed or {})
            mp = MixedParams(m["omega"], m["sweeps"], m["sweeps_per_exchange"], count_max,
                             epsilon, 0, None, *_restart(None, None, None))
            mp.flux_correction = int(bool(m["flux_correction"]))
        res = Result()
        st = lib().ffvgpu_update_p(self._h, ctypes.byref(sp),
                                   ctypes.byref(mp) if mp is not None else None,
                                   ctypes.byref(res))
        _check(st, "update_p", allow=(OK, NOT_CONVERGED))
        return dict(status=st, count=res.count, residual=res.residual, elapsed_ms=res.elapsed_ms,
                    bytes_moved=res.bytes_moved, kernel_launches=res.kernel_launches)

    def update_u(self, rhof=1.0, dt=0.002):
        """Solver::UpdateU (ffvgpu_update_u) with the sphere example's velocity BCs."""
        sp = self._step_params(rhof, dt, SOLVER_BICGSTAB, 1.0, 0, 0, 0.0, 0.0)
        _check(lib().ffvgpu_update_u(self._h, ctypes.byref(sp)), "update_u")

    # ---- pieces of a sharded solve -------------------------------------
    def rbgs_pass(self, blocks, residual, sweep, stored, omega):
        """One red-black pass over the first 'blocks' blocks (ffvgpu_rbgs_pass);
        returns the per-block residual partials when residual is set."""
        part = np.zeros(max(blocks, 1), np.float64) if residual else None
        _check(lib().ffvgpu_rbgs_pass(self._h, blocks, int(residual), int(sweep), int(stored),
                                      float(omega), _ptr(part) if residual else None),
               "rbgs_pass")
        return part

    def block_dots(self, fx, fy, blocks):
        part = np.zeros(max(blocks, 1), np.float64)
        _check(lib().ffvgpu_block_dots(self._h, FIELD[fx], FIELD[fy], blocks, _ptr(part)),
               "block_dots")
        return part

    def field_device(self, field="X"):
        """Device address of the current iterate (X) or of b (B): blocks x 4096 doubles."""
        v = ctypes.c_void_p()
        _check(lib().ffvgpu_pool_field_device(self._h, FIELD[field], ctypes.byref(v)),
               "pool_field_device")
        return v.value

    def generate_sphere(self, problem):
        """Device-generated u*, cut fields and flags only (ffvgpu_generate_sphere)."""
        _check(lib().ffvgpu_generate_sphere(self._h, ctypes.byref(problem)), "generate_sphere")

    def corr_u(self, rhof=1.0, dt=0.002):
        _check(lib().ffvgpu_corr_u(self._h, rhof, dt), "corr_u")

    def dump2(self, field, filename, vc=2):
        _check(lib().ffvgpu_dump2(self._h, FIELD[field], vc, filename.encode()), "dump2")

    def load2(self, field, filename, vc=2):
        _check(lib().ffvgpu_load2(self._h, FIELD[field], vc, filename.encode()), "load2")

    def set_stream(self, stream_handle):
        """Enqueue on a caller's CUDA stream (an int cudaStream_t, 0/None = own)."""
        _check(lib().ffvgpu_pool_set_stream(self._h, ctypes.c_void_p(stream_handle or None)),
               "pool_set_stream")

    def set_wait_limit(self, seconds):
        """Time limit of every bounded device wait (ffvgpu_pool_set_wait_limit)."""
        _check(lib().ffvgpu_pool_set_wait_limit(self._h, float(seconds)), "pool_set_wait_limit")

    def stall_next_solve(self):
        """Test hook: the next mixed solve's sweep waits for a copy never issued."""
        _check(lib().ffvgpu_pool_stall_next_solve(self._h), "pool_stall_next_solve")

    def cap_grids(self, ctas):
        """Test hook: at most ctas CTAs per persistent grid (0: none)."""
        _check(lib().ffvgpu_pool_cap_grids(self._h, int(ctas)), "pool_cap_grids")

    def stall_next_matvec(self):
        """Test hook: the next mixed solve's pipelined A*x issues no copy."""
        _check(lib().ffvgpu_pool_stall_next_matvec(self._h), "pool_stall_next_matvec")

    def fill(self, field, value):
        _check(lib().ffvgpu_fill(self._h, FIELD[field], float(value)), "fill")

    def rbgs_sweep(self, omega):
        _check(lib().ffvgpu_rbgs_sweep(self._h, omega), "rbgs_sweep")

    def calc_r2(self):
        v = ctypes.c_double()
        _check(lib().ffvgpu_calc_r2(self._h, ctypes.byref(v)), "calc_r2")
        return v.value

    def dot(self, fx, fy):
        v = ctypes.c_double()
        _check(lib().ffvgpu_dot(self._h, FIELD[fx], FIELD[fy], ctypes.byref(v)), "dot")
        return v.value

    def cf_flux_mismatch(self, per_cell=False):
        """Coarse-fine flux mismatch of X (ffvgpu_cf_flux_mismatch): dict with
        mismatch = sum V|delta|, flux = sum V|F|, cells, and with per_cell an
        array [cells][2] of (delta, F) in (block, face, position) order."""
        m, fl, n = ctypes.c_double(), ctypes.c_double(), ctypes.c_int32()
        _check(lib().ffvgpu_cf_flux_mismatch(self._h, ctypes.byref(m), ctypes.byref(fl),
                                             ctypes.byref(n), None, 0), "cf_flux_mismatch")
        out = dict(mismatch=m.value, flux=fl.value, cells=n.value)
        if per_cell:
            arr = np.zeros((max(n.value, 1), 2), np.float64)
            _check(lib().ffvgpu_cf_flux_mismatch(self._h, ctypes.byref(m), ctypes.byref(fl),
                                                 ctypes.byref(n), arr.ctypes.data, n.value),
                   "cf_flux_mismatch")
            out["per_cell"] = arr[:n.value]
        return out

    def assemble_sphere(self, problem):
        """Device-generated sphere-flow inputs + UpdateP P02-P05 (pool made from its grid)."""
        _check(lib().ffvgpu_assemble_sphere(self._h, ctypes.byref(problem)), "assemble_sphere")

    def solve_mixed(self, omega=1.5, sweeps=8, sweeps_per_exchange=4, count_max=1000,
                    epsilon=1e-8, history=True, check_every=0, restart_drop=None,
                    restart_growth=None, restart_every=None, flux_correction=False,
                    fp64_data=False, threads_per_block=0, stage_depth=0, sweep_threads=0,
                    matvec_form=0):
        """Mixed-precision solve (FP64 BiCGSTAB; RB-SOR preconditioner on 32-bit data).
        flux_correction: the FP64 residual and A*x use the coarse-fine
        flux-conserving operator; fp64_data: the same preconditioner on FP64 data;
        threads_per_block, stage_depth, sweep_threads, matvec_form: launch settings
        (0: defaults)."""
        hist = np.zeros(max(count_max, 1), np.float64) if history else None
        prm = MixedParams(omega, sweeps, sweeps_per_exchange, count_max, epsilon, check_every,
                          hist.ctypes.data if history else None,
                          *_restart(restart_drop, restart_growth, restart_every))
        prm.flux_correction = int(bool(flux_correction))
        prm.fp64_data = int(bool(fp64_data))
        prm.threads_per_block, prm.stage_depth = int(threads_per_block), int(stage_depth)
        prm.sweep_threads, prm.matvec_form = int(sweep_threads), int(matvec_form)
        res = Result()
        st = lib().ffvgpu_solve_mixed(self._h, ctypes.byref(prm), ctypes.byref(res))
        _check(st, "solve_mixed", allow=(OK, NOT_CONVERGED, NAN_DETECTED))
        out = dict(status=st, count=res.count, residual=res.residual, elapsed_ms=res.elapsed_ms,
                   sweep_ms=res.sweep_ms, kernel_launches=res.kernel_launches,
                   bytes_moved=res.bytes_moved, uniform_blocks=res.uniform_blocks)
        if history:
            n = res.count if 1 <= res.count <= count_max else (count_max if res.count > 0 else 0)
            out["history"] = hist[:n].copy()
        return out


def canonical_sum(partials):
    """The pool's cross-block reduction over per-block partials in block order."""
    a = np.ascontiguousarray(partials, np.float64)
    t = ctypes.c_double()
    _check(lib().ffvgpu_canonical_sum(_ptr(a), len(a), ctypes.byref(t)), "canonical_sum")
    return t.value


class Shard:
    """One rank's part of a grid sharded across ranks (ffvgpu_shard_*): its own
    blocks (local 0 .. owned-1), halo blocks, and the exchange lists per peer."""

    def __init__(self, desc, num_ranks, rank):
        self._h = ctypes.c_void_p()
        self._desc = desc
        _check(lib().ffvgpu_shard_create(ctypes.byref(desc), num_ranks, rank,
                                         ctypes.byref(self._h)), "shard_create")
        o, h = ctypes.c_int32(), ctypes.c_int32()
        _check(lib().ffvgpu_shard_info(self._h, ctypes.byref(o), ctypes.byref(h)), "shard_info")
        self.ranks, self.rank = num_ranks, rank
        self.owned, self.halo = o.value, h.value
        self.local = np.zeros(self.owned + self.halo, np.int32)
        _check(lib().ffvgpu_shard_local_blocks(self._h, _ptr(self.local)), "shard_local_blocks")
        n = desc.num_blocks
        self.zorder = np.zeros(n, np.int32)
        self.owner = np.zeros(n, np.int32)
        _check(lib().ffvgpu_shard_zorder(self._h, _ptr(self.zorder), _ptr(self.owner)),
               "shard_zorder")
        self.send, self.recv = {}, {}
        for p in range(num_ranks):
            if p == rank:
                continue
            ns, nr = ctypes.c_int32(), ctypes.c_int32()
            _check(lib().ffvgpu_shard_peer(self._h, p, ctypes.byref(ns), None, ctypes.byref(nr),
                                           None), "shard_peer")
            sl = np.zeros(max(ns.value, 1), np.int32)
            rl = np.zeros(max(nr.value, 1), np.int32)
            _check(lib().ffvgpu_shard_peer(self._h, p, ctypes.byref(ns), _ptr(sl),
                                           ctypes.byref(nr), _ptr(rl)), "shard_peer")
            self.send[p] = sl[:ns.value]
            self.recv[p] = rl[:nr.value]

    def desc(self):
        """The local grid description (pointers valid while this object lives)."""
        return lib().ffvgpu_shard_local_desc(self._h).contents

    def close(self):
        # the handle is cleared in place: at interpreter exit __del__ may run
        # after module globals such as ctypes are gone
        h = getattr(self, "_h", None)
        if h is not None and h.value and _lib is not None:
            _lib.ffvgpu_shard_destroy(h)
            h.value = None

    def __del__(self):
        self.close()


class _DeviceArray:
    """A device array for torch.as_tensor (__cuda_array_interface__, no copy)."""

    def __init__(self, ptr, shape):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": "<f8",
                                         "data": (int(ptr), False), "version": 3,
                                         "strides": None}


def pool_iterate(pool, blocks):
    """torch view [blocks][4096] of the pool's current iterate (device memory, no copy)."""
    import torch
    return torch.as_tensor(_DeviceArray(pool.field_device("X"), (blocks, 4096)), device="cuda")


def halo_exchange(dist, shard, x):
    """One exchange of a shard's halo blocks over torch.distributed: x is the
    rank's [local blocks][4096] iterate (a device view of the pool, or a host
    tensor); every rank sends each peer the blocks shard.send lists and
    stores what the peer sends into the blocks shard.recv lists, in list
    order.  Point-to-point only, the same steps on every rank."""
    import torch
    ops, recvs = [], []
    for p in sorted(set(shard.send) | set(shard.recv)):
        snd, rcv = shard.send.get(p, ()), shard.recv.get(p, ())
        if len(snd):
            idx = torch.as_tensor(np.asarray(snd, np.int64), device=x.device)
            ops.append(dist.P2POp(dist.isend, x.index_select(0, idx).contiguous(), p))
        if len(rcv):
            buf = torch.empty((len(rcv), x.shape[1]), dtype=x.dtype, device=x.device)
            ops.append(dist.P2POp(dist.irecv, buf, p))
            recvs.append((rcv, buf))
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()
    for rcv, buf in recvs:
        x.index_copy_(0, torch.as_tensor(np.asarray(rcv, np.int64), device=x.device), buf)


def sharded_rbgs(parts, omega, count, exchange, gather):
    """FFVILS::RBGS (ffvgpu_solve_rbgs's passes, epsilon 0) on a sharded grid.
    parts: the [(pool, shard)] this process drives (one per GPU: one part per
    rank over torch.distributed, or every part on one device); exchange():
    refreshes every part's halo blocks of the current iterate from their
    owners (halo_exchange); gather(list of per-block partials, one array per
    part, own blocks in local order): the per-block partials of every block
    of the grid in global block order.  Returns the residual history, bit for
    bit the unsharded pool's: same passes, same per-block sums, same
    cross-block tree."""
    tiny = float(np.finfo(np.float32).tiny)
    bb = canonical_sum(gather([P.block_dots("B", "B", S.owned) for P, S in parts]))

    def resid(partials):
        rr = canonical_sum(gather(partials))
        return float(np.sqrt(abs(rr) / abs(bb))) if abs(bb) > tiny else float(np.sqrt(abs(rr)))

    for P, S in parts:
        P.rbgs_pass(S.owned, 0, 1, 1, omega)
    hist = []
    for _ in range(2, count + 1):
        exchange()
        hist.append(resid([P.rbgs_pass(S.owned, 1, 1, 0, omega) for P, S in parts]))
    exchange()
    hist.append(resid([P.rbgs_pass(S.owned, 1, 0, 0, omega) for P, S in parts]))
    return np.array(hist)


def _restart(drop, growth, every):
    return (RESTART["restart_drop"] if drop is None else drop,
            RESTART["restart_growth"] if growth is None else growth,
            RESTART["restart_every"] if every is None else every)


def sphere_problem(max_level, seed=1, sigma=0.01, dt=0.002, rhof=1.0, **grid_kw):
    """ffvgpu_sphere_problem of the sphere-flow workload (grid keywords as SphereGrid)."""
    p = dict(FLOW_PAST_SPHERE)
    p.update(grid_kw)
    sp = SphereParams(p["domain_origin"], p["root_grid"], p["root_length"], max_level,
                      p["center"], p["radius"], p["margin"])
    pr = SphereProblem()
    pr.grid = sp
    pr.seed = seed
    pr.sigma = sigma
    pr.rhof = rhof
    pr.dt = dt
    for c, u in enumerate(("UX", "UY", "UZ")):
        for f in range(6):
            pr.u_bc_type[c][f] = U_BC_TYPE[f]
            pr.u_bc_value[c][f] = U_BC_VALUE[u][f]
    return pr


class Batch:
    """A batch pool: independent pressure problems sharing one device pool."""

    def __init__(self, capacity_blocks, max_instances=64, bc_type=P_BC_TYPE, bc_value=P_BC_VALUE):
        d = BatchDesc(capacity_blocks, max_instances, tuple(bc_type), tuple(bc_value))
        self._h = ctypes.c_void_p()
        _check(lib().ffvgpu_batch_create(ctypes.byref(d), ctypes.byref(self._h)), "batch_create")
        self.capacity = capacity_blocks

    def close(self):
        # the handle is cleared in place: at interpreter exit __del__ may run
        # after module globals such as ctypes are gone
        h = getattr(self, "_h", None)
        if h is not None and h.value and _lib is not None:
            _lib.ffvgpu_pool_destroy(h)
            h.value = None

    def __del__(self):
        self.close()

    @property
    def device_bytes(self):
        return lib().ffvgpu_pool_device_bytes(self._h)

    def admit_sphere(self, problem):
        """Instance id, or None when no block range or slot is free (FFVGPU_OOM)."""
        i = ctypes.c_int32()
        st = lib().ffvgpu_instance_admit_sphere(self._h, ctypes.byref(problem), ctypes.byref(i))
        if st == OOM:
            return None
        _check(st, "instance_admit_sphere")
        return i.value

    def admit(self, desc):
        i = ctypes.c_int32()
        st = lib().ffvgpu_instance_admit(self._h, ctypes.byref(desc), ctypes.byref(i))
        if st == OOM:
            return None
        _check(st, "instance_admit")
        return i.value

    def blocks(self, inst):
        return lib().ffvgpu_instance_blocks(self._h, inst)

    def free_blocks(self):
        t, r = ctypes.c_int32(), ctypes.c_int32()
        _check(lib().ffvgpu_pool_free_blocks(self._h, ctypes.byref(t), ctypes.byref(r)),
               "pool_free_blocks")
        return t.value, r.value

    def upload(self, inst, field, arr, vc=2):
        fid = FIELD[field]
        a = np.ascontiguousarray(arr, dtype=np.int32 if fid >= 100 else np.float64)
        assert a.size == self.blocks(inst) * (16 + 2 * vc) ** 3
        _check(lib().ffvgpu_instance_upload(self._h, inst, fid, _ptr(a), vc), f"upload {field}")

    def upload_ptr(self, inst, field, host_ptr, vc=2):
        """Upload from a raw host pointer (pinned memory is read directly)."""
        _check(lib().ffvgpu_instance_upload(self._h, inst, FIELD[field],
                                            ctypes.c_void_p(host_ptr), vc), f"upload {field}")

    def download(self, inst, field, vc=2):
        fid = FIELD[field]
        w = 16 + 2 * vc
        a = np.zeros((self.blocks(inst), w, w, w), np.int32 if fid >= 100 else np.float64)
        _check(lib().ffvgpu_instance_download(self._h, inst, fid, _ptr(a), vc),
               f"download {field}")
        return a

    def release(self, inst):
        _check(lib().ffvgpu_instance_release(self._h, inst), "instance_release")

    def fill(self, inst, field, value):
        _check(lib().ffvgpu_instance_fill(self._h, inst, FIELD[field], float(value)),
               "instance_fill")

    def set_stream(self, stream_handle):
        _check(lib().ffvgpu_pool_set_stream(self._h, ctypes.c_void_p(stream_handle or None)),
               "pool_set_stream")

    def set_wait_limit(self, seconds):
        _check(lib().ffvgpu_pool_set_wait_limit(self._h, float(seconds)), "pool_set_wait_limit")

    def cap_grids(self, ctas):
        """Test hook: at most ctas CTAs per persistent grid of the mixed form (0: none)."""
        _check(lib().ffvgpu_pool_cap_grids(self._h, int(ctas)), "pool_cap_grids")

    def solve_mixed(self, omega=1.5, sweeps=8, sweeps_per_exchange=4, count_max=1000,
                    epsilon=1e-8, check_every=0, restart_drop=None, restart_growth=None,
                    restart_every=None, flux_correction=False, fp64_data=False,
                    threads_per_block=0, stage_depth=0, sweep_threads=0, matvec_form=0):
        """Solves every admitted instance; returns the first instance's result."""
        prm = MixedParams(omega, sweeps, sweeps_per_exchange, count_max, epsilon, check_every,
                          None, *_restart(restart_drop, restart_growth, restart_every))
        prm.flux_correction = int(bool(flux_correction))
        prm.fp64_data = int(bool(fp64_data))
        prm.threads_per_block, prm.stage_depth = int(threads_per_block), int(stage_depth)
        prm.sweep_threads, prm.matvec_form = int(sweep_threads), int(matvec_form)
        res = Result()
        st = lib().ffvgpu_solve_mixed(self._h, ctypes.byref(prm), ctypes.byref(res))
        _check(st, "solve_mixed", allow=(OK, NOT_CONVERGED, NAN_DETECTED))
        return dict(status=st, count=res.count, residual=res.residual, elapsed_ms=res.elapsed_ms,
                    kernel_launches=res.kernel_launches, bytes_moved=res.bytes_moved)

    def serve(self, arrivals, problems, iterations_per_step=8, omega=1.5, sweeps=8,
              sweeps_per_exchange=4, count_max=5000, epsilon=1e-8, restart_drop=None,
              restart_growth=None, restart_every=None, cancels=None):
        """Request loop (ffvgpu_serve): per request admit/finish times, iterations,
        residual, status, blocks.  cancels: optional per-request cancel times (0: never)."""
        n = len(problems)
        req = (Request * n)()
        for i, (t, p) in enumerate(zip(arrivals, problems)):
            req[i].arrival_s = float(t)
            req[i].cancel_s = float(cancels[i]) if cancels is not None else 0.0
            req[i].problem = p
        out = (RequestResult * n)()
        prm = MixedParams(omega, sweeps, sweeps_per_exchange, count_max, epsilon, 0, None,
                          *_restart(restart_drop, restart_growth, restart_every))
        _check(lib().ffvgpu_serve(self._h, ctypes.byref(prm), n, req, iterations_per_step, out),
               "serve")
        return [dict(arrival_s=float(arrivals[i]), admit_s=out[i].admit_s,
                     finish_s=out[i].finish_s, count=out[i].count, residual=out[i].residual,
                     status=out[i].status, blocks=out[i].blocks) for i in range(n)]

    def _tune(self, ids, cands, count_max, epsilon):
        recs = (TuneRecord * len(cands))()
        for k, (om, sw, per, it, nt, dp, st, mv) in enumerate(cands):
            recs[k].omega, recs[k].sweeps = om, sw
            recs[k].sweeps_per_exchange, recs[k].iterations_per_replay = per, it
            recs[k].threads_per_block, recs[k].stage_depth = nt, dp
            recs[k].sweep_threads, recs[k].matvec_form = st, mv
        prm = MixedParams(1.5, 8, 4, count_max, epsilon, 0, None, *_restart(None, None, None))
        best = ctypes.c_int32()
        _check(lib().ffvgpu_mixed_autotune(self._h, _ptr(ids), len(ids), ctypes.byref(prm),
                                           recs, len(cands), ctypes.byref(best)), "autotune")
        out = [dict(omega=r.omega, sweeps=r.sweeps, sweeps_per_exchange=r.sweeps_per_exchange,
                    iterations_per_replay=r.iterations_per_replay,
                    threads_per_block=r.threads_per_block or 256, stage_depth=r.stage_depth or 1,
                    sweep_threads=r.sweep_threads or 256, matvec_form=r.matvec_form,
                    ms=r.ms, max_count=r.max_count, converged=bool(r.converged)) for r in recs]
        return out, best.value

    def autotune(self, instances, space=None, launch=None, count_max=1500, epsilon=1e-8):
        """ffvgpu_mixed_autotune in two stages: the numerical settings of space
        (omega, sweeps, per-exchange, replay iterations) at 256 threads and
        staging depth 1, then the fastest of them over launch (threads per
        block of the A*x and update kernels, staging depth, threads per block
        of the sweep kernel).  Returns (records as dicts, index of the best
        or -1)."""
        ids = np.ascontiguousarray(instances, np.int32)
        space = space or TUNE_SPACE
        launch = launch or TUNE_LAUNCH
        recs, best = self._tune(ids, [(om, sw, per, it) + TUNE_LAUNCH_DEFAULT
                                      for (om, sw, per, it) in space], count_max, epsilon)
        if best < 0:
            return recs, best
        b = recs[best]
        head = (b["omega"], b["sweeps"], b["sweeps_per_exchange"], b["iterations_per_replay"])
        more, best2 = self._tune(ids, [head + tuple(c) for c in launch
                                       if tuple(c) != TUNE_LAUNCH_DEFAULT], count_max, epsilon)
        recs2 = recs + more
        if best2 >= 0 and more[best2]["ms"] < b["ms"]:
            best = len(recs) + best2
        return recs2, best

    def begin(self, inst, omega=1.5, sweeps=8, sweeps_per_exchange=4, count_max=1000,
              epsilon=1e-8, restart_drop=None, restart_growth=None, restart_every=None,
              threads_per_block=0, stage_depth=0, sweep_threads=0, matvec_form=0):
        prm = MixedParams(omega, sweeps, sweeps_per_exchange, count_max, epsilon, 0, None,
                          *_restart(restart_drop, restart_growth, restart_every))
        prm.threads_per_block, prm.stage_depth = int(threads_per_block), int(stage_depth)
        prm.sweep_threads, prm.matvec_form = int(sweep_threads), int(matvec_form)
        _check(lib().ffvgpu_mixed_begin(self._h, inst, ctypes.byref(prm)), "mixed_begin")

    def cancel(self, inst):
        _check(lib().ffvgpu_mixed_cancel(self._h, inst), "mixed_cancel")

    def advance(self, iterations):
        _check(lib().ffvgpu_mixed_advance(self._h, iterations), "mixed_advance")

    def poll(self, capacity=4096):
        out = np.zeros(capacity, np.int32)
        n = ctypes.c_int32()
        _check(lib().ffvgpu_mixed_poll(self._h, _ptr(out), capacity, ctypes.byref(n)),
               "mixed_poll")
        return [int(v) for v in out[:n.value]]

    def result(self, inst, count_max=None):
        res = Result()
        hist = np.zeros(max(count_max or 1, 1), np.float64)
        st = lib().ffvgpu_instance_result(self._h, inst, ctypes.byref(res),
                                          _ptr(hist) if count_max else None)
        _check(st, "instance_result", allow=(OK, NOT_CONVERGED, NAN_DETECTED, CANCELLED))
        out = dict(status=st, count=res.count, residual=res.residual)
        if count_max:
            n = res.count if 1 <= res.count <= count_max else (count_max if res.count > 0 else 0)
            out["history"] = hist[:n].copy()
        return out
