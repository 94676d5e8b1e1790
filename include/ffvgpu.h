/* ffvgpu.h -- C ABI of the B200 pressure-Poisson path for FFV-HC.
 *
 * The reference calls its pressure solver once per time step through
 * FFVILS (src/FFV/FFVILS.h) on a BCMTools block manager whose leaf blocks
 * each hold (n+2*vc)^3 reals per field (src/FFV/LocalScalar3D.h:21-84).
 * This header replaces that per-solve surface with a device-resident block
 * pool: the caller describes the leaf blocks once, uploads fields in the
 * reference's own per-block layout, and calls the solve entry points, which
 * keep every iteration on the GPU.
 *
 * Conventions
 *  - All functions return ffvgpu_status; nothing calls exit().
 *  - One pool is used from one host thread at a time (thread-compatible).
 *  - Host arrays use the reference layout: per block (n+2*vc)^3 doubles
 *    (int32 for integer fields), i fastest, blocks back to back, with
 *    n = 16 and vc >= 1 (the reference default is vc = 2,
 *    src/FFV/FFVConfig.cpp:43-44).
 *  - Faces are numbered X_M=0, X_P=1, Y_M=2, Y_P=3, Z_M=4, Z_P=5 as in
 *    BCMTools' Face enum used by src/FFV/BlockScalar3D.h:42-172.
 */
#ifndef FFVGPU_H
#define FFVGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  FFVGPU_OK = 0,
  FFVGPU_NOT_CONVERGED = 1, /* countMax reached (reference: silent, FFVILS.h:44-45) */
  FFVGPU_NAN_DETECTED = 2,  /* residual NaN/Inf (reference: Exit(0), FFVILS.h:36-43) */
  FFVGPU_TIMEOUT = 3,       /* a bounded device wait gave up */
  FFVGPU_OOM = 4,           /* device allocation failed */
  FFVGPU_BAD_ARG = 5,       /* invalid argument or grid description */
  FFVGPU_CUDA_ERROR = 6,    /* a CUDA runtime call failed */
  FFVGPU_NO_DEVICE = 7,     /* no CUDA device visible */
  FFVGPU_CANCELLED = 8      /* the solve was stopped by ffvgpu_mixed_cancel or a serve
                               request's cancel time (no counterpart in the reference) */
} ffvgpu_status;

/* Outer boundary types, src/FFV/FFVBC.h:6-14. */
enum { FFVGPU_BC_DIRICHLET = 0, FFVGPU_BC_NEUMANN = 1 };

/* Neighbour kinds of one block face. */
enum {
  FFVGPU_NB_OUTER = 0,  /* outer boundary of the domain */
  FFVGPU_NB_SAME = 1,   /* one block of the same level */
  FFVGPU_NB_COARSE = 2, /* one block one level coarser (2:1) */
  FFVGPU_NB_FINE = 3    /* four blocks one level finer */
};

/* Pool fields.  Vectors carry guide cells; matrix fields are interior only. */
typedef enum {
  FFVGPU_FIELD_X = 0, /* pressure p (solution) */
  FFVGPU_FIELD_AP, FFVGPU_FIELD_AW, FFVGPU_FIELD_AE, FFVGPU_FIELD_AS,
  FFVGPU_FIELD_AN, FFVGPU_FIELD_AB, FFVGPU_FIELD_AT,
  FFVGPU_FIELD_B,
  FFVGPU_FIELD_UX, FFVGPU_FIELD_UY, FFVGPU_FIELD_UZ,
  FFVGPU_FIELD_C0, FFVGPU_FIELD_C1, FFVGPU_FIELD_C2, FFVGPU_FIELD_C3,
  FFVGPU_FIELD_C4, FFVGPU_FIELD_C5,
  FFVGPU_FIELD_VW, FFVGPU_FIELD_VE, FFVGPU_FIELD_VS, FFVGPU_FIELD_VN,
  FFVGPU_FIELD_VB, FFVGPU_FIELD_VT,
  FFVGPU_FIELD_LAPP, /* Laplacian of p written by ffvgpu_corr_u (bcut_corr_u's lapp) */
  FFVGPU_FIELD_NUM_REAL,
  /* integer fields */
  FFVGPU_IFIELD_CID0 = 100, FFVGPU_IFIELD_CID1, FFVGPU_IFIELD_CID2,
  FFVGPU_IFIELD_CID3, FFVGPU_IFIELD_CID4, FFVGPU_IFIELD_CID5,
  FFVGPU_IFIELD_PID
} ffvgpu_field;

/* Leaf-block layout, the information BCMTools' BlockManager holds
 * (BlockBase size/origin/level and NeighborInfo, used at
 * src/FFV/Solver.cpp:338-386). */
typedef struct {
  int32_t num_blocks;
  int32_t cells;               /* cells per block edge; must be 16 */
  const int32_t* level;        /* [num_blocks] octree level */
  const int32_t* block_index;  /* [num_blocks][3] block position, in units of
                                  this level's block edge, from domain_origin */
  double domain_origin[3];
  double root_length;          /* edge of a level-0 (root) block */
  int32_t root_grid[3];        /* root blocks per axis */
  /* Optional explicit neighbour table; NULL derives it from level and
   * block_index.  kind: [num_blocks][6]; ids: [num_blocks][6][4], where a
   * FINE face lists its four blocks in transverse order (u + 2v) and a
   * COARSE face lists the coarse block in ids[0]. */
  const int32_t* neighbor_kind;
  const int32_t* neighbor_ids;
  /* Outer boundary condition of the pressure, per face (FFVBC.h types).
   * Neumann values are multiplied by each block's cell size as in
   * src/FFV/BlockScalar3D.h:72-77. */
  int32_t bc_type[6];
  double bc_value[6];
} ffvgpu_grid_desc;

typedef struct ffvgpu_pool ffvgpu_pool;

/* Iteration parameters (src/FFV/FFVConfig.cpp:133-160 keys). */
typedef struct {
  double omega;          /* relaxation factor (Omega) */
  int32_t count_max;     /* MaxIteration */
  double epsilon;        /* ConvergenceCriterion (relative residual) */
  int32_t pre_count;     /* PreCount: Jacobi preconditioner sweeps (CG) */
  int32_t check_every;   /* host polls convergence every this many iterations
                            (0 = default); does not change results */
  double* history;       /* optional host array [count_max]: residual per iteration */
  double restart_drop;   /* BiCGSTAB only, no counterpart in the reference: restart the
                            recurrence (r0 = r, p = r) each time the residual has fallen by
                            this factor; 0 (the default) keeps the reference's recurrence */
} ffvgpu_iter_params;

typedef struct {
  int32_t count;         /* iterations, with the reference's loop-variable meaning */
  double residual;       /* sqrt(|rr|/|bb|) of the last iteration */
  double elapsed_ms;     /* device time of the solve (CUDA events) */
  double sweep_ms;       /* device time of the steady-state sweep passes only */
  int32_t sweep_launches;/* number of launches sweep_ms covers */
  int64_t bytes_moved;   /* algorithmic HBM bytes of the solve */
  int32_t kernel_launches;
  int32_t uniform_blocks;/* RBGS and the mixed form: blocks whose seven coefficients are the
                            same in every cell, which their kernels read once per block (the
                            results are the same); 0 otherwise */
} ffvgpu_result;

/* ---- pool lifetime ------------------------------------------------------ */

/* Creates a pool on the current CUDA device.  Replaces the per-field
 * LocalScalar3D allocation and VCUpdater registration
 * (src/FFV/LocalScalar3D.h:24-84, src/FFV/Solver.cpp:1967-2043). */
ffvgpu_status ffvgpu_pool_create(const ffvgpu_grid_desc* desc, ffvgpu_pool** out);
void ffvgpu_pool_destroy(ffvgpu_pool* pool);
int32_t ffvgpu_pool_num_blocks(const ffvgpu_pool* pool);
/* Runs the pool's work on the caller's CUDA stream (cudaStream_t passed as
 * void*; NULL = the pool's own stream).  All later calls enqueue there. */
ffvgpu_status ffvgpu_pool_set_stream(ffvgpu_pool* pool, void* stream);
/* Time limit, in seconds, of every bounded wait inside the pool's kernels
 * (default 4; 0 to 3600).  A wait that runs out ends the solve with
 * FFVGPU_TIMEOUT (ffvgpu_last_error names the roles that gave up) and leaves
 * the pool usable; copies already in flight are waited for before a kernel
 * exits, whatever the limit.  The reference has no device waits: its
 * counterpart is the MPI runtime's own timeouts. */
ffvgpu_status ffvgpu_pool_set_wait_limit(ffvgpu_pool* pool, double seconds);
/* Test hook for the timeout path (no counterpart in the reference): the next
 * mixed-form solve on the pool waits in its sweep kernel for a copy that is
 * never issued, so that wait runs out after the wait limit and the solve ends
 * with FFVGPU_TIMEOUT.  The hook covers that one solve. */
ffvgpu_status ffvgpu_pool_stall_next_solve(ffvgpu_pool* pool);
/* The same for the pipelined A*x kernel (matvec_form 0): its producer issues
 * no copy, so the consumers' first wait for a slot runs out. */
ffvgpu_status ffvgpu_pool_stall_next_matvec(ffvgpu_pool* pool);
/* Test hook: the persistent kernels (the mixed form's, and the FP64 CG and
 * BiCGSTAB's A*x and Jacobi sweeps) run at most 'ctas' CTAs (0: SMs x
 * resident CTAs, the default), so that each CTA walks more blocks -- with
 * one CTA, more than a chunk of its live-block list.  Results do not depend
 * on it.  Not while a stepped solve is running. */
ffvgpu_status ffvgpu_pool_cap_grids(ffvgpu_pool* pool, int32_t ctas);
/* Neighbour table as derived (kind [6], ids [6][4]); for tests. */
ffvgpu_status ffvgpu_pool_neighbors(const ffvgpu_pool* pool, int32_t block,
                                    int32_t* kind6, int32_t* ids24);
/* Device bytes held by the pool. */
int64_t ffvgpu_pool_device_bytes(const ffvgpu_pool* pool);

/* ---- host <-> device ------------------------------------------------------
 * host: num_blocks * (16+2*vc)^3 values, reference layout.  Upload reads the
 * interior and, for vector fields, the first guide layer.  Download writes
 * the interior and vc guide layers of every face (the values the
 * reference's exchange would hold, src/FFV/Scalar3DUpdater1.cpp); edge and
 * corner guide cells, which no kernel of the path reads, are written as 0. */
ffvgpu_status ffvgpu_pool_upload(ffvgpu_pool* pool, ffvgpu_field field,
                                 const void* host, int32_t vc);
ffvgpu_status ffvgpu_pool_download(ffvgpu_pool* pool, ffvgpu_field field,
                                   void* host, int32_t vc);

/* ---- operations -------------------------------------------------------- */

/* Guide-cell exchange of a vector field plus outer BC with the given types
 * and values: LocalScalar3D<real>::ImposeBoundaryCondition()
 * (src/FFV/LocalScalar3D.h:266-296) with updater 1
 * (src/FFV/Scalar3DUpdater1.cpp:9-661, src/CGMfuncs/sup.f90:1-179) and
 * src/CGMfuncs/bcx.f90.  bc_type/bc_value NULL = the pool's pressure BCs. */
ffvgpu_status ffvgpu_exchange(ffvgpu_pool* pool, ffvgpu_field field,
                              const int32_t* bc_type6, const double* bc_value6);

/* Cut-cell coefficients and RHS: per block bcut_calc_ab_p_
 * (src/FFV/bcut.f90:608-832) as called at src/FFV/Solver.cpp:5471-5481.
 * Reads UX/UY/UZ (with guide cells, exchange them first), C0..C5, CID0..5,
 * PID; writes AP..AT, B and VW..VT. */
ffvgpu_status ffvgpu_assemble_p(ffvgpu_pool* pool, double rhof, double dt);

/* Folds the pool's outer pressure BCs into A and b:
 * LocalScalar3D::ImposeBoundaryCondition(A..., b) (src/FFV/LocalScalar3D.h:298-323,
 * src/FFV/BlockScalar3D.h:183-190, src/CGMfuncs/bca.f90:5-388), as called
 * at src/FFV/Solver.cpp:5574. */
ffvgpu_status ffvgpu_fold_bc(ffvgpu_pool* pool);

/* Red-black SOR / Gauss-Seidel solve of A x = b on FIELD_X:
 * FFVILS::RBGS (src/FFV/FFVILS.h:547-594). */
ffvgpu_status ffvgpu_solve_rbgs(ffvgpu_pool* pool, const ffvgpu_iter_params* prm,
                                ffvgpu_result* res);

/* Jacobi-preconditioned CG on FIELD_X: FFVILS::CG (src/FFV/FFVILS.h:661-791). */
ffvgpu_status ffvgpu_solve_cg(ffvgpu_pool* pool, const ffvgpu_iter_params* prm,
                              ffvgpu_result* res);

/* FFVILS::Fill (src/FFV/FFVILS.h:425-445, blas.f90:5-33): every cell of a
 * real field, guide cells included, set to value. */
ffvgpu_status ffvgpu_fill(ffvgpu_pool* pool, ffvgpu_field field, double value);

/* FFVILS::RBGS_WithFixedAverage (src/FFV/FFVILS.h:596-659), the pressure
 * solver FFV uses for all-Neumann problems: each iteration an RB sweep, the
 * shift x += -sum(x)/ncells (LocalScalar3D::CalcSum / ShiftByA) and the
 * residual of the shifted x.  ncells: FFV passes numTotalCells, every
 * interior cell of every leaf block (Solver.cpp:1486-1490, 5601).  The
 * reference's xave argument is unused there and has no counterpart here. */
ffvgpu_status ffvgpu_solve_rbgs_fixed_average(ffvgpu_pool* pool, const ffvgpu_iter_params* prm,
                                              int64_t ncells, ffvgpu_result* res);

/* Jacobi-preconditioned BiCGSTAB on FIELD_X: FFVILS::BiCGSTAB
 * (src/FFV/FFVILS.h:793-974), the reference's default pressure solver
 * (src/FFV/Solver.cpp:5620-5676). */
ffvgpu_status ffvgpu_solve_bicgstab(ffvgpu_pool* pool, const ffvgpu_iter_params* prm,
                                    ffvgpu_result* res);

/* Single kernels of the path, for parity tests and for callers that drive
 * their own loop.  Each matches one FFVILS helper. */
/* RBGS_Smoother (FFVILS.h:104-162): both colours on every block + exchange. */
ffvgpu_status ffvgpu_rbgs_sweep(ffvgpu_pool* pool, double omega);
/* CalcR2 (FFVILS.h:247-296): sum over interior cells of (b - A x)^2. */
ffvgpu_status ffvgpu_calc_r2(ffvgpu_pool* pool, double* rr);
/* DOT (FFVILS.h:298-328) of two real fields. */
ffvgpu_status ffvgpu_dot(ffvgpu_pool* pool, ffvgpu_field x, ffvgpu_field y, double* xy);

/* Dot product of two device vectors that allocates nothing.  This entry
 * point has no counterpart in the reference.  It is for callers that cannot
 * call cudaMalloc: applications that hand the whole device memory to their
 * own allocator at start-up, and loops that must not stall on the device
 * synchronisation cudaMalloc/cudaFree bring.  x and y are caller-owned
 * device arrays of num_blocks * 4096 doubles in the pool's device layout
 * (per block, cells in the colour-split order of the pool, so the result is
 * bit for bit what ffvgpu_dot returns for the same fields); result is a
 * caller-owned device double; stream is a cudaStream_t (NULL = default).
 * The per-block partial sums live in one fixed array compiled into the
 * library, FFVGPU_NOALLOC_MAX_BLOCKS doubles per GPU, held until the process
 * exits; larger num_blocks is rejected with FFVGPU_BAD_ARG.  The first call
 * on a device looks the array up for that device, so make it before any
 * stream capture; the address is kept for the life of the process, which
 * assumes the device's primary context is never reset (no cudaDeviceReset
 * between calls).  stream must belong to the device current at the call.
 * Every call on a device shares the array: calls that overlap on the GPU
 * race and must be serialised by the caller.  The call is asynchronous on
 * the stream. */
#define FFVGPU_NOALLOC_MAX_BLOCKS 65536
ffvgpu_status ffvgpu_dot_noalloc(const double* x, const double* y, int32_t num_blocks,
                                 double* result, void* stream);

/* Sums (CalcR2, DOT, the norms inside the solves) use one fixed reduction
 * tree, so every result is bit-reproducible run to run. */
int32_t ffvgpu_version(void);
/* Last CUDA error string of this thread, for diagnostics. */
const char* ffvgpu_last_error(void);

/* Host-only neighbour derivation from a grid description (no device
 * needed): kind [num_blocks][6], ids [num_blocks][6][4] with the
 * conventions of ffvgpu_grid_desc.  Fails with BAD_ARG on a grid that is not
 * 2:1 face balanced. */
ffvgpu_status ffvgpu_grid_neighbors(const ffvgpu_grid_desc* desc, int32_t* kind,
                                    int32_t* ids);

/* ---- synthetic sphere grids (host only; no device needed) ----------------
 * Leaf blocks of a 2:1 face-balanced octree refined around a sphere, with
 * analytic cut-cell fractions in place of Cutlib (src/FFV/Solver.cpp:530-663)
 * and a seeded intermediate velocity u* = (1,0,0) + N(0, sigma^2). */
typedef struct {
  double domain_origin[3];
  int32_t root_grid[3];
  double root_length;
  int32_t max_level;
  double center[3];
  double radius;
  double margin;  /* refine while a block lies within radius + margin of center */
} ffvgpu_sphere_params;

typedef struct ffvgpu_sphere_grid ffvgpu_sphere_grid;

ffvgpu_status ffvgpu_sphere_grid_create(const ffvgpu_sphere_params* prm,
                                        ffvgpu_sphere_grid** out);
void ffvgpu_sphere_grid_destroy(ffvgpu_sphere_grid* g);
int32_t ffvgpu_sphere_grid_num_blocks(const ffvgpu_sphere_grid* g);
/* Copies level[num_blocks] and block_index[num_blocks][3]. */
void ffvgpu_sphere_grid_blocks(const ffvgpu_sphere_grid* g, int32_t* level,
                               int32_t* block_index);
/* Fills the per-cell inputs of the pressure assembly in the reference layout
 * (vc guide layers, guide cells set to 0):
 * ux,uy,uz: u*; c[6]: cut distance in (0,1] (1 where uncut, rounded through
 * float as Cutlib's CutPos32 does); cid[6]: 1 where cut; pid: 1 fluid, 0 solid.
 * Any pointer may be NULL to skip that output. */
ffvgpu_status ffvgpu_sphere_grid_fill(const ffvgpu_sphere_grid* g, uint64_t seed,
                                      double sigma, int32_t vc, double* ux,
                                      double* uy, double* uz, double* const* c6,
                                      int32_t* const* cid6, int32_t* pid);

/* ---- the projection either side of the solve ------------------------------
 * bcut_remove_p (src/FFV/bcut.f90:3879-4061; Solver.cpp:5378-5386, P01):
 * u* += dt grad(p)/rho on UX, UY, UZ with the cut-cell gradient rules, 0 in
 * solid cells.  bcut_corr_u (bcut.f90:4063-4297; Solver.cpp:5738-5748):
 * u -= dt grad(p)/rho on UX, UY, UZ and the face velocities VW..VT, LAPP = the
 * 7-point Laplacian of p (0 in solid and cut cells).  Both read p's stored
 * guide layer (what FIELD_X holds after its last exchange) and the cut fields;
 * the caller exchanges u afterwards, as UpdateP/UpdateU do. */
ffvgpu_status ffvgpu_remove_p(ffvgpu_pool* pool, double rhof, double dt);
ffvgpu_status ffvgpu_corr_u(ffvgpu_pool* pool, double rhof, double dt);

/* ---- block sharding across GPUs (one process per GPU) ---------------------
 * The reference spreads its leaf blocks over MPI ranks as contiguous ranges
 * of its ordered leaf list (Solver::InitTree / InitBlocks,
 * src/FFV/Solver.cpp:306-381) and exchanges guide faces between ranks.  A
 * shard plan puts the leaves in Z order (root blocks x fastest, then the
 * Morton order of each leaf's position in its root block at the finest
 * level), gives rank r the r-th of num_ranks contiguous ranges (sizes differ
 * by at most one) and describes r's local grid: its own blocks (local ids
 * 0 .. owned-1, in Z order), then halo blocks -- copies of other ranks'
 * blocks that its blocks' guide cells are computed from -- grouped by owner
 * rank, Z order within a group.  The local description carries an explicit
 * neighbour table (halo blocks have outer faces: they are never solved), so
 * ffvgpu_pool_create on it gives the shard's pool.  Before every pass that
 * reads neighbours, rank r sends peer p the interiors (ffvgpu_pool_field_device
 * layout, 4096 doubles per block) of the local blocks ffvgpu_shard_peer lists
 * under send, and stores what p sends into the blocks listed under recv, in
 * list order; the in-kernel exchange then gives the unsharded grid's guide
 * values.  Sums stay those of the unsharded pool when every rank's per-block
 * partials (ffvgpu_rbgs_pass, ffvgpu_block_dots) are gathered into global
 * block order and added by ffvgpu_canonical_sum. */
typedef struct ffvgpu_shard ffvgpu_shard;
ffvgpu_status ffvgpu_shard_create(const ffvgpu_grid_desc* global, int32_t num_ranks,
                                  int32_t rank, ffvgpu_shard** out);
void ffvgpu_shard_destroy(ffvgpu_shard* shard);
ffvgpu_status ffvgpu_shard_info(const ffvgpu_shard* shard, int32_t* owned, int32_t* halo);
/* global id of every local block, [owned + halo] */
ffvgpu_status ffvgpu_shard_local_blocks(const ffvgpu_shard* shard, int32_t* global_ids);
/* global ids in Z order [num_blocks] and the owner rank of every block [num_blocks] */
ffvgpu_status ffvgpu_shard_zorder(const ffvgpu_shard* shard, int32_t* order, int32_t* owner);
/* the local grid description (valid while the shard lives) */
const ffvgpu_grid_desc* ffvgpu_shard_local_desc(const ffvgpu_shard* shard);
/* exchange lists with one peer: local ids to send, local ids to receive into */
ffvgpu_status ffvgpu_shard_peer(const ffvgpu_shard* shard, int32_t peer, int32_t* n_send,
                                int32_t* send_local, int32_t* n_recv, int32_t* recv_local);
/* One pass of the red-black kernel over the pool's first 'blocks' blocks (a
 * shard's own blocks), the passes of ffvgpu_solve_rbgs: first sweep
 * (residual 0, sweep 1, stored 1: the guide layer stored with x), residual of
 * the current iterate + sweep (1, 1, 0), last residual (1, 0, 0).  A sweep
 * makes its result the current iterate; a residual writes each block's sum
 * of (b - A x)^2 (the pool's per-block tree) into partials[blocks]. */
ffvgpu_status ffvgpu_rbgs_pass(ffvgpu_pool* pool, int32_t blocks, int32_t residual,
                               int32_t sweep, int32_t stored, double omega, double* partials);
/* Per-block sums x.y (the pool's per-block tree) of the first 'blocks' blocks. */
ffvgpu_status ffvgpu_block_dots(ffvgpu_pool* pool, ffvgpu_field x, ffvgpu_field y,
                                int32_t blocks, double* partials);
/* Device address of the current iterate (FIELD_X) or of b (FIELD_B):
 * per block 4096 doubles in the pool's colour-split cell order. */
ffvgpu_status ffvgpu_pool_field_device(ffvgpu_pool* pool, ffvgpu_field field, void** ptr);
/* The cross-block stage of the pool's reduction tree over per-block partials
 * in block order (host only): the same bits as the pool's own sums. */
ffvgpu_status ffvgpu_canonical_sum(const double* partials, int32_t n, double* total);

/* ---- restart files: LocalScalar3D::Dump2 / Load2 -------------------------
 * (src/FFV/LocalScalar3D.cpp:216-354).  The file holds six native int32
 * (cells per block x, y, z = 16, guide width vc, 1, number of blocks) and then
 * every block's (16+2vc)^3 doubles in block order, guide cells included.
 * Dump2 exchanges the field first and writes it; Load2 reads a file of the
 * same shape, or of 8^3 blocks whose cells each fill 2x2x2 cells
 * (sf3d_copy_x2, src/CGMfuncs/bsf3d.f90:5-33), and exchanges the field.
 * Fields X, UX, UY, UZ.  A file that matches neither shape is refused
 * (the reference exits). */
ffvgpu_status ffvgpu_dump2(ffvgpu_pool* pool, ffvgpu_field field, int32_t vc,
                           const char* filename);
ffvgpu_status ffvgpu_load2(ffvgpu_pool* pool, ffvgpu_field field, int32_t vc,
                           const char* filename);
/* The reference's file name, path/prefix label-RRRRR-SSSSSSSSSS.bin
 * (LocalScalar3D.cpp:224-243); returns its length, or -1 when cap is too small. */
int32_t ffvgpu_restart_filename(char* out, int32_t cap, const char* path, const char* prefix,
                                const char* label, int32_t rank, int32_t step);

/* ---- mixed-precision form (no counterpart in the reference) -------------
 * FFVILS::BiCGSTAB's recurrence (src/FFV/FFVILS.h:793-974) in FP64 --
 * residuals, norms, dot products and the pressure update -- with the Jacobi
 * preconditioner (FFVILS.h:469-492) replaced by red-black SOR sweeps on
 * 32-bit data from zero: 'sweeps' colour pairs per application,
 * 'sweeps_per_exchange' of them between guide-cell exchanges (each block
 * sweeps on chip, in FP64 arithmetic, against fixed guide values in
 * between; the coefficients are kept as 32-bit words and the iterate is
 * stored in FP32 between exchanges).  sweeps must be a multiple of
 * sweeps_per_exchange.  Result fields as ffvgpu_solve_bicgstab; the solve
 * stops when sqrt(r.r / b.b) <= epsilon or after count_max iterations.
 * BiCGSTAB's recurrence stalls on the sphere grids (the reference's own FP64
 * BiCGSTAB stops by its breakdown test there) and the FP32 rounding of the
 * preconditioned vectors adds to it; restarts from the current residual each
 * time it has fallen by restart_drop (1e-3), and whenever it exceeds
 * restart_growth (100) times the smallest since the last restart, keep it
 * converging. */
typedef struct {
  double omega;                /* SOR relaxation factor of the sweeps */
  int32_t sweeps;              /* colour-pair sweeps per preconditioner application */
  int32_t sweeps_per_exchange; /* sweeps between guide-cell exchanges */
  int32_t count_max;
  double epsilon;
  int32_t check_every;         /* iterations between host polls (0: 8) */
  double* history;             /* optional host array [count_max]: residual per iteration */
  double restart_drop;         /* restart the recurrence (r0 = r, p = r) each time the
                                  residual has fallen by this factor; 0: never */
  double restart_growth;       /* also restart when the residual exceeds this factor times
                                  the cycle's smallest; 0: never */
  int32_t restart_every;       /* also restart after this many iterations of a cycle; 0: never */
  int32_t flux_correction;     /* 1: the FP64 residual and A*x products use the coarse-fine
                                  flux-conserving operator (ffvgpu_cf_flux_mismatch describes
                                  it); the sweeps keep the interpolating one.  0: the
                                  reference's operator */
  int32_t fp64_data;           /* 1: the same preconditioner on FP64 data -- coefficients and
                                  the iterate between exchanges in FP64, the preconditioned
                                  vectors in FP64 -- so that a comparison with the default
                                  (32-bit data) isolates what the 32-bit data buy */
  int32_t threads_per_block;   /* CTA size of the update kernel, and of the A*x kernel in
                                  matvec_form 1: 128, 256 or 512 (0: 256); results do not
                                  depend on it */
  int32_t stage_depth;         /* sweep kernel: how many blocks ahead a block's data are
                                  brought into L2 (1..3; 0: 1); results do not depend on it */
  int32_t sweep_threads;       /* CTA size of the sweep kernel: 512 (each thread a 4-cell
                                  column of one row) or 256 (of two rows); 0: 256; results
                                  do not depend on it */
  int32_t matvec_form;         /* A*x kernel: 0 pipelined (one CTA of 800 threads per SM;
                                  the next blocks' tiles and coefficients are staged while
                                  the current one is computed), 1 a block per CTA of
                                  threads_per_block threads; results do not depend on it */
} ffvgpu_mixed_params;

/* Solves every admitted instance of the pool (a pool made from one grid is
 * one instance); res receives instance 0's result when it is not NULL. */
ffvgpu_status ffvgpu_solve_mixed(ffvgpu_pool* pool, const ffvgpu_mixed_params* prm,
                                 ffvgpu_result* res);

/* Coarse-fine flux conservation (no counterpart in the reference, whose 2:1
 * exchange interpolates, src/CGMfuncs/sup.f90:54-179, and so does not
 * conserve flux across coarse-fine faces).  For every coarse cell P on a
 * face f whose neighbours are four finer blocks: the flux through f as the
 * four fine cells phi touching it see it, in P's equation,
 *   F = 0.125 * sum_{dv, du} A_fo(phi) * (x_phi - g_phi)
 * (fo the opposite face, g_phi phi's guide value across fo, the
 * prolongation; du inner, dv outer, summed from 0), and
 *   delta = F - A_f(P) * (g - x_P),
 * the difference from the coarse side's own term (g: P's guide value across
 * f, the restriction).  The flux-conserving operator of
 * ffvgpu_mixed_params.flux_correction adds delta to (A x)_P per such face in
 * face order.  This call evaluates both on FIELD_X (interior and stored
 * guide layer, as a solve leaves it) and returns mismatch = sum V_P |delta|
 * and flux = sum V_P |F| (V_P = dx^3), in FP64, over the n_cells such cells
 * in (block, face, position u + 16 v) order; per_cell (optional, capacity
 * pairs) receives (delta, F) per cell in that order. */
ffvgpu_status ffvgpu_cf_flux_mismatch(ffvgpu_pool* pool, double* mismatch, double* flux,
                                      int32_t* n_cells, double* per_cell, int32_t capacity);

/* ---- the pressure part of a fractional time step ---------------------------
 * Solver::UpdateP (src/FFV/Solver.cpp:5294-5688) and Solver::UpdateU
 * (Solver.cpp:5690-5771) on the device, in the reference's order:
 * update_p: P01 bcut_remove_p (the previous pressure), P02 exchange of UX,
 * UY, UZ with u_bc, P03 bcut_calc_ab_p, P05 BC folding, P06 the solve (x
 * starts from the previous pressure), P07 exchange of p;
 * update_u: U01 bcut_corr_u, U02 exchange of UX, UY, UZ, U03 exchange of p.
 * P04 (the reference-pressure pin, only active for all-Neumann problems,
 * Solver.cpp:5495-5566) and gravity/forcing (bcut_add_g, bcut_add_f) are not
 * part of this path; LapP's exchange in U03 is left out (no kernel of the
 * path reads its guide cells).  res receives the solve's result. */
enum { FFVGPU_SOLVER_RBGS = 0, FFVGPU_SOLVER_BICGSTAB = 1, FFVGPU_SOLVER_MIXED = 2 };
typedef struct {
  double rhof;
  double dt;
  int32_t u_bc_type[3][6];   /* per velocity component and face */
  double u_bc_value[3][6];
  int32_t solver;            /* FFVGPU_SOLVER_* */
  ffvgpu_iter_params iter;   /* RBGS, BiCGSTAB */
} ffvgpu_step_params;

/* mixed: the mixed-form settings when solver is FFVGPU_SOLVER_MIXED (else NULL). */
ffvgpu_status ffvgpu_update_p(ffvgpu_pool* pool, const ffvgpu_step_params* prm,
                              const ffvgpu_mixed_params* mixed, ffvgpu_result* res);
ffvgpu_status ffvgpu_update_u(ffvgpu_pool* pool, const ffvgpu_step_params* prm);

/* ---- batches: independent problems sharing one pool (no counterpart in the
 * reference) ---------------------------------------------------------------
 * A batch pool reserves capacity_blocks leaf blocks on the device and admits
 * instances -- each a complete pressure problem on its own grid -- into
 * free contiguous block ranges, up to max_instances at a time.  The
 * instances share the pressure BCs of the batch.  The kernels of a batched
 * solve run over all instances at once; every sum is taken per instance in
 * the same order as for the instance alone, so each instance's results are
 * bit-identical alone and in any mix.  The pool-wide entry points above
 * (uploads, assembly, the FFVILS-form solves) refuse batch pools. */
typedef struct {
  int32_t capacity_blocks;
  int32_t max_instances;
  int32_t bc_type[6];  /* pressure BCs */
  double bc_value[6];
} ffvgpu_batch_desc;

ffvgpu_status ffvgpu_batch_create(const ffvgpu_batch_desc* desc, ffvgpu_pool** out);

/* Admits an instance on its own grid (desc's BC fields are ignored: the
 * batch's apply).  A, b and x are then uploaded with ffvgpu_instance_upload.
 * FFVGPU_OOM when no free block range or instance slot is large enough (the
 * caller may retry after a release). */
ffvgpu_status ffvgpu_instance_admit(ffvgpu_pool* pool, const ffvgpu_grid_desc* desc,
                                   int32_t* instance);

/* A sphere-flow pressure problem generated and assembled on the device: the
 * grid of ffvgpu_sphere_grid_create, the inputs of ffvgpu_sphere_grid_fill
 * (same seed, same values), then UpdateP's P02-P05 (velocity exchange with
 * u_bc, bcut_calc_ab_p, BC folding) and x = 0. */
typedef struct {
  ffvgpu_sphere_params grid;
  uint64_t seed;
  double sigma;
  double rhof;
  double dt;
  int32_t u_bc_type[3][6];
  double u_bc_value[3][6];
} ffvgpu_sphere_problem;

ffvgpu_status ffvgpu_instance_admit_sphere(ffvgpu_pool* pool, const ffvgpu_sphere_problem* prob,
                                           int32_t* instance);
/* The same generation and assembly for a pool made from the problem's own
 * grid (ffvgpu_pool_create on the blocks of ffvgpu_sphere_grid_create). */
ffvgpu_status ffvgpu_assemble_sphere(ffvgpu_pool* pool, const ffvgpu_sphere_problem* prob);
/* Only the generation: u* (UX, UY, UZ interiors), the cut fields and the
 * phase flags of the problem, and the u BCs; no exchange, no assembly, the
 * pressure untouched.  The time-step loop below regenerates u* with it. */
ffvgpu_status ffvgpu_generate_sphere(ffvgpu_pool* pool, const ffvgpu_sphere_problem* prob);
/* Per-instance transfers in the reference layout of ffvgpu_pool_upload /
 * ffvgpu_pool_download (host buffers hold the instance's blocks only). */
ffvgpu_status ffvgpu_instance_upload(ffvgpu_pool* pool, int32_t instance, ffvgpu_field field,
                                     const void* host, int32_t vc);
ffvgpu_status ffvgpu_instance_download(ffvgpu_pool* pool, int32_t instance, ffvgpu_field field,
                                       void* host, int32_t vc);
/* FFVILS::Fill on one instance's blocks (interior and stored guide layer). */
ffvgpu_status ffvgpu_instance_fill(ffvgpu_pool* pool, int32_t instance, ffvgpu_field field,
                                   double value);
/* Frees the instance's blocks and slot; refused while its solve runs. */
ffvgpu_status ffvgpu_instance_release(ffvgpu_pool* pool, int32_t instance);
int32_t ffvgpu_instance_blocks(const ffvgpu_pool* pool, int32_t instance);
/* Free blocks in total and in the largest free contiguous range. */
ffvgpu_status ffvgpu_pool_free_blocks(const ffvgpu_pool* pool, int32_t* free_blocks,
                                      int32_t* largest_range);

/* Stepping form of the mixed solve, for request loops: begin starts an
 * instance's solve (its count_max, epsilon and history come from prm; the
 * preconditioner settings must equal those of instances already running);
 * advance enqueues 'iterations' iterations of every running instance (one
 * captured CUDA graph); poll returns the instances whose solves have ended
 * since the last poll (their x guide layer is exchanged, as FFVILS.h:973
 * does) and result reads one instance's outcome. */
ffvgpu_status ffvgpu_mixed_begin(ffvgpu_pool* pool, int32_t instance,
                                 const ffvgpu_mixed_params* prm);
ffvgpu_status ffvgpu_mixed_advance(ffvgpu_pool* pool, int32_t iterations);
ffvgpu_status ffvgpu_mixed_poll(ffvgpu_pool* pool, int32_t* finished, int32_t capacity,
                                int32_t* n_finished);
/* Stops one running instance before its next replay: its solve ends with
 * FFVGPU_CANCELLED, its result holds the iterations completed and the last
 * residual, its x is the iterate of the last completed iteration, and it can
 * be released or begun again. */
ffvgpu_status ffvgpu_mixed_cancel(ffvgpu_pool* pool, int32_t instance);
/* history: optional host array receiving min(count, count_max) residuals. */
ffvgpu_status ffvgpu_instance_result(const ffvgpu_pool* pool, int32_t instance,
                                     ffvgpu_result* res, double* history);

/* The autotuner (no counterpart in the reference): times the mixed solve of
 * the given admitted instances from x = 0 for each candidate setting --
 * omega, sweeps, sweeps_per_exchange, iterations per captured-graph replay,
 * threads per block of the A*x and update kernels and the sweep kernel's
 * staging depth -- with base's count_max, epsilon and restart settings, fills in
 * each record's device time (ms), its largest iteration count and whether
 * every instance reached epsilon, and sets *best to the fastest candidate
 * that converged them all (-1 if none did).  The instances end with x = 0. */
typedef struct {
  double omega;
  int32_t sweeps;
  int32_t sweeps_per_exchange;
  int32_t iterations_per_replay;
  double ms;          /* out */
  int32_t max_count;  /* out */
  int32_t converged;  /* out: 1 when every instance reached epsilon */
  int32_t threads_per_block;  /* as ffvgpu_mixed_params (0: 256) */
  int32_t stage_depth;        /* as ffvgpu_mixed_params (0: 1) */
  int32_t sweep_threads;      /* as ffvgpu_mixed_params (0: 256) */
  int32_t matvec_form;        /* as ffvgpu_mixed_params */
} ffvgpu_tune_record;

ffvgpu_status ffvgpu_mixed_autotune(ffvgpu_pool* pool, const int32_t* instances,
                                    int32_t n_instances, const ffvgpu_mixed_params* base,
                                    ffvgpu_tune_record* records, int32_t n_records,
                                    int32_t* best);

/* ---- serving (no counterpart in the reference) ---------------------------
 * A request loop with continuous batching on a batch pool: requests (sorted
 * by arrival time, seconds from the start of the call) are admitted in
 * arrival order as block ranges and instance slots free up -- one that does
 * not fit waits while later, smaller ones may pass it -- and join the
 * running solves at the next graph replay; every replay advances all running
 * solves by iterations_per_step iterations; a solve that ends has its
 * pressure copied to the host and its blocks released; a request whose
 * cancel time passes first is dropped or stopped instead.  out[i] receives
 * request i's admission and completion (or cancellation) times (same clock),
 * iterations, residual, status and block count.  On an error the pool may still hold
 * admitted instances: destroy it. */
typedef struct {
  double arrival_s;
  double cancel_s;  /* withdrawn at this time (same clock) if not finished by then:
                       dropped while waiting, stopped while solving (its blocks are
                       released); status FFVGPU_CANCELLED.  0: never */
  ffvgpu_sphere_problem problem;
} ffvgpu_request;

typedef struct {
  double admit_s;
  double finish_s;
  int32_t count;
  double residual;
  int32_t status;
  int32_t blocks;
} ffvgpu_request_result;

ffvgpu_status ffvgpu_serve(ffvgpu_pool* batch, const ffvgpu_mixed_params* prm, int32_t n,
                           const ffvgpu_request* requests, int32_t iterations_per_step,
                           ffvgpu_request_result* out);

#ifdef __cplusplus
}
#endif
#endif /* FFVGPU_H */
