// ffvgpu_layout.h -- plain structures and index maps shared by the host
// pool code and the device kernels of the pressure-Poisson path.
//
// Layout in HBM.  Every per-cell field of a 16^3 leaf block is stored as a
// dense 4096-double chunk with no guide cells, blocks back to back.  Cells
// are ordered by colour: storage index s = c*2048 + q with colour
// c = (i+j+k) & 1 (0-based interior indices; c equals the reference's
// red-black colour, src/CGMfuncs/bils.f90:90) and q = (k*16 + j)*8 + i/2.
// A colour sweep therefore reads and writes each coefficient array as one
// contiguous 16 KB run per block.  Guide cells are not stored for the
// solver's vectors: every stencil kernel computes them from the neighbours'
// interiors while it stages the block (the in-kernel block-to-block
// exchange), which is what the reference's exchange would have written
// (src/FFV/Scalar3DUpdater1.cpp:9-661, src/CGMfuncs/sup.f90:1-179,
// src/CGMfuncs/bcx.f90).  The caller-visible vectors (pressure and the three
// velocity components) also keep a stored copy of their first guide layer,
// [block][face][v][u], holding what the reference's field would hold in its
// guide cells: the uploaded values, or the last exchange.
#pragma once
#include <cstdint>

#ifdef __CUDACC__
#define FFVGPU_HD __host__ __device__
#else
#define FFVGPU_HD
#endif

namespace ffvgpu {

constexpr int NB_CELLS = 16;      // cells per block edge
constexpr int BLOCK_CELLS = 4096; // 16^3
constexpr int HALF_CELLS = 2048;  // cells of one colour
constexpr int FACE_CELLS = 256;   // 16^2
constexpr int THREADS = 256;      // threads per CTA of every block kernel
// Coefficient stream of the red-black sweep: per block 16 chunks (colour c,
// plane pair m -> chunk c*8 + m), each holding Ap, Aw, Ae, As, An, Ab, At, b
// of its 256 cells back to back (16 KB), so one bulk copy moves a chunk.
constexpr int STREAM_CHUNK = 8 * 256;
constexpr int STREAM_BLOCK = 16 * STREAM_CHUNK;
// Default limit of every bounded device wait (a pool setting,
// ffvgpu_pool_set_wait_limit): a wait that has not completed after it gives
// up and the solve reports a timeout.
constexpr uint64_t DEFAULT_WAIT_NS = 4000000000ull;

enum { X_M = 0, X_P, Y_M, Y_P, Z_M, Z_P };
enum { BC_DIRICHLET = 0, BC_NEUMANN = 1 };
enum { NB_OUTER = 0, NB_SAME = 1, NB_COARSE = 2, NB_FINE = 3 };

// One face of one block.  Transverse axes (u, v) of a face are the two
// other axes in increasing order: X faces (y, z), Y faces (x, z), Z faces
// (x, y).  COARSE: id[0] is the coarse block and (so_u, so_v) the half of
// its face this block covers.  FINE: id[qu + 2*qv] is the fine block
// covering half qu along u and qv along v.
struct FaceNbr {
  int32_t kind;
  int32_t id[4];
  int32_t so_u, so_v;
  int32_t pad;
};

// Outer boundary conditions of one field: type and value per face.  Neumann
// values are scaled by the block's cell size at use
// (src/FFV/BlockScalar3D.h:72-77).
struct BCSet {
  int32_t type[6];
  double value[6];
};

// Device-side solver state: scalars of the Krylov recurrences, convergence
// flag and the deterministic last-block reduction ticket.
struct SolveState {
  double bb, rr, residual;
  double rr0, rr1, alpha, beta, qp;
  double gamma, ts;  // BiCGSTAB: gamma = t.s / t.t, and t.s
  double eps;
  int32_t count;     // reference loop-variable value at exit
  int32_t done;      // 1 once the solve has stopped; later kernels return at entry
  int32_t status;    // 0 ok, 2 NaN/Inf
  int32_t count_max;
  uint32_t ticket;   // last-block-done counter of the current reduction
  int32_t timeout_where;  // roles whose bounded wait gave up (1 producer, 2 gatherer, 4 consumer)
  double* hist;      // device residual history [count_max] or null
  int32_t iter;      // mixed form: number of the iteration under way (1-based)
  int32_t cycle;     // mixed form: iteration within the current restart cycle (1: p = r)
  double drop;       // mixed form: restart when the residual has dropped by this factor
  double next_restart;  // mixed form: residual at which the next restart happens (< 0: none)
  double best;       // mixed form: smallest residual of the current cycle
  double growth;     // mixed form: restart when the residual exceeds growth * best (0: never)
  double scale;      // RBGS_WithFixedAverage: the cell count the sum is divided by
  int32_t max_cycle; // mixed form: restart after this many iterations of a cycle (0: never)
  int32_t ublocks;   // mixed form: blocks whose seven coefficients are the same in every cell
};

// Instances: independent problems that share one pool's blocks (a batch).
// Each owns the contiguous block range [first, first + count) and its own
// solver state; blocks of no instance carry -1.  A pool made from one grid
// is one instance covering every block.
struct InstTable {
  const int32_t* blk_inst;  // [capacity]
  const int32_t* first;     // [instances]
  const int32_t* count;     // [instances]
  SolveState* st;           // [instances]
};

// Sums over a block use one fixed tree of 512 virtual threads: virtual
// thread t sums, serially from 0.0, the cells c*2048 + t + 512*m (m = 0..3)
// of each colour c, and adds the two colour sums; the 32 virtual threads of
// each of the 16 virtual warps are combined by an xor butterfly (16, 8, 4,
// 2, 1); the 16 warp sums are added in order from 0.0.  Across blocks, 256
// threads sum the per-block partials t, t+256, ... serially, then the same
// butterfly and an in-order sum of the 8 warp sums.
// Finalisers run by the last CTA of a reduction.
enum Fin : int {
  FIN_STORE = 0,  // st->rr = total (plain dot product)
  FIN_BB,         // st->bb = total
  FIN_RBGS,       // residual of RBGS iteration 'iter' (FFVILS.h:547-594)
  FIN_CG_RR1,     // rr1 = r.z; early exit if |rr1| < FLT_MIN (FFVILS.h:712-724)
  FIN_CG_QP,      // qp = q.p; alpha = rr1/qp (FFVILS.h:750-758)
  FIN_CG_RR,      // residual of CG iteration 'iter'; rr0 = rr1 (FFVILS.h:774-788)
  FIN_BI_RR1,     // BiCGSTAB rr1 = r.r0; early exit; beta = rr1/rr0*alpha/gamma (FFVILS.h:845-859)
  FIN_BI_QR0,     // BiCGSTAB alpha = rr1 / (q_.r0) (FFVILS.h:890-896)
  FIN_BI_TS,      // BiCGSTAB t_.s (FFVILS.h:923-929)
  FIN_BI_TT,      // BiCGSTAB gamma = t_s / (t_.t_) (FFVILS.h:930-936)
  FIN_BI_RR,      // BiCGSTAB residual of iteration 'iter' (FFVILS.h:952-960), optional restart
  FIN_FA_SHIFT,   // RBGS_WithFixedAverage: alpha = -sum(x) / scale (FFVILS.h:636-639)
  // mixed form, per instance (two sums where noted)
  FIN_MX_INIT,    // b.b and r.r0: early exits of FFVILS.h:822-826 and 847-851
  FIN_MX_ALPHA,   // alpha = rr1 / (q.r0)
  FIN_MX_GAMMA,   // t.s and t.t: gamma = t.s / t.t
  FIN_MX_UPDATE   // r.r and r.r0: residual, convergence, next rr1 and beta
};

FFVGPU_HD inline int sidx(int i, int j, int k) {
  return (((i + j + k) & 1) << 11) | (((k << 4) | j) << 3) | (i >> 1);
}
FFVGPU_HD inline void cell_of(int s, int& i, int& j, int& k) {
  const int c = s >> 11, q = s & 2047;
  k = q >> 7;
  j = (q >> 3) & 15;
  i = 2 * (q & 7) + ((j + k + c) & 1);
}

}  // namespace ffvgpu
