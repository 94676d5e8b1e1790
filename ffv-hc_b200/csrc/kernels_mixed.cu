// kernels_mixed.cu -- the mixed-precision form of the pressure solve, with
// the per-instance bookkeeping that lets one launch serve a batch of
// independent problems (sm_100a).
//
// The outer iteration is FFVILS::BiCGSTAB's recurrence (src/FFV/FFVILS.h:
// 793-974) in FP64: residuals, norms, dot products and the pressure update
// keep the reference's per-cell expressions and are compiled with
// --fmad=false.  Its preconditioner -- FFVILS's Jacobi_PreConditioner
// (FFVILS.h:469-492) in the reference -- is replaced by red-black SOR sweeps
// on 32-bit data that solve A e = v approximately from e = 0: 'sweeps'
// colour pairs per application, grouped 'per_exchange' at a time between
// guide-cell exchanges (one pass of the sweep kernel per group).  Inside a
// pass a block sweeps against fixed guide values, so the whole pass runs on
// chip: one CTA per block keeps the block's coefficients in registers and
// its iterate in shared memory, and HBM sees one read of the coefficients
// and the right-hand side and one FP32 write of the iterate per pass.
//
// Data in HBM: the coefficients aw..at and dinv = 1 / Ap as 32-bit words
// (each FP64 value rounded to 20 fraction bits, kept as the high word of an
// FP64 number, so widening it is a register move), the iterate between
// passes and the preconditioned vectors in FP32, the right-hand side in
// FP64.  Arithmetic: FP64 throughout a pass, on an FP64 iterate (the tile);
// the iterate is rounded to FP32 once, at the end of the pass.  Sweep of
// one cell (colour order and neighbour terms as rbgs_smoother,
// src/CGMfuncs/bils.f90:57-108):
//   rc = v; rc = fma(-aw, eW, rc); ... fma(-ab, eB, rc); fma(-at, eT, rc)
//   xt = rc * dinv;  e = fma(-omega, e - xt, e)   (e - omega (e - xt))
// Forming rc in FP32 would cancel: once a block has nearly converged locally
// rc is far smaller than its terms, and its FP32 rounding error makes the
// preconditioner visibly nonlinear, which the BiCGSTAB recurrence does not
// survive; here the only nonlinearity left is the rounding of each pass's
// result.
// Guide cells of e: zero in the first pass; later, the exchange rules
// (same-level copy, 2:1 interpolation and restriction, src/CGMfuncs/sup.f90)
// evaluated in FP64 on the previous pass's FP32 values, with homogeneous
// Dirichlet values on outer faces.
//
// Every sum is the canonical tree of the layout header taken over one
// instance's blocks, so an instance gets the same bits alone or in a batch.
#include <algorithm>
#include <cfloat>
#include <cuda_runtime.h>

#include "ffvgpu_async.cuh"
#include "ffvgpu_internal.cuh"
#include "ffvgpu_mixed.h"

namespace ffvgpu {

namespace {

constexpr int MT = 256;  // FP64 kernels: 16 cells per thread

// Shared-memory tile of the sweep kernel: per colour a padded
// [k + 1][j + 1][ii] array of FP64 iterate values, k, j in -1..16 and
// ii = (i + 2) >> 1 for i in -1..16, with row pitch SP and plane pitch SQ;
// the first guide layer sits in the padding, in the half of its own colour
// (colour = (i + j + k) & 1).  With SQ = 2 mod 4 the two 8-cell groups of a
// half-warp's 64-bit accesses (k groups 4 planes apart: 4 SQ = 8 mod 16
// doubles) fall into disjoint banks.
constexpr int SP = 10, SQ = 190, SH = 18 * SQ;
constexpr int TILE = 2 * SH;
constexpr int COEF_WORDS = 7 * BLOCK_CELLS;  // coefficient words of one block
constexpr int GUIDES = 6 * FACE_CELLS;  // guide values of one block (FP64)
constexpr int SWEEP_SMEM = COEF_WORDS * 4 + TILE * 8 + BLOCK_CELLS * 8 + GUIDES * 8 + 16;

// Sweep-kernel geometry for PTS threads per CTA (512 or 256).  Thread t owns
// the cells (i, j, k) with i in {2 ih, 2 ih + 1}, j = JJ jp + jj (jj < JJ
// rows), k = 4 kg + h (h < 4), both colours: ih = t & 7, kg = (t >> 3) & 3,
// jp = t >> 5.  Its cell m < CPT is (colour c, row jj, plane h) with
// m = (c JJ + jj) 4 + h.
template <int PTS>
struct SweepGeom {
  static constexpr int JJ = 512 / PTS;  // rows per thread
  static constexpr int CPT = 8 * JJ;    // cells per thread
};
// Word of coefficient a of sweep thread t's cell m within a block.
template <int PTS>
__device__ __forceinline__ int coef_word(int a, int m, int t) {
  return ((a * (SweepGeom<PTS>::CPT / 4) + (m >> 2)) * PTS + t) * 4 + (m & 3);
}
__device__ __forceinline__ int tile_at(int i, int j, int k) {
  return (k + 1) * SQ + (j + 1) * SP + ((i + 2) >> 1);
}
// Storage slot of sweep thread t's cell m.
template <int PTS>
__host__ __device__ __forceinline__ int sweep_cell(int t, int m) {
  constexpr int JJ = SweepGeom<PTS>::JJ;
  const int ih = t & 7, kg = (t >> 3) & 3, jp = t >> 5;
  const int h = m & 3, jj = (m >> 2) % JJ, c = (m >> 2) / JJ;
  return c * HALF_CELLS + ((4 * kg + h) * 16 + JJ * jp + jj) * 8 + ih;
}

__device__ __forceinline__ int active_instance(const MixCtx& C, int blk) {
  const int i = C.inst.blk_inst[blk];
  if (i < 0) return -1;
  if (*((volatile const int32_t*)&C.inst.st[i].done)) return -1;
  return i;
}

// Per-instance finalisers, run by the CTA that finishes an instance's last
// block.
__device__ void mx_finalize(SolveState* S, const double* t, int fin) {
  switch (fin) {
    case FIN_MX_INIT:
      S->bb = t[0];
      if (fabs(t[0]) < (double)FLT_MIN) {  // FFVILS.h:822-826
        S->residual = 0.0;
        S->count = 0;
        S->done = 1;
        break;
      }
      S->rr1 = t[1];
      if (fabs(t[1]) < (double)FLT_MIN) {  // FFVILS.h:847-851 at count = 1
        S->residual = t[1];
        S->count = 0;
        S->done = 1;
        break;
      }
      S->rr0 = 1.0;
      S->alpha = 0.0;
      S->gamma = 1.0;
      S->iter = 1;
      S->cycle = 1;
      S->next_restart = (S->drop > 0.0) ? resid_of(t[1], t[0]) * S->drop : -1.0;
      S->best = resid_of(t[1], t[0]);
      break;
    case FIN_MX_ALPHA:
      S->qp = t[0];
      S->alpha = S->rr1 / t[0];
      break;
    case FIN_MX_GAMMA:
      S->ts = t[0];
      S->gamma = t[0] / t[1];
      break;
    case FIN_MX_UPDATE: {
      const int n = S->iter;
      const double res = resid_of(t[0], S->bb);  // IsConverged, FFVILS.h:24-47
      S->rr = t[0];
      S->residual = res;
      if (S->hist) S->hist[n - 1] = res;
      S->count = n;
      if (res <= S->eps) {
        S->done = 1;
      } else if (isnan(res) || isinf(res)) {
        S->done = 1;
        S->status = 2;
      } else if (n >= S->count_max) {
        S->done = 1;
        S->count = S->count_max + 1;
      } else {
        S->rr0 = S->rr1;  // FFVILS.h:960
        S->cycle += 1;
        double rr1 = t[1];  // next iteration's DOT(r, r0)
        const bool dropped = S->next_restart > 0.0 && res <= S->next_restart;
        const bool grew = S->growth > 0.0 && res > S->growth * S->best;
        const bool aged = S->max_cycle > 0 && S->cycle > S->max_cycle;
        if (res < S->best) S->best = res;
        if (dropped || grew || aged) {
          // restart from the current r: r0 = r (written by the next
          // iteration's first sweep pass), so DOT(r, r0) = r.r
          if (S->drop > 0.0) S->next_restart = res * S->drop;
          S->best = res;
          S->rr0 = 1.0;
          S->alpha = 0.0;
          S->gamma = 1.0;
          S->cycle = 1;
          rr1 = t[0];
        }
        S->rr1 = rr1;
        if (fabs(rr1) < (double)FLT_MIN) {
          S->residual = rr1;
          S->count = 0;
          S->done = 1;
        } else {
          S->beta = rr1 / S->rr0 * S->alpha / S->gamma;
          S->iter = n + 1;
        }
      }
      break;
    }
  }
}

// Canonical block sums of NV values and the last CTA's cross-block sums over
// the instance's blocks in block order, for CTAs of NT threads (128, 256 or
// 512).  Thread tid carries the sums of virtual threads tid + NT k of the
// block's 512-thread tree (acc[v][colour][k], k < 512 / NT), so the tree --
// and every result -- is the same for every NT; likewise the 256 lanes of
// the cross-block stage are threads tid + NT k below 256.
template <int NV, int NT>
__device__ void mx_reduce(double (&acc)[NV][2][512 / NT], const MixCtx& C, int blk, int inst,
                          int fin) {
  constexpr int VPT = 512 / NT, NW = NT / 32;
  constexpr int LPT = NT >= 256 ? 1 : 256 / NT;  // cross-block lanes per thread
  __shared__ double ws[NV][16];
  __shared__ int amlast;
  const int tid = threadIdx.x;
#pragma unroll
  for (int v = 0; v < NV; ++v)
#pragma unroll
    for (int k = 0; k < VPT; ++k) {
      double x = acc[v][0][k] + acc[v][1][k];
#pragma unroll
      for (int off = 16; off >= 1; off >>= 1) x += __shfl_xor_sync(0xffffffffu, x, off);
      if ((tid & 31) == 0) ws[v][(tid >> 5) + NW * k] = x;
    }
  __syncthreads();
  SolveState* S = C.inst.st + inst;
  const int first = C.inst.first[inst], cnt = C.inst.count[inst];
  if (tid == 0) {
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      double s = 0.0;
#pragma unroll
      for (int w = 0; w < 16; ++w) s += ws[v][w];
      __stcg(C.partials + (size_t)v * C.capacity + blk, s);
    }
    __threadfence();
    const unsigned t = atomicAdd(&S->ticket, 1u);
    amlast = (t == (unsigned)cnt - 1u);
  }
  __syncthreads();
  if (!amlast) return;
  __threadfence();
  double tot[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    double lv[LPT];
#pragma unroll
    for (int k = 0; k < LPT; ++k) {
      const int lane = tid + NT * k;
      double s = 0.0;
      if (lane < 256)
        for (int b = lane; b < cnt; b += 256)
          s += __ldcg(C.partials + (size_t)v * C.capacity + first + b);
#pragma unroll
      for (int off = 16; off >= 1; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
      lv[k] = s;
    }
    __syncthreads();
    if ((tid & 31) == 0)
#pragma unroll
      for (int k = 0; k < LPT; ++k)
        if (tid + NT * k < 256) ws[0][(tid + NT * k) >> 5] = lv[k];
    __syncthreads();
    double total = 0.0;
#pragma unroll
    for (int w = 0; w < 8; ++w) total += ws[0][w];
    tot[v] = total;
  }
  if (tid == 0) {
    mx_finalize(S, tot, fin);
    S->ticket = 0;
    __threadfence();
  }
}

// Stages block blk of an FP32 (or FP64) vector as FP64: the colour-split interior in
// O[4096] and the first guide layer in G[6][256], guides by the exchange
// rules in FP64 (outer faces by the field's BCs).
// nb: the block's six face records, already in shared memory (so each
// guide needs one round of global loads, not a dependent second).
template <int NT, typename ET>
__device__ __forceinline__ void stage_f32_as_f64(double* __restrict__ O, double* __restrict__ G,
                                                 const ET* __restrict__ x, int blk,
                                                 const FaceNbr* nb, double dx,
                                                 const MixCtx& C) {
  const int tid = threadIdx.x;
  const ET* xb = x + (size_t)blk * BLOCK_CELLS;
#pragma unroll
  for (int m = 0; m < BLOCK_CELLS / NT; ++m) O[tid + NT * m] = (double)__ldg(xb + tid + NT * m);
  // the guide pairs (face, p, p + 128), 768 of them, NT at a time: all the
  // pairs' loads in flight together
  constexpr int NP = (6 * 128 + NT - 1) / NT;
#pragma unroll
  for (int it = 0; it < NP; ++it) {
    const int w = tid + NT * it;
    if (NP * NT > 6 * 128 && w >= 6 * 128) break;
    const int f = w >> 7, p0 = w & 127, p1 = p0 + 128;
    const FaceNbr nf = nb[f];
    double v0, v1;
    guide_pair(x, blk, f, p0, p1, nf, C.bc, dx, v0, v1);
    G[f * FACE_CELLS + p0] = v0;
    G[f * FACE_CELLS + p1] = v1;
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// 32-bit coefficients of the sweeps.  Each is the FP64 value rounded to 20
// fraction bits (to nearest, ties away from zero) and stored as the high
// word of that FP64 number, so widening it back is a register move:
// aw, ae, as, an, ab, at and dinv = 1 / Ap (FP64 division, then rounded).
// Per block the words are laid out in the sweep kernel's thread order,
// [a][m / 4][t][m % 4] (coefficient a, the thread's cell m, thread t): 112 KB
// that one bulk copy moves into shared memory, where each thread reads its
// words as 14 16-byte vectors.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t hi_round(double x) {
  return (uint32_t)(((unsigned long long)__double_as_longlong(x) + 0x80000000ull) >> 32);
}
__device__ __forceinline__ double widen(uint32_t w) { return __hiloint2double((int)w, 0); }
// The same inside the sweep loop, kept there: hoisting the 56 widened
// coefficients out of the loop would need 112 registers.
__device__ __forceinline__ double widen_here(uint32_t w) {
  uint32_t v;
  asm volatile("mov.b32 %0, %1;" : "=r"(v) : "r"(w));
  return __hiloint2double((int)v, 0);
}

// D64 (the FP64-data variant): coef64 [blk][a][m][t] holds the FP64 values
// themselves (dinv = 1 / Ap in FP64), read at use by the sweep kernel.
template <bool D64, int PTS>
__global__ void __launch_bounds__(MT)
mx_pack_kernel(int first, const double* __restrict__ A, uint32_t* __restrict__ coef,
               double* __restrict__ coef64, double* __restrict__ ucoef, SolveState* st) {
  constexpr int CPT = SweepGeom<PTS>::CPT;
  const int blk = first + blockIdx.x;
  const double* Ab = A + (size_t)blk * 7 * BLOCK_CELLS;
  uint32_t* cb = D64 ? nullptr : coef + (size_t)blk * COEF_WORDS;
  double* cd = D64 ? coef64 + (size_t)blk * COEF_WORDS : nullptr;
  for (int w = threadIdx.x; w < BLOCK_CELLS; w += MT) {
    const int m = w / PTS, t = w % PTS;
    const int s = sweep_cell<PTS>(t, m);
    if (D64) {
#pragma unroll
      for (int a = 0; a < 6; ++a) cd[(a * CPT + m) * PTS + t] = Ab[(1 + a) * BLOCK_CELLS + s];
      cd[(6 * CPT + m) * PTS + t] = 1.0 / Ab[s];
    } else {
#pragma unroll
      for (int a = 0; a < 6; ++a)
        cb[coef_word<PTS>(a, m, t)] = hi_round(Ab[(1 + a) * BLOCK_CELLS + s]);
      cb[coef_word<PTS>(6, m, t)] = hi_round(1.0 / Ab[s]);
    }
  }
  // uniform block: all seven coefficients bitwise equal to cell 0's everywhere
  bool same = true;
  for (int s = threadIdx.x; s < BLOCK_CELLS; s += MT)
#pragma unroll
    for (int a = 0; a < 7; ++a)
      same = same && __double_as_longlong(Ab[a * BLOCK_CELLS + s]) ==
                         __double_as_longlong(Ab[a * BLOCK_CELLS]);
  same = __syncthreads_and(same);
  if (threadIdx.x < 8)
    ucoef[(size_t)blk * 8 + threadIdx.x] =
        threadIdx.x < 7 ? Ab[threadIdx.x * BLOCK_CELLS] : (same ? 1.0 : 0.0);
  if (threadIdx.x == 0 && same) atomicAdd(&st->ublocks, 1);
}

// ---------------------------------------------------------------------------
// Start of a solve (FFVILS.h:820-846): b.b, r = b - A x (calc_r,
// bils.f90:208-254, x's stored guide layer), r0 = r, r.r0.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(MT)
mx_init_kernel(MixCtx C, const double* __restrict__ x, const double* __restrict__ gx,
               const double* __restrict__ A, const double* __restrict__ bvec,
               double* __restrict__ r, double* __restrict__ r0) {
  const int blk = C.first + blockIdx.x;
  const int inst = active_instance(C, blk);
  if (inst < 0) return;
  __shared__ double O[BLOCK_CELLS];
  __shared__ double G[6 * FACE_CELLS];
  __shared__ FaceNbr snb[6];
  const int tid = threadIdx.x;
  const size_t base = (size_t)blk * BLOCK_CELLS;
  if (tid < 6) snb[tid] = C.nbr[blk * 6 + tid];
#pragma unroll 4
  for (int m = 0; m < 16; ++m) O[tid + MT * m] = __ldg(x + base + tid + MT * m);
#pragma unroll
  for (int f = 0; f < 6; ++f)
    G[f * FACE_CELLS + tid] = __ldg(gx + ((size_t)blk * 6 + f) * FACE_CELLS + tid);
  __syncthreads();
  const double* Ab = A + (size_t)blk * 7 * BLOCK_CELLS;
  double acc[2][2][2] = {};
#pragma unroll
  for (int c = 0; c < 2; ++c) {
#pragma unroll 2
    for (int m = 0; m < 8; ++m) {
      const int q = tid + MT * m, s = c * HALF_CELLS + q;
      const Nbrs v = split_neighbours(O + (1 - c) * HALF_CELLS, G, q, c);
      double rv = __ldg(bvec + base + s) - __ldg(Ab + 4096 + s) * v.w -
                        __ldg(Ab + 8192 + s) * v.e - __ldg(Ab + 12288 + s) * v.s -
                        __ldg(Ab + 16384 + s) * v.n - __ldg(Ab + 20480 + s) * v.b -
                        __ldg(Ab + 24576 + s) * v.t - __ldg(Ab + s) * O[s];
      if (C.cf)  // coarse-fine flux correction: r = b - (A x + delta)
        rv = cf_delta<true>(x, gx, A, C.nbr, C.dx, C.bc, snb, G, O[s], s, rv,
                            [&](int f) { return __ldg(Ab + (1 + f) * BLOCK_CELLS + s); });
      r[base + s] = rv;
      r0[base + s] = rv;
      const double bv = __ldg(bvec + base + s);
      acc[0][c][m & 1] += bv * bv;
      acc[1][c][m & 1] += rv * rv;
    }
  }
  mx_reduce<2, MT>(acc, C, blk, inst, FIN_MX_INIT);
}

// ---------------------------------------------------------------------------
// One pass of sweeps.  MODE 0: right-hand side p (FFVILS.h:853-871: p = r
// at the first iteration of a cycle, which also sets r0 = r, else
// p = r + beta*(p + (-gamma)*q)); MODE 1: right-hand side s = (-alpha)*q + r
// (FFVILS.h:898-903).  FIRST: the pass that forms the right-hand side
// (written to pv in FP64) and starts from e = 0 with zero guides; later
// passes read the right-hand side back from pv and start from ein with its
// exchanged guide layer.  Every pass writes its iterate to eout in FP32.
//
// Thread t owns the k-column (ih, j, 4 kg .. 4 kg + 3) of both colours
// (ih = t & 7, kg = (t >> 3) & 3, j = t >> 5): eight cells whose iterate
// and coefficients stay in registers for the whole pass (the right-hand
// side sits in shared memory in thread order).
// Of a cell's six neighbours (all of the other colour) the one at the same
// (ih, j) -- west or east by the row's parity -- and the z neighbours inside
// the column are this thread's own registers; the rest come from the tile.
// While this block sweeps, one bulk copy brings the next block's coefficient
// words (or, for a uniform block in a first pass, its right-hand-side vectors)
// and, in a later pass, its guide layer; vectors not copied are prefetched
// into L2.
// ---------------------------------------------------------------------------
// T and V are written by other threads between the barriers: no __restrict__
// on them, which would let the compiler move tile loads across
// __syncthreads().
// Where a cell's coefficients come from.  CS_UNI: a uniform block -- the
// seven coefficients ku (widened once) serve every cell.  CS_W32: each cell's
// 32-bit words cw[m] are widened at use.  CS_G64 (the FP64-data variant):
// each cell's FP64 coefficients are read at use from c64, the block's
// coefficients in thread order ([a][m][thread], c64 already offset to this
// thread).  For one data format the values, and so the results, do not
// depend on the source.
enum { CS_UNI = 0, CS_W32 = 1, CS_G64 = 2 };
// PTS threads: the cells m = (c JJ + jj) 4 + h of a thread (SweepGeom).  Of a
// cell's six neighbours (all of the other colour) the x neighbour at the same
// ih, the z neighbours inside the 4-cell column and, with two rows per thread
// (PTS 256), the y neighbour in the thread's other row are its own registers;
// the rest come from the tile.  The terms keep rbgs_smoother's order (w, e,
// s, n, b, t) whatever their source, so every PTS gives the same bits.
template <int CS, int PTS>
__device__ __forceinline__ void run_sweeps(double* T, const double* V, int o0, int p0,
                                           double (&E)[2][SweepGeom<PTS>::JJ][4],
                                           const uint32_t (&cw)[SweepGeom<PTS>::CPT][7],
                                           const double (&ku)[7],
                                           const double* __restrict__ c64, double mom,
                                           int nsweep) {
  constexpr bool UNI = CS == CS_UNI;
  constexpr int JJ = SweepGeom<PTS>::JJ, CPT = SweepGeom<PTS>::CPT;
#define MX_COEF(m, a)                                          \
  (CS == CS_UNI ? ku[a]                                        \
   : CS == CS_W32 ? widen_here(cw[m][a])                       \
                  : __ldg(c64 + ((a) * CPT + (m)) * PTS))
  // a uniform block has the registers to keep its right-hand side too (one
  // shared-memory read less per update)
  double vr[2][JJ][4];
#pragma unroll
  for (int c = 0; c < 2; ++c)
#pragma unroll
    for (int jj = 0; jj < JJ; ++jj)
#pragma unroll
      for (int h = 0; h < 4; ++h) vr[c][jj][h] = UNI ? V[((c * JJ + jj) * 4 + h) * PTS] : 0.0;
#pragma unroll 1
  for (int it = 0; it < nsweep; ++it) {
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      // the cells of this colour advance term by term, so their dependent
      // FP64 chains overlap (each chain keeps its own order)
      const double* O = T + o0 + (1 - c) * SH;  // cell (jj, h): O + jj SP + h SQ, other colour
      double rc[JJ][4], xo[JJ][4];
#pragma unroll
      for (int jj = 0; jj < JJ; ++jj)
#pragma unroll
        for (int h = 0; h < 4; ++h) {
          const int par = p0 ^ ((jj + h + c) & 1);  // x parity of the cell: i = 2 ih + par
          // the x neighbour at the same ih is this thread's own; the other one
          // is east (par 1) or west (par 0) of it in the tile
          xo[jj][h] = O[jj * SP + h * SQ + (par ? 1 : -1)];
          rc[jj][h] = UNI ? vr[c][jj][h] : V[((c * JJ + jj) * 4 + h) * PTS];
        }
#define MX_M(jj, h) ((c * JJ + (jj)) * 4 + (h))
#pragma unroll
      for (int jj = 0; jj < JJ; ++jj)
#pragma unroll
        for (int h = 0; h < 4; ++h) {
          const int par = p0 ^ ((jj + h + c) & 1);
          rc[jj][h] = __fma_rn(-MX_COEF(MX_M(jj, h), 0), par ? E[1 - c][jj][h] : xo[jj][h],
                               rc[jj][h]);
        }
#pragma unroll
      for (int jj = 0; jj < JJ; ++jj)
#pragma unroll
        for (int h = 0; h < 4; ++h) {
          const int par = p0 ^ ((jj + h + c) & 1);
          rc[jj][h] = __fma_rn(-MX_COEF(MX_M(jj, h), 1), par ? xo[jj][h] : E[1 - c][jj][h],
                               rc[jj][h]);
        }
#pragma unroll
      for (int jj = 0; jj < JJ; ++jj)
#pragma unroll
        for (int h = 0; h < 4; ++h)
          rc[jj][h] = __fma_rn(-MX_COEF(MX_M(jj, h), 2),
                               jj > 0 ? E[1 - c][jj - 1][h] : O[jj * SP + h * SQ - SP], rc[jj][h]);
#pragma unroll
      for (int jj = 0; jj < JJ; ++jj)
#pragma unroll
        for (int h = 0; h < 4; ++h)
          rc[jj][h] = __fma_rn(-MX_COEF(MX_M(jj, h), 3),
                               jj < JJ - 1 ? E[1 - c][jj + 1][h] : O[jj * SP + h * SQ + SP],
                               rc[jj][h]);
#pragma unroll
      for (int jj = 0; jj < JJ; ++jj)
#pragma unroll
        for (int h = 0; h < 4; ++h)
          rc[jj][h] = __fma_rn(-MX_COEF(MX_M(jj, h), 4),
                               h > 0 ? E[1 - c][jj][h - 1] : O[jj * SP - SQ], rc[jj][h]);
#pragma unroll
      for (int jj = 0; jj < JJ; ++jj)
#pragma unroll
        for (int h = 0; h < 4; ++h)
          rc[jj][h] = __fma_rn(-MX_COEF(MX_M(jj, h), 5),
                               h < 3 ? E[1 - c][jj][h + 1] : O[jj * SP + 4 * SQ], rc[jj][h]);
#pragma unroll
      for (int jj = 0; jj < JJ; ++jj)
#pragma unroll
        for (int h = 0; h < 4; ++h) {
          const double xt = __dmul_rn(rc[jj][h], MX_COEF(MX_M(jj, h), 6));
          const double e = E[c][jj][h];
          const double en = __fma_rn(mom, __dsub_rn(e, xt), e);
          E[c][jj][h] = en;
          T[o0 + c * SH + jj * SP + h * SQ] = en;
        }
#undef MX_M
      __syncthreads();
    }
  }
}
#undef MX_COEF

// Tile address of the guide cell at position p (u + 16 v) of a face.
__device__ __forceinline__ int guide_slot(int face, int p) {
  const int u = p & 15, v = p >> 4, out = (face & 1) ? 16 : -1;
  const int axis = face >> 1;
  const int i = axis == 0 ? out : u;
  const int j = axis == 0 ? u : (axis == 1 ? out : v);
  const int k = axis == 2 ? out : v;
  return ((i + j + k) & 1) * SH + tile_at(i, j, k);
}

constexpr int ROLE_SWEEP = 8;  // SolveState::timeout_where bit of this kernel's waits

// A CTA's live items, found once per chunk instead of a block ahead: entry
// (block, instance | flags) of the items blockIdx.x + k gridDim.x whose
// instance is still solving (the done flags change between launches only).
constexpr int LIST_CAP = 1024;           // entries per chunk (8 KB of shared memory)
constexpr int LF_UNI = 1 << 30;          // the block is uniform (MixCtx::ucoef)
constexpr int LF_COPY = 1 << 29;         // its instance starts a cycle (p = r, r0 = r)
constexpr int LF_INST = LF_COPY - 1;

// Called by every thread of a CTA of PTS: fills list[0, *n) from the
// candidates from, from + gridDim.x, ... (CAP of them, in item order) and
// sets *next to the first candidate after them.
template <int MODE, bool FIRST, int PTS, int CAP = LIST_CAP>
__device__ void build_live_list(const MixCtx& C, int from, int n_act, int2* list, int* n,
                                int* next, int* wcount) {
  static_assert(CAP % PTS == 0, "whole rounds of candidates");
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  int base = 0;
  for (int r = 0; r < CAP / PTS; ++r) {
    const int it = from + (r * PTS + tid) * gridDim.x;
    int b = -1, e = 0;
    bool live = false;
    if (it < n_act) {
      b = C.active[it];
      const int i = C.inst.blk_inst[b];
      live = i >= 0 && !*((volatile const int32_t*)&C.inst.st[i].done);
      if (live) {
        e = i;
        if (C.ucoef[(size_t)b * 8 + 7] != 0.0) e |= LF_UNI;
        if (FIRST && MODE == 0 && C.inst.st[i].cycle == 1) e |= LF_COPY;
      }
    }
    const unsigned m = __ballot_sync(0xffffffffu, live);
    if (lane == 0) wcount[warp] = __popc(m);
    __syncthreads();
    int off = base;
    for (int w = 0; w < warp; ++w) off += wcount[w];
    if (live) list[off + __popc(m & ((1u << lane) - 1u))] = make_int2(b, e);
    int tot = 0;
    for (int w = 0; w < PTS / 32; ++w) tot += wcount[w];
    base += tot;
    __syncthreads();  // wcount is refilled by the next round
  }
  if (tid == 0) {
    *n = base;
    *next = from + CAP * gridDim.x;
  }
  __syncthreads();
}

// ET: the iterate between passes, float (the mixed form) or double (the
// FP64-data variant, whose coefficients are FP64 too and read at use).
template <int MODE, bool FIRST, typename ET, int PTS>
__global__ void __launch_bounds__(PTS, 1)
mx_sweep_kernel(MixCtx C, float omega, int nsweep, const double* __restrict__ r,
                double* __restrict__ r0, double* __restrict__ pv, const double* __restrict__ q,
                const uint32_t* __restrict__ coef, const double* __restrict__ coef64,
                const ET* __restrict__ ein, const double* __restrict__ guides,
                ET* __restrict__ eout, int depth) {
  constexpr bool D64 = sizeof(ET) == 8;
  constexpr int JJ = SweepGeom<PTS>::JJ, CPT = SweepGeom<PTS>::CPT;
  extern __shared__ __align__(128) unsigned char smem[];
  uint32_t* slot = reinterpret_cast<uint32_t*>(smem);
  double* T = reinterpret_cast<double*>(smem + COEF_WORDS * 4);
  double* V = reinterpret_cast<double*>(smem + COEF_WORDS * 4 + TILE * 8);  // [m][t] rhs
  double* GB = V + BLOCK_CELLS;  // [face][p] guides of the block, copied with its coefficients
  uint64_t* bar = reinterpret_cast<uint64_t*>(GB + GUIDES);
  __shared__ int2 s_list[LIST_CAP];
  __shared__ int s_nlist, s_next_from, s_wcount[PTS / 32];
  __shared__ int abort_flag;
  __shared__ int s_copied[2];  // a copy was issued on the barrier for this parity
  // a uniform block's coefficient record (MixCtx::ucoef), copied with the block
  __shared__ __align__(16) double s_urec[2][8];
  // the copy of one block: its coefficient words unless the block is
  // uniform (then its coefficient record), and its guide layer in a later
  // pass; with none of them, the arrival alone completes the phase.  Run by
  // thread 0 for list entry e, copy parity p.  A uniform block needs no
  // coefficient words, so in a first pass its copy brings the block's
  // vectors into the slot instead and its staging reads shared memory: r
  // (slot doubles [0, 4096)), q ([4096, 8192)) and p ([8192, 12288)) as far
  // as it reads them.  (A later pass reads p and the FP32 iterate from global
  // memory, prefetched into L2 a block ahead: that measured faster than
  // copying them.)  Nothing here waits on a global load.
  auto issue = [&](int2 e, uint32_t p) {
    const int b = e.x;
    const bool uni = e.y & LF_UNI;
    // test hook (MixCtx::stall): nothing arrives on the barrier, so the wait
    // for this block runs out after the wait limit
    s_copied[p] = C.stall != 1;
    if (C.stall == 1) return;
    const size_t gb = (size_t)b * BLOCK_CELLS;
    constexpr uint32_t VB = BLOCK_CELLS * 8;  // bytes of one FP64 vector block
    constexpr uint32_t UB = 8 * 8;            // bytes of a coefficient record
    double* sd = reinterpret_cast<double*>(slot);
    if (uni) {
      if (FIRST) {
        const bool copy = e.y & LF_COPY;
        const bool needq = !copy, needp = MODE == 0 && !copy;
        async::mbar_expect_tx(bar, UB + VB + (needq ? VB : 0u) + (needp ? VB : 0u));
        async::bulk_g2s(s_urec[p], C.ucoef + (size_t)b * 8, UB, bar);
        async::bulk_g2s(sd, r + gb, VB, bar);
        if (needq) async::bulk_g2s(sd + BLOCK_CELLS, q + gb, VB, bar);
        if (needp) async::bulk_g2s(sd + 2 * BLOCK_CELLS, pv + gb, VB, bar);
      } else {
        async::mbar_expect_tx(bar, UB + GUIDES * 8u);
        async::bulk_g2s(s_urec[p], C.ucoef + (size_t)b * 8, UB, bar);
        async::bulk_g2s(GB, guides + (size_t)b * GUIDES, GUIDES * 8, bar);
      }
      return;
    }
    if (D64) {
      // FP64 coefficients are read at use (prefetched into L2); the copy
      // brings the guide layer only
      if (FIRST) {
        async::mbar_arrive(bar);
      } else {
        async::mbar_expect_tx(bar, GUIDES * 8u);
        async::bulk_g2s(GB, guides + (size_t)b * GUIDES, GUIDES * 8, bar);
      }
    } else {
      async::mbar_expect_tx(bar, COEF_WORDS * 4u + (FIRST ? 0u : GUIDES * 8u));
      async::bulk_g2s(slot, coef + (size_t)b * COEF_WORDS, COEF_WORDS * 4, bar);
      if (!FIRST) async::bulk_g2s(GB, guides + (size_t)b * GUIDES, GUIDES * 8, bar);
    }
  };
  // Brings into L2 what the copy and the staging of list entry e will read:
  // run for the entry 'depth' blocks ahead of the one being swept (depth 1:
  // the next block, whose copy is issued now).
  auto prefetch = [&](int2 e) {
    const int b = e.x;
    const bool uni = e.y & LF_UNI, copy = e.y & LF_COPY;
    const size_t gb = (size_t)b * BLOCK_CELLS;
    constexpr uint32_t VB = BLOCK_CELLS * 8;
    if (!uni) {
      if (D64)
        async::prefetch_l2(coef64 + (size_t)b * COEF_WORDS, COEF_WORDS * 8u);
      else if (depth > 1)
        async::prefetch_l2(coef + (size_t)b * COEF_WORDS, COEF_WORDS * 4u);
    }
    if (FIRST) {
      async::prefetch_l2(r + gb, VB);
      if (!copy) async::prefetch_l2(q + gb, VB);
      if (MODE == 0 && !copy) async::prefetch_l2(pv + gb, VB);
    } else {
      if (depth > 1) async::prefetch_l2(guides + (size_t)b * GUIDES, GUIDES * 8u);
      async::prefetch_l2(pv + gb, VB);
      async::prefetch_l2(ein + gb, BLOCK_CELLS * (uint32_t)sizeof(ET));
    }
  };
  const int tid = threadIdx.x;
  const int ih = tid & 7, kg = (tid >> 3) & 3, j0 = JJ * (tid >> 5);
  const int o0 = (4 * kg + 1) * SQ + (j0 + 1) * SP + ih + 1;  // tile slot of cell m = 0
  const int s0 = sweep_cell<PTS>(tid, 0);                      // its storage slot
  const double mom = -(double)omega;
  const int n_act = *C.n_active;
  if (tid == 0) {
    async::mbar_init(bar, 1);
    async::fence_mbar_init();
    abort_flag = 0;
  }
  if (FIRST)
    for (int g = tid; g < TILE; g += PTS) T[g] = 0.0;  // guides of e stay 0 in a first pass
  // The CTA visits the live items blockIdx.x + n gridDim.x of the active
  // list (blocks of instances still solving), found a chunk at a time, and
  // issues each block's copy while the block before it sweeps, so blocks of
  // instances that have stopped cost neither a copy nor a wait.
  build_live_list<MODE, FIRST, PTS>(C, blockIdx.x, n_act, s_list, &s_nlist, &s_next_from,
                                    s_wcount);
  while (s_nlist == 0 && s_next_from < n_act)  // a chunk with no live item
    build_live_list<MODE, FIRST, PTS>(C, s_next_from, n_act, s_list, &s_nlist, &s_next_from,
                                      s_wcount);
  if (tid == 0 && s_nlist > 0) {
    issue(s_list[0], 0);
    for (int k = 0; k < depth && k < s_nlist; ++k) prefetch(s_list[k]);
  }
  int pos = 0;         // list position of the current block
  uint32_t phase = 0;  // parity of the copy the current block waits on
  for (;; phase ^= 1u) {
    __syncthreads();
    if (pos >= s_nlist) break;
    const int2 ent = s_list[pos];
    const int blk = ent.x, inst = ent.y & LF_INST;
    const bool uni = ent.y & LF_UNI;
    const size_t base = (size_t)blk * BLOCK_CELLS + s0;
    double E[2][JJ][4] = {};
    // this block's copy (issued a block ago): coefficients and guides, or
    // for a uniform block its record, vectors or guides
    async::mbar_wait(bar, phase, &abort_flag, ROLE_SWEEP, C.wait_ns);
    const double* sd = reinterpret_cast<const double*>(slot);
    const size_t gbase = (size_t)blk * BLOCK_CELLS;
    if (FIRST) {
      const SolveState* S = C.inst.st + inst;
      const bool copy = ent.y & LF_COPY;  // first iteration of a (re)start: p = r, r0 = r
      const double mgamma = -S->gamma, beta = S->beta, malpha = -S->alpha;
      const double* rs = uni ? sd : r + gbase;
      const double* qs = uni ? sd + BLOCK_CELLS : q + gbase;
      const double* ps = uni ? sd + 2 * BLOCK_CELLS : pv + gbase;
      // With two rows per thread, threads of odd k groups take their rows in
      // the other order: the two 8-thread groups of a half-warp, 512 doubles
      // apart in the slot (the same banks), then read 8 doubles apart mod 16
      // (disjoint banks).  The iterate starts at 0, so only stores follow
      // the order.
      const int jsw = JJ == 2 ? (tid >> 3) & 1 : 0;
#pragma unroll
      for (int c = 0; c < 2; ++c)
#pragma unroll
        for (int jo = 0; jo < JJ; ++jo)
#pragma unroll
        for (int h = 0; h < 4; ++h) {
          const int jj = jo ^ jsw;
          const int sl = s0 + c * HALF_CELLS + jj * 8 + h * 128;
          const size_t s = gbase + sl;
          double rhs;
          if (MODE == 0) {
            if (copy) {
              rhs = rs[sl];
              r0[s] = rhs;
            } else {
              const double t = ps[sl] + mgamma * qs[sl];
              rhs = rs[sl] + beta * t;
            }
          } else {
            rhs = malpha * qs[sl] + rs[sl];
          }
          pv[s] = rhs;
          V[((c * JJ + jj) * 4 + h) * PTS + tid] = rhs;
          E[c][jo][h] = 0.0;
          T[o0 + c * SH + jo * SP + h * SQ] = 0.0;  // every cell of the thread, in row order
        }
    } else {
#pragma unroll
      for (int c = 0; c < 2; ++c)
#pragma unroll
        for (int jj = 0; jj < JJ; ++jj)
#pragma unroll
        for (int h = 0; h < 4; ++h) {
          const size_t s = base + c * HALF_CELLS + jj * 8 + h * 128;
          V[((c * JJ + jj) * 4 + h) * PTS + tid] = pv[s];
          E[c][jj][h] = (double)__ldg(ein + s);
          T[o0 + c * SH + jj * SP + h * SQ] = E[c][jj][h];
        }
#pragma unroll
      for (int g = tid; g < GUIDES; g += PTS) T[guide_slot(g >> 8, g & 255)] = GB[g];
    }
    uint32_t cw[CPT][7];
    double ku[7];
    if (uni) {
      const double* U = s_urec[phase];
      if (D64) {
#pragma unroll
        for (int a = 0; a < 6; ++a) ku[a] = U[1 + a];
        ku[6] = 1.0 / U[0];
      } else {
#pragma unroll
        for (int a = 0; a < 6; ++a) ku[a] = widen(hi_round(U[1 + a]));
        ku[6] = widen(hi_round(1.0 / U[0]));
      }
    } else if (!D64) {
#pragma unroll
      for (int a = 0; a < 7; ++a)
#pragma unroll
        for (int hq = 0; hq < CPT / 4; ++hq) {
          const uint4 w = reinterpret_cast<const uint4*>(slot)[(a * (CPT / 4) + hq) * PTS + tid];
          cw[4 * hq + 0][a] = w.x;
          cw[4 * hq + 1][a] = w.y;
          cw[4 * hq + 2][a] = w.z;
          cw[4 * hq + 3][a] = w.w;
        }
    }
    async::fence_proxy_async();
    __syncthreads();
    if (abort_flag) {
      // the copy did not land in time: wait (bounded by DRAIN_NS, whatever
      // the wait limit) until it has, so that the CTA never exits with a
      // copy into its shared memory in flight, stop every instance this CTA
      // still had to sweep, and leave.  Only one copy is ever in flight: the
      // next block's is issued after this check.
      if (tid == 0) {
        const bool drained = !s_copied[phase] || async::mbar_drain(bar, phase);
        const int where = ROLE_SWEEP | (drained ? 0 : async::ROLE_DRAIN);
        auto stop = [&](int i2) {
          atomicOr(&C.inst.st[i2].timeout_where, where);
          atomicExch(&C.inst.st[i2].status, 3);
          atomicExch(&C.inst.st[i2].done, 1);
        };
        for (int k = pos; k < s_nlist; ++k) stop(s_list[k].y & LF_INST);
        for (int it2 = s_next_from; it2 < n_act; it2 += gridDim.x) {
          const int i2 = C.inst.blk_inst[C.active[it2]];
          if (i2 >= 0) stop(i2);
        }
      }
      return;
    }
    // the next block: from this chunk, or from the next one (built by every
    // thread; this block's entry is already in registers)
    int npos = pos + 1;
    if (npos >= s_nlist && s_next_from < n_act) {
      do
        build_live_list<MODE, FIRST, PTS>(C, s_next_from, n_act, s_list, &s_nlist,
                                          &s_next_from, s_wcount);
      while (s_nlist == 0 && s_next_from < n_act);
      npos = 0;
    }
    // the next block's copy (thread 0) and the L2 prefetch 'depth' blocks
    // ahead (lane 0 of the second warp) are issued in parallel: every
    // thread waits for both at the sweeps' first barrier
    if (tid == 0 && npos < s_nlist) issue(s_list[npos], phase ^ 1u);
    if (tid == 32 && npos + depth - 1 < s_nlist) prefetch(s_list[npos + depth - 1]);
    pos = npos;
    const double* c64 = D64 ? coef64 + (size_t)blk * COEF_WORDS + tid : nullptr;
    if (uni)
      run_sweeps<CS_UNI, PTS>(T, V + tid, o0, j0 & 1, E, cw, ku, c64, mom, nsweep);
    else if constexpr (D64)
      run_sweeps<CS_G64, PTS>(T, V + tid, o0, j0 & 1, E, cw, ku, c64, mom, nsweep);
    else
      run_sweeps<CS_W32, PTS>(T, V + tid, o0, j0 & 1, E, cw, ku, c64, mom, nsweep);
#pragma unroll
    for (int c = 0; c < 2; ++c)
#pragma unroll
      for (int jj = 0; jj < JJ; ++jj)
#pragma unroll
        for (int h = 0; h < 4; ++h)
          eout[base + c * HALF_CELLS + jj * 8 + h * 128] = (ET)E[c][jj][h];
  }
}

// ---------------------------------------------------------------------------
// Guide layer of an FP32 iterate for the next sweep pass: per live block the
// first guide layer by the exchange rules (same-level copy, 2:1
// interpolation and restriction, src/CGMfuncs/sup.f90) evaluated in FP64,
// homogeneous Dirichlet values on outer faces; [blk][face][p] FP64, which
// the sweep kernel bulk-copies with the block's coefficients.
// ---------------------------------------------------------------------------
constexpr int GT = MT;  // guides kernel: three pairs (face, p, p + 128) per thread

template <typename ET>
__global__ void __launch_bounds__(GT)
mx_guides_kernel(MixCtx C, const ET* __restrict__ e, double* __restrict__ guides) {
  BCSet hom;
  for (int f = 0; f < 6; ++f) {
    hom.type[f] = BC_DIRICHLET;
    hom.value[f] = 0.0;
  }
  __shared__ FaceNbr snb[6];
  __shared__ double sdx;
  __shared__ int live;
  const int n_act = *C.n_active;
  for (int item = blockIdx.x; item < n_act; item += gridDim.x) {
    const int blk = C.active[item];
    if (threadIdx.x < 6) snb[threadIdx.x] = C.nbr[blk * 6 + threadIdx.x];
    if (threadIdx.x == 0) {
      live = active_instance(C, blk) >= 0;
      sdx = C.dx[blk];
    }
    __syncthreads();
    if (live) {
      double* gb = guides + (size_t)blk * GUIDES;
#pragma unroll
      for (int r = 0; r < 3; ++r) {  // the three pairs' loads in flight together
        const int w = threadIdx.x + GT * r, f = w >> 7, p0 = w & 127, p1 = p0 + 128;
        const FaceNbr nf = snb[f];
        double g0, g1;
        guide_pair(e, blk, f, p0, p1, nf, hom, sdx, g0, g1);
        gb[f * FACE_CELLS + p0] = g0;
        gb[f * FACE_CELLS + p1] = g1;
      }
    }
    __syncthreads();  // snb, sdx and live are refilled for the next block
  }
}

// ---------------------------------------------------------------------------
// y = A x for an FP32 x, in FP64 (calc_ax, bils.f90:162-206), with its dot
// products.  NV = 1: y.w0 (q_.r0, FFVILS.h:890-896).  NV = 2: y.w0 and y.y
// (t_.s and t_.t_, FFVILS.h:923-936).
// ---------------------------------------------------------------------------
template <int NV, bool CF, typename ET, int NT>
__global__ void __launch_bounds__(NT, 1024 / NT)
mx_matvec_kernel(MixCtx C, const ET* __restrict__ x, const double* __restrict__ A,
                 double* __restrict__ y, const double* __restrict__ w0) {
  __shared__ double O[BLOCK_CELLS];
  __shared__ double G[6 * FACE_CELLS];
  __shared__ FaceNbr snb[6];
  const int tid = threadIdx.x;
  const int n_act = *C.n_active;
  for (int item = blockIdx.x; item < n_act; item += gridDim.x) {
    const int blk = C.active[item];
    const int inst = active_instance(C, blk);
    if (inst < 0) continue;
    if (tid == 0 && item + (int)gridDim.x < n_act) {
      // the next block's vectors into L2 while this one is staged and summed
      const size_t nb = (size_t)C.active[item + gridDim.x] * BLOCK_CELLS;
      async::prefetch_l2(x + nb, BLOCK_CELLS * (uint32_t)sizeof(ET));
      async::prefetch_l2(w0 + nb, BLOCK_CELLS * 8u);
    }
    if (tid < 6) snb[tid] = C.nbr[blk * 6 + tid];
    const size_t base = (size_t)blk * BLOCK_CELLS;
    // with 8 cells per thread (NT 512) the registers hold the block's dot
    // partners and coefficient record, loaded before the staging so that
    // their latency overlaps it; with more cells per thread they are read
    // in the loop
    constexpr bool HOIST = NT >= 512;
    constexpr int CPC = HALF_CELLS / NT;  // cells per colour of a thread
    double wv[2][HOIST ? CPC : 1];
    double ur[8];
    if (HOIST) {
#pragma unroll
      for (int c = 0; c < 2; ++c)
#pragma unroll
        for (int m = 0; m < (HOIST ? CPC : 1); ++m)
          wv[c][m] = __ldg(w0 + base + c * HALF_CELLS + tid + NT * m);
#pragma unroll
      for (int a = 0; a < 8; ++a) ur[a] = __ldg(C.ucoef + (size_t)blk * 8 + a);
    }
    __syncthreads();
    stage_f32_as_f64<NT>(O, G, x, blk, snb, C.dx[blk], C);
    __syncthreads();
    const double* Ab = A + (size_t)blk * 7 * BLOCK_CELLS;
    const double* U = C.ucoef + (size_t)blk * 8;
    const bool uni = (HOIST ? ur[7] : U[7]) != 0.0;  // the same seven coefficients in every cell
    double u[7];
#pragma unroll
    for (int a = 0; a < 7; ++a) u[a] = uni ? (HOIST ? ur[a] : U[a]) : 0.0;
    constexpr int VPT = 512 / NT;
    double acc[NV][2][VPT] = {};
#pragma unroll
    for (int c = 0; c < 2; ++c) {
#pragma unroll 2
      for (int m = 0; m < HALF_CELLS / NT; ++m) {
        const int qd = tid + NT * m, s = c * HALF_CELLS + qd;
        const Nbrs v = split_neighbours(O + (1 - c) * HALF_CELLS, G, qd, c);
        double yv =
            uni ? u[1] * v.w + u[2] * v.e + u[3] * v.s + u[4] * v.n + u[5] * v.b + u[6] * v.t +
                      u[0] * O[s]
                : __ldg(Ab + 4096 + s) * v.w + __ldg(Ab + 8192 + s) * v.e +
                      __ldg(Ab + 12288 + s) * v.s + __ldg(Ab + 16384 + s) * v.n +
                      __ldg(Ab + 20480 + s) * v.b + __ldg(Ab + 24576 + s) * v.t +
                      __ldg(Ab + s) * O[s];
        if (CF)  // coarse-fine flux correction: y = A x + delta
          yv = cf_delta<false>(x, (const double*)nullptr, A, C.nbr, C.dx, C.bc, snb, G, O[s], s,
                               yv, [&](int f) {
                                 return uni ? u[1 + f] : __ldg(Ab + (1 + f) * BLOCK_CELLS + s);
                               });
        y[base + s] = yv;
        acc[0][c][m % VPT] += yv * (HOIST ? wv[c][HOIST ? m : 0] : __ldg(w0 + base + s));
        if (NV == 2) acc[NV - 1][c][m % VPT] += yv * yv;
      }
    }
    mx_reduce<NV, NT>(acc, C, blk, inst, NV == 1 ? FIN_MX_ALPHA : FIN_MX_GAMMA);
    __syncthreads();  // O and G are refilled for the next block
  }
}

// ---------------------------------------------------------------------------
// The same A*x and dot products as a persistent, warp-specialised kernel:
// one CTA of 800 threads per SM walks its live blocks.
//   producer (thread 0): through a ring of three 32 KB slots, by bulk copies,
//     the dot partner w0 (a uniform block: all of it in one slot) or, for a
//     block that streams its coefficients, eight slots of 512 cells with the
//     seven coefficient rows and w0.
//   gatherers (8 warps): a block ahead, its x widened to FP64 and its guide
//     layer by the exchange rules, written into a padded tile: per colour
//     [k + 1][j + 1][i >> 1] with rows of 8 values (k, j in -1..16), so every
//     neighbour of a cell is at a fixed offset but the x-face guides, which
//     sit in two arrays of their own; with rows of 8 the two rows a half-warp
//     reads fall into disjoint banks.  The loads are issued before the tile
//     frees up.
//   consumers (16 warps): consumer t takes cells q = 512 mm + t of each
//     colour, which makes it the block tree's virtual thread t: the per-block
//     sums are those of mx_reduce; the ticket of an instance is advanced once
//     per run of its blocks in the CTA's list, and the CTA that completes it
//     forms the cross-block sums (256 lanes, block order) and finalises.
// Every wait is bounded (MixCtx::wait_ns); a wait that gives up stops the
// instances of the CTA's list with TIMEOUT.
// With an FP64 x (ET double) and MixCtx::fin set it is also the A*x of the
// FP64 Krylov solvers (one instance over the pool): the same sums as their
// block-per-CTA trees, finalised by the FP64 solver's state machine.  With
// JAC the consumers form a Jacobi sweep of x instead (w0 = b; NV 0, or 1 for
// b.y), the second and later passes of the solvers' preconditioner.
// ---------------------------------------------------------------------------
namespace mvp {
constexpr int STAGES = 3;
constexpr int ROWS = 8;                            // A rows 0..6 (Ap, Aw..At), w0
constexpr int SLOT_CELLS = 512;
constexpr int SLOTS = BLOCK_CELLS / SLOT_CELLS;    // slots of a streamed block
constexpr uint32_t SLOT_BYTES = ROWS * SLOT_CELLS * 8;
constexpr int GATHER0 = 32, NGATHER = 256;
constexpr int CONS0 = GATHER0 + NGATHER, NCONS = 512, CONS_WARPS = NCONS / 32;
constexpr int NTHREADS = CONS0 + NCONS;            // 800
constexpr int CAP = NTHREADS;                      // list entries per chunk
constexpr int ROLE_MATVEC = 32;                    // SolveState::timeout_where bit
static_assert(SLOT_BYTES == BLOCK_CELLS * 8, "a slot holds a uniform block's w0");
// the tile: row pitch (i >> 1 in 0..7), plane pitch (rows j = -1..16) and
// colour half (planes k = -1..16)
constexpr int TR = 8, TP = 18 * TR, TH = 18 * TP, TT = 2 * TH;

struct __align__(128) Smem {
  double ring[STAGES][ROWS][SLOT_CELLS];  // 96 KB
  double tile[2][TT];                     // 81 KB: x of the current / next block, j/k guides
  double xg[2][2][FACE_CELLS];            // 8 KB: their x-face guides [face][j + 16 k]
  double urec[2][8];                      // coefficient records of the blocks in the tiles
  // warp sums of the block tree [block parity][sum][warp]: consumer 0 reads
  // block n's while the other warps may already write block n + 1's
  double ws[2][2][CONS_WARPS];
  int2 list[CAP];                         // the chunk's live entries
  FaceNbr snb[2][6];                      // face records (flux correction)
  // full/empty: ring slots; gfull: a tile ready; tempty: a tile free
  uint64_t full[STAGES], empty[STAGES], gfull[2], tempty[2];
  int wcount[NTHREADS / 32];
  int nlist, next_from, abort_flag, last_inst;
};
static_assert(sizeof(Smem) <= 227 * 1024, "shared memory of one CTA");

// Tile position of the j/k-face guide at (face, p = u + 16 v), face 2..5.
__device__ __forceinline__ int tile_guide(int face, int p) {
  const int u = p & 15, v = p >> 4, out = (face & 1) ? 16 : -1;
  return face < 4 ? ((u + out + v) & 1) * TH + (v + 1) * TP + (out + 1) * TR + (u >> 1)
                  : ((u + v + out) & 1) * TH + (out + 1) * TP + (v + 1) * TR + (u >> 1);
}
// The first guide layer of a tile read as [face][p] (flux correction).
struct TileGuides {
  const double* T;
  const double* XG;  // [2][256]
  __device__ double operator[](int g) const {
    const int f = g >> 8, p = g & 255;
    return f < 2 ? XG[f * FACE_CELLS + p] : T[tile_guide(f, p)];
  }
};

__device__ __forceinline__ void consumer_sync() {
  asm volatile("bar.sync 1, %0;" ::"n"(NCONS) : "memory");
}
__device__ __forceinline__ void release_slot(uint64_t* bar, int lane, bool live) {
  async::fence_proxy_async();
  __syncwarp();
  if (lane == 0 && live) async::mbar_arrive(bar);
}
}  // namespace mvp

template <int NV, bool CF, typename ET, bool JAC = false>
__global__ void __launch_bounds__(mvp::NTHREADS, 1)
mx_matvec_pipe_kernel(MixCtx C, const ET* __restrict__ x, const double* __restrict__ A,
                      double* __restrict__ y, const double* __restrict__ w0, double omega) {
  using namespace mvp;
  static_assert(!(JAC && CF), "the Jacobi sweep has no flux correction");
  static_assert(NV >= (JAC ? 0 : 1) && NV <= (JAC ? 1 : 2), "sums of the kernel");
  using async::mbar_wait;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  Smem& S = *reinterpret_cast<Smem*>(smem_raw);
  const int tid = threadIdx.x;
  volatile int* abort_flag = &S.abort_flag;
  const int n_act = *C.n_active;
  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) {
      async::mbar_init(&S.full[s], 1);
      async::mbar_init(&S.empty[s], CONS_WARPS);
    }
    for (int b = 0; b < 2; ++b) {
      async::mbar_init(&S.gfull[b], NGATHER);
      async::mbar_init(&S.tempty[b], 1);
    }
    S.abort_flag = 0;
    async::fence_mbar_init();
  }
  // Counters that run across the chunks: ring slots issued (producer) or
  // consumed (consumers), blocks of earlier chunks.
  uint32_t g = 0;
  int M0 = 0;
  int run = 0;  // consumer 0: blocks of the current instance not yet on its ticket
  bool live = true;
  for (int from = blockIdx.x; from < n_act;) {
    build_live_list<1, false, NTHREADS, CAP>(C, from, n_act, S.list, &S.nlist, &S.next_from,
                                             S.wcount);
    from = S.next_from;
    const int nl = S.nlist;
    auto is_uni = [&](int n) { return (S.list[n].y & LF_UNI) != 0; };
    if (tid == 0 && nl > 0 && !*abort_flag) {
      // ------------------------------------------------------------ producer
      // (test hook MixCtx::stall == 2: no copy is issued, so the consumers'
      // first wait for a slot runs out)
      for (int n = 0; n < nl && C.stall != 2; ++n) {
        const size_t blk = (size_t)S.list[n].x;
        const int ns = is_uni(n) ? 1 : SLOTS;
        bool ok = true;
        for (int j = 0; j < ns; ++j, ++g) {
          const int s = g % STAGES;
          if (!(ok = mbar_wait(&S.empty[s], ((g / STAGES) & 1) ^ 1, abort_flag, ROLE_MATVEC,
                               C.wait_ns)))
            break;
          async::mbar_expect_tx(&S.full[s], SLOT_BYTES);
          if (ns == 1) {
            async::bulk_g2s(S.ring[s], w0 + blk * BLOCK_CELLS, SLOT_BYTES, &S.full[s]);
          } else {
#pragma unroll 1
            for (int a = 0; a < 7; ++a)
              async::bulk_g2s(S.ring[s][a], A + (blk * 7 + a) * BLOCK_CELLS + j * SLOT_CELLS,
                              SLOT_CELLS * 8, &S.full[s]);
            async::bulk_g2s(S.ring[s][7], w0 + blk * BLOCK_CELLS + j * SLOT_CELLS,
                            SLOT_CELLS * 8, &S.full[s]);
          }
        }
        if (!ok) break;
      }
    } else if (tid >= GATHER0 && tid < CONS0) {
      // ----------------------------------------------------------- gatherers
      const int gt = tid - GATHER0, grp = gt >> 7, p0 = gt & 127, p1 = p0 + 128;
      for (int n = 0; n < nl; ++n) {
        const int Mg = M0 + n, b = Mg & 1;
        const int blk = S.list[n].x;
        const double dx = C.dx[blk];
        // everything this thread writes into the tile, loaded before the tile
        // (block Mg - 2) is free: 16 values of x (cells gt + 256 m: a
        // half-warp's stores then fill 16 consecutive tile positions, one
        // bank each), and two positions of alternate faces of the guide layer
        ET xv[16];
        const ET* xb = x + (size_t)blk * BLOCK_CELLS;
#pragma unroll
        for (int m = 0; m < 16; ++m) xv[m] = __ldg(xb + gt + NGATHER * m);
        double gv[3][2];
        FaceNbr nfs[CF ? 3 : 1];
#pragma unroll
        for (int r = 0; r < 3; ++r) {
          const int f = 2 * r + grp;
          const FaceNbr nf = C.nbr[blk * 6 + f];
          guide_pair(x, blk, f, p0, p1, nf, C.bc, dx, gv[r][0], gv[r][1]);
          if (CF) nfs[CF ? r : 0] = nf;
        }
        const double ur = gt < 8 ? __ldg(C.ucoef + (size_t)blk * 8 + gt) : 0.0;
        if (Mg >= 2 &&
            !mbar_wait(&S.tempty[b], ((Mg - 2) >> 1) & 1, abort_flag, ROLE_MATVEC, C.wait_ns))
          break;
        double* T = S.tile[b];
#pragma unroll
        for (int m = 0; m < 16; ++m) {
          const int s0 = gt + NGATHER * m;
          const int c = s0 >> 11, q = s0 & 2047;
          const int ih = q & 7, j = (q >> 3) & 15, k = q >> 7;
          T[c * TH + (k + 1) * TP + (j + 1) * TR + ih] = (double)xv[m];
        }
#pragma unroll
        for (int r = 0; r < 3; ++r) {
          const int f = 2 * r + grp;
          if (f < 2) {
            S.xg[b][f][p0] = gv[r][0];
            S.xg[b][f][p1] = gv[r][1];
          } else {
            T[tile_guide(f, p0)] = gv[r][0];
            T[tile_guide(f, p1)] = gv[r][1];
          }
          if (CF && p0 == 0) S.snb[b][f] = nfs[CF ? r : 0];
        }
        if (gt < 8) S.urec[b][gt] = ur;
        async::mbar_arrive(&S.gfull[b]);
      }
    } else if (tid >= CONS0) {
      // ----------------------------------------------------------- consumers
      // Every consumer runs the same sequence of named barriers and shuffles;
      // only the work is predicated on 'live'.
      const int ct = tid - CONS0, lane = ct & 31, warp = ct >> 5;
      // this thread's cells q = 512 mm + ct: (2 ih + p, j, k0 + 4 mm), where
      // the parity p of the row is the same for every mm
      const int ih = ct & 7, jr = (ct >> 3) & 15, k0 = ct >> 7;
      const int pos0 = (k0 + 1) * TP + (jr + 1) * TR + ih;  // tile position, mm = 0
      for (int n = 0; n < nl; ++n) {
        const int Mg = M0 + n, b = Mg & 1;
        const uint32_t par = (Mg >> 1) & 1;
        const int2 ent = S.list[n];
        const int blk = ent.x, inst = ent.y & LF_INST;
        const bool uni = ent.y & LF_UNI;
        live = live && mbar_wait(&S.gfull[b], par, abort_flag, ROLE_MATVEC, C.wait_ns);
        const double* T = S.tile[b];
        const double* XG = &S.xg[b][0][0];
        double u[7];
#pragma unroll
        for (int a = 0; a < 7; ++a) u[a] = uni ? S.urec[b][a] : 0.0;
        const int us = g % STAGES;
        if (uni)
          live = live && mbar_wait(&S.full[us], (g / STAGES) & 1, abort_flag, ROLE_MATVEC,
                                   C.wait_ns);
        const double* wflat = &S.ring[us][0][0];
        const size_t base = (size_t)blk * BLOCK_CELLS;
        double acc[NV > 0 ? NV : 1][2] = {};
#pragma unroll
        for (int c = 0; c < 2; ++c) {
          const int p = (jr + k0 + c) & 1;
          const double* own = T + c * TH + pos0;         // the cell
          const double* oth = T + (1 - c) * TH + pos0;   // its position in the other colour
          // the x-face guides take the place of the west (i = 0) and east
          // (i = 15) neighbours
          const bool gw = ih == 0 && p == 0, ge = ih == 7 && p == 1;
#pragma unroll 2
          for (int mm = 0; mm < SLOTS / 2; ++mm) {
            const int q = mm * NCONS + ct, s = c * HALF_CELLS + q, o = mm * 4 * TP;
            const int gq = jr + 16 * (k0 + 4 * mm);  // the x-face guides' position
            double k[7], wv = 0.0;
            if (uni) {
#pragma unroll
              for (int a = 0; a < 7; ++a) k[a] = u[a];
              if (live) wv = wflat[s];
            } else {
              const int sl = g % STAGES;
              live = live && mbar_wait(&S.full[sl], (g / STAGES) & 1, abort_flag, ROLE_MATVEC,
                                       C.wait_ns);
#pragma unroll
              for (int a = 0; a < 7; ++a) k[a] = live ? S.ring[sl][a][ct] : 0.0;
              if (live) wv = S.ring[sl][7][ct];
              asm volatile("" ::"d"(k[0]), "d"(k[1]), "d"(k[2]), "d"(k[3]), "d"(k[4]), "d"(k[5]),
                           "d"(k[6]), "d"(wv));
              release_slot(&S.empty[sl], lane, live);
              ++g;
            }
            if (!live) continue;
            // neighbours w, e (i -+ 1: other colour, columns ih + p - 1 and
            // ih + p of it), s, n (rows -+ 1), b, t (planes -+ 1); the j and k
            // guides sit in the tile's border rows and planes
            const double xw = gw ? XG[gq] : oth[o - 1 + p];
            const double xe = ge ? XG[FACE_CELLS + gq] : oth[o + p];
            const double xs = oth[o - TR], xn = oth[o + TR];
            const double xb = oth[o - TP], xt = oth[o + TP];
            const double xp = own[o];
            double yv;
            if (JAC) {  // Jacobi sweep (bils.f90:5-55) with b = w0
              const double r = wv - k[1] * xw - k[2] * xe - k[3] * xs - k[4] * xn - k[5] * xb -
                               k[6] * xt;
              const double x_tmp = r / k[0];
              yv = xp - omega * (xp - x_tmp);
            } else {
              yv = k[1] * xw + k[2] * xe + k[3] * xs + k[4] * xn + k[5] * xb + k[6] * xt +
                   k[0] * xp;
              if (CF)  // coarse-fine flux correction: y = A x + delta
                yv = cf_delta<false>(x, (const double*)nullptr, A, C.nbr, C.dx, C.bc, S.snb[b],
                                     TileGuides{T, XG}, xp, s, yv,
                                     [&](int f) { return k[1 + f]; });
            }
            y[base + s] = yv;
            if (NV > 0) acc[0][c] += yv * wv;
            if (NV == 2) acc[NV - 1][c] += yv * yv;
          }
        }
        if (uni) {  // w0 is in registers (the loads completed before its use)
          release_slot(&S.empty[us], lane, live);
          ++g;
        }
        // block tree (mx_reduce with 512 threads): warp butterflies, then the
        // 16 warp sums in order
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          double t = acc[v][0] + acc[v][1];
#pragma unroll
          for (int off = 16; off >= 1; off >>= 1) t += __shfl_xor_sync(0xffffffffu, t, off);
          if (lane == 0) S.ws[b][v][warp] = t;
        }
        consumer_sync();  // every consumer is done with tile b
        if (ct == 0 && live) {
          async::mbar_arrive(&S.tempty[b]);
#pragma unroll
          for (int v = 0; v < NV; ++v) {
            double sum = 0.0;
#pragma unroll
            for (int w = 0; w < CONS_WARPS; ++w) sum += S.ws[b][v][w];
            __stcg(C.partials + (size_t)v * C.capacity + blk, sum);
          }
          ++run;
        }
        // the instance's ticket, once per run of its blocks in this chunk
        if (NV > 0 && (n + 1 == nl || (S.list[n + 1].y & LF_INST) != inst)) {
          if (ct == 0) {
            int li = -1;
            if (live && run > 0) {
              __threadfence();
              const unsigned t = atomicAdd(&C.inst.st[inst].ticket, (unsigned)run);
              if (t + (unsigned)run == (unsigned)C.inst.count[inst]) li = inst;
            }
            run = 0;
            S.last_inst = li;
          }
          consumer_sync();
          const int li = S.last_inst;
          if (li >= 0) {
            // cross-block sums over the instance's blocks: lanes 0..255, block
            // order, butterfly, 8 warp sums in order
            __threadfence();
            const int first = C.inst.first[li], cnt = C.inst.count[li];
            double tot[NV > 0 ? NV : 1];
#pragma unroll
            for (int v = 0; v < NV; ++v) {
              double sv = 0.0;
              if (ct < 256)
                for (int bb = ct; bb < cnt; bb += 256)
                  sv += __ldcg(C.partials + (size_t)v * C.capacity + first + bb);
#pragma unroll
              for (int off = 16; off >= 1; off >>= 1) sv += __shfl_xor_sync(0xffffffffu, sv, off);
              consumer_sync();
              if (lane == 0 && ct < 256) S.ws[b][0][ct >> 5] = sv;
              consumer_sync();
              double total = 0.0;
#pragma unroll
              for (int w = 0; w < 8; ++w) total += S.ws[b][0][w];
              tot[v] = total;
            }
            if (ct == 0) {
              SolveState* St = C.inst.st + li;
              if (C.fin) {  // the FP64 solver
                finalize(St, tot[0], C.fin, 0);
                if (NV == 2) finalize(St, tot[NV - 1], FIN_BI_TT, 0);
              } else if (!JAC) {
                mx_finalize(St, tot, NV == 1 ? FIN_MX_ALPHA : FIN_MX_GAMMA);
              }
              St->ticket = 0;
              __threadfence();
            }
            consumer_sync();  // S.ws is rewritten by the next block
          }
        }
      }
    }
    M0 += nl;
    __syncthreads();  // every role is past the chunk before its list is rebuilt
    if (*abort_flag) break;
  }
  if (tid == 0) {
    // Drain: the last armed phase of every ring slot must complete before the
    // CTA may exit (each has at most one copy phase in flight: a slot is
    // refilled only after its copy landed and was used).
    bool drained = true;
    for (int s = 0; s < STAGES; ++s) {
      const uint32_t issued = (g > (uint32_t)s) ? (g - 1 - s) / STAGES + 1 : 0;
      if (issued) drained = async::mbar_drain(&S.full[s], (issued - 1) & 1) && drained;
    }
    if (*abort_flag) {
      // stop every instance of this CTA's chunk and of its later candidates
      const int where = *abort_flag | (drained ? 0 : async::ROLE_DRAIN);
      auto stop = [&](int i2) {
        atomicOr(&C.inst.st[i2].timeout_where, where);
        atomicExch(&C.inst.st[i2].status, 3);
        atomicExch(&C.inst.st[i2].done, 1);
      };
      for (int k = 0; k < S.nlist; ++k) stop(S.list[k].y & LF_INST);
      for (int it2 = S.next_from; it2 < n_act; it2 += gridDim.x) {
        const int i2 = C.inst.blk_inst[C.active[it2]];
        if (i2 >= 0) stop(i2);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// x = alpha*p_ + gamma*s_ + x (axpbypz, blas.f90:431-464, FFVILS.h:938-944);
// r = (-gamma)*t_ + s (axpyz, blas.f90:397-429, FFVILS.h:945-950); r.r and
// the next iteration's r.r0.
// ---------------------------------------------------------------------------
template <typename ET, int NT>
__global__ void __launch_bounds__(NT)
mx_update_kernel(MixCtx C, double* __restrict__ x, const ET* __restrict__ ph,
                 const ET* __restrict__ sh, double* __restrict__ r,
                 const double* __restrict__ t, const double* __restrict__ s,
                 const double* __restrict__ r0) {
  const int tid = threadIdx.x;
  const int n_act = *C.n_active;
  for (int item = blockIdx.x; item < n_act; item += gridDim.x) {
    const int blk = C.active[item];
    const int inst = active_instance(C, blk);
    if (inst < 0) continue;
    const SolveState* S = C.inst.st + inst;
    const double alpha = S->alpha, gamma = S->gamma, mgamma = -S->gamma;
    const size_t base = (size_t)blk * BLOCK_CELLS;
    constexpr int VPT = 512 / NT;
    double acc[2][2][VPT] = {};
#pragma unroll
    for (int c = 0; c < 2; ++c) {
#pragma unroll 4
      for (int m = 0; m < HALF_CELLS / NT; ++m) {
        const size_t i = base + c * HALF_CELLS + tid + NT * m;
        x[i] = alpha * (double)ph[i] + gamma * (double)sh[i] + x[i];
        const double rn = mgamma * t[i] + s[i];
        r[i] = rn;
        acc[0][c][m % VPT] += rn * rn;
        acc[1][c][m % VPT] += rn * __ldg(r0 + i);
      }
    }
    mx_reduce<2, NT>(acc, C, blk, inst, FIN_MX_UPDATE);
    __syncthreads();  // the reduction's shared words are reused for the next block
  }
}

// ---------------------------------------------------------------------------
// Coarse-fine flux mismatch of an FP64 field with its stored guide layer:
// per (block, face) pair of kind NB_FINE and face position p = a + 16 b, the
// fine-side flux F of the coarse cell there and delta = F - A_f (g - x_P),
// out[(pair * 256 + p) * 2 + {0, 1}] = delta, F.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(FACE_CELLS)
cf_mismatch_kernel(const double* __restrict__ x, const double* __restrict__ gx,
                   const double* __restrict__ A, const FaceNbr* __restrict__ nbr,
                   const double* __restrict__ dx, BCSet bc, const int32_t* __restrict__ pairs,
                   double* __restrict__ out) {
  const int blk = pairs[2 * blockIdx.x], f = pairs[2 * blockIdx.x + 1];
  const int p = threadIdx.x, a = p & 15, b = p >> 4;
  const int axis = f >> 1, ta = (axis == 0) ? 1 : 0, tb = (axis == 2) ? 1 : 2;
  int c[3];
  c[ta] = a;
  c[tb] = b;
  c[axis] = (f & 1) ? 15 : 0;
  const int s = sidx(c[0], c[1], c[2]);
  const FaceNbr nb = nbr[(size_t)blk * 6 + f];
  const double F = cf_fine_flux(x, gx, A, nbr, dx, bc, f, a, b, nb);
  const double xp = x[(size_t)blk * BLOCK_CELLS + s];
  const double g = gx[((size_t)blk * 6 + f) * FACE_CELLS + p];
  const double af = A[((size_t)blk * 7 + 1 + f) * BLOCK_CELLS + s];
  const double d = F - af * (g - xp);
  out[((size_t)blockIdx.x * FACE_CELLS + p) * 2] = d;
  out[((size_t)blockIdx.x * FACE_CELLS + p) * 2 + 1] = F;
}

void launch_cf_mismatch(cudaStream_t s, int npairs, const double* x, const double* gx,
                        const double* A, const FaceNbr* nbr, const double* dx, const BCSet& bc,
                        const int32_t* pairs, double* out) {
  if (npairs > 0) cf_mismatch_kernel<<<npairs, FACE_CELLS, 0, s>>>(x, gx, A, nbr, dx, bc, pairs, out);
}

// ---------------------------------------------------------------------------
// Launchers.
// ---------------------------------------------------------------------------
void launch_mx_pack(cudaStream_t s, int first, int count, const double* A, uint32_t* coef,
                    double* coef64, double* ucoef, SolveState* st, bool d64, int sweep_threads) {
  if (d64 && sweep_threads == 256)
    mx_pack_kernel<true, 256><<<count, MT, 0, s>>>(first, A, coef, coef64, ucoef, st);
  else if (d64)
    mx_pack_kernel<true, 512><<<count, MT, 0, s>>>(first, A, coef, coef64, ucoef, st);
  else if (sweep_threads == 256)
    mx_pack_kernel<false, 256><<<count, MT, 0, s>>>(first, A, coef, coef64, ucoef, st);
  else
    mx_pack_kernel<false, 512><<<count, MT, 0, s>>>(first, A, coef, coef64, ucoef, st);
}
void launch_mx_init(cudaStream_t s, const MixCtx& C, int count, const double* x,
                    const double* gx, const double* A, const double* b, double* r, double* r0) {
  mx_init_kernel<<<count, MT, 0, s>>>(C, x, gx, A, b, r, r0);
}

template <int MODE, bool FIRST, typename ET>
static void sweep_launch(cudaStream_t s, const MixCtx& C, int count, float omega, int nsweep,
                         const double* r, double* r0, double* pv, const double* q,
                         const uint32_t* coef, const double* coef64, const void* ein,
                         const double* guides, void* eout) {
  if (C.sweep_threads == 256)
    mx_sweep_kernel<MODE, FIRST, ET, 256><<<count, 256, SWEEP_SMEM, s>>>(
        C, omega, nsweep, r, r0, pv, q, coef, coef64, static_cast<const ET*>(ein), guides,
        static_cast<ET*>(eout), C.depth);
  else
    mx_sweep_kernel<MODE, FIRST, ET, 512><<<count, 512, SWEEP_SMEM, s>>>(
        C, omega, nsweep, r, r0, pv, q, coef, coef64, static_cast<const ET*>(ein), guides,
        static_cast<ET*>(eout), C.depth);
}

void launch_mx_sweep(cudaStream_t s, const MixCtx& C, int count, int mode, bool first,
                     float omega, int nsweep, const double* r, double* r0, double* pv,
                     const double* q, const uint32_t* coef, const double* coef64,
                     const void* ein, const double* guides, void* eout, bool d64) {
#define MX_SWEEP(M, F, T) \
  sweep_launch<M, F, T>(s, C, count, omega, nsweep, r, r0, pv, q, coef, coef64, ein, guides, eout)
  if (!d64) {
    if (mode == 0 && first) MX_SWEEP(0, true, float);
    if (mode == 0 && !first) MX_SWEEP(0, false, float);
    if (mode == 1 && first) MX_SWEEP(1, true, float);
    if (mode == 1 && !first) MX_SWEEP(1, false, float);
  } else {
    if (mode == 0 && first) MX_SWEEP(0, true, double);
    if (mode == 0 && !first) MX_SWEEP(0, false, double);
    if (mode == 1 && first) MX_SWEEP(1, true, double);
    if (mode == 1 && !first) MX_SWEEP(1, false, double);
  }
#undef MX_SWEEP
}

void launch_mx_guides(cudaStream_t s, const MixCtx& C, int count, const void* e, double* guides,
                      bool d64) {
  if (d64)
    mx_guides_kernel<double><<<count, GT, 0, s>>>(C, static_cast<const double*>(e), guides);
  else
    mx_guides_kernel<float><<<count, GT, 0, s>>>(C, static_cast<const float*>(e), guides);
}

template <typename K>
static void allow_sweep_smem(K kernel) {
  cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, SWEEP_SMEM);
}

void mx_grid_sizes(int threads, int* sweep, int* matvec, int* update, int* guides, int* mvpipe) {
  int dev = 0, sms = 0, a = 0, b = 0, c = 0, d = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // the sweep kernels' shared memory, on the calling device (before any launch)
#define MX_ALLOW(PTS)                                    \
  allow_sweep_smem(mx_sweep_kernel<0, true, float, PTS>);  \
  allow_sweep_smem(mx_sweep_kernel<0, false, float, PTS>); \
  allow_sweep_smem(mx_sweep_kernel<1, true, float, PTS>);  \
  allow_sweep_smem(mx_sweep_kernel<1, false, float, PTS>); \
  allow_sweep_smem(mx_sweep_kernel<0, true, double, PTS>); \
  allow_sweep_smem(mx_sweep_kernel<0, false, double, PTS>); \
  allow_sweep_smem(mx_sweep_kernel<1, true, double, PTS>); \
  allow_sweep_smem(mx_sweep_kernel<1, false, double, PTS>);
  MX_ALLOW(512)
  MX_ALLOW(256)
#undef MX_ALLOW
  // one CTA per SM for either thread count (its shared memory)
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, mx_sweep_kernel<0, true, float, 512>, 512,
                                                SWEEP_SMEM);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, mx_sweep_kernel<1, false, float, 256>, 256,
                                                SWEEP_SMEM);
  if (threads == 128) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c, mx_matvec_kernel<2, false, float, 128>,
                                                  128, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&d, mx_update_kernel<float, 128>, 128, 0);
  } else if (threads == 512) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c, mx_matvec_kernel<2, false, float, 512>,
                                                  512, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&d, mx_update_kernel<float, 512>, 512, 0);
  } else {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c, mx_matvec_kernel<2, false, float, 256>,
                                                  256, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&d, mx_update_kernel<float, 256>, 256, 0);
  }
  *sweep = sms * std::max(1, std::min(a, b));
  int g = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&g, mx_guides_kernel<float>, GT, 0);
  *guides = sms * std::max(1, g);
  *matvec = sms * std::max(1, c);
  *update = sms * std::max(1, d);
  // the pipelined A*x: its shared memory on this device, one CTA per SM
#define MV_ALLOW(NV, CF, ET, JAC)                                                      \
  cudaFuncSetAttribute(mx_matvec_pipe_kernel<NV, CF, ET, JAC>,                          \
                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(mvp::Smem));
  MV_ALLOW(1, false, float, false) MV_ALLOW(2, false, float, false)
  MV_ALLOW(1, true, float, false) MV_ALLOW(2, true, float, false)
  MV_ALLOW(1, false, double, false) MV_ALLOW(2, false, double, false)
  MV_ALLOW(1, true, double, false) MV_ALLOW(2, true, double, false)
  MV_ALLOW(0, false, double, true) MV_ALLOW(1, false, double, true)
#undef MV_ALLOW
  *mvpipe = sms;
}

template <typename ET, int NT>
static void matvec_launch(cudaStream_t s, const MixCtx& C, int count, int ndot, const ET* x,
                          const double* A, double* y, const double* w0) {
  if (ndot == 1 && !C.cf)
    mx_matvec_kernel<1, false, ET, NT><<<count, NT, 0, s>>>(C, x, A, y, w0);
  else if (!C.cf)
    mx_matvec_kernel<2, false, ET, NT><<<count, NT, 0, s>>>(C, x, A, y, w0);
  else if (ndot == 1)
    mx_matvec_kernel<1, true, ET, NT><<<count, NT, 0, s>>>(C, x, A, y, w0);
  else
    mx_matvec_kernel<2, true, ET, NT><<<count, NT, 0, s>>>(C, x, A, y, w0);
}

template <typename ET>
static void matvec_nt(cudaStream_t s, const MixCtx& C, int count, int ndot, int threads,
                      const ET* x, const double* A, double* y, const double* w0) {
  if (threads == 128)
    matvec_launch<ET, 128>(s, C, count, ndot, x, A, y, w0);
  else if (threads == 512)
    matvec_launch<ET, 512>(s, C, count, ndot, x, A, y, w0);
  else
    matvec_launch<ET, 256>(s, C, count, ndot, x, A, y, w0);
}

// The active list with the blocks that stream their coefficients first:
// one CTA, a stable partition chunk by chunk (warp ballots, warp offsets in
// order), so the order is the same on every run.
__global__ void __launch_bounds__(1024)
mx_order_active_kernel(const int32_t* __restrict__ raw, const double* __restrict__ ucoef,
                       int32_t* __restrict__ act) {
  __shared__ int ws[32], wu[32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int n = raw[0];
  auto streams = [&](int b) { return ucoef[(size_t)b * 8 + 7] == 0.0; };
  int cnt = 0;
  for (int i = tid; i < n; i += 1024) cnt += streams(raw[1 + i]) ? 1 : 0;
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, off);
  if (lane == 0) ws[warp] = cnt;
  __syncthreads();
  int nstream = 0;
  for (int w = 0; w < 32; ++w) nstream += ws[w];
  __syncthreads();
  int base_s = 0, base_u = nstream;
  const unsigned below = (1u << lane) - 1u;
  for (int c0 = 0; c0 < n; c0 += 1024) {
    const int i = c0 + tid;
    const int b = i < n ? raw[1 + i] : 0;
    const bool st = i < n && streams(b), un = i < n && !st;
    const unsigned ms = __ballot_sync(0xffffffffu, st), mu = __ballot_sync(0xffffffffu, un);
    if (lane == 0) {
      ws[warp] = __popc(ms);
      wu[warp] = __popc(mu);
    }
    __syncthreads();
    int os = base_s, ou = base_u, ts = 0, tu = 0;
    for (int w = 0; w < 32; ++w) {
      if (w < warp) {
        os += ws[w];
        ou += wu[w];
      }
      ts += ws[w];
      tu += wu[w];
    }
    if (st) act[1 + os + __popc(ms & below)] = b;
    if (un) act[1 + ou + __popc(mu & below)] = b;
    base_s += ts;
    base_u += tu;
    __syncthreads();  // ws, wu are rewritten by the next chunk
  }
  if (tid == 0) act[0] = n;
}

void launch_mx_order_active(cudaStream_t s, const int32_t* raw, const double* ucoef,
                            int32_t* act) {
  mx_order_active_kernel<<<1, 1024, 0, s>>>(raw, ucoef, act);
}

template <typename ET>
static void matvec_pipe(cudaStream_t s, const MixCtx& C, int count, int ndot, const ET* x,
                        const double* A, double* y, const double* w0) {
  constexpr int T = mvp::NTHREADS, B = (int)sizeof(mvp::Smem);
  if (ndot == 1 && !C.cf)
    mx_matvec_pipe_kernel<1, false, ET><<<count, T, B, s>>>(C, x, A, y, w0, 0.0);
  else if (!C.cf)
    mx_matvec_pipe_kernel<2, false, ET><<<count, T, B, s>>>(C, x, A, y, w0, 0.0);
  else if (ndot == 1)
    mx_matvec_pipe_kernel<1, true, ET><<<count, T, B, s>>>(C, x, A, y, w0, 0.0);
  else
    mx_matvec_pipe_kernel<2, true, ET><<<count, T, B, s>>>(C, x, A, y, w0, 0.0);
}

void launch_jacobi_pipe(cudaStream_t s, const MixCtx& C, int count, bool dot, const double* x,
                        const double* A, const double* b, double* y, double omega) {
  constexpr int T = mvp::NTHREADS, B = (int)sizeof(mvp::Smem);
  if (dot)
    mx_matvec_pipe_kernel<1, false, double, true><<<count, T, B, s>>>(C, x, A, y, b, omega);
  else
    mx_matvec_pipe_kernel<0, false, double, true><<<count, T, B, s>>>(C, x, A, y, b, omega);
}

void launch_mx_matvec(cudaStream_t s, const MixCtx& C, int count, int ndot, int threads, int form,
                      const void* x, const double* A, double* y, const double* w0, bool d64) {
  if (form == 0 && d64)
    matvec_pipe(s, C, count, ndot, static_cast<const double*>(x), A, y, w0);
  else if (form == 0)
    matvec_pipe(s, C, count, ndot, static_cast<const float*>(x), A, y, w0);
  else if (d64)
    matvec_nt(s, C, count, ndot, threads, static_cast<const double*>(x), A, y, w0);
  else
    matvec_nt(s, C, count, ndot, threads, static_cast<const float*>(x), A, y, w0);
}

template <typename ET>
static void update_nt(cudaStream_t s, const MixCtx& C, int count, int threads, double* x,
                      const ET* ph, const ET* sh, double* r, const double* t, const double* sv,
                      const double* r0) {
  if (threads == 128)
    mx_update_kernel<ET, 128><<<count, 128, 0, s>>>(C, x, ph, sh, r, t, sv, r0);
  else if (threads == 512)
    mx_update_kernel<ET, 512><<<count, 512, 0, s>>>(C, x, ph, sh, r, t, sv, r0);
  else
    mx_update_kernel<ET, 256><<<count, 256, 0, s>>>(C, x, ph, sh, r, t, sv, r0);
}

void launch_mx_update(cudaStream_t s, const MixCtx& C, int count, int threads, double* x,
                      const void* ph, const void* sh, double* r, const double* t,
                      const double* sv, const double* r0, bool d64) {
  if (d64)
    update_nt(s, C, count, threads, x, static_cast<const double*>(ph),
              static_cast<const double*>(sh), r, t, sv, r0);
  else
    update_nt(s, C, count, threads, x, static_cast<const float*>(ph),
              static_cast<const float*>(sh), r, t, sv, r0);
}

}  // namespace ffvgpu
