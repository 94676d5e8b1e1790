// kernels_mixed.cu -- the mixed-precision form of the pressure solve, with
// the per-instance bookkeeping that lets one launch serve a batch of
// independent problems (sm_100a).
//
// The outer iteration is FFVILS::BiCGSTAB's recurrence (src/FFV/FFVILS.h:
// 793-974) in FP64: residuals, norms, dot products and the pressure update
// keep the reference's per-cell expressions and are compiled with
// --fmad=false.  Its preconditioner -- FFVILS's Jacobi_PreConditioner
// (FFVILS.h:469-492) in the reference -- is replaced by red-black SOR sweeps
// in FP32 that solve A e = v approximately from e = 0: 'sweeps' colour pairs
// per application, grouped 'per_exchange' at a time between guide-cell
// exchanges.  Inside a group a block sweeps against fixed guide values, so
// the whole group runs on chip: one CTA per block keeps the block's FP32
// coefficients in registers and its iterate in shared memory, and HBM sees
// one read of the coefficients and one write of the result per group.
//
// Sweep of one cell (colour order and neighbour terms as rbgs_smoother,
// src/CGMfuncs/bils.f90:57-108) on FP32 data -- coefficients, right-hand
// side and iterate are FP32 values -- with the update formed in FP64 and
// rounded to FP32 once, when it is stored:
//   rc = v; rc = fma(-aw, eW, rc); ... fma(-ab, eB, rc); fma(-at, eT, rc)
//   xt = rc * dinv                       (dinv = (float)(1.0 / Ap))
//   e  = (float)fma(-omega, e - xt, e)   (e - omega (e - xt))
// Forming rc in FP32 would cancel: once a block has nearly converged locally
// rc is far smaller than its terms, and its FP32 rounding error (1e-5 and
// more relative) makes the preconditioner visibly nonlinear, which the
// BiCGSTAB recurrence does not survive; in FP64 the only nonlinearity left
// is the final rounding of each stored value.
// Guide cells of e: the exchange rules (same-level copy, 2:1 interpolation
// and restriction, src/CGMfuncs/sup.f90) evaluated in FP64 on the FP32
// values and rounded to FP32; outer faces take homogeneous Dirichlet values.
//
// Every sum is the canonical tree of the layout header taken over one
// instance's blocks, so an instance gets the same bits alone or in a batch.
#include <algorithm>
#include <cfloat>
#include <cuda_runtime.h>

#include "ffvgpu_internal.cuh"
#include "ffvgpu_mixed.h"

namespace ffvgpu {

namespace {

constexpr int MT = 256;  // FP64 kernels: 16 cells per thread
constexpr int PT = 512;  // FP32 sweep kernel: 8 cells per thread

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

// Canonical block sums of NV values (acc[v][colour][virtual thread r or
// r + 256]), per-instance ticket, and the last CTA's cross-block sums over
// the instance's blocks in block order.
template <int NV>
__device__ void mx_reduce(double (&acc)[NV][2][2], const MixCtx& C, int blk, int inst, int fin) {
  __shared__ double ws[NV][16];
  __shared__ int amlast;
  const int tid = threadIdx.x;
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    double v0 = acc[v][0][0] + acc[v][1][0], v1 = acc[v][0][1] + acc[v][1][1];
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) {
      v0 += __shfl_xor_sync(0xffffffffu, v0, off);
      v1 += __shfl_xor_sync(0xffffffffu, v1, off);
    }
    if ((tid & 31) == 0) {
      ws[v][tid >> 5] = v0;
      ws[v][8 + (tid >> 5)] = v1;
    }
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
    double s = 0.0;
    for (int b = tid; b < cnt; b += MT) s += __ldcg(C.partials + (size_t)v * C.capacity + first + b);
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    __syncthreads();
    if ((tid & 31) == 0) ws[0][tid >> 5] = s;
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

// Stages block blk of an FP32 vector as FP64: the colour-split interior in
// O[4096] and the first guide layer in G[6][256], guides by the exchange
// rules in FP64 (outer faces by the field's BCs).
__device__ __forceinline__ void stage_f32_as_f64(double* __restrict__ O, double* __restrict__ G,
                                                 const float* __restrict__ x, int blk,
                                                 const MixCtx& C) {
  const int tid = threadIdx.x;
  const float* xb = x + (size_t)blk * BLOCK_CELLS;
#pragma unroll 4
  for (int m = 0; m < 16; ++m) O[tid + MT * m] = (double)__ldg(xb + tid + MT * m);
  const double dx = C.dx[blk];
#pragma unroll 1
  for (int it = 0; it < 3; ++it) {
    const int f = 2 * it + (tid >> 7), p0 = tid & 127, p1 = p0 + 128;
    const FaceNbr nb = C.nbr[blk * 6 + f];
    double v0, v1;
    guide_pair(x, blk, f, p0, p1, nb, C.bc, dx, v0, v1);
    G[f * FACE_CELLS + p0] = v0;
    G[f * FACE_CELLS + p1] = v1;
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// FP32 coefficients of the sweeps: [blk][7][4096] = aw, ae, as, an, ab, at,
// dinv, colour-split like every field.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(MT)
mx_pack_kernel(int first, const double* __restrict__ A, float* __restrict__ coef) {
  const int blk = first + blockIdx.x;
  const double* Ab = A + (size_t)blk * 7 * BLOCK_CELLS;
  float* cb = coef + (size_t)blk * 7 * BLOCK_CELLS;
#pragma unroll 2
  for (int m = 0; m < 16; ++m) {
    const int s = threadIdx.x + MT * m;
#pragma unroll
    for (int a = 0; a < 6; ++a) cb[a * BLOCK_CELLS + s] = (float)Ab[(1 + a) * BLOCK_CELLS + s];
    cb[6 * BLOCK_CELLS + s] = (float)(1.0 / Ab[s]);
  }
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
  const int tid = threadIdx.x;
  const size_t base = (size_t)blk * BLOCK_CELLS;
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
      const double rv = __ldg(bvec + base + s) - __ldg(Ab + 4096 + s) * v.w -
                        __ldg(Ab + 8192 + s) * v.e - __ldg(Ab + 12288 + s) * v.s -
                        __ldg(Ab + 16384 + s) * v.n - __ldg(Ab + 20480 + s) * v.b -
                        __ldg(Ab + 24576 + s) * v.t - __ldg(Ab + s) * O[s];
      r[base + s] = rv;
      r0[base + s] = rv;
      const double bv = __ldg(bvec + base + s);
      acc[0][c][m & 1] += bv * bv;
      acc[1][c][m & 1] += rv * rv;
    }
  }
  mx_reduce<2>(acc, C, blk, inst, FIN_MX_INIT);
}

// ---------------------------------------------------------------------------
// One pass of FP32 sweeps.  MODE 0: right-hand side p (FFVILS.h:853-871:
// p = r at the first iteration of a cycle, which also sets r0 = r, else
// p = r + beta*(p + (-gamma)*q)); MODE 1: right-
// hand side s = (-alpha)*q + r (FFVILS.h:898-903).  FIRST: the pass that
// forms the right-hand side (writes p or s in FP64, and its FP32 copy when
// more passes follow) and starts from e = 0 with zero guides.  LAST: writes
// the preconditioned vector; otherwise the pass's iterate for the next.
// ---------------------------------------------------------------------------
template <int MODE, bool FIRST, bool LAST>
__global__ void __launch_bounds__(PT, 1)
mx_sweep_kernel(MixCtx C, float omega, int nsweep, const double* __restrict__ r,
                double* __restrict__ r0, double* __restrict__ pv, const double* __restrict__ q,
                const float* __restrict__ coef, float* __restrict__ v32,
                const float* __restrict__ ein, float* __restrict__ eout) {
  __shared__ float E[BLOCK_CELLS];
  __shared__ float G[6 * FACE_CELLS];
  const int tid = threadIdx.x;
  const double mom = -(double)omega;
  const int n_act = *C.n_active;
  for (int item = blockIdx.x; item < n_act; item += gridDim.x) {
    const int blk = C.active[item];
    const int inst = active_instance(C, blk);
    if (inst < 0) continue;
    const size_t base = (size_t)blk * BLOCK_CELLS;
    // this thread's cells: storage slots tid + 512*m, colour m >> 2
    float cf[8][7];
    const float* cb = coef + (size_t)blk * 7 * BLOCK_CELLS;
#pragma unroll
    for (int m = 0; m < 8; ++m)
#pragma unroll
      for (int a = 0; a < 7; ++a) cf[m][a] = __ldg(cb + a * BLOCK_CELLS + tid + PT * m);
    float v[8];
    if (FIRST) {
      const SolveState* S = C.inst.st + inst;
      const bool copy = S->cycle == 1;  // first iteration of a (re)start: p = r, r0 = r
      const double mgamma = -S->gamma, beta = S->beta, malpha = -S->alpha;
#pragma unroll
      for (int m = 0; m < 8; ++m) {
        const size_t s = base + tid + PT * m;
        double rhs;
        if (MODE == 0) {
          if (copy) {
            rhs = r[s];
            r0[s] = rhs;
          } else {
            const double t = pv[s] + mgamma * q[s];
            rhs = r[s] + beta * t;
          }
        } else {
          rhs = malpha * q[s] + r[s];
        }
        pv[s] = rhs;
        v[m] = (float)rhs;
        if (!LAST) v32[s] = v[m];
        E[tid + PT * m] = 0.0f;
      }
      for (int g = tid; g < 6 * FACE_CELLS; g += PT) G[g] = 0.0f;
    } else {
#pragma unroll
      for (int m = 0; m < 8; ++m) {
        v[m] = __ldg(v32 + base + tid + PT * m);
        E[tid + PT * m] = __ldg(ein + base + tid + PT * m);
      }
      BCSet hom;
      for (int f = 0; f < 6; ++f) {
        hom.type[f] = BC_DIRICHLET;
        hom.value[f] = 0.0;
      }
      const double dx = C.dx[blk];
      if (tid < 3 * 128) {
        const int f = 2 * (tid >> 7), p0 = tid & 127, p1 = p0 + 128;
        for (int h = 0; h < 2; ++h) {
          const FaceNbr nb = C.nbr[blk * 6 + f + h];
          double g0, g1;
          guide_pair(ein, blk, f + h, p0, p1, nb, hom, dx, g0, g1);
          G[(f + h) * FACE_CELLS + p0] = (float)g0;
          G[(f + h) * FACE_CELLS + p1] = (float)g1;
        }
      }
    }
    __syncthreads();
#pragma unroll 1
    for (int it = 0; it < nsweep; ++it) {
#pragma unroll
      for (int c = 0; c < 2; ++c) {
#pragma unroll
        for (int h = 0; h < 4; ++h) {
          const int m = 4 * c + h;
          const int qd = tid + PT * h;
          const NbrsT<float> nb = split_neighbours(E + (1 - c) * HALF_CELLS, G, qd, c);
          double rc = (double)v[m];
          rc = __fma_rn(-(double)cf[m][0], (double)nb.w, rc);
          rc = __fma_rn(-(double)cf[m][1], (double)nb.e, rc);
          rc = __fma_rn(-(double)cf[m][2], (double)nb.s, rc);
          rc = __fma_rn(-(double)cf[m][3], (double)nb.n, rc);
          rc = __fma_rn(-(double)cf[m][4], (double)nb.b, rc);
          rc = __fma_rn(-(double)cf[m][5], (double)nb.t, rc);
          const double xt = __dmul_rn(rc, (double)cf[m][6]);
          const double e = (double)E[c * HALF_CELLS + qd];
          E[c * HALF_CELLS + qd] = __double2float_rn(__fma_rn(mom, __dsub_rn(e, xt), e));
        }
        __syncthreads();
      }
    }
#pragma unroll
    for (int m = 0; m < 8; ++m) eout[base + tid + PT * m] = E[tid + PT * m];
    __syncthreads();  // E and G are refilled for the next block
  }
}

// ---------------------------------------------------------------------------
// y = A x for an FP32 x, in FP64 (calc_ax, bils.f90:162-206), with its dot
// products.  NV = 1: y.w0 (q_.r0, FFVILS.h:890-896).  NV = 2: y.w0 and y.y
// (t_.s and t_.t_, FFVILS.h:923-936).
// ---------------------------------------------------------------------------
template <int NV>
__global__ void __launch_bounds__(MT)
mx_matvec_kernel(MixCtx C, const float* __restrict__ x, const double* __restrict__ A,
                 double* __restrict__ y, const double* __restrict__ w0) {
  __shared__ double O[BLOCK_CELLS];
  __shared__ double G[6 * FACE_CELLS];
  const int tid = threadIdx.x;
  const int n_act = *C.n_active;
  for (int item = blockIdx.x; item < n_act; item += gridDim.x) {
    const int blk = C.active[item];
    const int inst = active_instance(C, blk);
    if (inst < 0) continue;
    stage_f32_as_f64(O, G, x, blk, C);
    __syncthreads();
    const size_t base = (size_t)blk * BLOCK_CELLS;
    const double* Ab = A + (size_t)blk * 7 * BLOCK_CELLS;
    double acc[NV][2][2] = {};
#pragma unroll
    for (int c = 0; c < 2; ++c) {
#pragma unroll 2
      for (int m = 0; m < 8; ++m) {
        const int qd = tid + MT * m, s = c * HALF_CELLS + qd;
        const Nbrs v = split_neighbours(O + (1 - c) * HALF_CELLS, G, qd, c);
        const double yv = __ldg(Ab + 4096 + s) * v.w + __ldg(Ab + 8192 + s) * v.e +
                          __ldg(Ab + 12288 + s) * v.s + __ldg(Ab + 16384 + s) * v.n +
                          __ldg(Ab + 20480 + s) * v.b + __ldg(Ab + 24576 + s) * v.t +
                          __ldg(Ab + s) * O[s];
        y[base + s] = yv;
        acc[0][c][m & 1] += yv * __ldg(w0 + base + s);
        if (NV == 2) acc[NV - 1][c][m & 1] += yv * yv;
      }
    }
    mx_reduce<NV>(acc, C, blk, inst, NV == 1 ? FIN_MX_ALPHA : FIN_MX_GAMMA);
    __syncthreads();  // O and G are refilled for the next block
  }
}

// ---------------------------------------------------------------------------
// x = alpha*p_ + gamma*s_ + x (axpbypz, blas.f90:431-464, FFVILS.h:938-944);
// r = (-gamma)*t_ + s (axpyz, blas.f90:397-429, FFVILS.h:945-950); r.r and
// the next iteration's r.r0.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(MT)
mx_update_kernel(MixCtx C, double* __restrict__ x, const float* __restrict__ ph,
                 const float* __restrict__ sh, double* __restrict__ r,
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
    double acc[2][2][2] = {};
#pragma unroll
    for (int c = 0; c < 2; ++c) {
#pragma unroll 4
      for (int m = 0; m < 8; ++m) {
        const size_t i = base + c * HALF_CELLS + tid + MT * m;
        x[i] = alpha * (double)ph[i] + gamma * (double)sh[i] + x[i];
        const double rn = mgamma * t[i] + s[i];
        r[i] = rn;
        acc[0][c][m & 1] += rn * rn;
        acc[1][c][m & 1] += rn * __ldg(r0 + i);
      }
    }
    mx_reduce<2>(acc, C, blk, inst, FIN_MX_UPDATE);
    __syncthreads();  // the reduction's shared words are reused for the next block
  }
}

// ---------------------------------------------------------------------------
// Launchers.
// ---------------------------------------------------------------------------
void launch_mx_pack(cudaStream_t s, int first, int count, const double* A, float* coef) {
  mx_pack_kernel<<<count, MT, 0, s>>>(first, A, coef);
}
void launch_mx_init(cudaStream_t s, const MixCtx& C, int count, const double* x,
                    const double* gx, const double* A, const double* b, double* r, double* r0) {
  mx_init_kernel<<<count, MT, 0, s>>>(C, x, gx, A, b, r, r0);
}

template <int MODE, bool FIRST, bool LAST>
static void sweep_launch(cudaStream_t s, const MixCtx& C, int count, float omega, int nsweep,
                         const double* r, double* r0, double* pv, const double* q,
                         const float* coef, float* v32, const float* ein, float* eout) {
  mx_sweep_kernel<MODE, FIRST, LAST>
      <<<count, PT, 0, s>>>(C, omega, nsweep, r, r0, pv, q, coef, v32, ein, eout);  // count: CTAs
}

void launch_mx_sweep(cudaStream_t s, const MixCtx& C, int count, int mode, bool first, bool last,
                     float omega, int nsweep, const double* r, double* r0, double* pv,
                     const double* q, const float* coef, float* v32, const float* ein,
                     float* eout) {
#define MX_CASE(M, F, L)                                                                   \
  if (mode == M && first == F && last == L) {                                              \
    sweep_launch<M, F, L>(s, C, count, omega, nsweep, r, r0, pv, q, coef, v32, ein, eout); \
    return;                                                                                \
  }
  MX_CASE(0, true, true) MX_CASE(0, true, false) MX_CASE(0, false, true) MX_CASE(0, false, false)
  MX_CASE(1, true, true) MX_CASE(1, true, false) MX_CASE(1, false, true) MX_CASE(1, false, false)
#undef MX_CASE
}

void mx_grid_sizes(int* sweep, int* matvec, int* update) {
  int dev = 0, sms = 0, a = 0, b = 0, c = 0, d = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, mx_sweep_kernel<0, true, true>, PT, 0);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, mx_sweep_kernel<1, false, true>, PT, 0);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c, mx_matvec_kernel<2>, MT, 0);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&d, mx_update_kernel, MT, 0);
  *sweep = sms * std::max(1, std::min(a, b));
  *matvec = sms * std::max(1, c);
  *update = sms * std::max(1, d);
}

void launch_mx_matvec(cudaStream_t s, const MixCtx& C, int count, int ndot, const float* x,
                      const double* A, double* y, const double* w0) {
  if (ndot == 1)
    mx_matvec_kernel<1><<<count, MT, 0, s>>>(C, x, A, y, w0);
  else
    mx_matvec_kernel<2><<<count, MT, 0, s>>>(C, x, A, y, w0);
}

void launch_mx_update(cudaStream_t s, const MixCtx& C, int count, double* x, const float* ph,
                      const float* sh, double* r, const double* t, const double* sv,
                      const double* r0) {
  mx_update_kernel<<<count, MT, 0, s>>>(C, x, ph, sh, r, t, sv, r0);
}

}  // namespace ffvgpu
