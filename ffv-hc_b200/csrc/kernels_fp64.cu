// kernels_fp64.cu -- FP64 kernels of the pressure-Poisson path (sm_100a).
//
// Compiled with --fmad=false: every product and sum is rounded separately,
// and every expression keeps the reference's left-to-right order, so a
// kernel's per-cell results equal the reference's bit for bit
// (src/CGMfuncs/bils.f90, blas.f90, sup.f90, bcx.f90, bca.f90 and
// src/FFV/bcut.f90, all built by the reference without FMA contraction).
//
// One CTA of 256 threads owns one 16^3 leaf block.  Stencil kernels stage
// the block's vector in shared memory as an 18^3 tile whose guide layer is
// computed from the neighbours' interiors (the exchange) or, on the first
// use of a field, read from its stored guide layer.  Sums use a fixed tree:
// per thread two serial sums over its 8 cells of each colour, an xor
// butterfly over the warp, a serial sum over the 8 warps, and across blocks
// the same shape over the per-block partials, run by the CTA that finishes
// last (ticket counter), which also advances the solver state.
#include <cfloat>
#include <cstdio>
#include <cuda_runtime.h>

#include "ffvgpu_internal.cuh"
#include "ffvgpu_kernels.h"

namespace ffvgpu {

constexpr int TW = 18;          // tile edge (16 + 2 guide cells)
constexpr int TP = TW * TW;     // tile plane
constexpr int TILE = TW * TW * TW;

__device__ __forceinline__ int tix(int i, int j, int k) {  // 0-based interior coords
  return (i + 1) + TW * (j + 1) + TP * (k + 1);
}

__device__ __forceinline__ bool solve_done(const SolveState* st) {
  return *((volatile const int32_t*)&st->done) != 0;
}

// Guide-cell position of face f at transverse (a, b), layer 1.
__device__ __forceinline__ int guide_tix(int f, int a, int b) {
  switch (f) {
    case X_M: return tix(-1, a, b);
    case X_P: return tix(16, a, b);
    case Y_M: return tix(a, -1, b);
    case Y_P: return tix(a, 16, b);
    case Z_M: return tix(a, b, -1);
    default:  return tix(a, b, 16);
  }
}

// Stage block 'blk' of x in the shared tile, guide layer included.  The
// interior's sixteen loads per thread are issued together, and the guide
// layer as pairs of positions of a face (guide_pair: the same values as
// guide_value) with the three pairs' loads in flight together.
__device__ __forceinline__ void stage_tile(double* __restrict__ xs, const double* __restrict__ x,
                                           int blk, const KCtx& C, const double* __restrict__ gst) {
  const int tid = threadIdx.x;
  const double* xb = x + (size_t)blk * BLOCK_CELLS;
  double v[16];
#pragma unroll
  for (int m = 0; m < 16; ++m) v[m] = __ldg(xb + tid + THREADS * m);
#pragma unroll
  for (int m = 0; m < 16; ++m) {
    int i, j, k;
    cell_of(tid + THREADS * m, i, j, k);
    xs[tix(i, j, k)] = v[m];
  }
#pragma unroll
  for (int it = 0; it < 3; ++it) {
    const int f = 2 * it + (tid >> 7), p0 = tid & 127, p1 = p0 + 128;
    double g0, g1;
    if (gst) {
      g0 = __ldg(gst + ((size_t)blk * 6 + f) * FACE_CELLS + p0);
      g1 = __ldg(gst + ((size_t)blk * 6 + f) * FACE_CELLS + p1);
    } else {
      const FaceNbr nb = C.nbr[blk * 6 + f];
      guide_pair(x, blk, f, p0, p1, nb, C.bc, C.dx[blk], g0, g1);
    }
    xs[guide_tix(f, p0 & 15, p0 >> 4)] = g0;
    xs[guide_tix(f, p1 & 15, p1 >> 4)] = g1;
  }
}

// Canonical block reduction + last-CTA cross-block reduction + finaliser.
// The block tree has 512 virtual threads (see the layout header); thread r
// of a 256-thread CTA carries virtual threads r and r + 256, whose serial
// per-colour sums are acc[c][0] and acc[c][1] (cells c*2048 + r + 256*m with
// m even and odd respectively).
__device__ void reduce_finalize(const double (&acc)[2][2], double* __restrict__ partials,
                                SolveState* st, int fin, int iter) {
  __shared__ double ws[16];
  __shared__ int amlast;
  const int tid = threadIdx.x;
  double v0 = acc[0][0] + acc[1][0], v1 = acc[0][1] + acc[1][1];
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1) {
    v0 += __shfl_xor_sync(0xffffffffu, v0, off);
    v1 += __shfl_xor_sync(0xffffffffu, v1, off);
  }
  if ((tid & 31) == 0) {
    ws[tid >> 5] = v0;
    ws[8 + (tid >> 5)] = v1;
  }
  __syncthreads();
  if (tid == 0) {
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < 16; ++w) s += ws[w];
    __stcg(partials + blockIdx.x, s);
    __threadfence();
    const unsigned t = atomicAdd(&st->ticket, 1u);
    amlast = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!amlast) return;
  __threadfence();
  double S = 0.0;
  for (int b = tid; b < (int)gridDim.x; b += THREADS) S += __ldcg(partials + b);
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1) S += __shfl_xor_sync(0xffffffffu, S, off);
  __syncthreads();
  if ((tid & 31) == 0) ws[tid >> 5] = S;
  __syncthreads();
  if (tid == 0) {
    double total = 0.0;
#pragma unroll
    for (int w = 0; w < 8; ++w) total += ws[w];
    finalize(st, total, fin, iter);
    st->ticket = 0;
    __threadfence();
  }
}

// ---------------------------------------------------------------------------
// Jacobi smoother (bils.f90:5-55) from the zero field of FFVILS::Fill(z, 0)
// (blas.f90:5-33, guides included) with b = bvec: the first pass of
// Jacobi_PreConditioner.  Later passes read a stored iterate and run on the
// pipelined kernel (launch_jacobi_pipe).  DOT: also forms b.x1
// (FFVILS.h:712-718 DOT(r, z), r = bvec).  Every neighbour is 0.0, and the
// products with it are kept, so the result has the reference's bits (the
// sign of a zero residual included).  A block whose uniform record
// (KCtx::urec) is set has the same seven coefficients in every cell: they
// are read once from the record, and the block moves b and x only.
// ---------------------------------------------------------------------------
template <bool DOT, bool UNI>
__device__ __forceinline__ void jacobi_cells(const double* __restrict__ Ab,
                                             const double* __restrict__ ur,
                                             const double* __restrict__ bb, double* __restrict__ xo,
                                             double omega, double (&acc)[2][2]) {
  const int tid = threadIdx.x;
  double u[7];
#pragma unroll
  for (int a = 0; a < 7; ++a) u[a] = UNI ? __ldg(ur + a) : 0.0;
  auto coef = [&](int a, int s) { return UNI ? u[a] : __ldg(Ab + a * BLOCK_CELLS + s); };
  const double x0 = 0.0;
  double bvs[16];  // the thread's 16 values of b, loads in flight together
#pragma unroll
  for (int m = 0; m < 16; ++m) bvs[m] = __ldg(bb + tid + THREADS * m);
#pragma unroll
  for (int c = 0; c < 2; ++c) {
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      const int s = c * HALF_CELLS + tid + THREADS * m;
      const double bv = bvs[c * 8 + m];
      const double r = bv - coef(1, s) * x0 - coef(2, s) * x0 - coef(3, s) * x0 -
                       coef(4, s) * x0 - coef(5, s) * x0 - coef(6, s) * x0;
      const double x_tmp = r / coef(0, s);
      const double x1 = x0 - omega * (x0 - x_tmp);
      xo[s] = x1;
      if (DOT) acc[c][m & 1] += bv * x1;
    }
  }
}

template <bool DOT>
__global__ void __launch_bounds__(THREADS, 3)
jacobi_kernel(KCtx C, double* __restrict__ xout, const double* __restrict__ A,
              const double* __restrict__ bvec, double omega, double* __restrict__ partials,
              SolveState* st) {
  if (solve_done(st)) return;
  const int blk = blockIdx.x;
  const double* ur = C.urec ? C.urec + (size_t)blk * 8 : nullptr;
  const bool uni = ur && __ldg(ur + 7) != 0.0;
  const double* Ab = A + (size_t)blk * 7 * BLOCK_CELLS;
  const double* bb = bvec + (size_t)blk * BLOCK_CELLS;
  double* xo = xout + (size_t)blk * BLOCK_CELLS;
  double acc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
  if (uni)
    jacobi_cells<DOT, true>(Ab, ur, bb, xo, omega, acc);
  else
    jacobi_cells<DOT, false>(Ab, ur, bb, xo, omega, acc);
  if (DOT) reduce_finalize(acc, partials, st, FIN_CG_RR1, 0);
}

// ---------------------------------------------------------------------------
// Element-wise and stencil helpers of FFVILS::CG.
// ---------------------------------------------------------------------------

// r = b - A x (calc_r, bils.f90:208-254); x guides from 'gst' when given.
__global__ void __launch_bounds__(THREADS, 3)
calc_r_kernel(KCtx C, const double* __restrict__ x, const double* __restrict__ gst,
              const double* __restrict__ A, const double* __restrict__ bvec,
              double* __restrict__ rout, SolveState* st) {
  if (st && solve_done(st)) return;
  __shared__ double xs[TILE];
  const int blk = blockIdx.x, tid = threadIdx.x;
  stage_tile(xs, x, blk, C, gst);
  __syncthreads();
  const double* Ab = A + (size_t)blk * 7 * BLOCK_CELLS;
  const double* bb = bvec + (size_t)blk * BLOCK_CELLS;
  double* ro = rout + (size_t)blk * BLOCK_CELLS;
#pragma unroll 4
  for (int m = 0; m < 16; ++m) {
    const int s = tid + THREADS * m;
    int i, j, k;
    cell_of(s, i, j, k);
    const int t = tix(i, j, k);
    ro[s] = __ldg(bb + s) - __ldg(Ab + 4096 + s) * xs[t - 1] - __ldg(Ab + 8192 + s) * xs[t + 1] -
            __ldg(Ab + 12288 + s) * xs[t - TW] - __ldg(Ab + 16384 + s) * xs[t + TW] -
            __ldg(Ab + 20480 + s) * xs[t - TP] - __ldg(Ab + 24576 + s) * xs[t + TP] -
            __ldg(Ab + s) * xs[t];
  }
}

// p = z (first iteration, copy) or p = z + beta*p (xpay, blas.f90:363-395).
__global__ void __launch_bounds__(THREADS)
p_update_kernel(const double* __restrict__ z, double* __restrict__ p, int first, SolveState* st) {
  if (solve_done(st)) return;
  const double beta = st->beta;
  const size_t base = (size_t)blockIdx.x * BLOCK_CELLS;
#pragma unroll 4
  for (int m = 0; m < 16; ++m) {
    const size_t s = base + threadIdx.x + THREADS * m;
    p[s] = first ? z[s] : (z[s] + beta * p[s]);
  }
}

// BiCGSTAB p update (FFVILS.h:853-871): first iteration p = r (copy); after
// it AXPY(p, q_, -gamma) then XPAY(p, r, beta), i.e. per cell
// t = p + (-gamma)*q_ ; p = r + beta*t (blas.f90:329-395).
__global__ void __launch_bounds__(THREADS)
bicg_p_kernel(const double* __restrict__ r, double* __restrict__ p, const double* __restrict__ q,
              SolveState* st) {
  if (solve_done(st)) return;
  const double beta = st->beta, mgamma = -st->gamma;
  const bool first = st->cycle == 1;  // iteration 1, or the first after a restart
  const size_t base = (size_t)blockIdx.x * BLOCK_CELLS;
#pragma unroll 4
  for (int m = 0; m < 16; ++m) {
    const size_t s = base + threadIdx.x + THREADS * m;
    if (first) {
      p[s] = r[s];
    } else {
      const double t = p[s] + mgamma * q[s];
      p[s] = r[s] + beta * t;
    }
  }
}

// AXPYZ (blas.f90:397-430): z = a*x + y with a = -alpha (FFVILS.h:898-903).
__global__ void __launch_bounds__(THREADS)
axpyz_kernel(double* __restrict__ z, const double* __restrict__ x, const double* __restrict__ y,
             SolveState* st) {
  if (solve_done(st)) return;
  const double a = -st->alpha;
  const size_t base = (size_t)blockIdx.x * BLOCK_CELLS;
#pragma unroll 4
  for (int m = 0; m < 16; ++m) {
    const size_t s = base + threadIdx.x + THREADS * m;
    z[s] = a * x[s] + y[s];
  }
}

// BiCGSTAB update (FFVILS.h:938-958): AXPBYPZ(x, p_, s_, alpha, gamma)
// (x = alpha*p_ + gamma*s_ + x, blas.f90:432-464), AXPYZ(r, t_, s, -gamma)
// (r = (-gamma)*t_ + s), and r.r for IsConverged.
__global__ void __launch_bounds__(THREADS)
bicg_update_kernel(double* __restrict__ x, const double* __restrict__ pz,
                   const double* __restrict__ sz, double* __restrict__ r,
                   const double* __restrict__ t, const double* __restrict__ s,
                   double* __restrict__ partials, SolveState* st, int iter) {
  if (solve_done(st)) return;
  const double alpha = st->alpha, gamma = st->gamma, mgamma = -st->gamma;
  const size_t base = (size_t)blockIdx.x * BLOCK_CELLS;
  double acc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
#pragma unroll
  for (int c = 0; c < 2; ++c) {
#pragma unroll 4
    for (int m = 0; m < 8; ++m) {
      const size_t i = base + c * HALF_CELLS + threadIdx.x + THREADS * m;
      x[i] = alpha * pz[i] + gamma * sz[i] + x[i];
      const double rn = mgamma * t[i] + s[i];
      r[i] = rn;
      acc[c][m & 1] += rn * rn;
    }
  }
  reduce_finalize(acc, partials, st, FIN_BI_RR, iter);
}

// x = x + alpha p; r = r + (-alpha) q (axpy, blas.f90:329-361); r.r.
__global__ void __launch_bounds__(THREADS)
cg_update_kernel(double* __restrict__ x, const double* __restrict__ p, double* __restrict__ r,
                 const double* __restrict__ q, double* __restrict__ partials, SolveState* st,
                 int iter) {
  if (solve_done(st)) return;
  const double alpha = st->alpha, malpha = -alpha;
  const size_t base = (size_t)blockIdx.x * BLOCK_CELLS;
  double acc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
#pragma unroll
  for (int c = 0; c < 2; ++c) {
#pragma unroll 4
    for (int m = 0; m < 8; ++m) {
      const size_t s = base + c * HALF_CELLS + threadIdx.x + THREADS * m;
      x[s] = x[s] + alpha * p[s];
      const double rn = r[s] + malpha * q[s];
      r[s] = rn;
      acc[c][m & 1] += rn * rn;
    }
  }
  reduce_finalize(acc, partials, st, FIN_CG_RR, iter);
}

// x.y over interior cells (dot, blas.f90:466-499) with a finaliser.
__global__ void __launch_bounds__(THREADS)
dot_kernel(const double* __restrict__ x, const double* __restrict__ y,
           double* __restrict__ partials, SolveState* st, int fin, int iter) {
  if (solve_done(st)) return;
  const size_t base = (size_t)blockIdx.x * BLOCK_CELLS;
  double acc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
#pragma unroll
  for (int c = 0; c < 2; ++c) {
#pragma unroll 4
    for (int m = 0; m < 8; ++m) {
      const size_t s = base + c * HALF_CELLS + threadIdx.x + THREADS * m;
      acc[c][m & 1] += __ldg(x + s) * __ldg(y + s);
    }
  }
  reduce_finalize(acc, partials, st, fin, iter);
}

// BiCGSTAB's DOT(r, r0) (FFVILS.h:845-846); on the first iteration of a
// cycle (iteration 1, or after a restart) r0 is first set to r.
__global__ void __launch_bounds__(THREADS)
dot_rr0_kernel(const double* __restrict__ r, double* __restrict__ r0, double* __restrict__ partials,
               SolveState* st, int fin, int iter) {
  if (solve_done(st)) return;
  const bool copy = st->cycle == 1;
  const size_t base = (size_t)blockIdx.x * BLOCK_CELLS + threadIdx.x;
  double acc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
  // the thread's 16 values of r (and of r0) with their loads in flight together
  double rv[16], yv[16];
#pragma unroll
  for (int m = 0; m < 16; ++m) rv[m] = __ldg(r + base + THREADS * m);
  if (copy) {
#pragma unroll
    for (int m = 0; m < 16; ++m) {
      r0[base + THREADS * m] = rv[m];
      yv[m] = rv[m];
    }
  } else {
#pragma unroll
    for (int m = 0; m < 16; ++m) yv[m] = r0[base + THREADS * m];
  }
#pragma unroll
  for (int c = 0; c < 2; ++c) {
#pragma unroll
    for (int m = 0; m < 8; ++m) acc[c][m & 1] += rv[c * 8 + m] * yv[c * 8 + m];
  }
  reduce_finalize(acc, partials, st, fin, iter);
}

// LocalScalar3D::CalcSum (LocalScalar3D.h:130-157, sf3d_calc_sum,
// src/CGMfuncs/bsf3d.f90:35-67): the sum of x over all interior cells.
__global__ void __launch_bounds__(THREADS)
sum_kernel(const double* __restrict__ x, double* __restrict__ partials, SolveState* st, int fin) {
  if (solve_done(st)) return;
  const size_t base = (size_t)blockIdx.x * BLOCK_CELLS;
  double acc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
#pragma unroll
  for (int c = 0; c < 2; ++c) {
#pragma unroll 4
    for (int m = 0; m < 8; ++m)
      acc[c][m & 1] += __ldg(x + base + c * HALF_CELLS + threadIdx.x + THREADS * m);
  }
  reduce_finalize(acc, partials, st, fin, 0);
}

// LocalScalar3D::ShiftByA (LocalScalar3D.h:159-178, adda, blas.f90:162-193):
// x = x + a on the interior with a = st->alpha.
__global__ void __launch_bounds__(THREADS)
shift_kernel(double* __restrict__ x, SolveState* st) {
  if (solve_done(st)) return;
  const double a = st->alpha;
  const size_t base = (size_t)blockIdx.x * BLOCK_CELLS;
#pragma unroll 4
  for (int m = 0; m < 16; ++m) {
    const size_t s = base + threadIdx.x + THREADS * m;
    x[s] = x[s] + a;
  }
}

// ---------------------------------------------------------------------------
// Exchange into a stored guide layer, layout conversion and set-up kernels.
// ---------------------------------------------------------------------------

// Writes layer-1 guide values of every face of every block into g.
__global__ void __launch_bounds__(THREADS)
exchange_kernel(KCtx C, const double* __restrict__ x, double* __restrict__ g) {
  const int blk = C.first + blockIdx.x, tid = threadIdx.x;
  const int a = tid & 15, b = tid >> 4;
  for (int f = 0; f < 6; ++f) {
    const FaceNbr nb = C.nbr[blk * 6 + f];
    g[((size_t)blk * 6 + f) * FACE_CELLS + b * 16 + a] =
        guide_value(x, blk, f, a, b, 1, nb, C.bc, C.dx[blk]);
  }
}

// Host layout block (n+2vc)^3 -> colour-split interior (+ layer-1 guides).
__global__ void __launch_bounds__(THREADS)
pack_kernel(const double* __restrict__ stage, int vc, double* __restrict__ dst, size_t stride,
            double* __restrict__ gdst) {
  const int blk = blockIdx.x, tid = threadIdx.x;
  const int w = 16 + 2 * vc;
  const double* sb = stage + (size_t)blk * w * w * w;
  // the interior row by row (16 threads read one row of 16 consecutive
  // values: whole sectors, also when 'stage' is pinned host memory read
  // across the link), every load in flight before the colour-split stores
  const int i = tid & 15, r0 = tid >> 4;
  double v[16];
#pragma unroll
  for (int m = 0; m < 16; ++m) {
    const int r = r0 + 16 * m, j = r & 15, k = r >> 4;
    v[m] = sb[(i + vc) + w * ((j + vc) + w * (k + vc))];
  }
#pragma unroll
  for (int m = 0; m < 16; ++m) {
    const int r = r0 + 16 * m, j = r & 15, k = r >> 4;
    dst[(size_t)blk * stride + ((i + j + k) & 1) * HALF_CELLS + (k * 16 + j) * 8 + (i >> 1)] = v[m];
  }
  if (gdst) {
    const int a = tid & 15, b = tid >> 4;
    for (int f = 0; f < 6; ++f) {
      int g[3];
      const int axis = f >> 1;
      if (axis == 0) { g[1] = a; g[2] = b; } else if (axis == 1) { g[0] = a; g[2] = b; } else { g[0] = a; g[1] = b; }
      g[axis] = (f & 1) ? 16 : -1;
      gdst[((size_t)blk * 6 + f) * FACE_CELLS + b * 16 + a] =
          sb[(g[0] + vc) + w * ((g[1] + vc) + w * (g[2] + vc))];
    }
  }
}

// Integer host field -> bit 'bit' of the per-cell flag byte.
// mode 0: bit set where value != 0 (cut ids); mode 1: bit set where value == 1 (fluid).
__global__ void __launch_bounds__(THREADS)
pack_flag_kernel(const int32_t* __restrict__ stage, int vc, uint8_t* __restrict__ flags, int bit,
                 int mode) {
  const int blk = blockIdx.x, tid = threadIdx.x;
  const int w = 16 + 2 * vc;
  const int32_t* sb = stage + (size_t)blk * w * w * w;
  for (int m = 0; m < 16; ++m) {
    const int s = tid + THREADS * m;
    int i, j, k;
    cell_of(s, i, j, k);
    const int32_t v = sb[(i + vc) + w * ((j + vc) + w * (k + vc))];
    const bool on = mode ? (v == 1) : (v != 0);
    uint8_t& f = flags[(size_t)blk * BLOCK_CELLS + s];
    f = on ? (uint8_t)(f | (1u << bit)) : (uint8_t)(f & ~(1u << bit));
  }
}

// Flag byte -> integer host field (inverse of pack_flag_kernel).
__global__ void __launch_bounds__(THREADS)
unpack_flag_kernel(const uint8_t* __restrict__ flags, int vc, int32_t* __restrict__ stage, int bit) {
  const int blk = blockIdx.x, tid = threadIdx.x;
  const int w = 16 + 2 * vc;
  int32_t* sb = stage + (size_t)blk * w * w * w;
  for (int m = tid; m < w * w * w; m += THREADS) sb[m] = 0;
  __syncthreads();
  for (int m = 0; m < 16; ++m) {
    const int s = tid + THREADS * m;
    int i, j, k;
    cell_of(s, i, j, k);
    sb[(i + vc) + w * ((j + vc) + w * (k + vc))] = (flags[(size_t)blk * BLOCK_CELLS + s] >> bit) & 1;
  }
}

// Colour-split interior -> host layout, with vc guide layers per face
// computed as the reference's exchange + outer BC would (layers 1..vc).
__global__ void __launch_bounds__(THREADS)
unpack_kernel(KCtx C, const double* __restrict__ src, size_t stride, int vc, int with_guides,
              double* __restrict__ stage) {
  const int blk = C.first + blockIdx.x, tid = threadIdx.x;
  const int w = 16 + 2 * vc;
  double* sb = stage + (size_t)blockIdx.x * w * w * w;
  for (int m = tid; m < w * w * w; m += THREADS) sb[m] = 0.0;
  __syncthreads();
  for (int m = 0; m < 16; ++m) {
    const int s = tid + THREADS * m;
    int i, j, k;
    cell_of(s, i, j, k);
    sb[(i + vc) + w * ((j + vc) + w * (k + vc))] = src[(size_t)blk * stride + s];
  }
  if (!with_guides) return;
  const int a = tid & 15, b = tid >> 4;
  for (int f = 0; f < 6; ++f) {
    const FaceNbr nb = C.nbr[blk * 6 + f];
    const int axis = f >> 1;
    for (int L = 1; L <= vc; ++L) {
      int g[3];
      if (axis == 0) { g[1] = a; g[2] = b; } else if (axis == 1) { g[0] = a; g[2] = b; } else { g[0] = a; g[1] = b; }
      g[axis] = (f & 1) ? (15 + L) : (-L);
      sb[(g[0] + vc) + w * ((g[1] + vc) + w * (g[2] + vc))] =
          guide_value(src, blk, f, a, b, L, nb, C.bc, C.dx[blk]);
    }
  }
}

// ---------------------------------------------------------------------------
// bcut_calc_ab_p (src/FFV/bcut.f90:608-832), one cell per thread-iteration.
// u guide values come from the stored guide layers of UX/UY/UZ.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double u_at(const double* __restrict__ u, const double* __restrict__ gu,
                                       int blk, int i, int j, int k) {
  int f = -1, a = 0, b = 0;
  if (i < 0) { f = X_M; a = j; b = k; } else if (i > 15) { f = X_P; a = j; b = k; }
  else if (j < 0) { f = Y_M; a = i; b = k; } else if (j > 15) { f = Y_P; a = i; b = k; }
  else if (k < 0) { f = Z_M; a = i; b = j; } else if (k > 15) { f = Z_P; a = i; b = j; }
  if (f < 0) return __ldg(u + (size_t)blk * BLOCK_CELLS + sidx(i, j, k));
  return __ldg(gu + ((size_t)blk * 6 + f) * FACE_CELLS + b * 16 + a);
}

__global__ void __launch_bounds__(THREADS)
assemble_kernel(KCtx C, const double* __restrict__ ux, const double* __restrict__ uy,
                const double* __restrict__ uz, const double* __restrict__ gux,
                const double* __restrict__ guy, const double* __restrict__ guz,
                const double* __restrict__ cut /* [6][nb*4096] */,
                const uint8_t* __restrict__ flags, double* __restrict__ A,
                double* __restrict__ bvec, double* __restrict__ vface /* [6][nb*4096] or null */,
                double rhof, double dt, size_t field_stride) {
  const int blk = C.first + blockIdx.x, tid = threadIdx.x;
  const double dx = C.dx[blk];
  double* Ab = A + (size_t)blk * 7 * BLOCK_CELLS;
  for (int m = 0; m < 16; ++m) {
    const int s = tid + THREADS * m;
    int i, j, k;
    cell_of(s, i, j, k);
    const size_t gs = (size_t)blk * BLOCK_CELLS + s;
    double r0 = 1.0 / rhof, r1 = 1.0 / rhof, r2 = 1.0 / rhof;
    double r3 = 1.0 / rhof, r4 = 1.0 / rhof, r5 = 1.0 / rhof;
    const double uxp = __ldg(ux + gs), uyp = __ldg(uy + gs), uzp = __ldg(uz + gs);
    double vx0 = 0.5 * (uxp + u_at(ux, gux, blk, i - 1, j, k));
    double vx1 = 0.5 * (uxp + u_at(ux, gux, blk, i + 1, j, k));
    double vy2 = 0.5 * (uyp + u_at(uy, guy, blk, i, j - 1, k));
    double vy3 = 0.5 * (uyp + u_at(uy, guy, blk, i, j + 1, k));
    double vz4 = 0.5 * (uzp + u_at(uz, guz, blk, i, j, k - 1));
    double vz5 = 0.5 * (uzp + u_at(uz, guz, blk, i, j, k + 1));
    const double d0 = __ldg(cut + gs), d1 = __ldg(cut + field_stride + gs);
    const double d2 = __ldg(cut + 2 * field_stride + gs), d3 = __ldg(cut + 3 * field_stride + gs);
    const double d4 = __ldg(cut + 4 * field_stride + gs), d5 = __ldg(cut + 5 * field_stride + gs);
    const unsigned fl = flags[gs];
    const bool c0 = fl & 1, c1 = fl & 2, c2 = fl & 4, c3 = fl & 8, c4 = fl & 16, c5 = fl & 32;
    const bool fluid = fl & 128;
    if (c0) { r0 = 0.0; vx0 = vx1 * (d0 - 0.5) / (d0 + 0.5); r1 = (1.0 / rhof) / (d0 + 0.5); }
    if (c1) { r1 = 0.0; vx1 = vx0 * (d1 - 0.5) / (d1 + 0.5); r0 = (1.0 / rhof) / (d1 + 0.5); }
    if (c2) { r2 = 0.0; vy2 = vy3 * (d2 - 0.5) / (d2 + 0.5); r3 = (1.0 / rhof) / (d2 + 0.5); }
    if (c3) { r3 = 0.0; vy3 = vy2 * (d3 - 0.5) / (d3 + 0.5); r2 = (1.0 / rhof) / (d3 + 0.5); }
    if (c4) { r4 = 0.0; vz4 = vz5 * (d4 - 0.5) / (d4 + 0.5); r5 = (1.0 / rhof) / (d4 + 0.5); }
    if (c5) { r5 = 0.0; vz5 = vz4 * (d5 - 0.5) / (d5 + 0.5); r4 = (1.0 / rhof) / (d5 + 0.5); }
    if (c0 && c1) { r0 = 0.0; r1 = 0.0; vx0 = 0.0; vx1 = 0.0; }
    if (c2 && c3) { r2 = 0.0; r3 = 0.0; vy2 = 0.0; vy3 = 0.0; }
    if (c4 && c5) { r4 = 0.0; r5 = 0.0; vz4 = 0.0; vz5 = 0.0; }
    const double l0 = r0 / (dx * dx), l1 = r1 / (dx * dx), l2 = r2 / (dx * dx);
    const double l3 = r3 / (dx * dx), l4 = r4 / (dx * dx), l5 = r5 / (dx * dx);
    const double divv = (vx1 - vx0 + vy3 - vy2 + vz5 - vz4) / dx;
    double ap = -(l0 + l1) - (l2 + l3) - (l4 + l5);
    double aw = l0, ae = l1, as = l2, an = l3, ab = l4, at = l5;
    double bv = divv / dt;
    if (!fluid) {
      ap = -6.0; aw = ae = as = an = ab = at = 1.0; bv = 0.0;
      vx0 = vx1 = vy2 = vy3 = vz4 = vz5 = 0.0;
    }
    Ab[s] = ap; Ab[4096 + s] = aw; Ab[8192 + s] = ae; Ab[12288 + s] = as;
    Ab[16384 + s] = an; Ab[20480 + s] = ab; Ab[24576 + s] = at;
    bvec[gs] = bv;
    if (vface) {
      vface[gs] = vx0; vface[field_stride + gs] = vx1; vface[2 * field_stride + gs] = vy2;
      vface[3 * field_stride + gs] = vy3; vface[4 * field_stride + gs] = vz4;
      vface[5 * field_stride + gs] = vz5;
    }
  }
}

// bcut_remove_p (bcut.f90:3879-4061, CORR false) and bcut_corr_u
// (bcut.f90:4063-4297, CORR true), one cell per thread-iteration, p staged
// with its stored guide layer.  Each expression in the reference's order.
template <bool CORR>
__global__ void __launch_bounds__(THREADS)
projection_kernel(KCtx C, const double* __restrict__ p, const double* __restrict__ gp,
                  const double* __restrict__ cut, const uint8_t* __restrict__ flags,
                  double* __restrict__ ux, double* __restrict__ uy, double* __restrict__ uz,
                  double* __restrict__ vface, double* __restrict__ lapp, double rhof, double dt,
                  size_t fs) {
  __shared__ double xs[TILE];
  const int blk = blockIdx.x, tid = threadIdx.x;
  stage_tile(xs, p, blk, C, gp);
  __syncthreads();
  const double dx = C.dx[blk];
  for (int m = 0; m < 16; ++m) {
    const int s = tid + THREADS * m;
    int i, j, k;
    cell_of(s, i, j, k);
    const int t = tix(i, j, k);
    const size_t gs = (size_t)blk * BLOCK_CELLS + s;
    const double r0 = 1.0 / rhof, r1 = 1.0 / rhof, r2 = 1.0 / rhof;
    const double r3 = 1.0 / rhof, r4 = 1.0 / rhof, r5 = 1.0 / rhof;
    double dpx0 = (xs[t] - xs[t - 1]) / dx;
    double dpx1 = (xs[t + 1] - xs[t]) / dx;
    double dpy2 = (xs[t] - xs[t - TW]) / dx;
    double dpy3 = (xs[t + TW] - xs[t]) / dx;
    double dpz4 = (xs[t] - xs[t - TP]) / dx;
    double dpz5 = (xs[t + TP] - xs[t]) / dx;
    double rdpx0 = r0 * dpx0, rdpx1 = r1 * dpx1, rdpy2 = r2 * dpy2;
    double rdpy3 = r3 * dpy3, rdpz4 = r4 * dpz4, rdpz5 = r5 * dpz5;
    const double d0 = __ldg(cut + gs), d1 = __ldg(cut + fs + gs), d2 = __ldg(cut + 2 * fs + gs);
    const double d3 = __ldg(cut + 3 * fs + gs), d4 = __ldg(cut + 4 * fs + gs);
    const double d5 = __ldg(cut + 5 * fs + gs);
    const unsigned fl = flags[gs];
    const bool c0 = fl & 1, c1 = fl & 2, c2 = fl & 4, c3 = fl & 8, c4 = fl & 16, c5 = fl & 32;
    const bool fluid = fl & 128;
    if (c0) { rdpx0 = rdpx1 * (d0 - 0.5) / (d0 + 0.5); dpx0 = dpx1 * (d0 - 0.5) / (d0 + 0.5); }
    if (c1) { rdpx1 = rdpx0 * (d1 - 0.5) / (d1 + 0.5); dpx1 = dpx0 * (d1 - 0.5) / (d1 + 0.5); }
    if (c2) { rdpy2 = rdpy3 * (d2 - 0.5) / (d2 + 0.5); dpy2 = dpy3 * (d2 - 0.5) / (d2 + 0.5); }
    if (c3) { rdpy3 = rdpy2 * (d3 - 0.5) / (d3 + 0.5); dpy3 = dpy2 * (d3 - 0.5) / (d3 + 0.5); }
    if (c4) { rdpz4 = rdpz5 * (d4 - 0.5) / (d4 + 0.5); dpz4 = dpz5 * (d4 - 0.5) / (d4 + 0.5); }
    if (c5) { rdpz5 = rdpz4 * (d5 - 0.5) / (d5 + 0.5); dpz5 = dpz4 * (d5 - 0.5) / (d5 + 0.5); }
    if (c0 && c1) { rdpx0 = 0.0; rdpx1 = 0.0; }
    if (c2 && c3) { rdpy2 = 0.0; rdpy3 = 0.0; }
    if (c4 && c5) { rdpz4 = 0.0; rdpz5 = 0.0; }
    const double rdpx = 0.5 * (rdpx0 + rdpx1);
    const double rdpy = 0.5 * (rdpy2 + rdpy3);
    const double rdpz = 0.5 * (rdpz4 + rdpz5);
    if (!CORR) {
      ux[gs] = fluid ? ux[gs] + rdpx * dt : 0.0;
      uy[gs] = fluid ? uy[gs] + rdpy * dt : 0.0;
      uz[gs] = fluid ? uz[gs] + rdpz * dt : 0.0;
    } else {
      ux[gs] = fluid ? ux[gs] - rdpx * dt : 0.0;
      uy[gs] = fluid ? uy[gs] - rdpy * dt : 0.0;
      uz[gs] = fluid ? uz[gs] - rdpz * dt : 0.0;
      vface[gs] = fluid ? vface[gs] - rdpx0 * dt : 0.0;
      vface[fs + gs] = fluid ? vface[fs + gs] - rdpx1 * dt : 0.0;
      vface[2 * fs + gs] = fluid ? vface[2 * fs + gs] - rdpy2 * dt : 0.0;
      vface[3 * fs + gs] = fluid ? vface[3 * fs + gs] - rdpy3 * dt : 0.0;
      vface[4 * fs + gs] = fluid ? vface[4 * fs + gs] - rdpz4 * dt : 0.0;
      vface[5 * fs + gs] = fluid ? vface[5 * fs + gs] - rdpz5 * dt : 0.0;
      const double lp = (xs[t + 1] + xs[t - 1] + xs[t + TW] + xs[t - TW] + xs[t + TP] +
                         xs[t - TP] - 6.0 * xs[t]) / (dx * dx);
      lapp[gs] = (!fluid || (fl & 63)) ? 0.0 : lp;
    }
  }
}

// Outer-BC folding (bca.f90:5-388) in the order w, e, s, n, b, t
// (BlockScalar3D.h:183-190) for every cell on an outer face.
__global__ void __launch_bounds__(THREADS)
fold_bc_kernel(KCtx C, double* __restrict__ A, double* __restrict__ bvec) {
  const int blk = C.first + blockIdx.x, tid = threadIdx.x;
  const double dx = C.dx[blk];
  int outer = 0;
  for (int f = 0; f < 6; ++f)
    if (C.nbr[blk * 6 + f].kind == NB_OUTER) outer |= 1 << f;
  if (!outer) return;
  double* Ab = A + (size_t)blk * 7 * BLOCK_CELLS;
  for (int m = 0; m < 16; ++m) {
    const int s = tid + THREADS * m;
    int i, j, k;
    cell_of(s, i, j, k);
    const int on[6] = {i == 0, i == 15, j == 0, j == 15, k == 0, k == 15};
    for (int f = 0; f < 6; ++f) {
      if (!((outer >> f) & 1) || !on[f]) continue;
      double* Af = Ab + (size_t)(1 + f) * BLOCK_CELLS;
      double* bp = bvec + (size_t)blk * BLOCK_CELLS + s;
      const double af = Af[s];
      if (C.bc.type[f] == BC_DIRICHLET) {
        const double xc = C.bc.value[f];
        Ab[s] = Ab[s] - af;
        *bp = *bp - af * xc * 2.0;
      } else {
        const double xc = C.bc.value[f] * dx;
        Ab[s] = Ab[s] + af;
        if (f & 1) *bp = *bp - af * xc;
        else *bp = *bp + af * xc;
      }
      Af[s] = 0.0;
    }
  }
}

// A (7 arrays) and b -> the sweep's coefficient stream (STREAM_BLOCK per block).
// Without STREAM only the uniform records are written.
template <bool STREAM>
__global__ void __launch_bounds__(THREADS)
pack_stream_kernel(const double* __restrict__ A, const double* __restrict__ b,
                   double* __restrict__ stream, double* __restrict__ urec,
                   int32_t* __restrict__ ucount) {
  const int blk = blockIdx.x, tid = threadIdx.x;
  const double* Ab = A + (size_t)blk * 7 * BLOCK_CELLS;
  double* sb = STREAM ? stream + (size_t)blk * STREAM_BLOCK : nullptr;
  bool same = true;
  for (int m = 0; m < 16; ++m) {
    const int s = tid + THREADS * m;  // chunk m, cell tid
    double* dst = STREAM ? sb + (size_t)m * STREAM_CHUNK + tid : nullptr;
    for (int a = 0; a < 7; ++a) {
      const double v = Ab[(size_t)a * BLOCK_CELLS + s];
      if (STREAM) dst[a * 256] = v;
      same = same && __double_as_longlong(v) == __double_as_longlong(Ab[(size_t)a * BLOCK_CELLS]);
    }
    if (STREAM) dst[7 * 256] = b[(size_t)blk * BLOCK_CELLS + s];
  }
  // a uniform block (all seven coefficients bitwise equal to cell 0's): the
  // sweep kernel copies only b of its stream and takes Ap..At from here
  same = __syncthreads_and(same);
  if (tid < 8) urec[(size_t)blk * 8 + tid] = tid < 7 ? Ab[(size_t)tid * BLOCK_CELLS] : (same ? 1.0 : 0.0);
  if (tid == 0 && same) atomicAdd(ucount, 1);
}

// FFVILS::Fill (blas.f90:5-33): interior and stored guide layer.
__global__ void __launch_bounds__(THREADS)
fill_kernel(double* __restrict__ x, size_t stride, double* __restrict__ g, double value) {
  const int blk = blockIdx.x, tid = threadIdx.x;
  for (int m = 0; m < 16; ++m) x[(size_t)blk * stride + tid + THREADS * m] = value;
  if (g)
    for (int f = 0; f < 6; ++f) g[((size_t)blk * 6 + f) * FACE_CELLS + tid] = value;
}

// ---------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------
void launch_jacobi(cudaStream_t s, const KCtx& C, bool dot, double* xout, const double* A,
                   const double* b, double omega, double* partials, SolveState* st) {
  if (dot)
    jacobi_kernel<true><<<C.nb, THREADS, 0, s>>>(C, xout, A, b, omega, partials, st);
  else
    jacobi_kernel<false><<<C.nb, THREADS, 0, s>>>(C, xout, A, b, omega, partials, st);
}

void launch_calc_r(cudaStream_t s, const KCtx& C, const double* x, const double* gst,
                   const double* A, const double* b, double* r, SolveState* st) {
  calc_r_kernel<<<C.nb, THREADS, 0, s>>>(C, x, gst, A, b, r, st);
}
void launch_p_update(cudaStream_t s, const KCtx& C, const double* z, double* p, int first,
                     SolveState* st) {
  p_update_kernel<<<C.nb, THREADS, 0, s>>>(z, p, first, st);
}
void launch_bicg_p(cudaStream_t s, const KCtx& C, const double* r, double* p, const double* q,
                   SolveState* st) {
  bicg_p_kernel<<<C.nb, THREADS, 0, s>>>(r, p, q, st);
}
void launch_axpyz(cudaStream_t s, const KCtx& C, double* z, const double* x, const double* y,
                  SolveState* st) {
  axpyz_kernel<<<C.nb, THREADS, 0, s>>>(z, x, y, st);
}
void launch_sum(cudaStream_t s, const KCtx& C, const double* x, double* partials, SolveState* st,
                int fin) {
  sum_kernel<<<C.nb, THREADS, 0, s>>>(x, partials, st, fin);
}
void launch_shift(cudaStream_t s, const KCtx& C, double* x, SolveState* st) {
  shift_kernel<<<C.nb, THREADS, 0, s>>>(x, st);
}
void launch_dot_rr0(cudaStream_t s, const KCtx& C, const double* r, double* r0, double* partials,
                    SolveState* st, int fin, int iter) {
  dot_rr0_kernel<<<C.nb, THREADS, 0, s>>>(r, r0, partials, st, fin, iter);
}
void launch_bicg_update(cudaStream_t s, const KCtx& C, double* x, const double* pz,
                        const double* sz, double* r, const double* t, const double* sv,
                        double* partials, SolveState* st, int iter) {
  bicg_update_kernel<<<C.nb, THREADS, 0, s>>>(x, pz, sz, r, t, sv, partials, st, iter);
}
void launch_cg_update(cudaStream_t s, const KCtx& C, double* x, const double* p, double* r,
                      const double* q, double* partials, SolveState* st, int iter) {
  cg_update_kernel<<<C.nb, THREADS, 0, s>>>(x, p, r, q, partials, st, iter);
}
void launch_dot(cudaStream_t s, const KCtx& C, const double* x, const double* y,
                double* partials, SolveState* st, int fin, int iter) {
  dot_kernel<<<C.nb, THREADS, 0, s>>>(x, y, partials, st, fin, iter);
}
void launch_exchange(cudaStream_t s, const KCtx& C, const double* x, double* g) {
  exchange_kernel<<<C.nb, THREADS, 0, s>>>(C, x, g);
}
void launch_pack(cudaStream_t s, int nb, const double* stage, int vc, double* dst, size_t stride,
                 double* gdst) {
  pack_kernel<<<nb, THREADS, 0, s>>>(stage, vc, dst, stride, gdst);
}
void launch_pack_flag(cudaStream_t s, int nb, const int32_t* stage, int vc, uint8_t* flags,
                      int bit, int mode) {
  pack_flag_kernel<<<nb, THREADS, 0, s>>>(stage, vc, flags, bit, mode);
}
void launch_unpack_flag(cudaStream_t s, int nb, const uint8_t* flags, int vc, int32_t* stage,
                        int bit) {
  unpack_flag_kernel<<<nb, THREADS, 0, s>>>(flags, vc, stage, bit);
}
void launch_unpack(cudaStream_t s, const KCtx& C, const double* src, size_t stride, int vc,
                   int with_guides, double* stage) {
  unpack_kernel<<<C.nb, THREADS, 0, s>>>(C, src, stride, vc, with_guides, stage);
}
void launch_assemble(cudaStream_t s, const KCtx& C, const double* ux, const double* uy,
                     const double* uz, const double* gux, const double* guy, const double* guz,
                     const double* cut, const uint8_t* flags, double* A, double* b,
                     double* vface, double rhof, double dt, size_t field_stride) {
  assemble_kernel<<<C.nb, THREADS, 0, s>>>(C, ux, uy, uz, gux, guy, guz, cut, flags, A, b, vface,
                                           rhof, dt, field_stride);
}
void launch_pack_stream(cudaStream_t s, int nb, const double* A, const double* b, double* stream,
                        double* urec, int32_t* ucount) {
  pack_stream_kernel<true><<<nb, THREADS, 0, s>>>(A, b, stream, urec, ucount);
}
void launch_urec(cudaStream_t s, int nb, const double* A, double* urec, int32_t* ucount) {
  pack_stream_kernel<false><<<nb, THREADS, 0, s>>>(A, nullptr, nullptr, urec, ucount);
}
void launch_fill(cudaStream_t s, int nb, double* x, size_t stride, double* g, double value) {
  fill_kernel<<<nb, THREADS, 0, s>>>(x, stride, g, value);
}
void launch_projection(cudaStream_t s, const KCtx& C, bool corr, const double* p,
                       const double* gp, const double* cut, const uint8_t* flags, double* ux,
                       double* uy, double* uz, double* vface, double* lapp, double rhof,
                       double dt, size_t field_stride) {
  if (corr)
    projection_kernel<true><<<C.nb, THREADS, 0, s>>>(C, p, gp, cut, flags, ux, uy, uz, vface,
                                                     lapp, rhof, dt, field_stride);
  else
    projection_kernel<false><<<C.nb, THREADS, 0, s>>>(C, p, gp, cut, flags, ux, uy, uz, vface,
                                                      lapp, rhof, dt, field_stride);
}
void launch_fold_bc(cudaStream_t s, const KCtx& C, double* A, double* b) {
  fold_bc_kernel<<<C.nb, THREADS, 0, s>>>(C, A, b);
}

}  // namespace ffvgpu
