// ffvgpu_internal.cuh -- device functions shared by the FP64 kernels:
// guide-cell values of the in-kernel block-to-block exchange.
#pragma once
#include <cfloat>

#include "ffvgpu_layout.h"

namespace ffvgpu {

// ---------------------------------------------------------------------------
// Guide-cell values (the exchange), one cell at a time.
// ---------------------------------------------------------------------------

// sup_get_intp_index (src/CGMfuncs/sup.f90:1-16), 1-based i in [1, 2n].
__device__ __forceinline__ void intp_index(int i, int n, int& ic, double& r) {
  ic = i / 2;
  r = 0.25 + 0.5 * (double)(i % 2);
  if (i < 2) {
    ic = 1;
    r = -0.25;
  } else if (i > 2 * n - 1) {
    ic = n - 1;
    r = 1.25;
  }
}

// Interior value of cell (i, j, k) of block blk, widened to double (exact
// for float sources, whose guide cells are formed in double arithmetic).
template <typename T>
__device__ __forceinline__ double ld(const T* __restrict__ x, int blk, int i, int j, int k) {
  return (double)__ldg(x + (size_t)blk * BLOCK_CELLS + sidx(i, j, k));
}

// Value of guide cell (layer L = 1 or 2) of face 'face' of block 'blk' at
// transverse position (a, b) in [0,16)^2, computed from interior values of x.
template <typename T>
static __device__ __noinline__ double guide_value(const T* __restrict__ x, int blk, int face,
                                           int a, int b, int L, const FaceNbr& nb,
                                           const BCSet& bc, double dx) {
  const int axis = face >> 1;
  const bool plus = face & 1;
  // 0-based coordinates of the guide cell in this block's frame
  int g[3];
  if (axis == 0) { g[1] = a; g[2] = b; } else if (axis == 1) { g[0] = a; g[2] = b; } else { g[0] = a; g[1] = b; }
  g[axis] = plus ? (15 + L) : (-L);
  switch (nb.kind) {
    case NB_SAME: {
      int s[3] = {g[0], g[1], g[2]};
      s[axis] = plus ? (L - 1) : (16 - L);
      return ld(x, nb.id[0], s[0], s[1], s[2]);
    }
    case NB_COARSE: {
      // sup_copy_from_neighbor_c2f (sup.f90:54-120) with the windows of
      // Scalar3DUpdater1::copyFromNeighborC2F (Scalar3DUpdater1.cpp:245-347):
      // 1-based fine positions inside the coarse block, in [1, 32].
      int f[3];
      const int ta = (axis == 0) ? 1 : 0, tb = (axis == 2) ? 1 : 2;
      f[ta] = g[ta] + 1 + 16 * nb.so_u;
      f[tb] = g[tb] + 1 + 16 * nb.so_v;
      f[axis] = plus ? L : (33 - L);
      int i1, j1, k1;
      double r, s, t;
      intp_index(f[0], 16, i1, r);
      intp_index(f[1], 16, j1, s);
      intp_index(f[2], 16, k1, t);
      const int c = nb.id[0];
      --i1; --j1; --k1;  // to 0-based interior indices
      const double nnn = ld(x, c, i1, j1, k1);
      const double pnn = ld(x, c, i1 + 1, j1, k1);
      const double npn = ld(x, c, i1, j1 + 1, k1);
      const double nnp = ld(x, c, i1, j1, k1 + 1);
      const double npp = ld(x, c, i1, j1 + 1, k1 + 1);
      const double pnp = ld(x, c, i1 + 1, j1, k1 + 1);
      const double ppn = ld(x, c, i1 + 1, j1 + 1, k1);
      const double ppp = ld(x, c, i1 + 1, j1 + 1, k1 + 1);
      return (1.0 - t) * ((1.0 - s) * ((1.0 - r) * nnn + r * pnn) +
                          s * ((1.0 - r) * npn + r * ppn)) +
             t * ((1.0 - s) * ((1.0 - r) * nnp + r * pnp) +
                  s * ((1.0 - r) * npp + r * ppp));
    }
    case NB_FINE: {
      // sup_copy_from_neighbor_f2c (sup.f90:122-179) with the windows of
      // Scalar3DUpdater1::copyFromNeighborF2C (Scalar3DUpdater1.cpp:430-520).
      const int ta = (axis == 0) ? 1 : 0, tb = (axis == 2) ? 1 : 2;
      const int qu = g[ta] >> 3, qv = g[tb] >> 3;
      const int fb = nb.id[qu + 2 * qv];
      int lo[3];
      lo[ta] = 2 * (g[ta] & 7);
      lo[tb] = 2 * (g[tb] & 7);
      lo[axis] = plus ? (2 * L - 2) : (16 - 2 * L);
      const int i1 = lo[0], j1 = lo[1], k1 = lo[2];
      const double nnn = ld(x, fb, i1, j1, k1);
      const double pnn = ld(x, fb, i1 + 1, j1, k1);
      const double npn = ld(x, fb, i1, j1 + 1, k1);
      const double nnp = ld(x, fb, i1, j1, k1 + 1);
      const double npp = ld(x, fb, i1, j1 + 1, k1 + 1);
      const double pnp = ld(x, fb, i1 + 1, j1, k1 + 1);
      const double ppn = ld(x, fb, i1 + 1, j1 + 1, k1);
      const double ppp = ld(x, fb, i1 + 1, j1 + 1, k1 + 1);
      return 0.125 * (nnn + pnn + npn + nnp + npp + pnp + ppn + ppp);
    }
    default: {
      // bcx.f90: bc_x?_d (5-147) / bc_x?_n (294-436) on the outer face
      int s[3] = {g[0], g[1], g[2]};
      s[axis] = plus ? 15 : 0;
      const double x0 = ld(x, blk, s[0], s[1], s[2]);
      const int type = bc.type[face];
      if (type == BC_DIRICHLET) {
        const double xc = bc.value[face];
        return (L == 1) ? (2.0 * xc - x0) : xc;
      }
      const double xc = bc.value[face] * dx;
      if (plus) return (L == 1) ? (x0 + xc) : (x0 + xc * 2.0);
      return (L == 1) ? (x0 - xc) : (x0 - xc * 2.0);
    }
  }
}

// Two guide cells (layer 1) of the same face, positions p0 and p1 in
// [0, 256) (p = v*16 + u), with every load of both issued before any is
// used: the batched form of guide_value for the pipelined kernels.  Same
// expressions, same evaluation order, same results as guide_value.
template <typename T>
__device__ __forceinline__ void guide_pair(const T* __restrict__ x, int blk, int face,
                                           int p0, int p1, const FaceNbr& nb, const BCSet& bc,
                                           double dx, double& v0, double& v1) {
  const int axis = face >> 1;
  const bool plus = face & 1;
  const int ta = (axis == 0) ? 1 : 0, tb = (axis == 2) ? 1 : 2;
  int g0[3], g1[3];
  g0[ta] = p0 & 15; g0[tb] = p0 >> 4; g0[axis] = plus ? 16 : -1;
  g1[ta] = p1 & 15; g1[tb] = p1 >> 4; g1[axis] = plus ? 16 : -1;
  if (nb.kind == NB_SAME) {
    g0[axis] = g1[axis] = plus ? 0 : 15;
    v0 = ld(x, nb.id[0], g0[0], g0[1], g0[2]);
    v1 = ld(x, nb.id[0], g1[0], g1[1], g1[2]);
    return;
  }
  if (nb.kind == NB_COARSE) {
    int f0[3], f1[3];
    f0[ta] = g0[ta] + 1 + 16 * nb.so_u; f0[tb] = g0[tb] + 1 + 16 * nb.so_v;
    f1[ta] = g1[ta] + 1 + 16 * nb.so_u; f1[tb] = g1[tb] + 1 + 16 * nb.so_v;
    f0[axis] = f1[axis] = plus ? 1 : 32;
    int i0, j0, k0, i1, j1, k1;
    double r0, s0, t0, r1, s1, t1;
    intp_index(f0[0], 16, i0, r0); intp_index(f0[1], 16, j0, s0); intp_index(f0[2], 16, k0, t0);
    intp_index(f1[0], 16, i1, r1); intp_index(f1[1], 16, j1, s1); intp_index(f1[2], 16, k1, t1);
    --i0; --j0; --k0; --i1; --j1; --k1;
    const int c = nb.id[0];
    const double a0 = ld(x, c, i0, j0, k0), a1 = ld(x, c, i0 + 1, j0, k0);
    const double a2 = ld(x, c, i0, j0 + 1, k0), a3 = ld(x, c, i0, j0, k0 + 1);
    const double a4 = ld(x, c, i0, j0 + 1, k0 + 1), a5 = ld(x, c, i0 + 1, j0, k0 + 1);
    const double a6 = ld(x, c, i0 + 1, j0 + 1, k0), a7 = ld(x, c, i0 + 1, j0 + 1, k0 + 1);
    const double b0 = ld(x, c, i1, j1, k1), b1 = ld(x, c, i1 + 1, j1, k1);
    const double b2 = ld(x, c, i1, j1 + 1, k1), b3 = ld(x, c, i1, j1, k1 + 1);
    const double b4 = ld(x, c, i1, j1 + 1, k1 + 1), b5 = ld(x, c, i1 + 1, j1, k1 + 1);
    const double b6 = ld(x, c, i1 + 1, j1 + 1, k1), b7 = ld(x, c, i1 + 1, j1 + 1, k1 + 1);
    // nnn, pnn, npn, nnp, npp, pnp, ppn, ppp = a0..a7
    v0 = (1.0 - t0) * ((1.0 - s0) * ((1.0 - r0) * a0 + r0 * a1) + s0 * ((1.0 - r0) * a2 + r0 * a6)) +
         t0 * ((1.0 - s0) * ((1.0 - r0) * a3 + r0 * a5) + s0 * ((1.0 - r0) * a4 + r0 * a7));
    v1 = (1.0 - t1) * ((1.0 - s1) * ((1.0 - r1) * b0 + r1 * b1) + s1 * ((1.0 - r1) * b2 + r1 * b6)) +
         t1 * ((1.0 - s1) * ((1.0 - r1) * b3 + r1 * b5) + s1 * ((1.0 - r1) * b4 + r1 * b7));
    return;
  }
  if (nb.kind == NB_FINE) {
    const int fb0 = nb.id[(g0[ta] >> 3) + 2 * (g0[tb] >> 3)];
    const int fb1 = nb.id[(g1[ta] >> 3) + 2 * (g1[tb] >> 3)];
    int l0[3], l1[3];
    l0[ta] = 2 * (g0[ta] & 7); l0[tb] = 2 * (g0[tb] & 7);
    l1[ta] = 2 * (g1[ta] & 7); l1[tb] = 2 * (g1[tb] & 7);
    l0[axis] = l1[axis] = plus ? 0 : 14;
    const int i0 = l0[0], j0 = l0[1], k0 = l0[2], i1 = l1[0], j1 = l1[1], k1 = l1[2];
    const double a0 = ld(x, fb0, i0, j0, k0), a1 = ld(x, fb0, i0 + 1, j0, k0);
    const double a2 = ld(x, fb0, i0, j0 + 1, k0), a3 = ld(x, fb0, i0, j0, k0 + 1);
    const double a4 = ld(x, fb0, i0, j0 + 1, k0 + 1), a5 = ld(x, fb0, i0 + 1, j0, k0 + 1);
    const double a6 = ld(x, fb0, i0 + 1, j0 + 1, k0), a7 = ld(x, fb0, i0 + 1, j0 + 1, k0 + 1);
    const double b0 = ld(x, fb1, i1, j1, k1), b1 = ld(x, fb1, i1 + 1, j1, k1);
    const double b2 = ld(x, fb1, i1, j1 + 1, k1), b3 = ld(x, fb1, i1, j1, k1 + 1);
    const double b4 = ld(x, fb1, i1, j1 + 1, k1 + 1), b5 = ld(x, fb1, i1 + 1, j1, k1 + 1);
    const double b6 = ld(x, fb1, i1 + 1, j1 + 1, k1), b7 = ld(x, fb1, i1 + 1, j1 + 1, k1 + 1);
    v0 = 0.125 * (a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7);
    v1 = 0.125 * (b0 + b1 + b2 + b3 + b4 + b5 + b6 + b7);
    return;
  }
  // outer face: bcx.f90 bc_x?_d (5-147) / bc_x?_n (294-436), layer 1
  g0[axis] = g1[axis] = plus ? 15 : 0;
  const double x0 = ld(x, blk, g0[0], g0[1], g0[2]);
  const double x1 = ld(x, blk, g1[0], g1[1], g1[2]);
  if (bc.type[face] == BC_DIRICHLET) {
    const double xc = bc.value[face];
    v0 = 2.0 * xc - x0;
    v1 = 2.0 * xc - x1;
  } else {
    const double xc = bc.value[face] * dx;
    v0 = plus ? (x0 + xc) : (x0 - xc);
    v1 = plus ? (x1 + xc) : (x1 - xc);
  }
}

// The six stencil neighbours of cell q (in [0, 2048)) of colour c, read from
// the other colour's half O of a colour-split block (every face neighbour
// has the other colour), or from the guide layer G ([face][v][u]) where the
// neighbour lies outside the block.
template <typename T>
struct NbrsT {
  T w, e, s, n, b, t;
};
using Nbrs = NbrsT<double>;
template <typename T>
__device__ __forceinline__ NbrsT<T> split_neighbours(const T* __restrict__ O,
                                               const T* __restrict__ G, int q, int c) {
  const int ih = q & 7, j = (q >> 3) & 15, k = q >> 7;
  const int p = (j + k + c) & 1;
  const int i = 2 * ih + p;
  NbrsT<T> r;
  const T ow = O[max(q - 1 + p, 0)], oe = O[min(q + p, HALF_CELLS - 1)];
  const T os = O[max(q - 8, 0)], on = O[min(q + 8, HALF_CELLS - 1)];
  const T ob = O[max(q - 128, 0)], ot = O[min(q + 128, HALF_CELLS - 1)];
  r.w = (i == 0) ? G[0 * FACE_CELLS + j + 16 * k] : ow;
  r.e = (i == 15) ? G[1 * FACE_CELLS + j + 16 * k] : oe;
  r.s = (j == 0) ? G[2 * FACE_CELLS + i + 16 * k] : os;
  r.n = (j == 15) ? G[3 * FACE_CELLS + i + 16 * k] : on;
  r.b = (k == 0) ? G[4 * FACE_CELLS + i + 16 * j] : ob;
  r.t = (k == 15) ? G[5 * FACE_CELLS + i + 16 * j] : ot;
  return r;
}

// ---------------------------------------------------------------------------
// Coarse-fine flux conservation (no counterpart in the reference).  The
// reference's 2:1 exchange interpolates (src/CGMfuncs/sup.f90:54-179), so the
// flux a coarse cell sees through a face shared with four fine cells,
// A_f (g - x_P) with g the restriction of eight fine cells, differs from the
// sum of what the four fine cells see through their quarter faces.  The
// correction replaces the coarse side's term by that sum: per coarse cell P
// on a face f whose neighbours are finer,
//   F = 0.125 * sum_{dv, du} A_fo(phi) * (x_phi - g_phi)
// over the four fine cells phi that touch P's face (du along the face's first
// transverse axis inner, dv outer, summed from 0.0 in that order), fo the
// opposite face, A_fo(phi) the fine cell's coefficient toward P and g_phi its
// guide value across fo (the 2:1 prolongation); 0.125 is the fine-to-coarse
// volume ratio.  The corrected operator adds delta = F - A_f(P) * (g - x_P)
// to (A x)_P for each such face, in face order 0..5.
// ---------------------------------------------------------------------------
// F of the coarse cell at transverse position (a, b) of face 'face' of block
// blk (kind NB_FINE, record nb).  gx: the stored first guide layer
// [block][face][p] of x, or null to evaluate the fine guides by the exchange
// rules from x.
template <typename T>
__device__ __noinline__ double cf_fine_flux(const T* __restrict__ x, const double* __restrict__ gx,
                                            const double* __restrict__ A,
                                            const FaceNbr* __restrict__ nbr,
                                            const double* __restrict__ dxs, const BCSet& bc,
                                            int face, int a, int b, const FaceNbr& nb) {
  const int axis = face >> 1, fo = face ^ 1;
  const bool plus = face & 1;
  const int ta = (axis == 0) ? 1 : 0, tb = (axis == 2) ? 1 : 2;
  const int fb = nb.id[(a >> 3) + 2 * (b >> 3)];
  double F = 0.0;
  for (int dv = 0; dv < 2; ++dv)
    for (int du = 0; du < 2; ++du) {
      const int fu = 2 * (a & 7) + du, fv = 2 * (b & 7) + dv;
      int c[3];
      c[ta] = fu;
      c[tb] = fv;
      c[axis] = plus ? 0 : 15;
      const int s = sidx(c[0], c[1], c[2]);
      const double xf = (double)x[(size_t)fb * BLOCK_CELLS + s];
      const double gf =
          gx ? gx[((size_t)fb * 6 + fo) * FACE_CELLS + fu + 16 * fv]
             : guide_value(x, fb, fo, fu, fv, 1, nbr[(size_t)fb * 6 + fo], bc, dxs[fb]);
      const double af = A[((size_t)fb * 7 + 1 + fo) * BLOCK_CELLS + s];
      F = F + af * (xf - gf);
    }
  return 0.125 * F;
}

// y plus (SUB: minus) the correction delta of each face of cell s (storage
// slot) whose neighbours are finer, in face order; y unchanged when it has
// none.  x_P and its guide layer G (read as G[face * 256 + p]: an array, or
// an accessor of a tile) as the stencil used them, its face coefficients af(f).
template <bool SUB, typename T, typename AF, typename GA>
__device__ __forceinline__ double cf_delta(const T* __restrict__ x, const double* __restrict__ gx,
                                           const double* __restrict__ A,
                                           const FaceNbr* __restrict__ nbr,
                                           const double* __restrict__ dxs, const BCSet& bc,
                                           const FaceNbr* snb, const GA& G, double xp,
                                           int s, double y, AF af) {
  int cc[3];
  cell_of(s, cc[0], cc[1], cc[2]);
#pragma unroll 1
  for (int f = 0; f < 6; ++f) {
    const int axis = f >> 1;
    if (cc[axis] != ((f & 1) ? 15 : 0) || snb[f].kind != NB_FINE) continue;
    const int a = cc[(axis == 0) ? 1 : 0], b = cc[(axis == 2) ? 1 : 2];
    const double F = cf_fine_flux(x, gx, A, nbr, dxs, bc, f, a, b, snb[f]);
    const double d = F - af(f) * (G[f * FACE_CELLS + a + 16 * b] - xp);
    y = SUB ? y - d : y + d;
  }
  return y;
}

// ---------------------------------------------------------------------------
// Convergence bookkeeping run by the last CTA of a reduction.
// ---------------------------------------------------------------------------
// FFVILS.h:24-47 IsConverged residual
__device__ __forceinline__ double resid_of(double rr, double bb) {
  return (fabs(bb) > (double)FLT_MIN) ? sqrt(fabs(rr) / fabs(bb)) : sqrt(fabs(rr));
}

__device__ __forceinline__ void finalize(SolveState* st, double total, int fin, int iter) {
  switch (fin) {
    case FIN_STORE:
      st->rr = total;
      break;
    case FIN_BB:
      st->bb = total;
      break;
    case FIN_RBGS:
    case FIN_CG_RR:
    case FIN_BI_RR: {
      const double res = resid_of(total, st->bb);
      st->rr = total;
      st->residual = res;
      if (st->hist) st->hist[iter - 1] = res;
      st->count = iter;
      st->iter = iter;  // last iteration with a residual (history length on an early exit)
      if (res <= st->eps) {
        st->done = 1;
      } else if (isnan(res) || isinf(res)) {
        st->done = 1;
        st->status = 2;
      } else if (iter >= st->count_max) {
        st->done = 1;
        st->count = st->count_max + 1;  // loop variable after the last pass
      } else if (fin == FIN_CG_RR) {
        st->rr0 = st->rr1;
      } else if (fin == FIN_BI_RR) {
        st->rr0 = st->rr1;  // FFVILS.h:960
        st->cycle += 1;
        if (st->next_restart > 0.0 && res <= st->next_restart) {
          // restart from the current r: the next DOT(r, r0) first sets r0 = r
          st->next_restart = res * st->drop;
          st->rr0 = 1.0;
          st->alpha = 0.0;
          st->gamma = 1.0;
          st->cycle = 1;
        }
      }
      break;
    }
    case FIN_CG_RR1:
      st->rr1 = total;
      if (fabs(total) < (double)FLT_MIN) {  // FFVILS.h:720-724
        st->residual = total;
        st->count = 0;
        st->done = 1;
      } else {
        st->beta = total / st->rr0;
      }
      break;
    case FIN_CG_QP:
      st->qp = total;
      st->alpha = st->rr1 / total;
      break;
    case FIN_BI_RR1:
      st->rr1 = total;
      if (fabs(total) < (double)FLT_MIN) {  // FFVILS.h:847-851
        st->residual = total;
        st->count = 0;
        st->done = 1;
      } else {
        st->beta = total / st->rr0 * st->alpha / st->gamma;
        if (st->drop > 0.0 && st->next_restart < 0.0)  // first iteration: r0 = r
          st->next_restart = resid_of(total, st->bb) * st->drop;
      }
      break;
    case FIN_BI_QR0:
      st->qp = total;
      st->alpha = st->rr1 / total;
      break;
    case FIN_BI_TS:
      st->ts = total;
      break;
    case FIN_BI_TT:
      st->gamma = st->ts / total;
      break;
    case FIN_FA_SHIFT:
      st->alpha = -total / st->scale;
      break;
  }
}

}  // namespace ffvgpu
