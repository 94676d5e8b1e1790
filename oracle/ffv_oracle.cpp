// ffv_oracle.cpp -- CPU restatement of FFV-HC's pressure-Poisson path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA path in
// ffv-hc_b200/: only tests/, __graft_entry__.smoke() and bench.py's
// cpu_baseline / reference legs may load it.  Nothing in the product links it.
//
// PARITY UNPINNED.  The reference ships no tests, fixtures or golden vectors
// for this path, and it cannot be compiled here (its kernels are Fortran 90,
// it needs MPI and the un-vendored BCMTools/Cutlib/Polylib/TextParser/PMlib/
// HDMlib libraries; this machine has no Fortran compiler and no MPI).  This
// restatement is therefore pinned only by reading: every routine below cites
// the reference file:line it follows, keeps the reference's storage (per-block
// arrays of (n+2g)^3 reals, i fastest, lower bound 1-g, g = 2) and evaluates
// every floating-point expression in the reference's source order.  Build it
// with -O2 -ffp-contract=off (no FMA contraction, no reassociation), matching
// the reference's default gnu build (-O3 without -ffast-math; x86-64 without
// -mfma, so gfortran never contracts).
//
// Block manager.  BCMTools (halo scheduling, neighbour discovery, subface
// numbering) is absent from the reference tree.  This file restates what its
// callers rely on: a neighbour per face that is the outer boundary, a block
// of the same level, a coarser block (2:1) or four finer blocks, found here
// from (level, block index) keys.  The exchange is order independent (no
// guide cell is read to fill another guide cell), so any correct table gives
// the reference's values.
//
// Reductions.  The reference sums each block serially (i fastest) and then
// sums blocks under an OpenMP reduction, whose order is not deterministic.
// RED_REFERENCE follows the per-block serial order and adds the block sums
// in id order (block sums taken on all threads, added by one).
// RED_CANONICAL reproduces the fixed two-level tree the CUDA path uses, so
// that Krylov scalars can be compared bit for bit.

#include <cmath>
#include <cfloat>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <tuple>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

enum { X_M = 0, X_P, Y_M, Y_P, Z_M, Z_P };
enum { BC_DIRICHLET = 0, BC_NEUMANN = 1 };
enum { NB_OUTER = 0, NB_SAME = 1, NB_COARSE = 2, NB_FINE = 3 };
enum { RED_REFERENCE = 0, RED_CANONICAL = 1 };

struct Block {
  int level;
  long idx[3];
  double org[3];
  double dx;
  int kind[6];
  int nbr[6][4];
  int so[6][2];  // subfaceOrigin0/1 as the reference's updater uses them
};

struct Grid {
  int nb = 0, n = 16, g = 2;
  long nc = 0;  // (n+2g)^3
  int root_grid[3];
  double dom_org[3];
  double root_len;
  std::vector<Block> blocks;
  // outer boundary conditions of the pressure field (FFVBC.h:6-14 types)
  int bc_type[6];
  double bc_value[6];
};

inline long IDX(const Grid& G, int i, int j, int k) {
  // Fortran x(1-g:n+g, 1-g:n+g, 1-g:n+g), i fastest.
  const int w = G.n + 2 * G.g;
  return (long)(i - 1 + G.g) + (long)w * ((j - 1 + G.g) + (long)w * (k - 1 + G.g));
}

// ---------------------------------------------------------------------------
// src/CGMfuncs/bils.f90
// ---------------------------------------------------------------------------

// bils.f90:57-108 rbgs_smoother
void rbgs_smoother(const Grid& G, double* x, const double* Ap, const double* Aw,
                   const double* Ae, const double* As, const double* An,
                   const double* Ab, const double* At, const double* b,
                   double omega, int color, int offset) {
  const int n = G.n;
  const long sx = 1, sy = n + 2 * G.g, sz = sy * sy;
  for (int k = 1; k <= n; ++k)
    for (int j = 1; j <= n; ++j)
      for (int i = 1 + (k + j + color + offset) % 2; i <= n; i += 2) {
        const long m = IDX(G, i, j, k);
        double r = b[m] - Aw[m] * x[m - sx] - Ae[m] * x[m + sx] -
                   As[m] * x[m - sy] - An[m] * x[m + sy] - Ab[m] * x[m - sz] -
                   At[m] * x[m + sz];
        double x_tmp = r / Ap[m];
        x[m] = x[m] - omega * (x[m] - x_tmp);
      }
}

// bils.f90:5-55 jacobi_smoother (x1 <- sweep of x0)
void jacobi_smoother(const Grid& G, double* x1, const double* x0,
                     const double* Ap, const double* Aw, const double* Ae,
                     const double* As, const double* An, const double* Ab,
                     const double* At, const double* b, double omega) {
  const int n = G.n;
  const long sx = 1, sy = n + 2 * G.g, sz = sy * sy;
  for (int k = 1; k <= n; ++k)
    for (int j = 1; j <= n; ++j)
      for (int i = 1; i <= n; ++i) {
        const long m = IDX(G, i, j, k);
        double r = b[m] - Aw[m] * x0[m - sx] - Ae[m] * x0[m + sx] -
                   As[m] * x0[m - sy] - An[m] * x0[m + sy] -
                   Ab[m] * x0[m - sz] - At[m] * x0[m + sz];
        double x_tmp = r / Ap[m];
        x1[m] = x0[m] - omega * (x0[m] - x_tmp);
      }
}

// bils.f90:162-206 calc_ax (note the leading unary plus: the sum starts at Aw*xW)
inline double ax_cell(const double* Ap, const double* Aw, const double* Ae,
                      const double* As, const double* An, const double* Ab,
                      const double* At, const double* x, long m, long sy, long sz) {
  return Aw[m] * x[m - 1] + Ae[m] * x[m + 1] + As[m] * x[m - sy] +
         An[m] * x[m + sy] + Ab[m] * x[m - sz] + At[m] * x[m + sz] +
         Ap[m] * x[m];
}

// bils.f90:208-254 calc_r / bils.f90:256-304 calc_r2 (same expression)
inline double r_cell(const double* Ap, const double* Aw, const double* Ae,
                     const double* As, const double* An, const double* Ab,
                     const double* At, const double* x, const double* b, long m,
                     long sy, long sz) {
  return b[m] - Aw[m] * x[m - 1] - Ae[m] * x[m + 1] - As[m] * x[m - sy] -
         An[m] * x[m + sy] - Ab[m] * x[m - sz] - At[m] * x[m + sz] -
         Ap[m] * x[m];
}

// ---------------------------------------------------------------------------
// Canonical reduction order (the CUDA path's fixed tree).
//   Storage index s = c*2048 + q of a 16^3 block, q = (k*16 + j)*8 + ih,
//   i = 2*ih + ((j + k + c) & 1) with 0-based (i, j, k).
//   Per block, 512 virtual threads t: S_c = sum_{m=0..3} v[c*2048 + t + 512m]
//   (serial, from 0.0) and T_t = S_0 + S_1; the 32 virtual threads of each
//   of the 16 virtual warps are combined by an xor butterfly (16, 8, 4, 2,
//   1); the 16 warp sums are added serially from 0.0.  Across blocks: thread
//   t in [0,256) sums partial[t + 256*r] serially from 0.0, then the same
//   butterfly per warp and a serial sum over the 8 warps.
// ---------------------------------------------------------------------------
inline void cell_of_storage(int s, int& i, int& j, int& k) {
  const int c = s >> 11, q = s & 2047;
  k = q >> 7;
  j = (q >> 3) & 15;
  const int ih = q & 7;
  i = 2 * ih + ((j + k + c) & 1);
}

double butterfly_warps(const double* T, int nwarps) {
  double block = 0.0;
  for (int w = 0; w < nwarps; ++w) {
    double v[32];
    for (int l = 0; l < 32; ++l) v[l] = T[32 * w + l];
    for (int off = 16; off >= 1; off >>= 1) {
      double nv[32];
      for (int l = 0; l < 32; ++l) nv[l] = v[l] + v[l ^ off];
      std::memcpy(v, nv, sizeof(v));
    }
    block += v[0];
  }
  return block;
}

double canonical_block(const double* v /* 4096 values in storage order */) {
  double T[512];
  for (int t = 0; t < 512; ++t) {
    double S0 = 0.0, S1 = 0.0;
    for (int m = 0; m < 4; ++m) S0 += v[t + 512 * m];
    for (int m = 0; m < 4; ++m) S1 += v[2048 + t + 512 * m];
    T[t] = S0 + S1;
  }
  return butterfly_warps(T, 16);
}

double canonical_blocks(const std::vector<double>& partial) {
  double T[256];
  for (int t = 0; t < 256; ++t) {
    double S = 0.0;
    for (size_t b = t; b < partial.size(); b += 256) S += partial[b];
    T[t] = S;
  }
  return butterfly_warps(T, 8);
}

// ---------------------------------------------------------------------------
// src/CGMfuncs/blas.f90
// ---------------------------------------------------------------------------

// blas.f90:5-33 fill (guide cells included)
void fill(const Grid& G, double* x, double a) {
  for (long m = 0; m < G.nc; ++m) x[m] = a;
}
// blas.f90:69-97 copy (guide cells included)
void copy(const Grid& G, double* y, const double* x) {
  for (long m = 0; m < G.nc; ++m) y[m] = x[m];
}
// blas.f90:329-361 axpy: y = y + a*x (interior)
void axpy(const Grid& G, double* y, const double* x, double a) {
  for (int k = 1; k <= G.n; ++k)
    for (int j = 1; j <= G.n; ++j)
      for (int i = 1; i <= G.n; ++i) {
        const long m = IDX(G, i, j, k);
        y[m] = y[m] + a * x[m];
      }
}
// blas.f90:363-395 xpay: y = x + a*y (interior)
void xpay(const Grid& G, double* y, const double* x, double a) {
  for (int k = 1; k <= G.n; ++k)
    for (int j = 1; j <= G.n; ++j)
      for (int i = 1; i <= G.n; ++i) {
        const long m = IDX(G, i, j, k);
        y[m] = x[m] + a * y[m];
      }
}
// blas.f90:397-430 axpyz: z = a*x + y (interior)
void axpyz(const Grid& G, double* z, const double* x, const double* y, double a) {
  for (int k = 1; k <= G.n; ++k)
    for (int j = 1; j <= G.n; ++j)
      for (int i = 1; i <= G.n; ++i) {
        const long m = IDX(G, i, j, k);
        z[m] = a * x[m] + y[m];
      }
}
// blas.f90:432-464 axpbypz: z = a*x + b*y + z (interior)
void axpbypz(const Grid& G, double* z, const double* x, const double* y,
             double a, double b) {
  for (int k = 1; k <= G.n; ++k)
    for (int j = 1; j <= G.n; ++j)
      for (int i = 1; i <= G.n; ++i) {
        const long m = IDX(G, i, j, k);
        z[m] = a * x[m] + b * y[m] + z[m];
      }
}

// ---------------------------------------------------------------------------
// src/CGMfuncs/sup.f90 and src/FFV/Scalar3DUpdater1.cpp (the exchange)
// ---------------------------------------------------------------------------

// sup.f90:1-16 sup_get_intp_index
inline void sup_get_intp_index(int& ic, double& r, int i, int n) {
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

// sup.f90:18-52 sup_copy_from_neighbor
void sup_copy_from_neighbor(const Grid& G, double* dst, const int* i1d,
                            const double* src, const int* i1s, const int* szc) {
  for (int k = 0; k < szc[2]; ++k)
    for (int j = 0; j < szc[1]; ++j)
      for (int i = 0; i < szc[0]; ++i)
        dst[IDX(G, i + i1d[0], j + i1d[1], k + i1d[2])] =
            src[IDX(G, i + i1s[0], j + i1s[1], k + i1s[2])];
}

// sup.f90:54-120 sup_copy_from_neighbor_c2f
void sup_copy_from_neighbor_c2f(const Grid& G, double* dst, const int* i1d,
                                const double* src, const int* i1s,
                                const int* szc) {
  const int n = G.n;
  for (int k = 0; k < szc[2]; ++k)
    for (int j = 0; j < szc[1]; ++j)
      for (int i = 0; i < szc[0]; ++i) {
        const int i0 = i + i1s[0], j0 = j + i1s[1], k0 = k + i1s[2];
        int i1, j1, k1;
        double r, s, t;
        sup_get_intp_index(i1, r, i0, n);
        sup_get_intp_index(j1, s, j0, n);
        sup_get_intp_index(k1, t, k0, n);
        const double nnn = src[IDX(G, i1, j1, k1)];
        const double pnn = src[IDX(G, i1 + 1, j1, k1)];
        const double npn = src[IDX(G, i1, j1 + 1, k1)];
        const double nnp = src[IDX(G, i1, j1, k1 + 1)];
        const double npp = src[IDX(G, i1, j1 + 1, k1 + 1)];
        const double pnp = src[IDX(G, i1 + 1, j1, k1 + 1)];
        const double ppn = src[IDX(G, i1 + 1, j1 + 1, k1)];
        const double ppp = src[IDX(G, i1 + 1, j1 + 1, k1 + 1)];
        dst[IDX(G, i + i1d[0], j + i1d[1], k + i1d[2])] =
            (1.0 - t) * ((1.0 - s) * ((1.0 - r) * nnn + r * pnn) +
                         s * ((1.0 - r) * npn + r * ppn)) +
            t * ((1.0 - s) * ((1.0 - r) * nnp + r * pnp) +
                 s * ((1.0 - r) * npp + r * ppp));
      }
}

// sup.f90:122-179 sup_copy_from_neighbor_f2c
void sup_copy_from_neighbor_f2c(const Grid& G, double* dst, const int* i1d,
                                const double* src, const int* i1s,
                                const int* szc) {
  for (int k = 0; k < szc[2]; ++k)
    for (int j = 0; j < szc[1]; ++j)
      for (int i = 0; i < szc[0]; ++i) {
        const int i0 = i + i1s[0], j0 = j + i1s[1], k0 = k + i1s[2];
        const int i1 = 2 * i0 - 1, j1 = 2 * j0 - 1, k1 = 2 * k0 - 1;
        const double nnn = src[IDX(G, i1, j1, k1)];
        const double pnn = src[IDX(G, i1 + 1, j1, k1)];
        const double npn = src[IDX(G, i1, j1 + 1, k1)];
        const double nnp = src[IDX(G, i1, j1, k1 + 1)];
        const double npp = src[IDX(G, i1, j1 + 1, k1 + 1)];
        const double pnp = src[IDX(G, i1 + 1, j1, k1 + 1)];
        const double ppn = src[IDX(G, i1 + 1, j1 + 1, k1)];
        const double ppp = src[IDX(G, i1 + 1, j1 + 1, k1 + 1)];
        dst[IDX(G, i + i1d[0], j + i1d[1], k + i1d[2])] =
            0.125 * (nnn + pnn + npn + nnp + npp + pnp + ppn + ppp);
      }
}

// Scalar3DUpdater1.cpp:9-98 copyFromNeighbor index windows (same level)
void copy_same(const Grid& G, int face, double* dst, const double* src) {
  const int n = G.n, vc = G.g;
  int i1d[3] = {1, 1, 1}, i1s[3] = {1, 1, 1}, szc[3] = {n, n, n};
  switch (face) {
    case X_M: i1d[0] = 1 - vc; i1s[0] = 1 + n - vc; szc[0] = vc; break;
    case X_P: i1d[0] = 1 + n;  i1s[0] = 1;          szc[0] = vc; break;
    case Y_M: i1d[1] = 1 - vc; i1s[1] = 1 + n - vc; szc[1] = vc; break;
    case Y_P: i1d[1] = 1 + n;  i1s[1] = 1;          szc[1] = vc; break;
    case Z_M: i1d[2] = 1 - vc; i1s[2] = 1 + n - vc; szc[2] = vc; break;
    case Z_P: i1d[2] = 1 + n;  i1s[2] = 1;          szc[2] = vc; break;
  }
  sup_copy_from_neighbor(G, dst, i1d, src, i1s, szc);
}

// Scalar3DUpdater1.cpp:245-347 copyFromNeighborC2F index windows
void copy_c2f(const Grid& G, int face, int so0, int so1, double* dst,
              const double* src) {
  const int n = G.n, vc = G.g;
  int i1d[3] = {1, 1, 1}, i1s[3] = {1, 1, 1}, szc[3] = {n, n, n};
  switch (face) {
    case X_M:
      i1d[0] = 1 - vc; i1s[0] = 1 + 2 * n - vc; i1s[1] = 1 + n * so0; i1s[2] = 1 + n * so1; szc[0] = vc; break;
    case X_P:
      i1d[0] = 1 + n;  i1s[0] = 1;              i1s[1] = 1 + n * so0; i1s[2] = 1 + n * so1; szc[0] = vc; break;
    case Y_M:
      i1d[1] = 1 - vc; i1s[0] = 1 + n * so1; i1s[1] = 1 + 2 * n - vc; i1s[2] = 1 + n * so0; szc[1] = vc; break;
    case Y_P:
      i1d[1] = 1 + n;  i1s[0] = 1 + n * so1; i1s[1] = 1;              i1s[2] = 1 + n * so0; szc[1] = vc; break;
    case Z_M:
      i1d[2] = 1 - vc; i1s[0] = 1 + n * so0; i1s[1] = 1 + n * so1; i1s[2] = 1 + 2 * n - vc; szc[2] = vc; break;
    case Z_P:
      i1d[2] = 1 + n;  i1s[0] = 1 + n * so0; i1s[1] = 1 + n * so1; i1s[2] = 1;              szc[2] = vc; break;
  }
  sup_copy_from_neighbor_c2f(G, dst, i1d, src, i1s, szc);
}

// Scalar3DUpdater1.cpp:430-520 copyFromNeighborF2C index windows
void copy_f2c(const Grid& G, int face, int so0, int so1, double* dst,
              const double* src) {
  const int n = G.n, vc = G.g, h = n / 2;
  int i1d[3] = {1, 1, 1}, i1s[3] = {1, 1, 1}, szc[3] = {h, h, h};
  switch (face) {
    case X_M: i1d[0] = 1 - vc; i1d[1] = 1 + h * so0; i1d[2] = 1 + h * so1; i1s[0] = 1 + h - vc; szc[0] = vc; break;
    case X_P: i1d[0] = 1 + n;  i1d[1] = 1 + h * so0; i1d[2] = 1 + h * so1; i1s[0] = 1;          szc[0] = vc; break;
    case Y_M: i1d[0] = 1 + h * so1; i1d[1] = 1 - vc; i1d[2] = 1 + h * so0; i1s[1] = 1 + h - vc; szc[1] = vc; break;
    case Y_P: i1d[0] = 1 + h * so1; i1d[1] = 1 + n;  i1d[2] = 1 + h * so0; i1s[1] = 1;          szc[1] = vc; break;
    case Z_M: i1d[0] = 1 + h * so0; i1d[1] = 1 + h * so1; i1d[2] = 1 - vc; i1s[2] = 1 + h - vc; szc[2] = vc; break;
    case Z_P: i1d[0] = 1 + h * so0; i1d[1] = 1 + h * so1; i1d[2] = 1 + n;  i1s[2] = 1;          szc[2] = vc; break;
  }
  sup_copy_from_neighbor_f2c(G, dst, i1d, src, i1s, szc);
}

// ---------------------------------------------------------------------------
// src/CGMfuncs/bcx.f90 (outer ghost values), dispatched per face as in
// src/FFV/BlockScalar3D.h:174-181, 201-253: x3=X_M, x1=X_P, x4=Y_M, x2=Y_P,
// x6=Z_M, x5=Z_P.  Loops run over the guide rows too, as the reference does.
// ---------------------------------------------------------------------------
void bc_x(const Grid& G, double* x, int face, int type, double xc) {
  const int n = G.n, g = G.g;
  for (int b2 = 1 - g; b2 <= n + g; ++b2)
    for (int b1 = 1 - g; b1 <= n + g; ++b1) {
      long m0, m1, m2;  // interior cell, guide layer 1, guide layer 2
      switch (face) {
        case X_P: m0 = IDX(G, n, b1, b2); m1 = IDX(G, n + 1, b1, b2); m2 = IDX(G, n + 2, b1, b2); break;
        case X_M: m0 = IDX(G, 1, b1, b2); m1 = IDX(G, 0, b1, b2);     m2 = IDX(G, -1, b1, b2);    break;
        case Y_P: m0 = IDX(G, b1, n, b2); m1 = IDX(G, b1, n + 1, b2); m2 = IDX(G, b1, n + 2, b2); break;
        case Y_M: m0 = IDX(G, b1, 1, b2); m1 = IDX(G, b1, 0, b2);     m2 = IDX(G, b1, -1, b2);    break;
        case Z_P: m0 = IDX(G, b1, b2, n); m1 = IDX(G, b1, b2, n + 1); m2 = IDX(G, b1, b2, n + 2); break;
        default:  m0 = IDX(G, b1, b2, 1); m1 = IDX(G, b1, b2, 0);     m2 = IDX(G, b1, b2, -1);    break;
      }
      const bool plus = (face == X_P || face == Y_P || face == Z_P);
      if (type == BC_DIRICHLET) {
        // bcx.f90:5-147 bc_x?_d
        x[m1] = 2.0 * xc - x[m0];
        x[m2] = xc;
      } else {
        // bcx.f90:294-436 bc_x?_n
        if (plus) {
          x[m1] = x[m0] + xc;
          x[m2] = x[m0] + xc * 2.0;
        } else {
          x[m1] = x[m0] - xc;
          x[m2] = x[m0] - xc * 2.0;
        }
      }
    }
}

// ---------------------------------------------------------------------------
// src/CGMfuncs/bca.f90 (fold outer BCs into A and b), dispatched per face as
// in src/FFV/BlockScalar3D.h:183-190 (w, e, s, n, b, t order).
// ---------------------------------------------------------------------------
void bc_a(const Grid& G, double* Ap, double* Aface, double* b, int face,
          int type, double xc) {
  const int n = G.n;
  for (int b2 = 1; b2 <= n; ++b2)
    for (int b1 = 1; b1 <= n; ++b1) {
      long m;
      switch (face) {
        case X_M: m = IDX(G, 1, b1, b2); break;
        case X_P: m = IDX(G, n, b1, b2); break;
        case Y_M: m = IDX(G, b1, 1, b2); break;
        case Y_P: m = IDX(G, b1, n, b2); break;
        case Z_M: m = IDX(G, b1, b2, 1); break;
        default:  m = IDX(G, b1, b2, n); break;
      }
      if (type == BC_DIRICHLET) {
        // bca.f90:5-195 bc_A?_d
        Ap[m] = Ap[m] - Aface[m];
        b[m] = b[m] - Aface[m] * xc * 2.0;
        Aface[m] = 0.0;
      } else {
        // bca.f90:197-387 bc_A?_n: '+' on the minus faces, '-' on the plus faces
        Ap[m] = Ap[m] + Aface[m];
        if (face == X_M || face == Y_M || face == Z_M)
          b[m] = b[m] + Aface[m] * xc;
        else
          b[m] = b[m] - Aface[m] * xc;
        Aface[m] = 0.0;
      }
    }
}

// ---------------------------------------------------------------------------
// src/FFV/bcut.f90:608-832 bcut_calc_ab_p
// ---------------------------------------------------------------------------
void bcut_calc_ab_p(const Grid& G, double* Ap, double* Aw, double* Ae,
                    double* As, double* An, double* Ab, double* At, double* b,
                    double* vw, double* ve, double* vs, double* vn, double* vb,
                    double* vt, const double* ux, const double* uy,
                    const double* uz, const double* const* c,
                    const int* const* cid, const int* pid, double rhof,
                    double dx, double dt) {
  const int n = G.n;
  const long sy = n + 2 * G.g, sz = sy * sy;
  for (int k = 1; k <= n; ++k)
    for (int j = 1; j <= n; ++j)
      for (int i = 1; i <= n; ++i) {
        const long m = IDX(G, i, j, k);
        double r0 = 1.0 / rhof, r1 = 1.0 / rhof, r2 = 1.0 / rhof;
        double r3 = 1.0 / rhof, r4 = 1.0 / rhof, r5 = 1.0 / rhof;
        double vx0 = 0.5 * (ux[m] + ux[m - 1]);
        double vx1 = 0.5 * (ux[m] + ux[m + 1]);
        double vy2 = 0.5 * (uy[m] + uy[m - sy]);
        double vy3 = 0.5 * (uy[m] + uy[m + sy]);
        double vz4 = 0.5 * (uz[m] + uz[m - sz]);
        double vz5 = 0.5 * (uz[m] + uz[m + sz]);
        const double d0 = c[0][m], d1 = c[1][m], d2 = c[2][m];
        const double d3 = c[3][m], d4 = c[4][m], d5 = c[5][m];
        const int cidp0 = cid[0][m], cidp1 = cid[1][m], cidp2 = cid[2][m];
        const int cidp3 = cid[3][m], cidp4 = cid[4][m], cidp5 = cid[5][m];
        const int pidp = pid[m];
        if (cidp0 != 0) { r0 = 0.0; vx0 = vx1 * (d0 - 0.5) / (d0 + 0.5); r1 = (1.0 / rhof) / (d0 + 0.5); }
        if (cidp1 != 0) { r1 = 0.0; vx1 = vx0 * (d1 - 0.5) / (d1 + 0.5); r0 = (1.0 / rhof) / (d1 + 0.5); }
        if (cidp2 != 0) { r2 = 0.0; vy2 = vy3 * (d2 - 0.5) / (d2 + 0.5); r3 = (1.0 / rhof) / (d2 + 0.5); }
        if (cidp3 != 0) { r3 = 0.0; vy3 = vy2 * (d3 - 0.5) / (d3 + 0.5); r2 = (1.0 / rhof) / (d3 + 0.5); }
        if (cidp4 != 0) { r4 = 0.0; vz4 = vz5 * (d4 - 0.5) / (d4 + 0.5); r5 = (1.0 / rhof) / (d4 + 0.5); }
        if (cidp5 != 0) { r5 = 0.0; vz5 = vz4 * (d5 - 0.5) / (d5 + 0.5); r4 = (1.0 / rhof) / (d5 + 0.5); }
        if (cidp0 != 0 && cidp1 != 0) { r0 = 0.0; r1 = 0.0; vx0 = 0.0; vx1 = 0.0; }
        if (cidp2 != 0 && cidp3 != 0) { r2 = 0.0; r3 = 0.0; vy2 = 0.0; vy3 = 0.0; }
        if (cidp4 != 0 && cidp5 != 0) { r4 = 0.0; r5 = 0.0; vz4 = 0.0; vz5 = 0.0; }
        const double l0 = r0 / (dx * dx), l1 = r1 / (dx * dx);
        const double l2 = r2 / (dx * dx), l3 = r3 / (dx * dx);
        const double l4 = r4 / (dx * dx), l5 = r5 / (dx * dx);
        const double divv = (vx1 - vx0 + vy3 - vy2 + vz5 - vz4) / dx;
        Ap[m] = -(l0 + l1) - (l2 + l3) - (l4 + l5);
        Aw[m] = l0; Ae[m] = l1; As[m] = l2; An[m] = l3; Ab[m] = l4; At[m] = l5;
        b[m] = divv / dt;
        vw[m] = vx0; ve[m] = vx1; vs[m] = vy2; vn[m] = vy3; vb[m] = vz4; vt[m] = vz5;
        if (pidp != 1) {
          Ap[m] = -6.0;
          Aw[m] = 1.0; Ae[m] = 1.0; As[m] = 1.0; An[m] = 1.0; Ab[m] = 1.0; At[m] = 1.0;
          b[m] = 0.0;
          vw[m] = 0.0; ve[m] = 0.0; vs[m] = 0.0; vn[m] = 0.0; vb[m] = 0.0; vt[m] = 0.0;
        }
      }
}

}  // namespace

// ===========================================================================
// Oracle object: a block pool in the reference's layout plus the FFVILS
// drivers (src/FFV/FFVILS.h) over it.
// ===========================================================================

enum OracleField {
  OF_X = 0, OF_AP, OF_AW, OF_AE, OF_AS, OF_AN, OF_AB, OF_AT, OF_B,
  OF_UX, OF_UY, OF_UZ,
  OF_C0, OF_C1, OF_C2, OF_C3, OF_C4, OF_C5,
  OF_VW, OF_VE, OF_VS, OF_VN, OF_VB, OF_VT,
  OF_R, OF_P, OF_Q, OF_Z, OF_X0, OF_R0, OF_P_, OF_Q_, OF_S, OF_S_, OF_T_, OF_LAPP,
  OF_NUM
};
enum OracleIField { OI_CID0 = 0, OI_CID1, OI_CID2, OI_CID3, OI_CID4, OI_CID5, OI_PID, OI_NUM };

struct Oracle {
  Grid G;
  std::vector<std::vector<double>> f;  // OF_NUM fields, nb*nc each
  std::vector<std::vector<int>> fi;    // OI_NUM int fields
  std::vector<int> slot;               // LSSwap indirection: field id -> storage
  int red_mode = RED_REFERENCE;
  int nthreads = 1;
  std::vector<double> history;
  long exchanges = 0;

  double* F(int id, int b) { return f[slot[id]].data() + (long)b * G.nc; }
  double* F(int id) { return f[slot[id]].data(); }
};

namespace {

// LocalScalar3D.h:266-296 ImposeBoundaryCondition(): AtOnce exchange of every
// face of every block, then BlockScalar3D.h:174-181 outer BC per block.
void impose_bc(Oracle& O, int fid, const int* type, const double* value) {
  Grid& G = O.G;
  O.exchanges++;
  for (int bi = 0; bi < G.nb; ++bi) {
    const Block& B = G.blocks[bi];
    double* dst = O.F(fid, bi);
    for (int face = 0; face < 6; ++face) {
      switch (B.kind[face]) {
        case NB_SAME:
          copy_same(G, face, dst, O.F(fid, B.nbr[face][0]));
          break;
        case NB_COARSE:
          copy_c2f(G, face, B.so[face][0], B.so[face][1], dst, O.F(fid, B.nbr[face][0]));
          break;
        case NB_FINE:
          for (int q = 0; q < 4; ++q) {
            // subface q: so0 = q & 1, so1 = q >> 1
            copy_f2c(G, face, q & 1, q >> 1, dst, O.F(fid, B.nbr[face][q]));
          }
          break;
        default:
          break;
      }
    }
  }
  for (int bi = 0; bi < G.nb; ++bi) {
    const Block& B = G.blocks[bi];
    double* x = O.F(fid, bi);
    for (int face = 0; face < 6; ++face) {
      if (B.kind[face] != NB_OUTER) continue;
      double v = value[face];
      // BlockScalar3D.h:72-77: Neumann values are scaled by the cell size.
      if (type[face] == BC_NEUMANN) v = value[face] * B.dx;
      bc_x(G, x, face, type[face], v);
    }
  }
}

void impose_bc_p(Oracle& O, int fid) { impose_bc(O, fid, O.G.bc_type, O.G.bc_value); }

// FFVILS.h:24-47 IsConverged; returns 1 converged, 0 not, -1 NaN/Inf.
int is_converged(double& residual, double rr, double bb, double eps) {
  residual = (std::fabs(bb) > FLT_MIN) ? std::sqrt(std::fabs(rr) / std::fabs(bb))
                                       : std::sqrt(std::fabs(rr));
  if (residual <= eps) return 1;
  if (std::isnan(residual) || std::isinf(residual)) return -1;
  return 0;
}

// FFVILS.h:298-328 DOT (+ comm_sum_ on one rank)
double DOT(Oracle& O, int fx, int fy) {
  Grid& G = O.G;
  const int n = G.n;
  if (O.red_mode == RED_REFERENCE) {
    // per-block sums on all threads, then added in block order: the same
    // bits as one thread doing both
    std::vector<double> part(G.nb);
#pragma omp parallel for num_threads(O.nthreads) schedule(static)
    for (int bi = 0; bi < G.nb; ++bi) {
      const double* x = O.F(fx, bi);
      const double* y = O.F(fy, bi);
      double xy = 0.0;  // blas.f90:466-499 dot
      for (int k = 1; k <= n; ++k)
        for (int j = 1; j <= n; ++j)
          for (int i = 1; i <= n; ++i) {
            const long m = IDX(G, i, j, k);
            xy = xy + x[m] * y[m];
          }
      part[bi] = xy;
    }
    double xy_local = 0.0;
    for (int bi = 0; bi < G.nb; ++bi) xy_local += part[bi];
    return xy_local;
  }
  std::vector<double> part(G.nb);
#pragma omp parallel for num_threads(O.nthreads) schedule(static)
  for (int bi = 0; bi < G.nb; ++bi) {
    const double* x = O.F(fx, bi);
    const double* y = O.F(fy, bi);
    double v[4096];
    for (int s = 0; s < 4096; ++s) {
      int i, j, k;
      cell_of_storage(s, i, j, k);
      const long m = IDX(G, i + 1, j + 1, k + 1);
      v[s] = x[m] * y[m];
    }
    part[bi] = canonical_block(v);
  }
  return canonical_blocks(part);
}

// LocalScalar3D.h:130-157 CalcSum: per block sf3d_calc_sum (bsf3d.f90:35-67,
// serial in i, j, k), blocks summed serially in block order (no OpenMP there).
double SUM(Oracle& O, int fx) {
  Grid& G = O.G;
  const int n = G.n;
  if (O.red_mode == RED_REFERENCE) {
    std::vector<double> part(G.nb);
#pragma omp parallel for num_threads(O.nthreads) schedule(static)
    for (int bi = 0; bi < G.nb; ++bi) {
      const double* x = O.F(fx, bi);
      double dsum = 0.0;
      for (int k = 1; k <= n; ++k)
        for (int j = 1; j <= n; ++j)
          for (int i = 1; i <= n; ++i) dsum = dsum + x[IDX(G, i, j, k)];
      part[bi] = dsum;
    }
    double sum_l = 0.0;
    for (int bi = 0; bi < G.nb; ++bi) sum_l += part[bi];
    return sum_l;
  }
  std::vector<double> part(G.nb);
#pragma omp parallel for num_threads(O.nthreads) schedule(static)
  for (int bi = 0; bi < G.nb; ++bi) {
    const double* x = O.F(fx, bi);
    double v[4096];
    for (int s = 0; s < 4096; ++s) {
      int i, j, k;
      cell_of_storage(s, i, j, k);
      v[s] = x[IDX(G, i + 1, j + 1, k + 1)];
    }
    part[bi] = canonical_block(v);
  }
  return canonical_blocks(part);
}

// FFVILS.h:247-296 CalcR2
double CalcR2(Oracle& O, int fx) {
  Grid& G = O.G;
  const int n = G.n;
  const long sy = n + 2 * G.g, sz = sy * sy;
  const double *Ap = nullptr;
  (void)Ap;
  if (O.red_mode == RED_REFERENCE) {
    std::vector<double> part(G.nb);
#pragma omp parallel for num_threads(O.nthreads) schedule(static)
    for (int bi = 0; bi < G.nb; ++bi) {
      const double* x = O.F(fx, bi);
      double rr = 0.0;  // bils.f90:256-304 calc_r2
      for (int k = 1; k <= n; ++k)
        for (int j = 1; j <= n; ++j)
          for (int i = 1; i <= n; ++i) {
            const long m = IDX(G, i, j, k);
            const double r = r_cell(O.F(OF_AP, bi), O.F(OF_AW, bi), O.F(OF_AE, bi),
                                    O.F(OF_AS, bi), O.F(OF_AN, bi), O.F(OF_AB, bi),
                                    O.F(OF_AT, bi), x, O.F(OF_B, bi), m, sy, sz);
            rr = rr + r * r;
          }
      part[bi] = rr;
    }
    double rr_local = 0.0;
    for (int bi = 0; bi < G.nb; ++bi) rr_local += part[bi];
    return rr_local;
  }
  std::vector<double> part(G.nb);
#pragma omp parallel for num_threads(O.nthreads) schedule(static)
  for (int bi = 0; bi < G.nb; ++bi) {
    const double* x = O.F(fx, bi);
    double v[4096];
    for (int s = 0; s < 4096; ++s) {
      int i, j, k;
      cell_of_storage(s, i, j, k);
      const long m = IDX(G, i + 1, j + 1, k + 1);
      const double r = r_cell(O.F(OF_AP, bi), O.F(OF_AW, bi), O.F(OF_AE, bi),
                              O.F(OF_AS, bi), O.F(OF_AN, bi), O.F(OF_AB, bi),
                              O.F(OF_AT, bi), x, O.F(OF_B, bi), m, sy, sz);
      v[s] = r * r;
    }
    part[bi] = canonical_block(v);
  }
  return canonical_blocks(part);
}

// FFVILS.h:104-162 RBGS_Smoother
void RBGS_Smoother(Oracle& O, int fx, double omega) {
  Grid& G = O.G;
#pragma omp parallel for num_threads(O.nthreads) schedule(static)
  for (int bi = 0; bi < G.nb; ++bi) {
    for (int color = 0; color < 2; ++color)
      rbgs_smoother(G, O.F(fx, bi), O.F(OF_AP, bi), O.F(OF_AW, bi), O.F(OF_AE, bi),
                    O.F(OF_AS, bi), O.F(OF_AN, bi), O.F(OF_AB, bi), O.F(OF_AT, bi),
                    O.F(OF_B, bi), omega, color, 0);
  }
  impose_bc_p(O, fx);
}

// FFVILS.h:49-102 Jacobi_Smoother: x0 <- sweep(x); LSSwap(x, x0); exchange x
void Jacobi_Smoother(Oracle& O, int fx, int fb, int fx0, double omega) {
  Grid& G = O.G;
#pragma omp parallel for num_threads(O.nthreads) schedule(static)
  for (int bi = 0; bi < G.nb; ++bi)
    jacobi_smoother(G, O.F(fx0, bi), O.F(fx, bi), O.F(OF_AP, bi), O.F(OF_AW, bi),
                    O.F(OF_AE, bi), O.F(OF_AS, bi), O.F(OF_AN, bi), O.F(OF_AB, bi),
                    O.F(OF_AT, bi), O.F(fb, bi), omega);
  std::swap(O.slot[fx], O.slot[fx0]);  // LocalScalar3D.h:115-119 LSSwap
  impose_bc_p(O, fx);
}

// FFVILS.h:164-202 CalcAx
void CalcAx(Oracle& O, int fax, int fx) {
  Grid& G = O.G;
  const int n = G.n;
  const long sy = n + 2 * G.g, sz = sy * sy;
#pragma omp parallel for num_threads(O.nthreads) schedule(static)
  for (int bi = 0; bi < G.nb; ++bi) {
    double* Ax = O.F(fax, bi);
    const double* x = O.F(fx, bi);
    for (int k = 1; k <= n; ++k)
      for (int j = 1; j <= n; ++j)
        for (int i = 1; i <= n; ++i) {
          const long m = IDX(G, i, j, k);
          Ax[m] = ax_cell(O.F(OF_AP, bi), O.F(OF_AW, bi), O.F(OF_AE, bi),
                          O.F(OF_AS, bi), O.F(OF_AN, bi), O.F(OF_AB, bi),
                          O.F(OF_AT, bi), x, m, sy, sz);
        }
  }
}

// FFVILS.h:204-245 CalcR
void CalcR(Oracle& O, int fr, int fx, int fb) {
  Grid& G = O.G;
  const int n = G.n;
  const long sy = n + 2 * G.g, sz = sy * sy;
#pragma omp parallel for num_threads(O.nthreads) schedule(static)
  for (int bi = 0; bi < G.nb; ++bi) {
    double* r = O.F(fr, bi);
    const double* x = O.F(fx, bi);
    for (int k = 1; k <= n; ++k)
      for (int j = 1; j <= n; ++j)
        for (int i = 1; i <= n; ++i) {
          const long m = IDX(G, i, j, k);
          r[m] = r_cell(O.F(OF_AP, bi), O.F(OF_AW, bi), O.F(OF_AE, bi),
                        O.F(OF_AS, bi), O.F(OF_AN, bi), O.F(OF_AB, bi),
                        O.F(OF_AT, bi), x, O.F(fb, bi), m, sy, sz);
        }
  }
}

void FILL(Oracle& O, int fx, double a) {
#pragma omp parallel for num_threads(O.nthreads) schedule(static)
  for (int bi = 0; bi < O.G.nb; ++bi) fill(O.G, O.F(fx, bi), a);
}
void COPY(Oracle& O, int fy, int fx) {
#pragma omp parallel for num_threads(O.nthreads) schedule(static)
  for (int bi = 0; bi < O.G.nb; ++bi) copy(O.G, O.F(fy, bi), O.F(fx, bi));
}
void AXPY(Oracle& O, int fy, int fx, double a) {
#pragma omp parallel for num_threads(O.nthreads) schedule(static)
  for (int bi = 0; bi < O.G.nb; ++bi) axpy(O.G, O.F(fy, bi), O.F(fx, bi), a);
}
void XPAY(Oracle& O, int fy, int fx, double a) {
#pragma omp parallel for num_threads(O.nthreads) schedule(static)
  for (int bi = 0; bi < O.G.nb; ++bi) xpay(O.G, O.F(fy, bi), O.F(fx, bi), a);
}
void AXPYZ(Oracle& O, int fz, int fx, int fy, double a) {
#pragma omp parallel for num_threads(O.nthreads) schedule(static)
  for (int bi = 0; bi < O.G.nb; ++bi) axpyz(O.G, O.F(fz, bi), O.F(fx, bi), O.F(fy, bi), a);
}
void AXPBYPZ(Oracle& O, int fz, int fx, int fy, double a, double b) {
#pragma omp parallel for num_threads(O.nthreads) schedule(static)
  for (int bi = 0; bi < O.G.nb; ++bi)
    axpbypz(O.G, O.F(fz, bi), O.F(fx, bi), O.F(fy, bi), a, b);
}

// FFVILS.h:469-492 Jacobi_PreConditioner
void Jacobi_PreConditioner(Oracle& O, int fx, int fb, int fx0, double omega, int countPre) {
  for (int c = 0; c < countPre; ++c) Jacobi_Smoother(O, fx, fb, fx0, omega);
}

}  // namespace

// ===========================================================================
// extern "C" API for the test harness (ctypes).
// ===========================================================================
extern "C" {

Oracle* orc_create(int nb, int n, int g, const int* level, const long* idx3,
                   const double* dom_org, double root_len, const int* root_grid) {
  Oracle* O = new Oracle();
  Grid& G = O->G;
  G.nb = nb;
  G.n = n;
  G.g = g;
  const long w = n + 2 * g;
  G.nc = w * w * w;
  for (int a = 0; a < 3; ++a) {
    G.root_grid[a] = root_grid[a];
    G.dom_org[a] = dom_org[a];
  }
  G.root_len = root_len;
  for (int f = 0; f < 6; ++f) {
    G.bc_type[f] = BC_NEUMANN;
    G.bc_value[f] = 0.0;
  }
  G.blocks.resize(nb);
  std::map<std::tuple<int, long, long, long>, int> key;
  for (int b = 0; b < nb; ++b) {
    Block& B = G.blocks[b];
    B.level = level[b];
    const double bl = root_len / (double)(1L << B.level);
    for (int a = 0; a < 3; ++a) {
      B.idx[a] = idx3[3 * b + a];
      B.org[a] = dom_org[a] + bl * (double)B.idx[a];
    }
    B.dx = bl / (double)n;
    key[std::make_tuple(B.level, B.idx[0], B.idx[1], B.idx[2])] = b;
  }
  auto find = [&](int L, long x, long y, long z) -> int {
    auto it = key.find(std::make_tuple(L, x, y, z));
    return it == key.end() ? -1 : it->second;
  };
  int bad = 0;
  for (int b = 0; b < nb; ++b) {
    Block& B = G.blocks[b];
    for (int face = 0; face < 6; ++face) {
      const int ax = face / 2, dir = (face & 1) ? 1 : -1;
      long nI[3] = {B.idx[0], B.idx[1], B.idx[2]};
      nI[ax] += dir;
      const long ext = (long)root_grid[ax] << B.level;
      for (int q = 0; q < 4; ++q) B.nbr[face][q] = -1;
      B.so[face][0] = B.so[face][1] = 0;
      // transverse axes in the reference's subfaceOrigin order
      // (Scalar3DUpdater1.cpp:263-341): X -> (j, k), Y -> (k, i), Z -> (i, j)
      int t0, t1;
      if (ax == 0) { t0 = 1; t1 = 2; } else if (ax == 1) { t0 = 2; t1 = 0; } else { t0 = 0; t1 = 1; }
      if (nI[ax] < 0 || nI[ax] >= ext) {
        B.kind[face] = NB_OUTER;
        continue;
      }
      int s = find(B.level, nI[0], nI[1], nI[2]);
      if (s >= 0) {
        B.kind[face] = NB_SAME;
        B.nbr[face][0] = s;
        continue;
      }
      if (B.level > 0) {
        int c = find(B.level - 1, nI[0] >> 1, nI[1] >> 1, nI[2] >> 1);
        if (c >= 0) {
          B.kind[face] = NB_COARSE;
          B.nbr[face][0] = c;
          B.so[face][0] = (int)(B.idx[t0] & 1);
          B.so[face][1] = (int)(B.idx[t1] & 1);
          continue;
        }
      }
      B.kind[face] = NB_FINE;
      for (int q = 0; q < 4; ++q) {
        const int s0 = q & 1, s1 = q >> 1;
        long c[3];
        c[ax] = 2 * nI[ax] + (dir > 0 ? 0 : 1);
        c[t0] = 2 * nI[t0] + s0;
        c[t1] = 2 * nI[t1] + s1;
        const int fb = find(B.level + 1, c[0], c[1], c[2]);
        if (fb < 0) bad++;
        B.nbr[face][q] = fb;
      }
    }
  }
  if (bad) {
    std::fprintf(stderr, "orc_create: grid is not 2:1 face balanced (%d)\n", bad);
    delete O;
    return nullptr;
  }
  O->f.assign(OF_NUM, std::vector<double>((size_t)nb * G.nc, 0.0));
  O->fi.assign(OI_NUM, std::vector<int>((size_t)nb * G.nc, 0));
  O->slot.resize(OF_NUM);
  for (int i = 0; i < OF_NUM; ++i) O->slot[i] = i;
  return O;
}

void orc_destroy(Oracle* O) { delete O; }
double* orc_field(Oracle* O, int id) { return O->F(id); }
int* orc_ifield(Oracle* O, int id) { return O->fi[id].data(); }
long orc_cells_per_block(Oracle* O) { return O->G.nc; }
void orc_set_threads(Oracle* O, int n) { O->nthreads = n > 0 ? n : 1; }
void orc_set_reduction(Oracle* O, int mode) { O->red_mode = mode; }
int orc_neighbor(Oracle* O, int b, int face, int* kind, int* nbr4, int* so2) {
  const Block& B = O->G.blocks[b];
  *kind = B.kind[face];
  for (int q = 0; q < 4; ++q) nbr4[q] = B.nbr[face][q];
  so2[0] = B.so[face][0];
  so2[1] = B.so[face][1];
  return 0;
}
double orc_block_dx(Oracle* O, int b) { return O->G.blocks[b].dx; }
void orc_set_bc(Oracle* O, const int* type6, const double* value6) {
  for (int f = 0; f < 6; ++f) {
    O->G.bc_type[f] = type6[f];
    O->G.bc_value[f] = value6[f];
  }
}
// Exchange + outer BC of any field with explicit BCs (e.g. velocity, P02).
void orc_exchange(Oracle* O, int fid, const int* type6, const double* value6) {
  impose_bc(*O, fid, type6, value6);
}
// Solver.cpp:5404-5484 (P03): per block bcut_calc_ab_p_
void orc_assemble_p(Oracle* O, double rhof, double dt) {
  Grid& G = O->G;
#pragma omp parallel for num_threads(O->nthreads) schedule(static)
  for (int bi = 0; bi < G.nb; ++bi) {
    const double* c[6];
    const int* cid[6];
    for (int f = 0; f < 6; ++f) {
      c[f] = O->F(OF_C0 + f, bi);
      cid[f] = O->fi[OI_CID0 + f].data() + (long)bi * G.nc;
    }
    bcut_calc_ab_p(G, O->F(OF_AP, bi), O->F(OF_AW, bi), O->F(OF_AE, bi),
                   O->F(OF_AS, bi), O->F(OF_AN, bi), O->F(OF_AB, bi),
                   O->F(OF_AT, bi), O->F(OF_B, bi), O->F(OF_VW, bi),
                   O->F(OF_VE, bi), O->F(OF_VS, bi), O->F(OF_VN, bi),
                   O->F(OF_VB, bi), O->F(OF_VT, bi), O->F(OF_UX, bi),
                   O->F(OF_UY, bi), O->F(OF_UZ, bi), c, cid,
                   O->fi[OI_PID].data() + (long)bi * G.nc, rhof, G.blocks[bi].dx, dt);
  }
}
// Solver.cpp:5574 (P05) -> LocalScalar3D.h:298-323 -> BlockScalar3D.h:183-190
void orc_fold_bc(Oracle* O) {
  Grid& G = O->G;
  static const int face_of[6] = {X_M, X_P, Y_M, Y_P, Z_M, Z_P};
  static const int coef_of[6] = {OF_AW, OF_AE, OF_AS, OF_AN, OF_AB, OF_AT};
  for (int bi = 0; bi < G.nb; ++bi) {
    const Block& B = G.blocks[bi];
    for (int q = 0; q < 6; ++q) {
      const int face = face_of[q];
      if (B.kind[face] != NB_OUTER) continue;
      double v = G.bc_value[face];
      if (G.bc_type[face] == BC_NEUMANN) v = G.bc_value[face] * B.dx;
      bc_a(G, O->F(OF_AP, bi), O->F(coef_of[q], bi), O->F(OF_B, bi), face,
           G.bc_type[face], v);
    }
  }
}

// Single RBGS smoother pass (both colours + exchange), FFVILS.h:104-162.
void orc_rbgs_sweep(Oracle* O, double omega) { RBGS_Smoother(*O, OF_X, omega); }
double orc_calc_r2(Oracle* O) { return CalcR2(*O, OF_X); }
double orc_dot(Oracle* O, int fx, int fy) { return DOT(*O, fx, fy); }
void orc_calc_ax(Oracle* O, int fax, int fx) { CalcAx(*O, fax, fx); }
void orc_calc_r(Oracle* O, int fr, int fx, int fb) { CalcR(*O, fr, fx, fb); }
void orc_jacobi_smoother(Oracle* O, int fx, int fb, int fx0, double omega) {
  Jacobi_Smoother(*O, fx, fb, fx0, omega);
}
int orc_slot(Oracle* O, int id) { return O->slot[id]; }

// FFVILS.h:547-594 RBGS.  Returns 0 ok, 2 NaN/Inf (reference: Exit(0)).
int orc_rbgs(Oracle* O, double omega, int countMax, double epsilon, int* count,
             double* residual, double* hist) {
  Oracle& R = *O;
  double bb = DOT(R, OF_B, OF_B);
  int c;
  for (c = 1; c <= countMax; ++c) {
    RBGS_Smoother(R, OF_X, omega);
    double rr = CalcR2(R, OF_X);
    int st = is_converged(*residual, rr, bb, epsilon);
    if (hist) hist[c - 1] = *residual;
    if (st < 0) {
      *count = c;
      return 2;
    }
    if (st == 1) break;
  }
  *count = (c > countMax) ? countMax + 1 : c;  // loop variable as in the reference
  return 0;
}

// FFVILS.h:661-791 CG (Jacobi-preconditioned).  Returns 0 ok, 2 NaN/Inf.
int orc_cg(Oracle* O, double omega, int countPre, int countMax, double epsilon,
           int* count, double* residual, double* hist) {
  Oracle& R = *O;
  double bb = DOT(R, OF_B, OF_B);
  if (std::fabs(bb) < FLT_MIN) {
    *residual = 0.0;
    *count = 0;
    return 0;
  }
  CalcR(R, OF_R, OF_X, OF_B);
  impose_bc_p(R, OF_R);
  double rr0 = 1.0, rr1 = 0.0;
  int c;
  for (c = 1; c <= countMax; ++c) {
    FILL(R, OF_Z, 0.0);
    Jacobi_PreConditioner(R, OF_Z, OF_R, OF_X0, omega, countPre);
    rr1 = DOT(R, OF_R, OF_Z);
    if (std::fabs(rr1) < FLT_MIN) {
      *residual = rr1;
      c = 0;
      break;
    }
    double beta = rr1 / rr0;
    if (c == 1)
      COPY(R, OF_P, OF_Z);
    else
      XPAY(R, OF_P, OF_Z, beta);
    impose_bc_p(R, OF_P);
    CalcAx(R, OF_Q, OF_P);
    double qp = DOT(R, OF_Q, OF_P);
    double alpha = rr1 / qp;
    AXPY(R, OF_X, OF_P, alpha);
    AXPY(R, OF_R, OF_Q, -alpha);
    impose_bc_p(R, OF_R);
    double rr = DOT(R, OF_R, OF_R);
    int st = is_converged(*residual, rr, bb, epsilon);
    if (hist) hist[c - 1] = *residual;
    if (st < 0) {
      *count = c;
      return 2;
    }
    if (st == 1) break;
    rr0 = rr1;
  }
  impose_bc_p(R, OF_X);
  *count = (c > countMax) ? countMax + 1 : c;
  return 0;
}

// FFVILS.h:793-974 BiCGSTAB (Jacobi-preconditioned).  Returns 0 ok, 2 NaN/Inf.
int orc_bicgstab_restart(Oracle* O, double omega, int countPre, int countMax, double epsilon,
                         double restart_drop, int* count, double* residual, double* hist);

// bcut.f90:3879-4061 bcut_remove_p (corr = 0) and bcut.f90:4063-4297
// bcut_corr_u (corr = 1), per block in i, j, k order, on the reference
// layout: p = X with the guide values it holds.
void orc_projection(Oracle* O, int corr, double rhof, double dt) {
  Oracle& R = *O;
  Grid& G = R.G;
  const int n = G.n;
  const long sy = n + 2 * G.g, sz = sy * sy;
#pragma omp parallel for num_threads(R.nthreads) schedule(static)
  for (int bi = 0; bi < G.nb; ++bi) {
    const double dx = G.blocks[bi].dx;
    const double* p = R.F(OF_X, bi);
    double* ux = R.F(OF_UX, bi);
    double* uy = R.F(OF_UY, bi);
    double* uz = R.F(OF_UZ, bi);
    double* vw = R.F(OF_VW, bi);
    double* ve = R.F(OF_VE, bi);
    double* vs = R.F(OF_VS, bi);
    double* vn = R.F(OF_VN, bi);
    double* vb = R.F(OF_VB, bi);
    double* vt = R.F(OF_VT, bi);
    double* lapp = R.F(OF_LAPP, bi);
    const double* c[6] = {R.F(OF_C0, bi), R.F(OF_C1, bi), R.F(OF_C2, bi),
                          R.F(OF_C3, bi), R.F(OF_C4, bi), R.F(OF_C5, bi)};
    const int* cid[6];
    for (int f = 0; f < 6; ++f) cid[f] = R.fi[OI_CID0 + f].data() + (long)bi * G.nc;
    const int* pid = R.fi[OI_PID].data() + (long)bi * G.nc;
    for (int k = 1; k <= n; ++k)
      for (int j = 1; j <= n; ++j)
        for (int i = 1; i <= n; ++i) {
          const long m = IDX(G, i, j, k);
          const double r0 = 1.0 / rhof, r1 = 1.0 / rhof, r2 = 1.0 / rhof;
          const double r3 = 1.0 / rhof, r4 = 1.0 / rhof, r5 = 1.0 / rhof;
          double dpx0 = (p[m] - p[m - 1]) / dx;
          double dpx1 = (p[m + 1] - p[m]) / dx;
          double dpy2 = (p[m] - p[m - sy]) / dx;
          double dpy3 = (p[m + sy] - p[m]) / dx;
          double dpz4 = (p[m] - p[m - sz]) / dx;
          double dpz5 = (p[m + sz] - p[m]) / dx;
          double rdpx0 = r0 * dpx0, rdpx1 = r1 * dpx1, rdpy2 = r2 * dpy2;
          double rdpy3 = r3 * dpy3, rdpz4 = r4 * dpz4, rdpz5 = r5 * dpz5;
          const double d0 = c[0][m], d1 = c[1][m], d2 = c[2][m];
          const double d3 = c[3][m], d4 = c[4][m], d5 = c[5][m];
          const int cp0 = cid[0][m], cp1 = cid[1][m], cp2 = cid[2][m];
          const int cp3 = cid[3][m], cp4 = cid[4][m], cp5 = cid[5][m];
          if (cp0 != 0) { rdpx0 = rdpx1 * (d0 - 0.5) / (d0 + 0.5); dpx0 = dpx1 * (d0 - 0.5) / (d0 + 0.5); }
          if (cp1 != 0) { rdpx1 = rdpx0 * (d1 - 0.5) / (d1 + 0.5); dpx1 = dpx0 * (d1 - 0.5) / (d1 + 0.5); }
          if (cp2 != 0) { rdpy2 = rdpy3 * (d2 - 0.5) / (d2 + 0.5); dpy2 = dpy3 * (d2 - 0.5) / (d2 + 0.5); }
          if (cp3 != 0) { rdpy3 = rdpy2 * (d3 - 0.5) / (d3 + 0.5); dpy3 = dpy2 * (d3 - 0.5) / (d3 + 0.5); }
          if (cp4 != 0) { rdpz4 = rdpz5 * (d4 - 0.5) / (d4 + 0.5); dpz4 = dpz5 * (d4 - 0.5) / (d4 + 0.5); }
          if (cp5 != 0) { rdpz5 = rdpz4 * (d5 - 0.5) / (d5 + 0.5); dpz5 = dpz4 * (d5 - 0.5) / (d5 + 0.5); }
          if (cp0 != 0 && cp1 != 0) { rdpx0 = 0.0; rdpx1 = 0.0; }
          if (cp2 != 0 && cp3 != 0) { rdpy2 = 0.0; rdpy3 = 0.0; }
          if (cp4 != 0 && cp5 != 0) { rdpz4 = 0.0; rdpz5 = 0.0; }
          const double rdpx = 0.5 * (rdpx0 + rdpx1);
          const double rdpy = 0.5 * (rdpy2 + rdpy3);
          const double rdpz = 0.5 * (rdpz4 + rdpz5);
          (void)dpx0; (void)dpx1; (void)dpy2; (void)dpy3; (void)dpz4; (void)dpz5;
          if (!corr) {
            ux[m] = ux[m] + rdpx * dt;
            uy[m] = uy[m] + rdpy * dt;
            uz[m] = uz[m] + rdpz * dt;
            if (pid[m] != 1) ux[m] = uy[m] = uz[m] = 0.0;
          } else {
            ux[m] = ux[m] - rdpx * dt;
            uy[m] = uy[m] - rdpy * dt;
            uz[m] = uz[m] - rdpz * dt;
            vw[m] = vw[m] - rdpx0 * dt;
            ve[m] = ve[m] - rdpx1 * dt;
            vs[m] = vs[m] - rdpy2 * dt;
            vn[m] = vn[m] - rdpy3 * dt;
            vb[m] = vb[m] - rdpz4 * dt;
            vt[m] = vt[m] - rdpz5 * dt;
            lapp[m] = (p[m + 1] + p[m - 1] + p[m + sy] + p[m - sy] + p[m + sz] + p[m - sz] -
                       6.0 * p[m]) / (dx * dx);
            if (pid[m] != 1) {
              ux[m] = uy[m] = uz[m] = 0.0;
              vw[m] = ve[m] = vs[m] = vn[m] = vb[m] = vt[m] = 0.0;
              lapp[m] = 0.0;
            }
            if (cp0 != 0 || cp1 != 0 || cp2 != 0 || cp3 != 0 || cp4 != 0 || cp5 != 0)
              lapp[m] = 0.0;
          }
        }
  }
}

// FFVILS.h:596-659 RBGS_WithFixedAverage (the reference's xave is unused).
int orc_rbgs_fixed_average(Oracle* O, double omega, long ncells, int countMax, double epsilon,
                           int* count, double* residual, double* hist) {
  Oracle& R = *O;
  const double bb = DOT(R, OF_B, OF_B);
  int c;
  for (c = 1; c <= countMax; ++c) {
    RBGS_Smoother(R, OF_X, omega);
    const double sum_x1 = SUM(R, OF_X);
    const double a = -sum_x1 / (double)ncells;
    for (int bi = 0; bi < R.G.nb; ++bi) {  // adda, blas.f90:162-193
      double* x = R.F(OF_X, bi);
      for (int k = 1; k <= R.G.n; ++k)
        for (int j = 1; j <= R.G.n; ++j)
          for (int i = 1; i <= R.G.n; ++i) {
            const long m = IDX(R.G, i, j, k);
            x[m] = x[m] + a;
          }
    }
    impose_bc_p(R, OF_X);
    const double rr = CalcR2(R, OF_X);
    const int st = is_converged(*residual, rr, bb, epsilon);
    if (hist) hist[c - 1] = *residual;
    if (st < 0) {
      *count = c;
      return 2;
    }
    if (st == 1) break;
  }
  *count = (c > countMax) ? countMax + 1 : c;
  return 0;
}

int orc_bicgstab(Oracle* O, double omega, int countPre, int countMax,
                 double epsilon, int* count, double* residual, double* hist) {
  return orc_bicgstab_restart(O, omega, countPre, countMax, epsilon, 0.0, count, residual, hist);
}

// FFVILS::BiCGSTAB; restart_drop > 0 (no counterpart in the reference)
// restarts the recurrence (r0 = r, p = r) each time the residual has fallen
// by that factor since the last (re)start, as the GPU's restart option does.
int orc_bicgstab_restart(Oracle* O, double omega, int countPre, int countMax, double epsilon,
                         double restart_drop, int* count, double* residual, double* hist) {
  Oracle& R = *O;
  double bb = DOT(R, OF_B, OF_B);
  if (std::fabs(bb) < FLT_MIN) {
    *residual = 0.0;
    *count = 0;
    return 0;
  }
  CalcR(R, OF_R, OF_X, OF_B);
  COPY(R, OF_R0, OF_R);
  double rr0 = 1.0, alpha = 0.0, gamma = 1.0;
  double next_restart = -1.0;
  int cycle = 1;
  int c;
  for (c = 1; c <= countMax; ++c) {
    double rr1 = DOT(R, OF_R, OF_R0);
    if (std::fabs(rr1) < FLT_MIN) {
      *residual = rr1;
      c = 0;
      break;
    }
    if (c == 1 && restart_drop > 0.0) {
      double r_init;
      is_converged(r_init, rr1, bb, 0.0);
      next_restart = r_init * restart_drop;
    }
    if (cycle == 1) {
      COPY(R, OF_P, OF_R);
    } else {
      double beta = rr1 / rr0 * alpha / gamma;
      AXPY(R, OF_P, OF_Q_, -gamma);
      XPAY(R, OF_P, OF_R, beta);
    }
    impose_bc_p(R, OF_P);
    FILL(R, OF_P_, 0.0);
    Jacobi_PreConditioner(R, OF_P_, OF_P, OF_X0, omega, countPre);
    CalcAx(R, OF_Q_, OF_P_);
    double q_r0 = DOT(R, OF_Q_, OF_R0);
    alpha = rr1 / q_r0;
    AXPYZ(R, OF_S, OF_Q_, OF_R, -alpha);
    impose_bc_p(R, OF_S);
    FILL(R, OF_S_, 0.0);
    Jacobi_PreConditioner(R, OF_S_, OF_S, OF_X0, omega, countPre);
    CalcAx(R, OF_T_, OF_S_);
    double t_s = DOT(R, OF_T_, OF_S);
    double t_t_ = DOT(R, OF_T_, OF_T_);
    gamma = t_s / t_t_;
    AXPBYPZ(R, OF_X, OF_P_, OF_S_, alpha, gamma);
    AXPYZ(R, OF_R, OF_T_, OF_S, -gamma);
    double rr = DOT(R, OF_R, OF_R);
    int st = is_converged(*residual, rr, bb, epsilon);
    if (hist) hist[c - 1] = *residual;
    if (st < 0) {
      *count = c;
      return 2;
    }
    if (st == 1) break;
    rr0 = rr1;
    ++cycle;
    if (next_restart > 0.0 && *residual <= next_restart && c < countMax) {
      next_restart = *residual * restart_drop;
      COPY(R, OF_R0, OF_R);
      rr0 = 1.0;
      alpha = 0.0;
      gamma = 1.0;
      cycle = 1;
    }
  }
  impose_bc_p(R, OF_X);
  *count = (c > countMax) ? countMax + 1 : c;
  return 0;
}

// ---------------------------------------------------------------------------
// Mixed-precision form (no counterpart in the reference): orc_bicgstab's
// recurrence (FFVILS.h:793-974) with Jacobi_PreConditioner replaced by
// red-black SOR sweeps from zero on 32-bit data, 'per' sweeps between guide
// exchanges.  Restates ffv-hc_b200/csrc/kernels_mixed.cu:
//   coefficients aw..at and dinv = 1.0 / Ap, each rounded to 20 fraction
//   bits (the FP64 bit pattern plus 2^31, low word cleared) -- the 32-bit
//   words the kernel keeps;
//   per pass, the iterate in FP64: zero (interior and guides) in the first
//   pass; later, the FP32 iterate of the previous pass widened and its
//   first guide layer by the exchange (homogeneous Dirichlet outer faces),
//   in FP64;
//   per cell of colour c (colour 0 first, rbgs_smoother's order of terms),
//   with the FP64 right-hand side v:
//     rc = fma(-aw, eW, v) ... fma(-at, eT, rc); xt = rc * dinv;
//     e = fma(-omega, e - xt, e)
//   at the end of a pass the iterate is rounded to FP32.
// The preconditioned vectors' guides come from the pressure-BC exchange
// before CalcAx, and every dot product is DOT.  The FP64-data variant
// (data64) keeps the coefficients unrounded and the iterate in FP64 between
// passes; the arithmetic is the same.  With cf, the FP64 residual and both
// A*x products add the coarse-fine flux correction (cf_apply).
// ---------------------------------------------------------------------------
namespace {

struct Coef32 {
  std::vector<double> a[7];  // aw, ae, as, an, ab, at, dinv (rounded); reference layout
};

double round_hi(double x) {
  uint64_t u;
  std::memcpy(&u, &x, 8);
  u = (u + 0x80000000ull) & 0xFFFFFFFF00000000ull;
  double d;
  std::memcpy(&d, &u, 8);
  return d;
}

// data64 (the FP64-data variant): the FP64 values themselves, unrounded.
void mixed_coef(Oracle& O, Coef32& C, bool data64) {
  const long N = (long)O.G.nb * O.G.nc;
  const int src[6] = {OF_AW, OF_AE, OF_AS, OF_AN, OF_AB, OF_AT};
  auto rnd = [data64](double v) { return data64 ? v : round_hi(v); };
  for (int a = 0; a < 7; ++a) C.a[a].assign(N, 0.0);
  for (int bi = 0; bi < O.G.nb; ++bi)
    for (long m = 0; m < O.G.nc; ++m) {
      const long g = (long)bi * O.G.nc + m;
      for (int a = 0; a < 6; ++a) C.a[a][g] = rnd(O.F(src[a], bi)[m]);
      C.a[6][g] = rnd(1.0 / O.F(OF_AP, bi)[m]);
    }
}

// out = M(v), widened to double (interior).  The pass's FP64 iterate with
// its guide layer lives in the scratch field Z.  Between passes the iterate
// is rounded to FP32 (data64: kept in FP64).
void mixed_precondition(Oracle& O, const Coef32& C, int fv, int fout, float omega, int sweeps,
                        int per, bool data64) {
  Grid& G = O.G;
  const int n = G.n;
  const long sy = n + 2 * G.g, sz = sy * sy;
  const long N = (long)G.nb * G.nc;
  std::vector<double> e(N, 0.0);  // the iterate between passes (interior)
  auto store = [data64](double v) { return data64 ? v : (double)(float)v; };
  const int hom_t[6] = {BC_DIRICHLET, BC_DIRICHLET, BC_DIRICHLET,
                        BC_DIRICHLET, BC_DIRICHLET, BC_DIRICHLET};
  const double hom_v[6] = {0, 0, 0, 0, 0, 0};
  for (int ps = 0; ps < sweeps / per; ++ps) {
    for (int bi = 0; bi < G.nb; ++bi) {
      double* z = O.F(OF_Z, bi);
      for (long m = 0; m < G.nc; ++m) z[m] = (ps == 0) ? 0.0 : e[(long)bi * G.nc + m];
    }
    if (ps > 0) impose_bc(O, OF_Z, hom_t, hom_v);  // guide layer 1 of the iterate, in double
    for (int it = 0; it < per; ++it)
      for (int c = 0; c < 2; ++c) {
#pragma omp parallel for num_threads(O.nthreads) schedule(static)
        for (int bi = 0; bi < G.nb; ++bi) {
          double* eb = O.F(OF_Z, bi);
          const double* vb = O.F(fv, bi);
          const long o = (long)bi * G.nc;
          for (int k = 1; k <= n; ++k)
            for (int j = 1; j <= n; ++j)
              for (int i = 1; i <= n; ++i) {
                if ((((i - 1) + (j - 1) + (k - 1)) & 1) != c) continue;
                const long m = IDX(G, i, j, k);
                double rc = vb[m];
                rc = std::fma(-C.a[0][o + m], eb[m - 1], rc);
                rc = std::fma(-C.a[1][o + m], eb[m + 1], rc);
                rc = std::fma(-C.a[2][o + m], eb[m - sy], rc);
                rc = std::fma(-C.a[3][o + m], eb[m + sy], rc);
                rc = std::fma(-C.a[4][o + m], eb[m - sz], rc);
                rc = std::fma(-C.a[5][o + m], eb[m + sz], rc);
                const double xt = rc * C.a[6][o + m];
                const double ev = eb[m];
                eb[m] = std::fma(-(double)omega, ev - xt, ev);
              }
        }
      }
    for (int bi = 0; bi < G.nb; ++bi) {
      const double* z = O.F(OF_Z, bi);
      for (int k = 1; k <= n; ++k)
        for (int j = 1; j <= n; ++j)
          for (int i = 1; i <= n; ++i) {
            const long m = IDX(G, i, j, k);
            e[(long)bi * G.nc + m] = store(z[m]);
          }
    }
  }
  for (int bi = 0; bi < G.nb; ++bi) {
    double* out = O.F(fout, bi);
    for (int k = 1; k <= n; ++k)
      for (int j = 1; j <= n; ++j)
        for (int i = 1; i <= n; ++i) {
          const long m = IDX(G, i, j, k);
          out[m] = e[(long)bi * G.nc + m];
        }
  }
}

// Coarse-fine flux correction (no counterpart in the reference; restates
// ffv-hc_b200/csrc/ffvgpu_internal.cuh cf_fine_flux and cf_delta).  For the
// coarse cell at 0-based transverse position (a, b) of face f of block bi,
// whose neighbours across f are finer: F = 0.125 * sum over the four fine
// cells phi touching the face (du inner, dv outer, from 0.0) of
// A_fo(phi) * (x_phi - g_phi), g_phi phi's guide cell across the opposite
// face fo; delta = F - A_f(P) * (g - x_P).  Guide cells as field fx holds them.
void cf_cell(Oracle& O, int fx, int bi, int f, int a, int b, double& delta, double& F) {
  const Grid& G = O.G;
  const Block& B = G.blocks[bi];
  const int coef_of[6] = {OF_AW, OF_AE, OF_AS, OF_AN, OF_AB, OF_AT};
  const int axis = f >> 1, fo = f ^ 1;
  const bool plus = f & 1;
  const int ta = (axis == 0) ? 1 : 0, tb = (axis == 2) ? 1 : 2;
  // subface of the quarter (a >> 3, b >> 3) as the reference's updater
  // numbers them (so0 + 2 so1, Scalar3DUpdater1.cpp:430-520): so0 along the
  // face's first transverse axis, except on Y faces, where so0 runs along z
  const int qa = a >> 3, qb = b >> 3;
  const int fb = B.nbr[f][axis == 1 ? qb + 2 * qa : qa + 2 * qb];
  const int gstep = (fo & 1) ? 1 : -1;  // the fine cell's guide across fo
  double Fs = 0.0;
  for (int dv = 0; dv < 2; ++dv)
    for (int du = 0; du < 2; ++du) {
      int c[3];
      c[ta] = 2 * (a & 7) + du;
      c[tb] = 2 * (b & 7) + dv;
      c[axis] = plus ? 0 : 15;
      const long m = IDX(G, c[0] + 1, c[1] + 1, c[2] + 1);
      c[axis] += gstep;
      const long gm = IDX(G, c[0] + 1, c[1] + 1, c[2] + 1);
      const double* xf = O.F(fx, fb);
      Fs = Fs + O.F(coef_of[fo], fb)[m] * (xf[m] - xf[gm]);
    }
  F = 0.125 * Fs;
  int c[3];
  c[ta] = a;
  c[tb] = b;
  c[axis] = plus ? 15 : 0;
  const long m = IDX(G, c[0] + 1, c[1] + 1, c[2] + 1);
  c[axis] += plus ? 1 : -1;
  const long gm = IDX(G, c[0] + 1, c[1] + 1, c[2] + 1);
  const double* x = O.F(fx, bi);
  delta = F - O.F(coef_of[f], bi)[m] * (x[gm] - x[m]);
}

// y +/- delta (sign > 0: A x + delta; sign < 0: b - A x - delta) on every
// coarse cell at a face with finer neighbours, faces in order 0..5.
void cf_apply(Oracle& O, int fy, int fx, int sign) {
  const Grid& G = O.G;
  for (int bi = 0; bi < G.nb; ++bi)
    for (int f = 0; f < 6; ++f) {
      if (G.blocks[bi].kind[f] != NB_FINE) continue;
      const int axis = f >> 1, ta = (axis == 0) ? 1 : 0, tb = (axis == 2) ? 1 : 2;
      for (int b = 0; b < 16; ++b)
        for (int a = 0; a < 16; ++a) {
          double d, F;
          cf_cell(O, fx, bi, f, a, b, d, F);
          int c[3];
          c[ta] = a;
          c[tb] = b;
          c[axis] = (f & 1) ? 15 : 0;
          double& y = O.F(fy, bi)[IDX(G, c[0] + 1, c[1] + 1, c[2] + 1)];
          y = sign > 0 ? y + d : y - d;
        }
    }
}

}  // namespace

// y = y + delta (sign > 0) or y - delta (sign < 0) of field fx on every
// coarse cell at a face with finer neighbours (the flux-conserving operator
// applied after orc_calc_ax / orc_calc_r).
void orc_cf_apply(Oracle* O, int fy, int fx, int sign) { cf_apply(*O, fy, fx, sign); }

// Per coarse cell at a face with finer neighbours, in (block, face,
// position a + 16 b) order: (delta, F) of field fx into out[2 * n] (when
// out and capacity allow); returns the number of such cells.
long orc_cf_cells(Oracle* O, int fx, double* out, long capacity) {
  const Grid& G = O->G;
  long n = 0;
  for (int bi = 0; bi < G.nb; ++bi)
    for (int f = 0; f < 6; ++f) {
      if (G.blocks[bi].kind[f] != NB_FINE) continue;
      for (int p = 0; p < 256; ++p, ++n) {
        double d, F;
        cf_cell(*O, fx, bi, f, p & 15, p >> 4, d, F);
        if (out && n < capacity) {
          out[2 * n] = d;
          out[2 * n + 1] = F;
        }
      }
    }
  return n;
}

int orc_mixed(Oracle* O, double omega, int sweeps, int per, int countMax, double epsilon,
              double restart_drop, double restart_growth, int restart_every, int cf,
              int data64, int* count, double* residual, double* hist) {
  Oracle& R = *O;
  if (countMax <= 0) {
    *count = 1;
    *residual = 0.0;
    return 0;
  }
  double bb = DOT(R, OF_B, OF_B);
  if (std::fabs(bb) < FLT_MIN) {
    *residual = 0.0;
    *count = 0;
    return 0;
  }
  Coef32 C;
  mixed_coef(R, C, data64 != 0);
  const float om = (float)omega;
  CalcR(R, OF_R, OF_X, OF_B);
  if (cf) cf_apply(R, OF_R, OF_X, -1);
  COPY(R, OF_R0, OF_R);
  double rr0 = 1.0, alpha = 0.0, gamma = 1.0;
  // restarts: when the residual has dropped by restart_drop since the last
  // (re)start, the recurrence starts again from the current r (r0 = r, p = r)
  double next_restart = -1.0, best = 0.0;
  int cycle = 1;
  int c;
  for (c = 1; c <= countMax; ++c) {
    double rr1 = DOT(R, OF_R, OF_R0);
    if (std::fabs(rr1) < FLT_MIN) {
      *residual = rr1;
      c = 0;
      break;
    }
    if (c == 1) {
      double r_init;
      is_converged(r_init, rr1, bb, 0.0);
      if (restart_drop > 0.0) next_restart = r_init * restart_drop;
      best = r_init;
    }
    if (cycle == 1) {
      COPY(R, OF_P, OF_R);
    } else {
      double beta = rr1 / rr0 * alpha / gamma;
      AXPY(R, OF_P, OF_Q_, -gamma);
      XPAY(R, OF_P, OF_R, beta);
    }
    mixed_precondition(R, C, OF_P, OF_P_, om, sweeps, per, data64 != 0);
    impose_bc_p(R, OF_P_);
    CalcAx(R, OF_Q_, OF_P_);
    if (cf) cf_apply(R, OF_Q_, OF_P_, 1);
    double q_r0 = DOT(R, OF_Q_, OF_R0);
    alpha = rr1 / q_r0;
    AXPYZ(R, OF_S, OF_Q_, OF_R, -alpha);
    mixed_precondition(R, C, OF_S, OF_S_, om, sweeps, per, data64 != 0);
    impose_bc_p(R, OF_S_);
    CalcAx(R, OF_T_, OF_S_);
    if (cf) cf_apply(R, OF_T_, OF_S_, 1);
    double t_s = DOT(R, OF_T_, OF_S);
    double t_t_ = DOT(R, OF_T_, OF_T_);
    gamma = t_s / t_t_;
    AXPBYPZ(R, OF_X, OF_P_, OF_S_, alpha, gamma);
    AXPYZ(R, OF_R, OF_T_, OF_S, -gamma);
    double rr = DOT(R, OF_R, OF_R);
    int st = is_converged(*residual, rr, bb, epsilon);
    if (hist) hist[c - 1] = *residual;
    if (st < 0) {
      *count = c;
      return 2;
    }
    if (st == 1) break;
    rr0 = rr1;
    ++cycle;
    const bool dropped = next_restart > 0.0 && *residual <= next_restart;
    const bool grew = restart_growth > 0.0 && *residual > restart_growth * best;
    const bool aged = restart_every > 0 && cycle > restart_every;
    if (*residual < best) best = *residual;
    if ((dropped || grew || aged) && c < countMax) {
      if (restart_drop > 0.0) next_restart = *residual * restart_drop;
      best = *residual;
      COPY(R, OF_R0, OF_R);
      rr0 = 1.0;
      alpha = 0.0;
      gamma = 1.0;
      cycle = 1;
    }
  }
  impose_bc_p(R, OF_X);
  *count = (c > countMax) ? countMax + 1 : c;
  return 0;
}

// The precision form as a defect correction (no counterpart in the
// reference): r = b - A x in FP64 (CalcR, FFVILS.h:204-245, with x's guide
// layer exchanged first); e = M(r), the RB-SOR preconditioner of orc_mixed on
// 32-bit data (mixed_precondition, e from 0, widened to double); x = x + e
// (axpy with a = 1, blas.f90:329-361); until sqrt(r.r / b.b) <= epsilon
// (IsConverged, FFVILS.h:24-47).  hist[c - 1] is the residual after c
// corrections; the early exits mirror orc_mixed's (b.b, then r.r, below
// FLT_MIN: count 0).
int orc_mixed_dc(Oracle* O, double omega, int sweeps, int per, int countMax, double epsilon,
                 int data64, int* count, double* residual, double* hist) {
  Oracle& R = *O;
  if (countMax <= 0) {
    *count = 1;
    *residual = 0.0;
    return 0;
  }
  const double bb = DOT(R, OF_B, OF_B);
  if (std::fabs(bb) < FLT_MIN) {
    *residual = 0.0;
    *count = 0;
    return 0;
  }
  Coef32 C;
  mixed_coef(R, C, data64 != 0);
  const float om = (float)omega;
  CalcR(R, OF_R, OF_X, OF_B);
  double rr = DOT(R, OF_R, OF_R);
  if (std::fabs(rr) < FLT_MIN) {
    *residual = rr;
    *count = 0;
    return 0;
  }
  int c;
  for (c = 1; c <= countMax; ++c) {
    mixed_precondition(R, C, OF_R, OF_P_, om, sweeps, per, data64 != 0);
    AXPY(R, OF_X, OF_P_, 1.0);
    impose_bc_p(R, OF_X);
    CalcR(R, OF_R, OF_X, OF_B);
    rr = DOT(R, OF_R, OF_R);
    const int st = is_converged(*residual, rr, bb, epsilon);
    if (hist) hist[c - 1] = *residual;
    if (st < 0) {
      *count = c;
      return 2;
    }
    if (st == 1) break;
  }
  impose_bc_p(R, OF_X);
  *count = (c > countMax) ? countMax + 1 : c;
  return 0;
}

}  // extern "C"
