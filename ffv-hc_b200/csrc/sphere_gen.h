// sphere_gen.h -- per-cell synthetic inputs of the sphere-flow workload: one
// definition compiled for the host generator (sphere_grid.cpp) and for the
// device generator (kernels_gen.cu), producing the same bits on both.  Only
// integer arithmetic, IEEE-rounded +, -, *, / and sqrt appear, evaluated in
// a fixed order (the host is built with -ffp-contract=off, the device with
// --fmad=false).
//
// Cut information per cell and direction f (0:-x 1:+x 2:-y 3:+y 4:-z 5:+z)
// follows the meaning bcut_calc_ab_p gives it (src/FFV/bcut.f90:608-832):
// cid_f != 0 when the segment from the cell centre to the neighbour centre
// crosses the sphere, and c_f in (0,1] is the distance to the nearest
// crossing in cell widths, rounded through float as Cutlib's CutPos32Array
// stores it (src/FFV/Solver.cpp:618-637); uncut faces keep c_f = 1
// (Solver::ClearCut, src/FFV/Solver.cpp:514-527).  A cell is fluid (pid 1)
// when its centre lies outside the sphere.
//
// Noise: Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random
// numbers: as easy as 1, 2, 3", SC'11), one counter stream per (cell,
// component), turned into a standard normal draw by Marsaglia's polar
// method with a natural logarithm from the series ln m = 2 atanh((m-1)/(m+1)).
#pragma once
#include <cmath>
#include <cstdint>

#include "ffvgpu_layout.h"

namespace ffvgpu {

FFVGPU_HD inline void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
    const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
    c[0] = n0;
    c[1] = lo1;
    c[2] = n2;
    c[3] = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

// Natural logarithm of u > 0 (finite, normal): u = m * 2^e with m in
// [sqrt(1/2), sqrt(2)), ln m = 2 (z + z^3/3 + ... + z^23/23), z = (m-1)/(m+1),
// |z| < 0.172 (truncation below 1e-19 relative).
FFVGPU_HD inline double ln_series(double u) {
  int e = 0;
  double m = frexp(u, &e);  // m in [0.5, 1)
  if (m < 0.70710678118654752) {
    m = m * 2.0;
    e = e - 1;
  }
  const double z = (m - 1.0) / (m + 1.0);
  const double w = z * z;
  double s = 1.0 / 23.0;
  s = s * w + 1.0 / 21.0;
  s = s * w + 1.0 / 19.0;
  s = s * w + 1.0 / 17.0;
  s = s * w + 1.0 / 15.0;
  s = s * w + 1.0 / 13.0;
  s = s * w + 1.0 / 11.0;
  s = s * w + 1.0 / 9.0;
  s = s * w + 1.0 / 7.0;
  s = s * w + 1.0 / 5.0;
  s = s * w + 1.0 / 3.0;
  s = s * w + 1.0;
  const double ln2 = 0.69314718055994531;
  return (double)e * ln2 + 2.0 * z * s;
}

// Uniform in (0, 1) with 53 random bits from two 32-bit words.
FFVGPU_HD inline double uniform53(uint32_t a, uint32_t b) {
  return ((double)(a >> 5) * 67108864.0 + (double)(b >> 6) + 0.5) / 9007199254740992.0;
}

// Standard normal draw for (seed, cell, component): polar method on the
// counter stream (cell, comp, attempt).
FFVGPU_HD inline double normal_draw(uint64_t seed, uint64_t cell, uint32_t comp) {
  for (uint32_t attempt = 0; attempt < 64; ++attempt) {
    uint32_t c[4] = {(uint32_t)cell, (uint32_t)(cell >> 32), comp, attempt};
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    const double v1 = 2.0 * uniform53(c[0], c[1]) - 1.0;
    const double v2 = 2.0 * uniform53(c[2], c[3]) - 1.0;
    const double s = v1 * v1 + v2 * v2;
    if (s >= 1.0 || s == 0.0) continue;
    return v1 * sqrt(-2.0 * ln_series(s) / s);
  }
  return 0.0;
}

// Geometry of one cell: fluid flag, cut bits (bit f: direction f crosses the
// sphere) and cut distances c[6] (1.0 where uncut).
struct CellCut {
  int fluid;
  int cid;
  double c[6];
};

// Cell (i, j, k) of a block whose lower corner is org and whose cells have
// edge dx; sphere of centre cen and radius R.
FFVGPU_HD inline CellCut sphere_cell(const double org[3], double dx, int i, int j, int k,
                                     const double cen[3], double R) {
  CellCut out;
  const double R2 = R * R;
  const double P[3] = {org[0] + ((double)i + 0.5) * dx, org[1] + ((double)j + 0.5) * dx,
                       org[2] + ((double)k + 0.5) * dx};
  double D[3], d2 = 0.0;
  for (int a = 0; a < 3; ++a) {
    D[a] = P[a] - cen[a];
    d2 += D[a] * D[a];
  }
  out.fluid = (d2 >= R2) ? 1 : 0;
  out.cid = 0;
  for (int f = 0; f < 6; ++f) {
    out.c[f] = 1.0;
    const int a = f / 2;
    const double s = (f & 1) ? 1.0 : -1.0;
    const double bq = s * D[a];
    const double disc = bq * bq - (d2 - R2);
    if (disc < 0.0) continue;
    const double sq = sqrt(disc);
    const double t1 = -bq - sq, t2 = -bq + sq;
    double t = -1.0;
    if (t1 > 0.0 && t1 <= dx) t = t1;
    else if (t2 > 0.0 && t2 <= dx) t = t2;
    if (t <= 0.0) continue;
    double d = (double)(float)(t / dx);
    if (d <= 0.0) d = 1.0e-6;
    if (d > 1.0) d = 1.0;
    out.c[f] = d;
    out.cid |= 1 << f;
  }
  return out;
}

// Lower corner and cell edge of block (level L, index idx) of a domain.
FFVGPU_HD inline double block_geometry(const double dom_org[3], double root_len, int L,
                                       const int32_t idx[3], double org[3]) {
  const double bl = root_len / (double)(1LL << L);
  for (int a = 0; a < 3; ++a) org[a] = dom_org[a] + bl * (double)idx[a];
  return bl / 16.0;
}

}  // namespace ffvgpu
