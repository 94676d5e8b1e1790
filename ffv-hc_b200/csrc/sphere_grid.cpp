// sphere_grid.cpp -- synthetic leaf-block grids around a sphere (host only).
//
// Stands in for the reference's grid generation chain, which depends on
// libraries absent from the reference tree: BCMTools' BCMOctree/Divider
// (src/FFV/Solver.cpp:219-386, src/FFV/SphereDivider2.h:21-161) for the
// octree and Cutlib's CalcCutInfo (src/FFV/Solver.cpp:530-663) for cut
// positions.  The octree refines a block while its level is below max_level
// and the block's box lies within radius + margin of the sphere centre (the
// box-distance test of SphereDivider2::checkOuter, SphereDivider2.h:129-157),
// then refines further until every face neighbour differs by at most one
// level (2:1 face balance).  Leaves are listed in depth-first Z order.
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
// The intermediate velocity u* = (1,0,0) + N(0, sigma^2) draws one
// Philox4x32-10 counter per (cell, component) (Salmon, Moraes, Dror, Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC'11) and a Box-Muller
// transform, so any subset of cells can be regenerated independently.

#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <set>
#include <tuple>
#include <vector>

#include "../../include/ffvgpu.h"

struct ffvgpu_sphere_grid {
  ffvgpu_sphere_params prm;
  std::vector<int32_t> level;
  std::vector<int32_t> index;  // [nb][3]
};

namespace {

using Key = std::tuple<int, long, long, long>;

struct Tree {
  const ffvgpu_sphere_params& p;
  std::set<Key> leaves;
  explicit Tree(const ffvgpu_sphere_params& prm) : p(prm) {}

  double block_len(int L) const { return p.root_length / (double)(1L << L); }

  bool near_sphere(int L, long ix, long iy, long iz) const {
    const double bl = block_len(L);
    const long id[3] = {ix, iy, iz};
    double d2 = 0.0;
    for (int a = 0; a < 3; ++a) {
      const double lo = p.domain_origin[a] + bl * (double)id[a];
      const double hi = lo + bl;
      double d = 0.0;
      if (p.center[a] < lo) d = lo - p.center[a];
      else if (p.center[a] > hi) d = p.center[a] - hi;
      d2 += d * d;
    }
    const double rr = p.radius + p.margin;
    return d2 <= rr * rr;
  }

  void build(int L, long ix, long iy, long iz) {
    if (L < p.max_level && near_sphere(L, ix, iy, iz)) {
      for (int c = 0; c < 8; ++c)
        build(L + 1, 2 * ix + (c & 1), 2 * iy + ((c >> 1) & 1), 2 * iz + (c >> 2));
    } else {
      leaves.insert(Key(L, ix, iy, iz));
    }
  }

  // Level of the leaf covering block position (L, idx), or -1 if that
  // position is covered by finer leaves (it is a branch).
  int covering_level(int L, long ix, long iy, long iz) const {
    for (int l = L; l >= 0; --l) {
      const int s = L - l;
      if (leaves.count(Key(l, ix >> s, iy >> s, iz >> s))) return l;
    }
    return -1;
  }

  void balance() {
    bool changed = true;
    while (changed) {
      changed = false;
      std::vector<Key> split;
      for (const Key& k : leaves) {
        const int L = std::get<0>(k);
        const long id[3] = {std::get<1>(k), std::get<2>(k), std::get<3>(k)};
        for (int f = 0; f < 6; ++f) {
          const int a = f / 2;
          long n[3] = {id[0], id[1], id[2]};
          n[a] += (f & 1) ? 1 : -1;
          const long ext = (long)p.root_grid[a] << L;
          if (n[a] < 0 || n[a] >= ext) continue;
          const int lc = covering_level(L, n[0], n[1], n[2]);
          if (lc >= 0 && lc < L - 1) {
            const int s = L - lc;
            split.push_back(Key(lc, n[0] >> s, n[1] >> s, n[2] >> s));
          }
        }
      }
      for (const Key& k : split) {
        if (!leaves.erase(k)) continue;
        const int L = std::get<0>(k);
        for (int c = 0; c < 8; ++c)
          leaves.insert(Key(L + 1, 2 * std::get<1>(k) + (c & 1),
                            2 * std::get<2>(k) + ((c >> 1) & 1),
                            2 * std::get<3>(k) + (c >> 2)));
        changed = true;
      }
    }
  }

  void emit(int L, long ix, long iy, long iz, std::vector<int32_t>& lev,
            std::vector<int32_t>& idx) const {
    if (leaves.count(Key(L, ix, iy, iz))) {
      lev.push_back(L);
      idx.push_back((int32_t)ix);
      idx.push_back((int32_t)iy);
      idx.push_back((int32_t)iz);
      return;
    }
    if (L > 40) return;
    for (int c = 0; c < 8; ++c)
      emit(L + 1, 2 * ix + (c & 1), 2 * iy + ((c >> 1) & 1), 2 * iz + (c >> 2), lev, idx);
  }
};

inline void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
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

inline double normal_draw(uint64_t seed, uint64_t cell, uint32_t comp) {
  uint32_t c[4] = {(uint32_t)cell, (uint32_t)(cell >> 32), comp, 0u};
  philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  const double two53 = 9007199254740992.0;
  const double u1 = ((double)(c[0] >> 5) * 67108864.0 + (double)(c[1] >> 6) + 0.5) / two53;
  const double u2 = ((double)(c[2] >> 5) * 67108864.0 + (double)(c[3] >> 6) + 0.5) / two53;
  return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
}

}  // namespace

extern "C" {

ffvgpu_status ffvgpu_sphere_grid_create(const ffvgpu_sphere_params* prm,
                                        ffvgpu_sphere_grid** out) {
  if (!prm || !out || prm->root_length <= 0.0 || prm->max_level < 0 ||
      prm->max_level > 12 || prm->radius < 0.0)
    return FFVGPU_BAD_ARG;
  for (int a = 0; a < 3; ++a)
    if (prm->root_grid[a] <= 0) return FFVGPU_BAD_ARG;
  Tree T(*prm);
  for (long z = 0; z < prm->root_grid[2]; ++z)
    for (long y = 0; y < prm->root_grid[1]; ++y)
      for (long x = 0; x < prm->root_grid[0]; ++x) T.build(0, x, y, z);
  T.balance();
  ffvgpu_sphere_grid* g = new ffvgpu_sphere_grid();
  g->prm = *prm;
  for (long z = 0; z < prm->root_grid[2]; ++z)
    for (long y = 0; y < prm->root_grid[1]; ++y)
      for (long x = 0; x < prm->root_grid[0]; ++x) T.emit(0, x, y, z, g->level, g->index);
  *out = g;
  return FFVGPU_OK;
}

void ffvgpu_sphere_grid_destroy(ffvgpu_sphere_grid* g) { delete g; }

int32_t ffvgpu_sphere_grid_num_blocks(const ffvgpu_sphere_grid* g) {
  return (int32_t)g->level.size();
}

void ffvgpu_sphere_grid_blocks(const ffvgpu_sphere_grid* g, int32_t* level,
                               int32_t* block_index) {
  if (level) std::memcpy(level, g->level.data(), g->level.size() * sizeof(int32_t));
  if (block_index)
    std::memcpy(block_index, g->index.data(), g->index.size() * sizeof(int32_t));
}

ffvgpu_status ffvgpu_sphere_grid_fill(const ffvgpu_sphere_grid* g, uint64_t seed,
                                      double sigma, int32_t vc, double* ux,
                                      double* uy, double* uz, double* const* c6,
                                      int32_t* const* cid6, int32_t* pid) {
  if (!g || vc < 1 || vc > 4) return FFVGPU_BAD_ARG;
  const ffvgpu_sphere_params& p = g->prm;
  const int n = 16;
  const long w = n + 2 * vc;
  const long nc = w * w * w;
  const long nb = (long)g->level.size();
  const double R = p.radius, R2 = R * R;
#pragma omp parallel for schedule(dynamic, 4)
  for (long b = 0; b < nb; ++b) {
    const int L = g->level[b];
    const double bl = p.root_length / (double)(1L << L);
    const double dx = bl / (double)n;
    double org[3];
    for (int a = 0; a < 3; ++a) org[a] = p.domain_origin[a] + bl * (double)g->index[3 * b + a];
    const long base = b * nc;
    // guide cells are zero
    if (ux) std::memset(ux + base, 0, nc * sizeof(double));
    if (uy) std::memset(uy + base, 0, nc * sizeof(double));
    if (uz) std::memset(uz + base, 0, nc * sizeof(double));
    for (int f = 0; f < 6; ++f) {
      if (c6 && c6[f])
        for (long m = 0; m < nc; ++m) c6[f][base + m] = 1.0;
      if (cid6 && cid6[f]) std::memset(cid6[f] + base, 0, nc * sizeof(int32_t));
    }
    if (pid) std::memset(pid + base, 0, nc * sizeof(int32_t));
    for (int k = 0; k < n; ++k)
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
          const long m = base + (i + vc) + w * ((j + vc) + w * (k + vc));
          const uint64_t cell = (uint64_t)b * 4096u + (uint64_t)(i + 16 * (j + 16 * k));
          if (ux) ux[m] = 1.0 + sigma * normal_draw(seed, cell, 0);
          if (uy) uy[m] = sigma * normal_draw(seed, cell, 1);
          if (uz) uz[m] = sigma * normal_draw(seed, cell, 2);
          const double P[3] = {org[0] + ((double)i + 0.5) * dx,
                               org[1] + ((double)j + 0.5) * dx,
                               org[2] + ((double)k + 0.5) * dx};
          double D[3], d2 = 0.0;
          for (int a = 0; a < 3; ++a) {
            D[a] = P[a] - p.center[a];
            d2 += D[a] * D[a];
          }
          if (pid) pid[m] = (d2 >= R2) ? 1 : 0;
          for (int f = 0; f < 6; ++f) {
            const int a = f / 2;
            const double s = (f & 1) ? 1.0 : -1.0;
            const double bq = s * D[a];
            const double disc = bq * bq - (d2 - R2);
            if (disc < 0.0) continue;
            const double sq = std::sqrt(disc);
            const double t1 = -bq - sq, t2 = -bq + sq;
            double t = -1.0;
            if (t1 > 0.0 && t1 <= dx) t = t1;
            else if (t2 > 0.0 && t2 <= dx) t = t2;
            if (t <= 0.0) continue;
            double d = (double)(float)(t / dx);
            if (d <= 0.0) d = 1.0e-6;
            if (d > 1.0) d = 1.0;
            if (c6 && c6[f]) c6[f][m] = d;
            if (cid6 && cid6[f]) cid6[f][m] = 1;
          }
        }
  }
  return FFVGPU_OK;
}

}  // extern "C"
