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
// Per-cell inputs (cut positions, fluid flags, u* = (1,0,0) + N(0, sigma^2))
// come from sphere_gen.h, shared with the device generator; cell (i, j, k) of
// the grid's block b draws from counter b*4096 + i + 16*(j + 16*k), so any
// subset of cells can be regenerated independently.

#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <set>
#include <tuple>
#include <vector>

#include "../../include/ffvgpu.h"
#include "sphere_gen.h"

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
#pragma omp parallel for schedule(dynamic, 4)
  for (long b = 0; b < nb; ++b) {
    double org[3];
    const double dx = ffvgpu::block_geometry(p.domain_origin, p.root_length, g->level[b],
                                             &g->index[3 * b], org);
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
          if (ux) ux[m] = 1.0 + sigma * ffvgpu::normal_draw(seed, cell, 0);
          if (uy) uy[m] = sigma * ffvgpu::normal_draw(seed, cell, 1);
          if (uz) uz[m] = sigma * ffvgpu::normal_draw(seed, cell, 2);
          const ffvgpu::CellCut cc = ffvgpu::sphere_cell(org, dx, i, j, k, p.center, p.radius);
          if (pid) pid[m] = cc.fluid;
          for (int f = 0; f < 6; ++f) {
            if (!((cc.cid >> f) & 1)) continue;
            if (c6 && c6[f]) c6[f][m] = cc.c[f];
            if (cid6 && cid6[f]) cid6[f][m] = 1;
          }
        }
  }
  return FFVGPU_OK;
}

}  // extern "C"
