// Host-side check of the device exchange's index arithmetic: compiles
// ffvgpu_internal.cuh for the host with a bounds-checking load and evaluates
// guide_value for every block, face, transverse position and layer of a
// grid given on stdin (nb, then per block: level ix iy iz, then the
// neighbour table as kind id0 id1 id2 id3 so_u so_v per face).  Prints the
// number of out-of-range loads (must be 0).
#include <cmath>
#include <cstdio>
#include <cstdint>
#include <algorithm>
#include <vector>

using std::fabs;
using std::isinf;
using std::isnan;
using std::sqrt;
#define __device__
#define __host__
#define __forceinline__ inline
#define __noinline__
#define __restrict__
using std::max;
using std::min;
static const double* g_base = nullptr;
static size_t g_count = 0;
static long g_bad = 0;
static inline double __ldg(const double* p) {
  if (p < g_base || p >= g_base + g_count) {
    ++g_bad;
    return 0.0;
  }
  return *p;
}
#include "../../ffv-hc_b200/csrc/ffvgpu_internal.cuh"

using namespace ffvgpu;

int main() {
  int nb;
  if (std::scanf("%d", &nb) != 1) return 2;
  std::vector<FaceNbr> nbr((size_t)nb * 6);
  for (int b = 0; b < nb; ++b)
    for (int f = 0; f < 6; ++f) {
      FaceNbr& F = nbr[b * 6 + f];
      if (std::scanf("%d %d %d %d %d %d %d", &F.kind, &F.id[0], &F.id[1], &F.id[2], &F.id[3],
                     &F.so_u, &F.so_v) != 7)
        return 2;
    }
  std::vector<double> x((size_t)nb * BLOCK_CELLS, 1.0);
  g_base = x.data();
  g_count = x.size();
  BCSet bc;
  for (int f = 0; f < 6; ++f) {
    bc.type[f] = f & 1;
    bc.value[f] = 0.5;
  }
  long evals = 0, nonfinite = 0;
  for (int b = 0; b < nb; ++b)
    for (int f = 0; f < 6; ++f)
      for (int L = 1; L <= 2; ++L)
        for (int v = 0; v < 16; ++v)
          for (int u = 0; u < 16; ++u) {
            const FaceNbr& F = nbr[b * 6 + f];
            if ((F.kind == NB_SAME || F.kind == NB_COARSE) && (F.id[0] < 0 || F.id[0] >= nb)) {
              ++g_bad;
              continue;
            }
            const double val = guide_value(x.data(), b, f, u, v, L, F, bc, 0.1);
            ++evals;
            if (!std::isfinite(val)) ++nonfinite;
            // a constant field must be reproduced by same/c2f/f2c exactly
            if (F.kind != NB_OUTER && val != 1.0) ++nonfinite;
          }
  // guide_pair (the batched form used by the pipelined kernel) must equal
  // guide_value bit for bit on arbitrary data
  long pair_mismatch = 0;
  uint64_t st = 88172645463325252ull;
  for (double& v : x) {
    st ^= st << 13; st ^= st >> 7; st ^= st << 17;
    v = (double)(int64_t)(st >> 11) * 1.0e-15 - 4.0;
  }
  for (int b = 0; b < nb; ++b)
    for (int f = 0; f < 6; ++f)
      for (int p = 0; p < 128; ++p) {
        const FaceNbr& F = nbr[b * 6 + f];
        double v0, v1;
        guide_pair(x.data(), b, f, p, p + 128, F, bc, 0.1, v0, v1);
        const double w0 = guide_value(x.data(), b, f, p & 15, p >> 4, 1, F, bc, 0.1);
        const double w1 = guide_value(x.data(), b, f, (p + 128) & 15, (p + 128) >> 4, 1, F, bc, 0.1);
        pair_mismatch += (v0 != w0) + (v1 != w1);
      }
  nonfinite += pair_mismatch;
  // split_neighbours (colour-split tile + guide layer) must return the same
  // cells as direct (i, j, k) indexing with guide cells outside the block
  long nbr_mismatch = 0;
  {
    std::vector<double> blkx(BLOCK_CELLS), G(6 * FACE_CELLS);
    for (int s = 0; s < BLOCK_CELLS; ++s) blkx[s] = 1000.0 + s;
    for (int q = 0; q < 6 * FACE_CELLS; ++q) G[q] = -1.0 - q;
    auto at = [&](int i, int j, int k) -> double {
      if (i < 0) return G[0 * 256 + j + 16 * k];
      if (i > 15) return G[1 * 256 + j + 16 * k];
      if (j < 0) return G[2 * 256 + i + 16 * k];
      if (j > 15) return G[3 * 256 + i + 16 * k];
      if (k < 0) return G[4 * 256 + i + 16 * j];
      if (k > 15) return G[5 * 256 + i + 16 * j];
      return blkx[sidx(i, j, k)];
    };
    for (int c = 0; c < 2; ++c)
      for (int q = 0; q < HALF_CELLS; ++q) {
        int i, j, k;
        cell_of(c * HALF_CELLS + q, i, j, k);
        const Nbrs r = split_neighbours(blkx.data() + (1 - c) * HALF_CELLS, G.data(), q, c);
        nbr_mismatch += (r.w != at(i - 1, j, k)) + (r.e != at(i + 1, j, k)) +
                        (r.s != at(i, j - 1, k)) + (r.n != at(i, j + 1, k)) +
                        (r.b != at(i, j, k - 1)) + (r.t != at(i, j, k + 1));
      }
  }
  g_bad += nbr_mismatch;
  // sidx must be a bijection onto [0, 4096)
  std::vector<int> seen(BLOCK_CELLS, 0);
  for (int k = 0; k < 16; ++k)
    for (int j = 0; j < 16; ++j)
      for (int i = 0; i < 16; ++i) {
        const int s = sidx(i, j, k);
        if (s < 0 || s >= BLOCK_CELLS) ++g_bad;
        else seen[s]++;
        int a, bq, c;
        cell_of(s, a, bq, c);
        if (a != i || bq != j || c != k) ++g_bad;
      }
  for (int s = 0; s < BLOCK_CELLS; ++s)
    if (seen[s] != 1) ++g_bad;
  std::printf("%ld %ld %ld\n", evals, g_bad, nonfinite);
  return g_bad ? 1 : 0;
}
