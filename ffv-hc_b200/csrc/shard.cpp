// shard.cpp -- block sharding of one grid across ranks (one process per GPU).
//
// The reference distributes its leaf blocks over MPI ranks as contiguous
// ranges of the octree's ordered leaf list (Solver::InitTree / InitBlocks,
// src/FFV/Solver.cpp:306-381: BCMOctree ordering, BCMTools' Partition), each
// rank holding its blocks and exchanging guide faces with the others.  Here
// the leaves are put in Z order -- root blocks in x-fastest order, then the
// Morton order of each leaf's position inside its root block at the finest
// level -- and cut into num_ranks contiguous ranges whose sizes differ by at
// most one.  A rank's pool holds its own blocks (local ids 0 .. owned-1, in
// that order), then halo blocks: copies of the other ranks' blocks that its
// blocks' guide cells are computed from (every face neighbour), grouped by
// owner rank and in Z order within a group.  The halo blocks are never
// solved; before every pass that reads neighbours, each rank sends the
// interiors of the blocks its peers hold as halos, in the order the peer
// lists them, and the unchanged in-kernel exchange then gives the guide
// values of the unsharded grid bit for bit.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <map>
#include <new>
#include <set>
#include <tuple>
#include <vector>

#include "../../include/ffvgpu.h"
#include "ffvgpu_layout.h"
#include "pool_internal.h"

using namespace ffvgpu;
using namespace ffvgpu::detail;

struct ffvgpu_shard {
  int ranks = 0, rank = 0;
  std::vector<int32_t> order;       // global ids in Z order
  std::vector<int32_t> owner;       // [global] rank
  std::vector<int32_t> local;       // local id -> global id (owned, then halo)
  int owned = 0;
  std::vector<int32_t> level, index;             // local grid
  std::vector<int32_t> nkind, nids;              // local neighbour table
  std::vector<std::vector<int32_t>> send, recv;  // [peer] local ids
  ffvgpu_grid_desc desc{};
};

namespace {

uint64_t spread3(uint64_t v) {  // bit b of v -> bit 3b
  uint64_t r = 0;
  for (int b = 0; b < 21; ++b) r |= ((v >> b) & 1ull) << (3 * b);
  return r;
}

}  // namespace

ffvgpu_status ffvgpu_shard_create(const ffvgpu_grid_desc* d, int32_t num_ranks, int32_t rank,
                                  ffvgpu_shard** out) {
  if (!d || !out) return bad("null argument");
  *out = nullptr;
  if (num_ranks < 1 || rank < 0 || rank >= num_ranks) return bad("bad rank or rank count");
  if (d->num_blocks < num_ranks) return bad("fewer blocks than ranks");
  const int nb = d->num_blocks;
  std::vector<FaceNbr> nbr;
  ffvgpu_status s;
  if (d->neighbor_kind || d->neighbor_ids) return bad("shards derive the neighbour table");
  if ((s = derive_neighbors(nb, d->level, d->block_index, d, nbr))) return s;
  int lmax = 0;
  for (int b = 0; b < nb; ++b) lmax = std::max(lmax, (int)d->level[b]);
  if (lmax > 20) return bad("block level out of range");
  ffvgpu_shard* S = new (std::nothrow) ffvgpu_shard();
  if (!S) return bad("out of host memory");
  S->ranks = num_ranks;
  S->rank = rank;
  // Z order: root block (x fastest), then Morton position at the finest level
  std::vector<std::pair<std::pair<uint64_t, uint64_t>, int32_t>> keys(nb);
  for (int b = 0; b < nb; ++b) {
    const int L = d->level[b];
    uint64_t root = 0, m = 0;
    int64_t r[3];
    uint64_t loc[3];
    for (int a = 0; a < 3; ++a) {
      r[a] = (int64_t)d->block_index[3 * b + a] >> L;
      loc[a] = ((uint64_t)d->block_index[3 * b + a] & ((1ull << L) - 1)) << (lmax - L);
    }
    root = (uint64_t)(r[0] + (int64_t)d->root_grid[0] * (r[1] + (int64_t)d->root_grid[1] * r[2]));
    m = spread3(loc[0]) | (spread3(loc[1]) << 1) | (spread3(loc[2]) << 2);
    keys[b] = {{root, m}, b};
  }
  std::sort(keys.begin(), keys.end());
  S->order.resize(nb);
  S->owner.resize(nb);
  std::vector<int32_t> pos(nb);
  for (int k = 0; k < nb; ++k) {
    S->order[k] = keys[k].second;
    pos[keys[k].second] = k;
  }
  const int base = nb / num_ranks, rem = nb % num_ranks;
  auto start = [&](int r) { return r * base + std::min(r, rem); };
  for (int r = 0; r < num_ranks; ++r)
    for (int k = start(r); k < start(r + 1); ++k) S->owner[S->order[k]] = r;
  // local blocks: owned in Z order, then halos grouped by owner, Z order within
  std::set<std::pair<int, int>> halo;  // (owner, Z position)
  for (int k = start(rank); k < start(rank + 1); ++k) {
    const int b = S->order[k];
    for (int f = 0; f < 6; ++f) {
      const FaceNbr& F = nbr[(size_t)b * 6 + f];
      const int n = F.kind == NB_FINE ? 4 : (F.kind == NB_OUTER ? 0 : 1);
      for (int q = 0; q < n; ++q)
        if (S->owner[F.id[q]] != rank) halo.insert({S->owner[F.id[q]], pos[F.id[q]]});
    }
  }
  S->owned = start(rank + 1) - start(rank);
  for (int k = start(rank); k < start(rank + 1); ++k) S->local.push_back(S->order[k]);
  for (const auto& h : halo) S->local.push_back(S->order[h.second]);
  const int nl = (int)S->local.size();
  std::vector<int32_t> to_local(nb, -1);
  for (int l = 0; l < nl; ++l) to_local[S->local[l]] = l;
  S->level.resize(nl);
  S->index.resize(3 * (size_t)nl);
  S->nkind.assign((size_t)nl * 6, NB_OUTER);
  S->nids.assign((size_t)nl * 24, -1);
  for (int l = 0; l < nl; ++l) {
    const int b = S->local[l];
    S->level[l] = d->level[b];
    for (int a = 0; a < 3; ++a) S->index[3 * l + a] = d->block_index[3 * b + a];
    if (l >= S->owned) continue;  // halo blocks are never solved: outer faces
    for (int f = 0; f < 6; ++f) {
      const FaceNbr& F = nbr[(size_t)b * 6 + f];
      S->nkind[(size_t)l * 6 + f] = F.kind;
      const int n = F.kind == NB_FINE ? 4 : (F.kind == NB_OUTER ? 0 : 1);
      for (int q = 0; q < n; ++q) S->nids[((size_t)l * 6 + f) * 4 + q] = to_local[F.id[q]];
    }
  }
  // exchange lists: what this rank receives from peer p is its halo group of
  // p (in local order); what it sends to p is its owned blocks in p's halo
  // set, in Z order -- the order p lists them
  S->send.assign(num_ranks, {});
  S->recv.assign(num_ranks, {});
  for (int l = S->owned; l < nl; ++l) S->recv[S->owner[S->local[l]]].push_back(l);
  for (int p = 0; p < num_ranks; ++p) {
    if (p == rank) continue;
    std::set<int> need;  // Z positions of this rank's blocks that p's blocks read
    for (int k = start(p); k < start(p + 1); ++k) {
      const int b = S->order[k];
      for (int f = 0; f < 6; ++f) {
        const FaceNbr& F = nbr[(size_t)b * 6 + f];
        const int n = F.kind == NB_FINE ? 4 : (F.kind == NB_OUTER ? 0 : 1);
        for (int q = 0; q < n; ++q)
          if (S->owner[F.id[q]] == rank) need.insert(pos[F.id[q]]);
      }
    }
    for (int z : need) S->send[p].push_back(to_local[S->order[z]]);
  }
  ffvgpu_grid_desc& L = S->desc;
  L = *d;
  L.num_blocks = nl;
  L.level = S->level.data();
  L.block_index = S->index.data();
  L.neighbor_kind = S->nkind.data();
  L.neighbor_ids = S->nids.data();
  *out = S;
  return FFVGPU_OK;
}

void ffvgpu_shard_destroy(ffvgpu_shard* S) { delete S; }

ffvgpu_status ffvgpu_shard_info(const ffvgpu_shard* S, int32_t* owned, int32_t* halo) {
  if (!S || !owned || !halo) return bad("null argument");
  *owned = S->owned;
  *halo = (int32_t)S->local.size() - S->owned;
  return FFVGPU_OK;
}

ffvgpu_status ffvgpu_shard_local_blocks(const ffvgpu_shard* S, int32_t* global_ids) {
  if (!S || !global_ids) return bad("null argument");
  std::memcpy(global_ids, S->local.data(), sizeof(int32_t) * S->local.size());
  return FFVGPU_OK;
}

ffvgpu_status ffvgpu_shard_zorder(const ffvgpu_shard* S, int32_t* order, int32_t* owner) {
  if (!S || !order || !owner) return bad("null argument");
  std::memcpy(order, S->order.data(), sizeof(int32_t) * S->order.size());
  std::memcpy(owner, S->owner.data(), sizeof(int32_t) * S->owner.size());
  return FFVGPU_OK;
}

const ffvgpu_grid_desc* ffvgpu_shard_local_desc(const ffvgpu_shard* S) {
  return S ? &S->desc : nullptr;
}

ffvgpu_status ffvgpu_shard_peer(const ffvgpu_shard* S, int32_t peer, int32_t* n_send,
                                int32_t* send_local, int32_t* n_recv, int32_t* recv_local) {
  if (!S || !n_send || !n_recv) return bad("null argument");
  if (peer < 0 || peer >= S->ranks) return bad("bad peer");
  *n_send = (int32_t)S->send[peer].size();
  *n_recv = (int32_t)S->recv[peer].size();
  if (send_local) std::memcpy(send_local, S->send[peer].data(), sizeof(int32_t) * *n_send);
  if (recv_local) std::memcpy(recv_local, S->recv[peer].data(), sizeof(int32_t) * *n_recv);
  return FFVGPU_OK;
}

// The cross-block stage of the pool's fixed reduction tree over per-block
// partial sums in block order: 256 lanes sum partials t, t + 256, ...
// serially from 0; each warp of 32 lanes is combined by an xor butterfly
// (16, 8, 4, 2, 1) and lane 0's value taken; the 8 warp sums are added in
// order from 0.  The same bits as the device's last-block reduction.
ffvgpu_status ffvgpu_canonical_sum(const double* partials, int32_t n, double* total) {
  if (!partials || !total || n < 0) return bad("bad argument");
  double T[256];
  for (int t = 0; t < 256; ++t) {
    double s = 0.0;
    for (int b = t; b < n; b += 256) s += partials[b];
    T[t] = s;
  }
  double sum = 0.0;
  for (int w = 0; w < 8; ++w) {
    double v[32], nv[32];
    for (int l = 0; l < 32; ++l) v[l] = T[32 * w + l];
    for (int off = 16; off >= 1; off >>= 1) {
      for (int l = 0; l < 32; ++l) nv[l] = v[l] + v[l ^ off];
      std::memcpy(v, nv, sizeof(v));
    }
    sum += v[0];
  }
  *total = sum;
  return FFVGPU_OK;
}
