// instances.cpp -- batches of independent pressure problems in one pool, and
// the mixed-precision solve that runs them (include/ffvgpu.h).
//
// A batch pool reserves a block capacity on the device and admits
// instances into free contiguous block ranges (first fit).  Every kernel of
// the mixed solve covers the whole capacity; a block looks up its instance
// and returns at once when the block is free or its instance is not
// solving.  Each instance has its own solver state, its own reduction
// ticket and its own sums, taken in block order over its range, so its
// results do not depend on what else shares the pool.  One iteration of all
// running instances is a fixed sequence of launches, captured once as a
// CUDA graph and replayed; the host polls the per-instance states between
// replays, and an instance admitted while others run joins at the next
// replay.
#include <cfloat>
#include <cstddef>
#include <cmath>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/ffvgpu.h"
#include "ffvgpu_gen.h"
#include "ffvgpu_kernels.h"
#include "ffvgpu_layout.h"
#include "ffvgpu_mixed.h"
#include "pool_internal.h"

using namespace ffvgpu;
using namespace ffvgpu::detail;

namespace ffvgpu {
namespace detail {

void release_instances(ffvgpu_pool* P) {
  if (P->mgraph) cudaGraphExecDestroy(P->mgraph);
  P->mgraph = nullptr;
  void* ptrs[] = {P->blk_inst_d, P->inst_first_d, P->inst_count_d, P->blk_geo_d, P->mst,
                  P->mpartials, P->mhist, P->mcoef, P->mguide, P->mucoef, P->me[0], P->me[1], P->mph,
                  P->msh, P->mcoef64, P->me64[0], P->me64[1], P->mph64, P->msh64};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (P->act_d) cudaFree(P->act_d);
  if (P->act_raw_d) cudaFree(P->act_raw_d);
  for (int k = 0; k < 2; ++k) {
    if (P->act_h[k]) cudaFreeHost(P->act_h[k]);
    if (P->act_ev[k]) cudaEventDestroy(P->act_ev[k]);
  }
  if (P->mst_h) cudaFreeHost(P->mst_h);
  P->mst_h = nullptr;
}

}  // namespace detail
}  // namespace ffvgpu

namespace {

int num_inst(const ffvgpu_pool* P) { return (int)P->inst.size(); }

// Device copies of the instance tables (allocated once, sized by capacity).
ffvgpu_status ensure_inst_device(ffvgpu_pool* P) {
  ffvgpu_status s;
  const int ni = num_inst(P);
  if ((s = dalloc_t(P, &P->blk_inst_d, (size_t)P->nb)) ||
      (s = dalloc_t(P, &P->inst_first_d, (size_t)ni)) ||
      (s = dalloc_t(P, &P->inst_count_d, (size_t)ni)) ||
      (s = dalloc_t(P, &P->blk_geo_d, (size_t)P->nb * 4)) ||
      (s = dalloc_t(P, &P->mst, (size_t)ni)) || (s = dalloc_t(P, &P->mpartials, 2 * (size_t)P->nb)))
    return s;
  if (!P->mst_h) {
    cudaError_t e = cudaMallocHost(&P->mst_h, sizeof(SolveState) * ni);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMallocHost");
    std::memset(P->mst_h, 0, sizeof(SolveState) * ni);
    for (int i = 0; i < ni; ++i) P->mst_h[i].done = 1;  // idle until a solve begins
    CK(upload(P, P->mst, P->mst_h, sizeof(SolveState) * ni));
    CK(cudaStreamSynchronize(P->stream));  // mst_h is pinned: rewritten only after the copy
  }
  if (P->inst_dirty) {
    std::vector<int32_t> first(ni), count(ni), geo((size_t)P->nb * 4);
    for (int i = 0; i < ni; ++i) {
      first[i] = P->inst[i].first;
      count[i] = P->inst[i].count;
    }
    for (int b = 0; b < P->nb; ++b) {
      geo[4 * b] = P->level[b];
      for (int a = 0; a < 3; ++a) geo[4 * b + 1 + a] = P->index[3 * b + a];
    }
    CK(upload(P, P->blk_inst_d, P->blk_inst_h.data(), sizeof(int32_t) * P->nb));
    CK(upload(P, P->inst_first_d, first.data(), sizeof(int32_t) * ni));
    CK(upload(P, P->inst_count_d, count.data(), sizeof(int32_t) * ni));
    CK(upload(P, P->blk_geo_d, geo.data(), sizeof(int32_t) * 4 * P->nb));
    P->inst_dirty = false;
  }
  return FFVGPU_OK;
}

// Publishes the blocks of every running instance to the persistent kernels
// (stream-ordered: work enqueued later sees the new list), the blocks that
// stream their coefficients first (launch_mx_order_active), so that the
// persistent grids deal them out evenly.  A staging buffer is rewritten only
// after its previous copy has been consumed.
ffvgpu_status publish_active(ffvgpu_pool* P) {
  const int k = P->act_next;
  P->act_next ^= 1;
  CK(cudaEventSynchronize(P->act_ev[k]));
  int32_t* h = P->act_h[k];
  int n = 0;
  for (const ffvgpu_instance& I : P->inst)
    if (I.running)
      for (int b = 0; b < I.count; ++b) h[1 + n++] = I.first + b;
  h[0] = n;
  CK(cudaMemcpyAsync(P->act_raw_d, h, sizeof(int32_t) * (size_t)(n + 1),
                     cudaMemcpyHostToDevice, P->stream));
  CK(cudaEventRecord(P->act_ev[k], P->stream));
  launch_mx_order_active(P->stream, P->act_raw_d, P->mucoef, P->act_d);
  CK(cudaGetLastError());
  return FFVGPU_OK;
}

ffvgpu_status ensure_mixed_buffers(ffvgpu_pool* P, bool d64) {
  ffvgpu_status s;
  const size_t n = field_count(P);
  if (!P->act_d) {
    if ((s = dalloc_t(P, &P->act_d, n / BC + 1)) || (s = dalloc_t(P, &P->act_raw_d, n / BC + 1)))
      return s;
    CK(cudaMemsetAsync(P->act_d, 0, sizeof(int32_t), P->stream));
    for (int k = 0; k < 2; ++k) {
      CK(cudaMallocHost(&P->act_h[k], sizeof(int32_t) * (n / BC + 1)));
      CK(cudaEventCreateWithFlags(&P->act_ev[k], cudaEventDisableTiming));
      CK(cudaEventRecord(P->act_ev[k], P->stream));
    }
    mx_grid_sizes(P->m_threads, &P->grid_sweep, &P->grid_matvec, &P->grid_update,
                  &P->grid_guides, &P->grid_mvpipe);
    P->grid_threads = P->m_threads;
  }
  if ((s = dalloc_t(P, &P->mcoef, 7 * n)) || (s = dalloc_t(P, &P->mguide, n / BC * 6 * 256)) ||
      (s = dalloc_t(P, &P->mucoef, n / BC * 8)) ||
      (s = dalloc_t(P, &P->me[0], n)) ||
      (s = dalloc_t(P, &P->me[1], n)) || (s = dalloc_t(P, &P->mph, n)) ||
      (s = dalloc_t(P, &P->msh, n)) ||
      (s = dalloc_t(P, &P->r, n)) || (s = dalloc_t(P, &P->r0, n)) || (s = dalloc_t(P, &P->p, n)) ||
      (s = dalloc_t(P, &P->q, n)) || (s = dalloc_t(P, &P->sv, n)) || (s = dalloc_t(P, &P->tv, n)))
    return s;
  if (d64 && ((s = dalloc_t(P, &P->mcoef64, 7 * n)) || (s = dalloc_t(P, &P->me64[0], n)) ||
              (s = dalloc_t(P, &P->me64[1], n)) || (s = dalloc_t(P, &P->mph64, n)) ||
              (s = dalloc_t(P, &P->msh64, n))))
    return s;
  return FFVGPU_OK;
}

ffvgpu_status ensure_mhist(ffvgpu_pool* P, int n) {
  if (n <= P->mhist_cap) return FFVGPU_OK;
  if (P->mhist) {
    for (const ffvgpu_instance& I : P->inst)
      if (I.running) return bad("history length grows while solves run");
    cudaFree(P->mhist);
    P->bytes -= (int64_t)P->mhist_cap * num_inst(P) * 8;
    P->mhist = nullptr;
  }
  P->mhist_cap = 0;
  ffvgpu_status s = dalloc_t(P, &P->mhist, (size_t)n * num_inst(P));
  if (s == FFVGPU_OK) P->mhist_cap = n;
  return s;
}

MixCtx mix_ctx(const ffvgpu_pool* P) {
  MixCtx C;
  C.nbr = P->nbr_d;
  C.dx = P->dx_d;
  C.bc = P->bc_p;
  C.inst.blk_inst = P->blk_inst_d;
  C.inst.first = P->inst_first_d;
  C.inst.count = P->inst_count_d;
  C.inst.st = P->mst;
  C.partials = P->mpartials;
  C.ucoef = P->mucoef;
  C.capacity = P->nb;
  C.first = 0;
  C.n_active = P->act_d;
  C.active = P->act_d + 1;
  C.wait_ns = P->wait_ns;
  C.stall = P->stall_sweep;
  C.cf = P->m_cf;
  C.depth = P->m_depth;
  C.sweep_threads = P->m_sweep_threads;
  return C;
}

KCtx range_ctx(const ffvgpu_pool* P, const BCSet& bc, const ffvgpu_instance& I) {
  KCtx C = P->ctx(bc);
  C.first = I.first;
  C.nb = I.count;
  return C;
}

int stage_depth_of(const ffvgpu_mixed_params* prm) {
  return prm->stage_depth > 0 ? prm->stage_depth : 1;
}
int threads_of(const ffvgpu_mixed_params* prm) {
  return prm->threads_per_block > 0 ? prm->threads_per_block : 256;
}
int sweep_threads_of(const ffvgpu_mixed_params* prm) {
  return prm->sweep_threads > 0 ? prm->sweep_threads : 256;
}

ffvgpu_status check_mixed(const ffvgpu_mixed_params* prm) {
  if (!prm) return bad("null parameters");
  if (prm->sweeps < 1 || prm->sweeps_per_exchange < 1 ||
      prm->sweeps % prm->sweeps_per_exchange != 0)
    return bad("sweeps must be a positive multiple of sweeps_per_exchange");
  if (prm->sweeps_per_exchange > 64) return bad("sweeps_per_exchange must be at most 64");
  if (!(prm->omega > 0.0 && prm->omega < 2.0)) return bad("omega must lie in (0, 2)");
  if (!(prm->restart_drop >= 0.0 && prm->restart_drop < 1.0))
    return bad("restart_drop must lie in [0, 1)");
  if (!(prm->restart_growth == 0.0 || prm->restart_growth > 1.0))
    return bad("restart_growth must be 0 or greater than 1");
  if (prm->restart_every < 0) return bad("restart_every must not be negative");
  if (prm->count_max < 0) return bad("count_max must not be negative");
  if (prm->stage_depth < 0 || prm->stage_depth > 3) return bad("stage_depth must lie in 0..3");
  if (prm->sweep_threads != 0 && prm->sweep_threads != 256 && prm->sweep_threads != 512)
    return bad("sweep_threads must be 0, 256 or 512");
  if (prm->matvec_form != 0 && prm->matvec_form != 1) return bad("matvec_form must be 0 or 1");
  if (prm->threads_per_block != 0 && prm->threads_per_block != 128 &&
      prm->threads_per_block != 256 && prm->threads_per_block != 512)
    return bad("threads_per_block must be 0, 128, 256 or 512");
  return FFVGPU_OK;
}

// Algorithmic HBM bytes of one iteration per cell: two preconditioner
// applications, two A*x with dot products, the update.  cw: coefficient bytes
// of a cell in a sweep pass (28 as 32-bit words, 56 in FP64), ew: bytes of one
// iterate or preconditioned-vector value (4 in FP32, 8 in FP64).
// Of those, the per-cell coefficient bytes that a uniform block does not move
// (its seven values come from one per-block record).
int64_t uniform_saving_per_cell(int passes, bool d64) {
  return 2 * passes * (d64 ? 56 : 28) + 2 * 56;
}

int64_t iteration_bytes_per_cell(int passes, bool d64) {
  const int64_t cw = d64 ? 56 : 28, ew = d64 ? 8 : 4;
  const int64_t first_p = cw + 8 + 16 + 8 + ew;  // coefficients, r, p and q, p, e
  const int64_t first_s = cw + 16 + 8 + ew;      // coefficients, q and r, s, e
  const int64_t later = cw + 8 + ew + ew;        // coefficients, p or s, e in, e out
  const int64_t matvec = 56 + ew + 8 + 8;
  const int64_t update = ew + ew + 8 + 8 + 8 + 8 + 8 + 8;
  return first_p + first_s + 2 * (passes - 1) * later + 2 * matvec + update;
}

// One iteration of every running instance (all blocks of the pool).
void enqueue_iteration(ffvgpu_pool* P, cudaStream_t s) {
  const MixCtx C = mix_ctx(P);
  // CTAs of a persistent grid: SMs x resident CTAs, or the test cap
  auto cap = [&](int n) { return P->grid_cap > 0 ? std::min(n, P->grid_cap) : n; };
  const int passes = P->m_sweeps / P->m_per_exchange;
  const float om = (float)P->m_omega;
  const bool d64 = P->m_d64 != 0;
  double* x = P->x[P->xcur];
  void* e[2] = {d64 ? (void*)P->me64[0] : (void*)P->me[0],
                d64 ? (void*)P->me64[1] : (void*)P->me[1]};
  void* ph = d64 ? (void*)P->mph64 : (void*)P->mph;
  void* sh = d64 ? (void*)P->msh64 : (void*)P->msh;
  for (int mode = 0; mode < 2; ++mode) {
    double* rhs = mode == 0 ? P->p : P->sv;
    void* hat = mode == 0 ? ph : sh;
    for (int ps = 0; ps < passes; ++ps) {
      const bool last = ps == passes - 1;
      const void* ein = ps > 0 ? e[(ps - 1) & 1] : nullptr;
      if (ps > 0) launch_mx_guides(s, C, cap(P->grid_guides), ein, P->mguide, d64);
      launch_mx_sweep(s, C, cap(P->grid_sweep), mode, ps == 0, om, P->m_per_exchange, P->r, P->r0,
                      rhs, P->q, P->mcoef, P->mcoef64, ein, P->mguide, last ? hat : e[ps & 1],
                      d64);
    }
    const int mvc = cap(P->m_mvform == 0 ? P->grid_mvpipe : P->grid_matvec);
    if (mode == 0)
      launch_mx_matvec(s, C, mvc, 1, P->m_threads, P->m_mvform, ph, P->A, P->q, P->r0, d64);
    else
      launch_mx_matvec(s, C, mvc, 2, P->m_threads, P->m_mvform, sh, P->A, P->tv, P->sv, d64);
  }
  launch_mx_update(s, C, cap(P->grid_update), P->m_threads, x, ph, sh, P->r, P->tv, P->sv, P->r0,
                   d64);
}

int launches_per_iteration(const ffvgpu_pool* P) {
  const int passes = P->m_sweeps / P->m_per_exchange;
  return 2 * passes + 2 * (passes - 1) + 3;  // sweeps, guide layers, A*x (2), update
}

ffvgpu_status result_status(const ffvgpu_result& R, int status_code, double eps, int count_max,
                            int timeout_where) {
  if (status_code == 3) {
    g_last_error = timeout_message(timeout_where);
    return FFVGPU_TIMEOUT;
  }
  if (status_code == 4) {
    g_last_error = "the solve was cancelled";
    return FFVGPU_CANCELLED;
  }
  if (status_code == 2) {
    g_last_error = "residual is NaN or Inf";
    return FFVGPU_NAN_DETECTED;
  }
  if (eps > 0.0 && R.count > count_max) return FFVGPU_NOT_CONVERGED;
  return FFVGPU_OK;
}

ffvgpu_status admit_range(ffvgpu_pool* P, const ffvgpu_grid_desc* d, int32_t* instance) {
  if (!P->batch) return bad("instances are admitted into batch pools");
  if (!d || !instance || !d->level || !d->block_index || d->num_blocks <= 0)
    return bad("empty grid");
  if (d->cells != 16) return bad("only 16^3 leaf blocks are supported");
  if (d->root_length <= 0.0) return bad("root_length must be positive");
  const int n = d->num_blocks;
  for (int b = 0; b < n; ++b) {
    if (d->level[b] < 0 || d->level[b] > 20) return bad("block level out of range");
    for (int a = 0; a < 3; ++a) {
      const long ext = (long)d->root_grid[a] << d->level[b];
      if (d->block_index[3 * b + a] < 0 || d->block_index[3 * b + a] >= ext)
        return bad("block index outside the root grid");
    }
  }
  std::vector<FaceNbr> nbr;
  ffvgpu_status s = derive_neighbors(n, d->level, d->block_index, d, nbr);
  if (s != FFVGPU_OK) return s;
  int slot = -1;
  for (int i = 0; i < num_inst(P); ++i)
    if (!P->inst[i].used) {
      slot = i;
      break;
    }
  if (slot < 0) {
    g_last_error = "no free instance slot";
    return FFVGPU_OOM;
  }
  int first = -1;
  for (int b = 0, run = 0; b < P->nb; ++b) {
    run = (P->blk_inst_h[b] < 0) ? run + 1 : 0;
    if (run == n) {
      first = b - n + 1;
      break;
    }
  }
  if (first < 0) {
    g_last_error = "no free block range of " + std::to_string(n) + " blocks";
    return FFVGPU_OOM;
  }
  if ((s = ensure_inst_device(P))) return s;
  ffvgpu_instance& I = P->inst[slot];
  I = ffvgpu_instance();
  I.used = true;
  I.first = first;
  I.count = n;
  I.level.assign(d->level, d->level + n);
  I.index.assign(d->block_index, d->block_index + 3 * n);
  I.desc = *d;
  I.desc.level = I.level.data();
  I.desc.block_index = I.index.data();
  I.desc.neighbor_kind = nullptr;
  I.desc.neighbor_ids = nullptr;
  for (int b = 0; b < n; ++b) {
    const int g = first + b;
    P->blk_inst_h[g] = slot;
    P->level[g] = d->level[b];
    for (int a = 0; a < 3; ++a) P->index[3 * g + a] = d->block_index[3 * b + a];
    P->dx_h[g] = d->root_length / (double)(1L << d->level[b]) / 16.0;
    for (int f = 0; f < 6; ++f) {
      FaceNbr F = nbr[(size_t)b * 6 + f];
      for (int q = 0; q < 4; ++q)
        if (F.id[q] >= 0) F.id[q] += first;
      P->nbr_h[(size_t)g * 6 + f] = F;
    }
  }
  // the instance's state stays idle (done) while its tables go live
  SolveState idle;
  std::memset(&idle, 0, sizeof(idle));
  idle.done = 1;
  CK(upload(P, P->mst + slot, &idle, sizeof(idle)));
  CK(upload(P, P->nbr_d + (size_t)first * 6, P->nbr_h.data() + (size_t)first * 6,
            sizeof(FaceNbr) * 6 * n));
  CK(upload(P, P->dx_d + first, P->dx_h.data() + first, sizeof(double) * n));
  P->inst_dirty = true;
  if ((s = ensure_inst_device(P))) return s;
  *instance = slot;
  return FFVGPU_OK;
}

// UpdateP's P02-P05 for the blocks of instance I from device-generated
// sphere-flow inputs: u*, cuts and flags (kernels_gen.cu), the velocity
// exchange, bcut_calc_ab_p, the BC folding, and x = 0.
// assemble false: only u*, the cut fields and the flags (and the u BCs).
ffvgpu_status generate_and_assemble(ffvgpu_pool* P, const ffvgpu_instance& I,
                                    const ffvgpu_sphere_problem* prob, bool assemble = true) {
  ffvgpu_status s;
  if ((s = ensure_inst_device(P))) return s;
  // fields the generator and the assembly write (pool-wide, allocated once)
  double *ux, *uy, *uz, *c0, *xp, *dummy;
  size_t stride;
  if ((s = field_ptr(P, FFVGPU_FIELD_UX, true, &ux, &stride, &dummy)) ||
      (s = field_ptr(P, FFVGPU_FIELD_UY, true, &uy, &stride, &dummy)) ||
      (s = field_ptr(P, FFVGPU_FIELD_UZ, true, &uz, &stride, &dummy)) ||
      (s = field_ptr(P, FFVGPU_FIELD_C0, true, &c0, &stride, &dummy)) ||
      (s = field_ptr(P, FFVGPU_FIELD_X, true, &xp, &stride, &dummy)) ||
      (s = dalloc_t(P, &P->flags, field_count(P))) ||
      (s = dalloc_t(P, &P->A, 7 * field_count(P))) || (s = dalloc_t(P, &P->b, field_count(P))))
    return s;
  SphereGenParams G;
  for (int a = 0; a < 3; ++a) {
    G.domain_origin[a] = prob->grid.domain_origin[a];
    G.center[a] = prob->grid.center[a];
  }
  G.root_length = prob->grid.root_length;
  G.radius = prob->grid.radius;
  G.seed = prob->seed;
  G.sigma = prob->sigma;
  launch_gen_sphere(P->stream, I.first, I.count, P->blk_geo_d, G, ux, uy, uz, c0, field_count(P),
                    P->flags);
  for (int c = 0; c < 3; ++c) {
    BCSet bu;
    for (int f = 0; f < 6; ++f) {
      bu.type[f] = prob->u_bc_type[c][f];
      bu.value[f] = prob->u_bc_value[c][f];
    }
    P->bc_u[c] = bu;
    if (assemble) launch_exchange(P->stream, range_ctx(P, bu, I), P->u[c], P->gu[c]);
  }
  if (!assemble) {
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(P->stream));
    return FFVGPU_OK;
  }
  launch_assemble(P->stream, range_ctx(P, P->bc_p, I), P->u[0], P->u[1], P->u[2], P->gu[0],
                  P->gu[1], P->gu[2], P->cut, P->flags, P->A, P->b, nullptr, prob->rhof,
                  prob->dt, field_count(P));
  launch_fold_bc(P->stream, range_ctx(P, P->bc_p, I), P->A, P->b);
  launch_fill(P->stream, I.count, P->x[P->xcur] + (size_t)I.first * BC, BC,
              P->gx + (size_t)I.first * 6 * FACE_CELLS, 0.0);
  P->sys_version++;
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(P->stream));
  return FFVGPU_OK;
}

ffvgpu_instance* get_inst(ffvgpu_pool* P, int32_t i) {
  if (!P || i < 0 || i >= num_inst(P) || !P->inst[i].used) return nullptr;
  return &P->inst[i];
}

}  // namespace

extern "C" {

ffvgpu_status ffvgpu_batch_create(const ffvgpu_batch_desc* d, ffvgpu_pool** out) {
  if (!d || !out) return bad("null argument");
  *out = nullptr;
  if (d->capacity_blocks <= 0) return bad("capacity_blocks must be positive");
  if (d->max_instances <= 0 || d->max_instances > 65536)
    return bad("max_instances must lie in [1, 65536]");
  for (int f = 0; f < 6; ++f)
    if (d->bc_type[f] != FFVGPU_BC_DIRICHLET && d->bc_type[f] != FFVGPU_BC_NEUMANN)
      return bad("outer BC type must be Dirichlet or Neumann");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    g_last_error = "no CUDA device";
    return FFVGPU_NO_DEVICE;
  }
  ffvgpu_pool* P = new ffvgpu_pool();
  cudaGetDevice(&P->device);
  P->batch = true;
  P->nb = d->capacity_blocks;
  P->level.assign(P->nb, 0);
  P->index.assign((size_t)P->nb * 3, 0);
  P->dx_h.assign(P->nb, 1.0);
  FaceNbr outer;
  std::memset(&outer, 0, sizeof(outer));
  outer.kind = NB_OUTER;
  for (int q = 0; q < 4; ++q) outer.id[q] = -1;
  P->nbr_h.assign((size_t)P->nb * 6, outer);
  for (int f = 0; f < 6; ++f) {
    P->bc_p.type[f] = d->bc_type[f];
    P->bc_p.value[f] = d->bc_value[f];
    for (int c = 0; c < 3; ++c) {
      P->bc_u[c].type[f] = FFVGPU_BC_NEUMANN;
      P->bc_u[c].value[f] = 0.0;
    }
  }
  P->inst.resize(d->max_instances);
  P->blk_inst_h.assign(P->nb, -1);
  ffvgpu_status s;
  if ((s = pool_init_device(P)) || (s = ensure_inst_device(P))) {
    ffvgpu_pool_destroy(P);
    return s;
  }
  *out = P;
  return FFVGPU_OK;
}

ffvgpu_status ffvgpu_instance_admit(ffvgpu_pool* P, const ffvgpu_grid_desc* d,
                                    int32_t* instance) {
  if (!P) return bad("null pool");
  cudaSetDevice(P->device);
  return admit_range(P, d, instance);
}

ffvgpu_status ffvgpu_instance_admit_sphere(ffvgpu_pool* P, const ffvgpu_sphere_problem* prob,
                                           int32_t* instance) {
  if (!P || !prob || !instance) return bad("null argument");
  if (!(prob->rhof > 0.0) || !(prob->dt > 0.0)) return bad("rhof and dt must be positive");
  cudaSetDevice(P->device);
  ffvgpu_sphere_grid* g = nullptr;
  ffvgpu_status s = ffvgpu_sphere_grid_create(&prob->grid, &g);
  if (s != FFVGPU_OK) return s == FFVGPU_BAD_ARG ? bad("bad sphere grid parameters") : s;
  const int n = ffvgpu_sphere_grid_num_blocks(g);
  std::vector<int32_t> lev(n), idx(3 * (size_t)n);
  ffvgpu_sphere_grid_blocks(g, lev.data(), idx.data());
  ffvgpu_sphere_grid_destroy(g);
  ffvgpu_grid_desc d;
  std::memset(&d, 0, sizeof(d));
  d.num_blocks = n;
  d.cells = 16;
  d.level = lev.data();
  d.block_index = idx.data();
  for (int a = 0; a < 3; ++a) {
    d.domain_origin[a] = prob->grid.domain_origin[a];
    d.root_grid[a] = prob->grid.root_grid[a];
  }
  d.root_length = prob->grid.root_length;
  int32_t slot = -1;
  if ((s = admit_range(P, &d, &slot))) return s;
  if ((s = generate_and_assemble(P, P->inst[slot], prob))) {
    ffvgpu_instance_release(P, slot);
    return s;
  }
  *instance = slot;
  return FFVGPU_OK;
}

static ffvgpu_status sphere_on_pool(ffvgpu_pool* P, const ffvgpu_sphere_problem* prob,
                                    bool assemble);

ffvgpu_status ffvgpu_assemble_sphere(ffvgpu_pool* P, const ffvgpu_sphere_problem* prob) {
  return sphere_on_pool(P, prob, true);
}

ffvgpu_status ffvgpu_generate_sphere(ffvgpu_pool* P, const ffvgpu_sphere_problem* prob) {
  return sphere_on_pool(P, prob, false);
}

static ffvgpu_status sphere_on_pool(ffvgpu_pool* P, const ffvgpu_sphere_problem* prob,
                                    bool assemble) {
  if (!P || !prob) return bad("null argument");
  if (P->batch) return bad("a batch pool admits sphere problems with ffvgpu_instance_admit_sphere");
  if (!(prob->rhof > 0.0) || !(prob->dt > 0.0)) return bad("rhof and dt must be positive");
  cudaSetDevice(P->device);
  // the pool's grid must be the problem's grid
  ffvgpu_sphere_grid* g = nullptr;
  ffvgpu_status s = ffvgpu_sphere_grid_create(&prob->grid, &g);
  if (s != FFVGPU_OK) return bad("bad sphere grid parameters");
  const int n = ffvgpu_sphere_grid_num_blocks(g);
  std::vector<int32_t> lev(n), idx(3 * (size_t)n);
  ffvgpu_sphere_grid_blocks(g, lev.data(), idx.data());
  ffvgpu_sphere_grid_destroy(g);
  if (n != P->nb || lev != P->level || idx != P->index)
    return bad("the pool was not created from this sphere problem's grid");
  for (int a = 0; a < 3; ++a)
    if (P->inst[0].desc.domain_origin[a] != prob->grid.domain_origin[a])
      return bad("the pool's domain origin differs from the problem's");
  return generate_and_assemble(P, P->inst[0], prob, assemble);
}

ffvgpu_status ffvgpu_instance_upload(ffvgpu_pool* P, int32_t inst, ffvgpu_field f,
                                     const void* host, int32_t vc) {
  ffvgpu_instance* I = get_inst(P, inst);
  if (!I || !host) return bad("bad instance or null buffer");
  if (I->running) return bad("instance is solving");
  if (vc < 1 || vc > 4) return bad("vc must be in [1,4]");
  cudaSetDevice(P->device);
  const size_t w = 16 + 2 * (size_t)vc;
  const size_t per = w * w * w;
  ffvgpu_status s;
  if (f >= FFVGPU_IFIELD_CID0 && f <= FFVGPU_IFIELD_PID) {
    if ((s = dalloc_t(P, &P->flags, field_count(P)))) return s;
    if ((s = ensure_stage(P, per * I->count * sizeof(int32_t)))) return s;
    CK(cudaMemcpyAsync(P->stage, host, per * I->count * sizeof(int32_t), cudaMemcpyHostToDevice,
                       P->stream));
    const int bit = (f == FFVGPU_IFIELD_PID) ? 7 : (f - FFVGPU_IFIELD_CID0);
    launch_pack_flag(P->stream, I->count, (const int32_t*)P->stage, vc,
                     P->flags + (size_t)I->first * BC, bit, f == FFVGPU_IFIELD_PID ? 1 : 0);
  } else {
    double *dst, *g;
    size_t stride;
    if ((s = field_ptr(P, f, true, &dst, &stride, &g))) return s;
    const double* src;
    if ((s = host_source(P, host, per * I->count * sizeof(double), &src))) return s;
    launch_pack(P->stream, I->count, src, vc, dst + (size_t)I->first * stride, stride,
                g ? g + (size_t)I->first * 6 * FACE_CELLS : nullptr);
  }
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(P->stream));
  return FFVGPU_OK;
}

ffvgpu_status ffvgpu_instance_download(ffvgpu_pool* P, int32_t inst, ffvgpu_field f, void* host,
                                       int32_t vc) {
  ffvgpu_instance* I = get_inst(P, inst);
  if (!I || !host) return bad("bad instance or null buffer");
  if (vc < 1 || vc > 2) return bad("download supports vc = 1 or 2");
  cudaSetDevice(P->device);
  const size_t w = 16 + 2 * (size_t)vc;
  const size_t per = w * w * w;
  ffvgpu_status s;
  if (f >= FFVGPU_IFIELD_CID0 && f <= FFVGPU_IFIELD_PID) {
    if (!P->flags) return bad("integer fields have not been uploaded");
    if ((s = ensure_stage(P, per * I->count * sizeof(int32_t)))) return s;
    const int bit = (f == FFVGPU_IFIELD_PID) ? 7 : (f - FFVGPU_IFIELD_CID0);
    launch_unpack_flag(P->stream, I->count, P->flags + (size_t)I->first * BC, vc,
                       (int32_t*)P->stage, bit);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(host, P->stage, per * I->count * sizeof(int32_t), cudaMemcpyDeviceToHost,
                       P->stream));
    CK(cudaStreamSynchronize(P->stream));
    return FFVGPU_OK;
  }
  double *src, *g;
  size_t stride;
  if ((s = field_ptr(P, f, false, &src, &stride, &g))) return s;
  if ((s = ensure_stage(P, per * I->count * sizeof(double)))) return s;
  const bool vec = (f == FFVGPU_FIELD_X) || (f >= FFVGPU_FIELD_UX && f <= FFVGPU_FIELD_UZ);
  launch_unpack(P->stream, range_ctx(P, field_bc(P, f), *I), src, stride, vc, vec ? 1 : 0,
                (double*)P->stage);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(host, P->stage, per * I->count * sizeof(double), cudaMemcpyDeviceToHost,
                     P->stream));
  CK(cudaStreamSynchronize(P->stream));
  return FFVGPU_OK;
}

ffvgpu_status ffvgpu_instance_fill(ffvgpu_pool* P, int32_t inst, ffvgpu_field f, double value) {
  ffvgpu_instance* I = get_inst(P, inst);
  if (!I) return bad("bad instance");
  if (I->running) return bad("instance is solving");
  cudaSetDevice(P->device);
  double *x, *g;
  size_t stride;
  ffvgpu_status s;
  if ((s = field_ptr(P, f, true, &x, &stride, &g))) return s;
  launch_fill(P->stream, I->count, x + (size_t)I->first * stride, stride,
              g ? g + (size_t)I->first * 6 * FACE_CELLS : nullptr, value);
  if ((f >= FFVGPU_FIELD_AP && f <= FFVGPU_FIELD_AT) || f == FFVGPU_FIELD_B) P->sys_version++;
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(P->stream));
  return FFVGPU_OK;
}

ffvgpu_status ffvgpu_instance_release(ffvgpu_pool* P, int32_t inst) {
  ffvgpu_instance* I = get_inst(P, inst);
  if (!I) return bad("bad instance");
  if (!P->batch) return bad("the instance of a one-grid pool is the pool");
  if (I->running) return bad("instance is solving");
  cudaSetDevice(P->device);
  CK(cudaStreamSynchronize(P->stream));
  for (int b = I->first; b < I->first + I->count; ++b) P->blk_inst_h[b] = -1;
  CK(upload(P, P->blk_inst_d + I->first, P->blk_inst_h.data() + I->first,
            sizeof(int32_t) * I->count));
  *I = ffvgpu_instance();
  return FFVGPU_OK;
}

int32_t ffvgpu_instance_blocks(const ffvgpu_pool* P, int32_t inst) {
  if (!P || inst < 0 || inst >= (int)P->inst.size() || !P->inst[inst].used) return 0;
  return P->inst[inst].count;
}

ffvgpu_status ffvgpu_pool_free_blocks(const ffvgpu_pool* P, int32_t* free_blocks,
                                      int32_t* largest_range) {
  if (!P) return bad("null pool");
  int32_t total = 0, best = 0, run = 0;
  for (int b = 0; b < P->nb; ++b) {
    if (P->blk_inst_h[b] < 0) {
      ++total;
      ++run;
      if (run > best) best = run;
    } else {
      run = 0;
    }
  }
  if (free_blocks) *free_blocks = total;
  if (largest_range) *largest_range = best;
  return FFVGPU_OK;
}

ffvgpu_status ffvgpu_mixed_begin(ffvgpu_pool* P, int32_t inst, const ffvgpu_mixed_params* prm) {
  ffvgpu_instance* I = get_inst(P, inst);
  if (!I) return bad("bad instance");
  if (I->running) return bad("instance is already solving");
  ffvgpu_status s;
  if ((s = check_mixed(prm))) return s;
  if (!P->A || !P->b) return bad("A and b must be uploaded or assembled before a solve");
  cudaSetDevice(P->device);
  bool others = false;
  for (const ffvgpu_instance& J : P->inst) others = others || J.running;
  if (others && (prm->omega != P->m_omega || prm->sweeps != P->m_sweeps ||
                 prm->sweeps_per_exchange != P->m_per_exchange ||
                 (prm->flux_correction != 0) != (P->m_cf != 0) ||
                 (prm->fp64_data != 0) != (P->m_d64 != 0) ||
                 stage_depth_of(prm) != P->m_depth || threads_of(prm) != P->m_threads ||
                 sweep_threads_of(prm) != P->m_sweep_threads || prm->matvec_form != P->m_mvform))
    return bad("running instances use other preconditioner settings");
  double *xp, *g;
  size_t stride;
  if ((s = field_ptr(P, FFVGPU_FIELD_X, true, &xp, &stride, &g))) return s;
  if ((s = ensure_inst_device(P)) || (s = ensure_mixed_buffers(P, prm->fp64_data != 0)) ||
      (s = ensure_mhist(P, prm->count_max > 0 ? prm->count_max : 1)))
    return s;
  P->m_omega = prm->omega;
  P->m_sweeps = prm->sweeps;
  P->m_per_exchange = prm->sweeps_per_exchange;
  P->m_cf = prm->flux_correction != 0;
  P->m_d64 = prm->fp64_data != 0;
  P->m_depth = stage_depth_of(prm);
  P->m_threads = threads_of(prm);
  P->m_sweep_threads = sweep_threads_of(prm);
  P->m_mvform = prm->matvec_form;
  if (P->grid_threads != P->m_threads) {  // the persistent grids of this CTA size
    mx_grid_sizes(P->m_threads, &P->grid_sweep, &P->grid_matvec, &P->grid_update,
                  &P->grid_guides, &P->grid_mvpipe);
    P->grid_threads = P->m_threads;
  }
  I->count_max = prm->count_max;
  I->epsilon = prm->epsilon;
  I->result = ffvgpu_result();
  SolveState& h = P->mst_h[inst];  // pinned staging of the state copy
  std::memset(&h, 0, sizeof(h));
  h.eps = prm->epsilon;
  h.count_max = prm->count_max;
  h.drop = prm->restart_drop;
  h.growth = prm->restart_growth;
  h.max_cycle = prm->restart_every;
  h.hist = P->mhist + (size_t)inst * P->mhist_cap;
  h.done = 0;
  if (prm->count_max <= 0) {  // for(count=1; count<=countMax; ...) runs no iteration
    I->result.count = 1;
    I->status = 0;
    I->running = false;
    return FFVGPU_OK;
  }
  // the instance's state, its 32-bit coefficients and uniform-block records
  // (counted into the state), then b.b / r / r0 / r.r0
  I->ublocks = 0;
  CK(cudaMemcpyAsync(P->mst + inst, &h, sizeof(h), cudaMemcpyHostToDevice, P->stream));
  launch_mx_pack(P->stream, I->first, I->count, P->A, P->mcoef, P->mcoef64, P->mucoef,
                 P->mst + inst, P->m_d64 != 0, P->m_sweep_threads);
  MixCtx C = mix_ctx(P);
  C.first = I->first;
  launch_mx_init(P->stream, C, I->count, P->x[P->xcur], P->gx, P->A, P->b, P->r, P->r0);
  CK(cudaGetLastError());
  P->m_launches += 2;
  P->m_bytes += (int64_t)I->count * BC * (7 * 8 + 7 * (P->m_d64 ? 8 : 4) + 8 * 9 + 16);
  I->running = true;
  return publish_active(P);
}

ffvgpu_status ffvgpu_mixed_advance(ffvgpu_pool* P, int32_t iterations) {
  if (!P) return bad("null pool");
  if (iterations <= 0) return FFVGPU_OK;
  int running = 0;
  int64_t cells = 0, ucells = 0;
  for (const ffvgpu_instance& I : P->inst)
    if (I.running) {
      ++running;
      cells += (int64_t)I.count * BC;
      ucells += (int64_t)I.ublocks * BC;
    }
  if (!running) return FFVGPU_OK;
  cudaSetDevice(P->device);
  // kernel arguments (the wait limit among them) are fixed at capture
  if (!P->mgraph || P->mgraph_iters != iterations || P->mgraph_omega != P->m_omega ||
      P->mgraph_sweeps != P->m_sweeps || P->mgraph_per != P->m_per_exchange ||
      P->mgraph_wait_ns != P->wait_ns || P->mgraph_stall != P->stall_sweep ||
      P->mgraph_cap != P->grid_cap ||
      P->mgraph_cf != P->m_cf || P->mgraph_d64 != P->m_d64 ||
      P->mgraph_depth != P->m_depth || P->mgraph_threads != P->m_threads ||
      P->mgraph_sweep_threads != P->m_sweep_threads || P->mgraph_mvform != P->m_mvform) {
    if (P->mgraph) cudaGraphExecDestroy(P->mgraph);
    P->mgraph = nullptr;
    cudaGraph_t graph;
    CK(cudaStreamBeginCapture(P->own_stream, cudaStreamCaptureModeThreadLocal));
    for (int it = 0; it < iterations; ++it) enqueue_iteration(P, P->own_stream);
    CK(cudaStreamEndCapture(P->own_stream, &graph));
    cudaError_t e = cudaGraphInstantiate(&P->mgraph, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate");
    P->mgraph_iters = iterations;
    P->mgraph_omega = P->m_omega;
    P->mgraph_sweeps = P->m_sweeps;
    P->mgraph_per = P->m_per_exchange;
    P->mgraph_wait_ns = P->wait_ns;
    P->mgraph_stall = P->stall_sweep;
    P->mgraph_cap = P->grid_cap;
    P->mgraph_cf = P->m_cf;
    P->mgraph_d64 = P->m_d64;
    P->mgraph_depth = P->m_depth;
    P->mgraph_threads = P->m_threads;
    P->mgraph_sweep_threads = P->m_sweep_threads;
    P->mgraph_mvform = P->m_mvform;
  }
  CK(cudaGraphLaunch(P->mgraph, P->stream));
  P->m_launches += (int64_t)iterations * launches_per_iteration(P);
  const int passes = P->m_sweeps / P->m_per_exchange;
  P->m_bytes += (int64_t)iterations *
                (cells * iteration_bytes_per_cell(passes, P->m_d64 != 0) -
                 ucells * uniform_saving_per_cell(passes, P->m_d64 != 0));
  return FFVGPU_OK;
}

ffvgpu_status ffvgpu_mixed_poll(ffvgpu_pool* P, int32_t* finished, int32_t capacity,
                                int32_t* n_finished) {
  if (!P) return bad("null pool");
  if (n_finished) *n_finished = 0;
  bool any = false;
  for (const ffvgpu_instance& I : P->inst) any = any || I.running;
  if (!any) return FFVGPU_OK;
  cudaSetDevice(P->device);
  const int ni = num_inst(P);
  CK(cudaMemcpyAsync(P->mst_h, P->mst, sizeof(SolveState) * ni, cudaMemcpyDeviceToHost,
                     P->stream));
  CK(cudaStreamSynchronize(P->stream));
  int nf = 0;
  for (int i = 0; i < ni; ++i) {
    ffvgpu_instance& I = P->inst[i];
    if (I.running) I.ublocks = I.result.uniform_blocks = P->mst_h[i].ublocks;  // from the packing
    if (!I.running || !P->mst_h[i].done) continue;
    const SolveState& h = P->mst_h[i];
    I.running = false;
    I.result.count = h.count;
    I.result.residual = h.residual;
    I.status = h.status;
    I.timeout_where = h.timeout_where;
    P->stall_sweep = 0;  // the test hook covers one solve
    I.last_iter = (h.count == 0) ? h.iter : 0;  // 0 when the exit came before iteration 1
    launch_exchange(P->stream, range_ctx(P, P->bc_p, I), P->x[P->xcur], P->gx);  // FFVILS.h:973
    if (finished && nf < capacity) finished[nf] = i;
    ++nf;
  }
  CK(cudaGetLastError());
  if (nf) {
    ffvgpu_status s = publish_active(P);
    if (s != FFVGPU_OK) return s;
    CK(cudaStreamSynchronize(P->stream));
  }
  if (n_finished) *n_finished = nf;
  return FFVGPU_OK;
}

// Test hook: the next mixed solve's sweep kernel waits for a copy it never
// issues, so the wait runs out after the pool's wait limit and the solve ends
// with FFVGPU_TIMEOUT; nothing is in flight, so nothing is drained.
ffvgpu_status ffvgpu_pool_stall_next_solve(ffvgpu_pool* P) {
  if (!P) return bad("null pool");
  P->stall_sweep = 1;
  return FFVGPU_OK;
}

ffvgpu_status ffvgpu_pool_stall_next_matvec(ffvgpu_pool* P) {
  if (!P) return bad("null pool");
  P->stall_sweep = 2;
  return FFVGPU_OK;
}

ffvgpu_status ffvgpu_pool_cap_grids(ffvgpu_pool* P, int32_t ctas) {
  if (!P) return bad("null pool");
  if (ctas < 0) return bad("ctas must not be negative");
  for (const ffvgpu_instance& I : P->inst)
    if (I.running) return bad("a stepped mixed solve is running on this pool");
  P->grid_cap = ctas;
  return FFVGPU_OK;
}

// Stops one running instance: its device state is marked done (status 4,
// stream-ordered, so the next replay skips its blocks), its blocks leave the
// active list, and its result records the iterations completed so far.
ffvgpu_status ffvgpu_mixed_cancel(ffvgpu_pool* P, int32_t inst) {
  ffvgpu_instance* I = get_inst(P, inst);
  if (!I) return bad("bad instance");
  if (!I->running) return bad("instance is not solving");
  cudaSetDevice(P->device);
  // done and status are adjacent int32 fields of SolveState
  static_assert(offsetof(SolveState, status) == offsetof(SolveState, done) + 4,
                "SolveState layout");
  int32_t* flags = reinterpret_cast<int32_t*>(P->host_done);  // pinned
  flags[0] = 1;
  flags[1] = 4;
  CK(cudaMemcpyAsync(&P->mst[inst].done, flags, 2 * sizeof(int32_t), cudaMemcpyHostToDevice,
                     P->stream));
  CK(cudaMemcpyAsync(P->mst_h + inst, P->mst + inst, sizeof(SolveState), cudaMemcpyDeviceToHost,
                     P->stream));
  CK(cudaStreamSynchronize(P->stream));
  const SolveState& h = P->mst_h[inst];
  I->running = false;
  I->status = 4;
  I->timeout_where = 0;
  I->result.count = h.iter > 1 ? h.iter - 1 : 0;  // iterations with a residual
  I->result.residual = h.residual;
  I->last_iter = I->result.count;
  return publish_active(P);
}

ffvgpu_status ffvgpu_instance_result(const ffvgpu_pool* P, int32_t inst, ffvgpu_result* res,
                                     double* history) {
  if (!P || inst < 0 || inst >= (int)P->inst.size() || !P->inst[inst].used)
    return bad("bad instance");
  const ffvgpu_instance& I = P->inst[inst];
  if (I.running) return bad("instance is solving");
  if (res) *res = I.result;
  if (history && I.count_max > 0 && P->mhist) {
    const int c = I.result.count;
    // an early exit (count 0) keeps the residuals of the iterations before it
    const int nh = (c >= 1 && c <= I.count_max) ? c : (c == 0 ? I.last_iter : I.count_max);
    if (nh > 0)
      CK(download_sync(const_cast<ffvgpu_pool*>(P), history,
                       P->mhist + (size_t)inst * P->mhist_cap, sizeof(double) * nh));
  }
  return result_status(I.result, I.status, I.epsilon, I.count_max, I.timeout_where);
}

ffvgpu_status ffvgpu_solve_mixed(ffvgpu_pool* P, const ffvgpu_mixed_params* prm,
                                 ffvgpu_result* res) {
  if (!P) return bad("null pool");
  ffvgpu_status s;
  if ((s = check_mixed(prm))) return s;
  cudaSetDevice(P->device);
  for (const ffvgpu_instance& I : P->inst)
    if (I.running) return bad("a stepped mixed solve is running on this pool");
  const int64_t l0 = P->m_launches, b0 = P->m_bytes;
  CK(cudaEventRecord(P->ev0, P->stream));
  std::vector<int> mine;
  for (int i = 0; i < num_inst(P); ++i) {
    if (!P->inst[i].used) continue;
    if ((s = ffvgpu_mixed_begin(P, i, prm))) return s;
    mine.push_back(i);
  }
  CK(cudaEventRecord(P->ev2, P->stream));
  const int every = prm->check_every > 0 ? prm->check_every : 8;
  for (;;) {
    int32_t nf = 0;
    if ((s = ffvgpu_mixed_poll(P, nullptr, 0, &nf))) return s;
    bool any = false;
    for (int i : mine) any = any || P->inst[i].running;
    if (!any) break;
    if ((s = ffvgpu_mixed_advance(P, every))) return s;
  }
  CK(cudaEventRecord(P->ev1, P->stream));
  CK(cudaEventSynchronize(P->ev1));
  float ms = 0.f, sms = 0.f;
  cudaEventElapsedTime(&ms, P->ev0, P->ev1);
  cudaEventElapsedTime(&sms, P->ev2, P->ev1);
  ffvgpu_status first_status = FFVGPU_OK;
  bool first = true;
  for (int i : mine) {
    ffvgpu_instance& I = P->inst[i];
    I.result.elapsed_ms = ms;
    I.result.sweep_ms = sms;
    I.result.sweep_launches = (int32_t)(P->m_launches - l0);
    I.result.kernel_launches = (int32_t)(P->m_launches - l0);
    I.result.bytes_moved = P->m_bytes - b0;
    if (first) {
      first = false;
      first_status = ffvgpu_instance_result(P, i, res, prm->history);
    }
  }
  return first_status;
}

// Times the mixed solve of the given instances, from x = 0, for each
// candidate setting in records (omega, sweeps, sweeps_per_exchange,
// iterations per graph replay), with base's count_max, epsilon and restart
// settings; fills in each record's time, largest iteration count and whether
// every instance converged, and returns in *best the fastest candidate that
// converged them all (-1 if none did).  The instances end with x = 0.
ffvgpu_status ffvgpu_mixed_autotune(ffvgpu_pool* P, const int32_t* instances, int32_t n,
                                    const ffvgpu_mixed_params* base, ffvgpu_tune_record* rec,
                                    int32_t n_rec, int32_t* best) {
  if (!P || !instances || n <= 0 || !base || !rec || n_rec <= 0 || !best)
    return bad("null or empty argument");
  cudaSetDevice(P->device);
  for (const ffvgpu_instance& I : P->inst)
    if (I.running) return bad("a stepped mixed solve is running on this pool");
  for (int i = 0; i < n; ++i)
    if (!get_inst(P, instances[i])) return bad("bad instance");
  ffvgpu_status s;
  *best = -1;
  double best_ms = 0.0;
  for (int c = 0; c < n_rec; ++c) {
    ffvgpu_tune_record& R = rec[c];
    ffvgpu_mixed_params prm = *base;
    prm.omega = R.omega;
    prm.sweeps = R.sweeps;
    prm.sweeps_per_exchange = R.sweeps_per_exchange;
    prm.threads_per_block = R.threads_per_block;
    prm.stage_depth = R.stage_depth;
    prm.sweep_threads = R.sweep_threads;
    prm.matvec_form = R.matvec_form;
    prm.history = nullptr;
    R.ms = 0.0;
    R.max_count = 0;
    R.converged = 0;
    if ((s = check_mixed(&prm))) return s;
    if (R.iterations_per_replay <= 0) return bad("iterations_per_replay must be positive");
    for (int i = 0; i < n; ++i)
      if ((s = ffvgpu_instance_fill(P, instances[i], FFVGPU_FIELD_X, 0.0))) return s;
    CK(cudaEventRecord(P->ev0, P->stream));
    for (int i = 0; i < n; ++i)
      if ((s = ffvgpu_mixed_begin(P, instances[i], &prm))) return s;
    for (;;) {
      int32_t nf = 0;
      if ((s = ffvgpu_mixed_poll(P, nullptr, 0, &nf))) return s;
      bool any = false;
      for (int i = 0; i < n; ++i) any = any || P->inst[instances[i]].running;
      if (!any) break;
      if ((s = ffvgpu_mixed_advance(P, R.iterations_per_replay))) return s;
    }
    CK(cudaEventRecord(P->ev1, P->stream));
    CK(cudaEventSynchronize(P->ev1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, P->ev0, P->ev1);
    R.ms = ms;
    bool all = true;
    for (int i = 0; i < n; ++i) {
      const ffvgpu_instance& I = P->inst[instances[i]];
      const int cnt = I.result.count;
      if (cnt > R.max_count) R.max_count = cnt;
      const bool ok = I.status == 0 && cnt >= 1 && cnt <= prm.count_max &&
                      I.result.residual <= prm.epsilon;
      all = all && ok;
    }
    R.converged = all ? 1 : 0;
    if (all && (*best < 0 || R.ms < best_ms)) {
      *best = c;
      best_ms = R.ms;
    }
  }
  for (int i = 0; i < n; ++i)
    if ((s = ffvgpu_instance_fill(P, instances[i], FFVGPU_FIELD_X, 0.0))) return s;
  return FFVGPU_OK;
}

}  // extern "C"

// Coarse-fine flux mismatch of FIELD_X (interior and stored guide layer):
// per coarse cell on a face whose neighbours are finer, the fine-side flux F
// and delta = F - A_f (g - x_P); sums of V_P |delta| and V_P |F| in (block,
// face, position) order.
ffvgpu_status ffvgpu_cf_flux_mismatch(ffvgpu_pool* P, double* mismatch, double* flux,
                                      int32_t* n_cells, double* per_cell, int32_t capacity) {
  if (!P || !mismatch || !flux || !n_cells) return bad("null argument");
  if (!P->A) return bad("A must be uploaded or assembled first");
  cudaSetDevice(P->device);
  double *xp, *g;
  size_t stride;
  ffvgpu_status s;
  if ((s = field_ptr(P, FFVGPU_FIELD_X, false, &xp, &stride, &g))) return s;
  if (!xp || !g) return bad("pressure field not allocated");
  std::vector<int32_t> pairs;
  for (int b = 0; b < P->nb; ++b) {
    if (b < (int)P->blk_inst_h.size() && P->blk_inst_h[b] < 0) continue;
    for (int f = 0; f < 6; ++f)
      if (P->nbr_h[(size_t)b * 6 + f].kind == NB_FINE) {
        pairs.push_back(b);
        pairs.push_back(f);
      }
  }
  const int np = (int)pairs.size() / 2;
  const int64_t nc = (int64_t)np * FACE_CELLS;
  *n_cells = (int32_t)nc;
  *mismatch = 0.0;
  *flux = 0.0;
  if (per_cell && capacity < nc) return bad("per_cell capacity below the number of cells");
  if (np == 0) return FFVGPU_OK;
  int32_t* pd = nullptr;
  double* od = nullptr;
  cudaError_t e = cudaMalloc(&pd, sizeof(int32_t) * pairs.size());
  if (e == cudaSuccess) e = cudaMalloc(&od, sizeof(double) * 2 * nc);
  std::vector<double> out(2 * nc);
  if (e == cudaSuccess) e = upload(P, pd, pairs.data(), sizeof(int32_t) * pairs.size());
  if (e == cudaSuccess) {
    launch_cf_mismatch(P->stream, np, xp, g, P->A, P->nbr_d, P->dx_d, P->bc_p, pd, od);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = download_sync(P, out.data(), od, sizeof(double) * 2 * nc);
  cudaFree(pd);
  cudaFree(od);
  if (e != cudaSuccess) return cuda_fail(e, "cf_flux_mismatch");
  double m = 0.0, fl = 0.0;
  for (int i = 0; i < np; ++i) {
    const double dx = P->dx_h[pairs[2 * i]], vol = dx * dx * dx;
    for (int p = 0; p < FACE_CELLS; ++p) {
      const size_t c = (size_t)i * FACE_CELLS + p;
      m += vol * std::fabs(out[2 * c]);
      fl += vol * std::fabs(out[2 * c + 1]);
    }
  }
  if (per_cell) std::memcpy(per_cell, out.data(), sizeof(double) * 2 * nc);
  *mismatch = m;
  *flux = fl;
  return FFVGPU_OK;
}
