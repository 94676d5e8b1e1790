// pool.cpp -- device block pool and the extern "C" entry points of
// include/ffvgpu.h.
//
// The pool plays the role of the reference's per-rank LocalScalar3D fields
// on a BCMTools BlockManager (src/FFV/LocalScalar3D.h:21-460): it owns every
// field of every leaf block, resident in HBM, plus the neighbour table the
// in-kernel exchange reads.  The solve entry points follow FFVILS
// (src/FFV/FFVILS.h) iteration by iteration; all scalars of the recurrences
// live on the device, so the host only enqueues kernels and, when a
// convergence criterion is set, polls the done flag every few iterations.
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/ffvgpu.h"
#include "ffvgpu_kernels.h"
#include "ffvgpu_layout.h"
#include "ffvgpu_mixed.h"
#include "pool_internal.h"

using namespace ffvgpu;
using namespace ffvgpu::detail;

namespace ffvgpu {
namespace detail {

ffvgpu_status dalloc(ffvgpu_pool* P, void** ptr, size_t bytes) {
  if (*ptr) return FFVGPU_OK;
  cudaError_t e = cudaMalloc(ptr, bytes);
  if (e != cudaSuccess) {
    *ptr = nullptr;
    return cuda_fail(e, "cudaMalloc");
  }
  P->bytes += (int64_t)bytes;
  return FFVGPU_OK;
}


ffvgpu_status ensure_stage(ffvgpu_pool* P, size_t bytes) {
  if (P->stage_bytes >= bytes) return FFVGPU_OK;
  if (P->stage) {
    cudaFree(P->stage);
    P->bytes -= (int64_t)P->stage_bytes;
    P->stage = nullptr;
  }
  P->stage_bytes = 0;
  ffvgpu_status s = dalloc(P, &P->stage, bytes);
  if (s == FFVGPU_OK) P->stage_bytes = bytes;
  return s;
}

ffvgpu_status host_source(ffvgpu_pool* P, const void* host, size_t bytes, const double** src) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, host) == cudaSuccess && at.type == cudaMemoryTypeHost &&
      at.devicePointer) {
    *src = static_cast<const double*>(at.devicePointer);
    return FFVGPU_OK;
  }
  cudaGetLastError();  // a pageable buffer is not an error here
  ffvgpu_status s;
  if ((s = ensure_stage(P, bytes))) return s;
  CK(cudaMemcpyAsync(P->stage, host, bytes, cudaMemcpyHostToDevice, P->stream));
  *src = static_cast<const double*>(P->stage);
  return FFVGPU_OK;
}

size_t field_count(const ffvgpu_pool* P) { return (size_t)P->nb * BC; }

// Device pointer and block stride of a real field's interior.
ffvgpu_status field_ptr(ffvgpu_pool* P, int f, bool alloc, double** ptr, size_t* stride,
                        double** guides) {
  const size_t n = field_count(P);
  *stride = BC;
  if (guides) *guides = nullptr;
  ffvgpu_status s = FFVGPU_OK;
  if (f == FFVGPU_FIELD_X) {
    if (alloc) {
      if ((s = dalloc_t(P, &P->x[0], n)) || (s = dalloc_t(P, &P->x[1], n)) ||
          (s = dalloc_t(P, &P->gx, (size_t)P->nb * 6 * FACE_CELLS)))
        return s;
    }
    *ptr = P->x[P->xcur];
    if (guides) *guides = P->gx;
  } else if (f >= FFVGPU_FIELD_AP && f <= FFVGPU_FIELD_AT) {
    if (alloc && (s = dalloc_t(P, &P->A, 7 * n))) return s;
    *ptr = P->A ? P->A + (size_t)(f - FFVGPU_FIELD_AP) * BC : nullptr;
    *stride = 7 * BC;
  } else if (f == FFVGPU_FIELD_B) {
    if (alloc && (s = dalloc_t(P, &P->b, n))) return s;
    *ptr = P->b;
  } else if (f >= FFVGPU_FIELD_UX && f <= FFVGPU_FIELD_UZ) {
    const int c = f - FFVGPU_FIELD_UX;
    if (alloc && ((s = dalloc_t(P, &P->u[c], n)) ||
                  (s = dalloc_t(P, &P->gu[c], (size_t)P->nb * 6 * FACE_CELLS))))
      return s;
    *ptr = P->u[c];
    if (guides) *guides = P->gu[c];
  } else if (f >= FFVGPU_FIELD_C0 && f <= FFVGPU_FIELD_C5) {
    if (alloc && (s = dalloc_t(P, &P->cut, 6 * n))) return s;
    *ptr = P->cut ? P->cut + (size_t)(f - FFVGPU_FIELD_C0) * n : nullptr;
  } else if (f >= FFVGPU_FIELD_VW && f <= FFVGPU_FIELD_VT) {
    if (alloc && (s = dalloc_t(P, &P->vface, 6 * n))) return s;
    *ptr = P->vface ? P->vface + (size_t)(f - FFVGPU_FIELD_VW) * n : nullptr;
  } else if (f == FFVGPU_FIELD_LAPP) {
    if (alloc && (s = dalloc_t(P, &P->lapp, n))) return s;
    *ptr = P->lapp;
  } else {
    return bad("unknown real field");
  }
  if (!*ptr) return bad("field has not been uploaded or computed");
  return FFVGPU_OK;
}

const BCSet& field_bc(const ffvgpu_pool* P, int f) {
  if (f >= FFVGPU_FIELD_UX && f <= FFVGPU_FIELD_UZ) return P->bc_u[f - FFVGPU_FIELD_UX];
  return P->bc_p;
}

ffvgpu_status ensure_solver(ffvgpu_pool* P) {
  ffvgpu_status s;
  if ((s = dalloc_t(P, &P->partials, (size_t)P->nb + 1)) || (s = dalloc_t(P, &P->st, 1)))
    return s;
  if (!P->host_done) {
    cudaError_t e = cudaMallocHost(&P->host_done, sizeof(SolveState));
    if (e != cudaSuccess) return cuda_fail(e, "cudaMallocHost");
  }
  return FFVGPU_OK;
}

ffvgpu_status reset_state(ffvgpu_pool* P, double eps, int count_max, double* hist,
                          double drop = 0.0) {
  SolveState h;
  std::memset(&h, 0, sizeof(h));
  h.eps = eps;
  h.count_max = count_max;
  h.rr0 = 1.0;
  h.gamma = 1.0;  // FFVILS.h:841-842: alpha = 0, gamma = 1 before the first iteration
  h.hist = hist;
  h.cycle = 1;
  h.drop = drop;
  h.next_restart = -1.0;
  CK(cudaMemcpyAsync(P->st, &h, sizeof(h), cudaMemcpyHostToDevice, P->stream));
  return FFVGPU_OK;
}

ffvgpu_status read_state(ffvgpu_pool* P, SolveState* h) {
  CK(cudaMemcpyAsync(P->host_done, P->st, sizeof(SolveState), cudaMemcpyDeviceToHost, P->stream));
  CK(cudaStreamSynchronize(P->stream));
  std::memcpy(h, P->host_done, sizeof(SolveState));
  return FFVGPU_OK;
}

ffvgpu_status poll_done(ffvgpu_pool* P, bool* done) {
  SolveState h;
  ffvgpu_status s = read_state(P, &h);
  *done = h.done != 0;
  return s;
}

ffvgpu_status ensure_hist(ffvgpu_pool* P, int n) {
  if (n <= P->hist_cap) return FFVGPU_OK;
  if (P->hist_d) {
    cudaFree(P->hist_d);
    P->bytes -= (int64_t)P->hist_cap * 8;
    P->hist_d = nullptr;
  }
  P->hist_cap = 0;
  ffvgpu_status s = dalloc_t(P, &P->hist_d, (size_t)n);
  if (s == FFVGPU_OK) P->hist_cap = n;
  return s;
}

ffvgpu_status require_system(ffvgpu_pool* P) {
  if (!P->A || !P->b) return bad("A and b must be uploaded or assembled before a solve");
  double* xp;
  size_t st;
  return field_ptr(P, FFVGPU_FIELD_X, true, &xp, &st, nullptr);
}

// Repacks A and b into the sweep's coefficient stream when they changed.
ffvgpu_status ensure_stream(ffvgpu_pool* P) {
  ffvgpu_status s;
  if ((s = dalloc_t(P, &P->coef, (size_t)P->nb * STREAM_BLOCK)) ||
      (s = dalloc_t(P, &P->urec, (size_t)P->nb * 8)) || (s = dalloc_t(P, &P->ucount_d, 1)))
    return s;
  if (P->stream_version != P->sys_version) {
    CK(cudaMemsetAsync(P->ucount_d, 0, sizeof(int32_t), P->stream));
    launch_pack_stream(P->stream, P->nb, P->A, P->b, P->coef, P->urec, P->ucount_d);
    CK(cudaGetLastError());
    CK(download_sync(P, &P->ucount_h, P->ucount_d, sizeof(int32_t)));
    P->stream_version = P->sys_version;
    P->urec_version = P->sys_version;
    P->ucount_version = P->sys_version;
  }
  return FFVGPU_OK;
}

// The uniform records of A (KCtx::urec) when A changed.
ffvgpu_status ensure_urec(ffvgpu_pool* P) {
  ffvgpu_status s;
  if ((s = dalloc_t(P, &P->urec, (size_t)P->nb * 8)) || (s = dalloc_t(P, &P->ucount_d, 1)))
    return s;
  if (P->urec_version != P->sys_version) {
    CK(cudaMemsetAsync(P->ucount_d, 0, sizeof(int32_t), P->stream));
    launch_urec(P->stream, P->nb, P->A, P->urec, P->ucount_d);
    CK(cudaGetLastError());
    P->urec_version = P->sys_version;
  }
  return FFVGPU_OK;
}

// The FP64 solvers' pipelined A*x over the pool as one instance: its block
// list (the blocks that stream their coefficients first, so the persistent
// grid deals them out evenly), instance tables and per-block sums.
ffvgpu_status ensure_kpipe(ffvgpu_pool* P) {
  ffvgpu_status s;
  if ((s = ensure_urec(P))) return s;
  const int nb = P->nb;
  if (!P->kpipe_ready) {  // allocations already made are kept by dalloc on a retry
    if ((s = dalloc_t(P, &P->kpipe, (size_t)2 * nb + 3)) ||
        (s = dalloc_t(P, &P->kraw, (size_t)nb + 1)) ||
        (s = dalloc_t(P, &P->kpart, (size_t)2 * nb)))
      return s;
    std::vector<int32_t> h((size_t)2 * nb + 3, 0);
    h[0] = nb;
    for (int b = 0; b < nb; ++b) h[1 + b] = b;
    h[(size_t)2 * nb + 2] = nb;  // count; blk_inst and first stay 0
    CK(upload(P, P->kraw, h.data(), sizeof(int32_t) * ((size_t)nb + 1)));
    CK(upload(P, P->kpipe + 1 + nb, h.data() + 1 + nb, sizeof(int32_t) * ((size_t)nb + 2)));
    if (!P->grid_mvpipe) {
      int a, b, c, d, e;
      mx_grid_sizes(P->m_threads, &a, &b, &c, &d, &e);
      P->grid_mvpipe = e;
    }
    P->kpipe_version = 0;
    P->kpipe_ready = true;
  }
  if (P->kpipe_version != P->sys_version) {
    launch_mx_order_active(P->stream, P->kraw, P->urec, P->kpipe);
    CK(cudaGetLastError());
    P->kpipe_version = P->sys_version;
  }
  return FFVGPU_OK;
}

MixCtx krylov_mix_ctx(const ffvgpu_pool* P, int fin) {
  const int nb = P->nb;
  MixCtx C;
  C.active = P->kpipe + 1;
  C.n_active = P->kpipe;
  C.nbr = P->nbr_d;
  C.dx = P->dx_d;
  C.bc = P->bc_p;
  C.inst.blk_inst = P->kpipe + 1 + nb;
  C.inst.first = P->kpipe + 1 + 2 * nb;
  C.inst.count = P->kpipe + 2 + 2 * nb;
  C.inst.st = P->st;
  C.partials = P->kpart;
  C.ucoef = P->urec;
  C.capacity = nb;
  C.first = 0;
  C.wait_ns = P->wait_ns;
  C.stall = 0;
  C.cf = 0;
  C.depth = 1;
  C.sweep_threads = P->m_sweep_threads;
  C.fin = fin;
  return C;
}

// q = A x and q.w (fin FIN_BI_QR0 or FIN_CG_QP), or with t.t as well
// (FIN_BI_TS, then FIN_BI_TT) when 'two'.
void krylov_matvec(ffvgpu_pool* P, const double* x, double* q, const double* w, int fin,
                   bool two) {
  int grid = P->grid_mvpipe;
  if (P->grid_cap > 0 && P->grid_cap < grid) grid = P->grid_cap;
  launch_mx_matvec(P->stream, krylov_mix_ctx(P, fin), grid, two ? 2 : 1, 0, 0, x, P->A, q, w,
                   true);
}

// A Jacobi sweep from a stored iterate, y = J(x; A, b), on the same kernel;
// with dot also b.y (FIN_CG_RR1).
void krylov_jacobi(ffvgpu_pool* P, const double* x, double* y, const double* b, double omega,
                   bool dot) {
  int grid = P->grid_mvpipe;
  if (P->grid_cap > 0 && P->grid_cap < grid) grid = P->grid_cap;
  launch_jacobi_pipe(P->stream, krylov_mix_ctx(P, dot ? FIN_CG_RR1 : 0), grid, dot, x, P->A, b,
                     y, omega);
}

// Derives the neighbour table from levels and block indices.
ffvgpu_status derive_neighbors(int nb, const int32_t* level, const int32_t* index,
                               const ffvgpu_grid_desc* d, std::vector<FaceNbr>& out) {
  out.resize((size_t)nb * 6);
  std::map<std::tuple<int, long, long, long>, int> key;
  for (int b = 0; b < nb; ++b)
    key[std::make_tuple(level[b], (long)index[3 * b], (long)index[3 * b + 1],
                        (long)index[3 * b + 2])] = b;
  auto find = [&](int L, long x, long y, long z) {
    auto it = key.find(std::make_tuple(L, x, y, z));
    return it == key.end() ? -1 : it->second;
  };
  for (int b = 0; b < nb; ++b) {
    const int L = level[b];
    const long id[3] = {index[3 * b], index[3 * b + 1], index[3 * b + 2]};
    for (int f = 0; f < 6; ++f) {
      FaceNbr& F = out[b * 6 + f];
      std::memset(&F, 0, sizeof(F));
      for (int q = 0; q < 4; ++q) F.id[q] = -1;
      const int ax = f >> 1, dir = (f & 1) ? 1 : -1;
      const int ta = (ax == 0) ? 1 : 0, tb = (ax == 2) ? 1 : 2;
      long n[3] = {id[0], id[1], id[2]};
      n[ax] += dir;
      const long ext = (long)d->root_grid[ax] << L;
      if (n[ax] < 0 || n[ax] >= ext) {
        F.kind = NB_OUTER;
        continue;
      }
      int s = find(L, n[0], n[1], n[2]);
      if (s >= 0) {
        F.kind = NB_SAME;
        F.id[0] = s;
        continue;
      }
      if (L > 0 && (s = find(L - 1, n[0] >> 1, n[1] >> 1, n[2] >> 1)) >= 0) {
        F.kind = NB_COARSE;
        F.id[0] = s;
        F.so_u = (int)(id[ta] & 1);
        F.so_v = (int)(id[tb] & 1);
        continue;
      }
      F.kind = NB_FINE;
      for (int q = 0; q < 4; ++q) {
        long c[3];
        c[ax] = 2 * n[ax] + (dir > 0 ? 0 : 1);
        c[ta] = 2 * n[ta] + (q & 1);
        c[tb] = 2 * n[tb] + (q >> 1);
        F.id[q] = find(L + 1, c[0], c[1], c[2]);
        if (F.id[q] < 0) return bad("grid is not 2:1 face balanced or has a hole");
      }
    }
  }
  return FFVGPU_OK;
}

ffvgpu_status explicit_neighbors(ffvgpu_pool* P, const ffvgpu_grid_desc* d) {
  for (int b = 0; b < P->nb; ++b)
    for (int f = 0; f < 6; ++f) {
      FaceNbr& F = P->nbr_h[b * 6 + f];
      std::memset(&F, 0, sizeof(F));
      F.kind = d->neighbor_kind[b * 6 + f];
      for (int q = 0; q < 4; ++q) F.id[q] = d->neighbor_ids[(b * 6 + f) * 4 + q];
      const int ax = f >> 1;
      const int ta = (ax == 0) ? 1 : 0, tb = (ax == 2) ? 1 : 2;
      if (F.kind < NB_OUTER || F.kind > NB_FINE) return bad("bad neighbour kind");
      const int need = (F.kind == NB_FINE) ? 4 : (F.kind == NB_OUTER ? 0 : 1);
      for (int q = 0; q < need; ++q)
        if (F.id[q] < 0 || F.id[q] >= P->nb) return bad("neighbour id out of range");
      if (F.kind == NB_COARSE) {
        F.so_u = P->index[3 * b + ta] & 1;
        F.so_v = P->index[3 * b + tb] & 1;
        if (P->level[F.id[0]] != P->level[b] - 1) return bad("coarse neighbour level mismatch");
      }
      if (F.kind == NB_SAME && P->level[F.id[0]] != P->level[b])
        return bad("same-level neighbour level mismatch");
      if (F.kind == NB_FINE)
        for (int q = 0; q < 4; ++q)
          if (P->level[F.id[q]] != P->level[b] + 1) return bad("fine neighbour level mismatch");
    }
  return FFVGPU_OK;
}

ffvgpu_status solve_status(const SolveState& h, const ffvgpu_iter_params* prm, int N, int count) {
  if (h.status == 3) {
    g_last_error = timeout_message(h.timeout_where);
    return FFVGPU_TIMEOUT;
  }
  if (h.status == 2) {
    g_last_error = "residual is NaN or Inf";
    return FFVGPU_NAN_DETECTED;
  }
  if (prm->epsilon > 0.0 && count > N) return FFVGPU_NOT_CONVERGED;
  return FFVGPU_OK;
}

int64_t interior_bytes(const ffvgpu_pool* P, int words) {
  return (int64_t)P->nb * (int64_t)BC * 8 * words;
}
// Bytes of one pass of the red-black kernel: 'words' per cell (10 for a
// sweep with its residual, 9 for a residual alone) in a block that streams
// its coefficients, 'words' - 7 in a uniform block (b and x only).
int64_t rbgs_pass_bytes(const ffvgpu_pool* P, int words) {
  const int64_t u = P->ucount_h, n = P->nb;
  return ((n - u) * words + u * (words - 7)) * (int64_t)BC * 8;
}
// Bytes the kernels of an FP64 Krylov solve moved: 'words' values per cell
// over every block, less 'coef' per-cell coefficient words in each uniform
// block (the Jacobi and A*x kernels read its seven coefficients once from
// its record).  The uniform count is read back once per assembled A.
ffvgpu_status krylov_bytes(ffvgpu_pool* P, int64_t words, int64_t coef, int64_t* bytes) {
  if (P->ucount_version != P->sys_version) {
    CK(download_sync(P, &P->ucount_h, P->ucount_d, sizeof(int32_t)));
    P->ucount_version = P->sys_version;
  }
  *bytes = ((int64_t)P->nb * words - (int64_t)P->ucount_h * coef) * (int64_t)BC * 8;
  return FFVGPU_OK;
}

// Stream, events, neighbour table, cell sizes and the solver state of a
// pool whose host tables are filled in.
ffvgpu_status pool_init_device(ffvgpu_pool* P) {
  cudaError_t e;
  if ((e = cudaStreamCreateWithFlags(&P->own_stream, cudaStreamNonBlocking)) != cudaSuccess ||
      (e = cudaEventCreate(&P->ev0)) != cudaSuccess ||
      (e = cudaEventCreate(&P->ev1)) != cudaSuccess ||
      (e = cudaEventCreate(&P->ev2)) != cudaSuccess ||
      (e = cudaEventCreate(&P->ev3)) != cudaSuccess)
    return cuda_fail(e, "stream/event create");
  P->stream = P->own_stream;
  ffvgpu_status s;
  if ((s = dalloc_t(P, &P->nbr_d, P->nbr_h.size())) || (s = dalloc_t(P, &P->dx_d, P->dx_h.size())))
    return s;
  CK(upload(P, P->nbr_d, P->nbr_h.data(), P->nbr_h.size() * sizeof(FaceNbr)));
  CK(upload(P, P->dx_d, P->dx_h.data(), P->dx_h.size() * sizeof(double)));
  return ensure_solver(P);
}

}  // namespace detail
}  // namespace ffvgpu

void ffvgpu::set_last_error(const std::string& msg) { g_last_error = msg; }

extern "C" {

int32_t ffvgpu_version(void) { return 1; }
const char* ffvgpu_last_error(void) { return g_last_error.c_str(); }

ffvgpu_status ffvgpu_pool_create(const ffvgpu_grid_desc* d, ffvgpu_pool** out) {
  if (!d || !out) return bad("null argument");
  *out = nullptr;
  if (d->cells != 16) return bad("only 16^3 leaf blocks are supported");
  if (d->num_blocks <= 0 || !d->level || !d->block_index) return bad("empty grid");
  if (d->root_length <= 0.0) return bad("root_length must be positive");
  for (int f = 0; f < 6; ++f)
    if (d->bc_type[f] != FFVGPU_BC_DIRICHLET && d->bc_type[f] != FFVGPU_BC_NEUMANN)
      return bad("outer BC type must be Dirichlet or Neumann");
  // every check of the description runs on the host, before the device is
  // touched, so a malformed grid is BAD_ARG whether or not a device is there
  ffvgpu_pool* P = new ffvgpu_pool();
  P->nb = d->num_blocks;
  P->level.assign(d->level, d->level + P->nb);
  P->index.assign(d->block_index, d->block_index + 3 * P->nb);
  for (int b = 0; b < P->nb; ++b) {
    if (P->level[b] < 0 || P->level[b] > 20) {
      delete P;
      return bad("block level out of range");
    }
    for (int a = 0; a < 3; ++a) {
      const long ext = (long)d->root_grid[a] << P->level[b];
      if (P->index[3 * b + a] < 0 || P->index[3 * b + a] >= ext) {
        delete P;
        return bad("block index outside the root grid");
      }
    }
  }
  P->nbr_h.resize((size_t)P->nb * 6);
  P->dx_h.resize(P->nb);
  for (int b = 0; b < P->nb; ++b)
    P->dx_h[b] = d->root_length / (double)(1L << P->level[b]) / 16.0;
  for (int f = 0; f < 6; ++f) {
    P->bc_p.type[f] = d->bc_type[f];
    P->bc_p.value[f] = d->bc_value[f];
    for (int c = 0; c < 3; ++c) {
      P->bc_u[c].type[f] = FFVGPU_BC_NEUMANN;
      P->bc_u[c].value[f] = 0.0;
    }
  }
  ffvgpu_status s = (d->neighbor_kind && d->neighbor_ids)
                        ? explicit_neighbors(P, d)
                        : derive_neighbors(P->nb, P->level.data(), P->index.data(), d, P->nbr_h);
  if (s != FFVGPU_OK) {
    delete P;
    return s;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    delete P;
    g_last_error = "no CUDA device";
    return FFVGPU_NO_DEVICE;
  }
  cudaGetDevice(&P->device);
  // the grid is instance 0 of its own pool
  P->inst.resize(1);
  ffvgpu_instance& I = P->inst[0];
  I.used = true;
  I.first = 0;
  I.count = P->nb;
  I.level = P->level;
  I.index = P->index;
  I.desc = *d;
  I.desc.level = I.level.data();
  I.desc.block_index = I.index.data();
  I.desc.neighbor_kind = nullptr;
  I.desc.neighbor_ids = nullptr;
  P->blk_inst_h.assign(P->nb, 0);
  if ((s = pool_init_device(P)) != FFVGPU_OK) {
    ffvgpu_pool_destroy(P);
    return s;
  }
  *out = P;
  return FFVGPU_OK;
}

void ffvgpu_pool_destroy(ffvgpu_pool* P) {
  if (!P) return;
  cudaSetDevice(P->device);
  if (P->stream) cudaStreamSynchronize(P->stream);
  if (P->own_stream) cudaStreamSynchronize(P->own_stream);
  release_instances(P);
  void* ptrs[] = {P->x[0], P->x[1], P->gx, P->A, P->coef, P->urec, P->ucount_d, P->b, P->u[0], P->u[1], P->u[2],
                  P->gu[0], P->gu[1], P->gu[2], P->cut, P->vface, P->lapp, P->flags, P->r,
                  P->p, P->q, P->z[0], P->z[1], P->r0, P->sv, P->tv, P->zb[0], P->zb[1],
                  P->partials, P->st, P->hist_d, P->kpipe, P->kraw, P->kpart,
                  P->stage, P->nbr_d, P->dx_d};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (P->host_done) cudaFreeHost(P->host_done);
  for (cudaEvent_t ev : {P->ev0, P->ev1, P->ev2, P->ev3})
    if (ev) cudaEventDestroy(ev);
  if (P->own_stream) cudaStreamDestroy(P->own_stream);
  delete P;
}

int32_t ffvgpu_pool_num_blocks(const ffvgpu_pool* P) { return P ? P->nb : 0; }
int64_t ffvgpu_pool_device_bytes(const ffvgpu_pool* P) { return P ? P->bytes : 0; }

ffvgpu_status ffvgpu_pool_set_stream(ffvgpu_pool* P, void* stream) {
  if (!P) return bad("null pool");
  cudaSetDevice(P->device);
  CK(cudaStreamSynchronize(P->stream));
  P->stream = stream ? (cudaStream_t)stream : P->own_stream;
  return FFVGPU_OK;
}

ffvgpu_status ffvgpu_pool_set_wait_limit(ffvgpu_pool* P, double seconds) {
  if (!P) return bad("null pool");
  if (!(seconds >= 0.0 && seconds <= 3600.0)) return bad("wait limit must lie in [0, 3600] s");
  P->wait_ns = (uint64_t)(seconds * 1e9);
  return FFVGPU_OK;
}

ffvgpu_status ffvgpu_grid_neighbors(const ffvgpu_grid_desc* d, int32_t* kind, int32_t* ids) {
  if (!d || !d->level || !d->block_index || d->num_blocks <= 0) return bad("empty grid");
  std::vector<FaceNbr> t;
  ffvgpu_status s = derive_neighbors(d->num_blocks, d->level, d->block_index, d, t);
  if (s != FFVGPU_OK) return s;
  for (size_t i = 0; i < t.size(); ++i) {
    if (kind) kind[i] = t[i].kind;
    if (ids)
      for (int q = 0; q < 4; ++q) ids[i * 4 + q] = t[i].id[q];
  }
  return FFVGPU_OK;
}

ffvgpu_status ffvgpu_fill(ffvgpu_pool* P, ffvgpu_field f, double value) {
  if (!P) return bad("null pool");
  if (P->batch) return bad("a batch pool is used through the instance entry points");
  cudaSetDevice(P->device);
  double *x, *g;
  size_t stride;
  ffvgpu_status s;
  if ((s = field_ptr(P, f, true, &x, &stride, &g))) return s;
  launch_fill(P->stream, P->nb, x, stride, g, value);
  if ((f >= FFVGPU_FIELD_AP && f <= FFVGPU_FIELD_AT) || f == FFVGPU_FIELD_B) P->sys_version++;
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(P->stream));
  return FFVGPU_OK;
}

ffvgpu_status ffvgpu_pool_neighbors(const ffvgpu_pool* P, int32_t b, int32_t* kind6,
                                    int32_t* ids24) {
  if (!P || b < 0 || b >= P->nb) return bad("bad block");
  for (int f = 0; f < 6; ++f) {
    const FaceNbr& F = P->nbr_h[b * 6 + f];
    if (kind6) kind6[f] = F.kind;
    if (ids24)
      for (int q = 0; q < 4; ++q) ids24[f * 4 + q] = F.id[q];
  }
  return FFVGPU_OK;
}

ffvgpu_status ffvgpu_pool_upload(ffvgpu_pool* P, ffvgpu_field f, const void* host, int32_t vc) {
  if (!P || !host) return bad("null argument");
  if (P->batch) return bad("a batch pool is used through the instance entry points");
  if (vc < 1 || vc > 4) return bad("vc must be in [1,4]");
  cudaSetDevice(P->device);
  const size_t w = 16 + 2 * (size_t)vc;
  const size_t per = w * w * w;
  ffvgpu_status s;
  if (f >= FFVGPU_IFIELD_CID0 && f <= FFVGPU_IFIELD_PID) {
    if ((s = dalloc_t(P, &P->flags, field_count(P)))) return s;
    if ((s = ensure_stage(P, per * P->nb * sizeof(int32_t)))) return s;
    CK(cudaMemcpyAsync(P->stage, host, per * P->nb * sizeof(int32_t), cudaMemcpyHostToDevice,
                       P->stream));
    const int bit = (f == FFVGPU_IFIELD_PID) ? 7 : (f - FFVGPU_IFIELD_CID0);
    launch_pack_flag(P->stream, P->nb, (const int32_t*)P->stage, vc, P->flags, bit,
                     f == FFVGPU_IFIELD_PID ? 1 : 0);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(P->stream));
    return FFVGPU_OK;
  }
  double* dst;
  double* g;
  size_t stride;
  if ((s = field_ptr(P, f, true, &dst, &stride, &g))) return s;
  const double* src;
  if ((s = host_source(P, host, per * P->nb * sizeof(double), &src))) return s;
  launch_pack(P->stream, P->nb, src, vc, dst, stride, g);
  CK(cudaGetLastError());
  if ((f >= FFVGPU_FIELD_AP && f <= FFVGPU_FIELD_AT) || f == FFVGPU_FIELD_B) P->sys_version++;
  CK(cudaStreamSynchronize(P->stream));
  return FFVGPU_OK;
}

ffvgpu_status ffvgpu_pool_download(ffvgpu_pool* P, ffvgpu_field f, void* host, int32_t vc) {
  if (!P || !host) return bad("null argument");
  if (P->batch) return bad("a batch pool is used through the instance entry points");
  if (vc < 1 || vc > 2) return bad("download supports vc = 1 or 2");
  cudaSetDevice(P->device);
  const size_t w = 16 + 2 * (size_t)vc;
  const size_t per = w * w * w;
  ffvgpu_status s;
  if (f >= FFVGPU_IFIELD_CID0 && f <= FFVGPU_IFIELD_PID) {
    if (!P->flags) return bad("integer fields have not been uploaded");
    if ((s = ensure_stage(P, per * P->nb * sizeof(int32_t)))) return s;
    const int bit = (f == FFVGPU_IFIELD_PID) ? 7 : (f - FFVGPU_IFIELD_CID0);
    launch_unpack_flag(P->stream, P->nb, P->flags, vc, (int32_t*)P->stage, bit);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(host, P->stage, per * P->nb * sizeof(int32_t), cudaMemcpyDeviceToHost,
                       P->stream));
    CK(cudaStreamSynchronize(P->stream));
    return FFVGPU_OK;
  }
  double* src;
  double* g;
  size_t stride;
  if ((s = field_ptr(P, f, false, &src, &stride, &g))) return s;
  if ((s = ensure_stage(P, per * P->nb * sizeof(double)))) return s;
  const bool vec = (f == FFVGPU_FIELD_X) || (f >= FFVGPU_FIELD_UX && f <= FFVGPU_FIELD_UZ);
  launch_unpack(P->stream, P->ctx(field_bc(P, f)), src, stride, vc, vec ? 1 : 0,
                (double*)P->stage);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(host, P->stage, per * P->nb * sizeof(double), cudaMemcpyDeviceToHost,
                     P->stream));
  CK(cudaStreamSynchronize(P->stream));
  return FFVGPU_OK;
}

ffvgpu_status ffvgpu_exchange(ffvgpu_pool* P, ffvgpu_field f, const int32_t* bc_type6,
                              const double* bc_value6) {
  if (!P) return bad("null pool");
  if (P->batch) return bad("a batch pool is used through the instance entry points");
  cudaSetDevice(P->device);
  BCSet bc = P->bc_p;
  if (bc_type6 && bc_value6)
    for (int i = 0; i < 6; ++i) {
      if (bc_type6[i] != FFVGPU_BC_DIRICHLET && bc_type6[i] != FFVGPU_BC_NEUMANN)
        return bad("BC type must be Dirichlet or Neumann");
      bc.type[i] = bc_type6[i];
      bc.value[i] = bc_value6[i];
    }
  double* x;
  double* g;
  size_t stride;
  ffvgpu_status s;
  if ((s = field_ptr(P, f, false, &x, &stride, &g))) return s;
  if (!g) return bad("field has no guide cells");
  if (f >= FFVGPU_FIELD_UX && f <= FFVGPU_FIELD_UZ) P->bc_u[f - FFVGPU_FIELD_UX] = bc;
  launch_exchange(P->stream, P->ctx(bc), x, g);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(P->stream));
  return FFVGPU_OK;
}

ffvgpu_status ffvgpu_assemble_p(ffvgpu_pool* P, double rhof, double dt) {
  if (!P) return bad("null pool");
  if (P->batch) return bad("a batch pool is used through the instance entry points");
  if (!(rhof > 0.0) || !(dt > 0.0)) return bad("rhof and dt must be positive");
  cudaSetDevice(P->device);
  for (int c = 0; c < 3; ++c)
    if (!P->u[c]) return bad("UX, UY, UZ must be uploaded before assembly");
  if (!P->cut || !P->flags) return bad("cut fields C0..C5, CID0..5 and PID must be uploaded");
  ffvgpu_status s;
  const size_t n = field_count(P);
  if ((s = dalloc_t(P, &P->A, 7 * n)) || (s = dalloc_t(P, &P->b, n)) ||
      (s = dalloc_t(P, &P->vface, 6 * n)))
    return s;
  launch_assemble(P->stream, P->ctx(P->bc_p), P->u[0], P->u[1], P->u[2], P->gu[0], P->gu[1],
                  P->gu[2], P->cut, P->flags, P->A, P->b, P->vface, rhof, dt, n);
  P->sys_version++;
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(P->stream));
  return FFVGPU_OK;
}

static ffvgpu_status projection(ffvgpu_pool* P, double rhof, double dt, bool corr) {
  if (!P) return bad("null pool");
  if (P->batch) return bad("a batch pool is used through the instance entry points");
  if (!(rhof > 0.0) || !(dt > 0.0)) return bad("rhof and dt must be positive");
  cudaSetDevice(P->device);
  for (int c = 0; c < 3; ++c)
    if (!P->u[c]) return bad("UX, UY, UZ must exist");
  if (!P->cut || !P->flags) return bad("cut fields C0..C5, CID0..5 and PID must be uploaded");
  if (!P->x[P->xcur]) return bad("the pressure must exist");
  ffvgpu_status s;
  const size_t n = field_count(P);
  if (corr && ((s = dalloc_t(P, &P->vface, 6 * n)) || (s = dalloc_t(P, &P->lapp, n)))) return s;
  launch_projection(P->stream, P->ctx(P->bc_p), corr, P->x[P->xcur], P->gx, P->cut, P->flags,
                    P->u[0], P->u[1], P->u[2], corr ? P->vface : nullptr,
                    corr ? P->lapp : nullptr, rhof, dt, n);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(P->stream));
  return FFVGPU_OK;
}

ffvgpu_status ffvgpu_remove_p(ffvgpu_pool* P, double rhof, double dt) {
  return projection(P, rhof, dt, false);
}

ffvgpu_status ffvgpu_corr_u(ffvgpu_pool* P, double rhof, double dt) {
  return projection(P, rhof, dt, true);
}

ffvgpu_status ffvgpu_fold_bc(ffvgpu_pool* P) {
  if (!P) return bad("null pool");
  if (P->batch) return bad("a batch pool is used through the instance entry points");
  if (!P->A || !P->b) return bad("A and b must exist before folding BCs");
  cudaSetDevice(P->device);
  launch_fold_bc(P->stream, P->ctx(P->bc_p), P->A, P->b);
  P->sys_version++;
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(P->stream));
  return FFVGPU_OK;
}

// Solver::UpdateP's pressure sequence (Solver.cpp:5294-5688): P01, P02, P03,
// P05, P06, P07.
ffvgpu_status ffvgpu_update_p(ffvgpu_pool* P, const ffvgpu_step_params* prm,
                              const ffvgpu_mixed_params* mixed, ffvgpu_result* res) {
  if (!P || !prm) return bad("null argument");
  if (P->batch) return bad("a batch pool is used through the instance entry points");
  if (prm->solver == FFVGPU_SOLVER_MIXED && !mixed) return bad("mixed settings missing");
  if (prm->solver < FFVGPU_SOLVER_RBGS || prm->solver > FFVGPU_SOLVER_MIXED)
    return bad("unknown solver");
  ffvgpu_status s;
  if ((s = ffvgpu_remove_p(P, prm->rhof, prm->dt))) return s;  // P01
  for (int c = 0; c < 3; ++c)                                    // P02
    if ((s = ffvgpu_exchange(P, (ffvgpu_field)(FFVGPU_FIELD_UX + c), prm->u_bc_type[c],
                             prm->u_bc_value[c])))
      return s;
  if ((s = ffvgpu_assemble_p(P, prm->rhof, prm->dt))) return s;  // P03
  if ((s = ffvgpu_fold_bc(P))) return s;                           // P05
  ffvgpu_status solved;                                            // P06
  if (prm->solver == FFVGPU_SOLVER_RBGS)
    solved = ffvgpu_solve_rbgs(P, &prm->iter, res);
  else if (prm->solver == FFVGPU_SOLVER_BICGSTAB)
    solved = ffvgpu_solve_bicgstab(P, &prm->iter, res);
  else
    solved = ffvgpu_solve_mixed(P, mixed, res);
  if (solved != FFVGPU_OK && solved != FFVGPU_NOT_CONVERGED) return solved;
  if ((s = ffvgpu_exchange(P, FFVGPU_FIELD_X, nullptr, nullptr))) return s;  // P07
  return solved;
}

// Solver::UpdateU (Solver.cpp:5690-5771): U01, U02, U03 (p only).
ffvgpu_status ffvgpu_update_u(ffvgpu_pool* P, const ffvgpu_step_params* prm) {
  if (!P || !prm) return bad("null argument");
  ffvgpu_status s;
  if ((s = ffvgpu_corr_u(P, prm->rhof, prm->dt))) return s;  // U01
  for (int c = 0; c < 3; ++c)                                 // U02
    if ((s = ffvgpu_exchange(P, (ffvgpu_field)(FFVGPU_FIELD_UX + c), prm->u_bc_type[c],
                             prm->u_bc_value[c])))
      return s;
  return ffvgpu_exchange(P, FFVGPU_FIELD_X, nullptr, nullptr);  // U03
}

ffvgpu_status ffvgpu_dot(ffvgpu_pool* P, ffvgpu_field fx, ffvgpu_field fy, double* xy) {
  if (!P || !xy) return bad("null argument");
  if (P->batch) return bad("a batch pool is used through the instance entry points");
  cudaSetDevice(P->device);
  double *x, *y, *g;
  size_t sx, sy;
  ffvgpu_status s;
  if ((s = field_ptr(P, fx, false, &x, &sx, &g)) || (s = field_ptr(P, fy, false, &y, &sy, &g)))
    return s;
  if (sx != BC || sy != BC) return bad("dot of matrix fields is not supported");
  if ((s = reset_state(P, 0.0, 0, nullptr))) return s;
  launch_dot(P->stream, P->ctx(P->bc_p), x, y, P->partials, P->st, FIN_STORE, 0);
  CK(cudaGetLastError());
  SolveState h;
  if ((s = read_state(P, &h))) return s;
  *xy = h.rr;
  return FFVGPU_OK;
}

ffvgpu_status ffvgpu_calc_r2(ffvgpu_pool* P, double* rr) {
  if (!P || !rr) return bad("null argument");
  if (P->batch) return bad("a batch pool is used through the instance entry points");
  cudaSetDevice(P->device);
  ffvgpu_status s;
  if ((s = require_system(P))) return s;
  if ((s = reset_state(P, 0.0, 0, nullptr))) return s;
  if ((s = ensure_stream(P))) return s;
  launch_rbgs(P->stream, P->ctx(P->bc_p), true, false, P->x[P->xcur], nullptr, P->coef, P->gx,
              0.0, P->partials, P->st, FIN_STORE, 0);
  CK(cudaGetLastError());
  SolveState h;
  if ((s = read_state(P, &h))) return s;
  *rr = h.rr;
  if (h.status == 3) {
    g_last_error = timeout_message(h.timeout_where);
    return FFVGPU_TIMEOUT;
  }
  return FFVGPU_OK;
}

ffvgpu_status ffvgpu_rbgs_sweep(ffvgpu_pool* P, double omega) {
  if (!P) return bad("null pool");
  if (P->batch) return bad("a batch pool is used through the instance entry points");
  cudaSetDevice(P->device);
  ffvgpu_status s;
  if ((s = require_system(P))) return s;
  if ((s = reset_state(P, 0.0, 0, nullptr))) return s;
  if ((s = ensure_stream(P))) return s;
  launch_rbgs(P->stream, P->ctx(P->bc_p), false, true, P->x[P->xcur], P->x[1 - P->xcur],
              P->coef, P->gx, omega, P->partials, P->st, FIN_STORE, 0);
  P->xcur = 1 - P->xcur;
  launch_exchange(P->stream, P->ctx(P->bc_p), P->x[P->xcur], P->gx);
  CK(cudaGetLastError());
  SolveState h;
  if ((s = read_state(P, &h))) return s;
  if (h.status == 3) {
    g_last_error = timeout_message(h.timeout_where);
    return FFVGPU_TIMEOUT;
  }
  return FFVGPU_OK;
}

// FFVILS::RBGS (src/FFV/FFVILS.h:547-594).  Kernel n (n >= 2) forms the
// residual of iterate n-1 and sweeps to iterate n in one pass; the residual
// of the last iterate comes from a residual-only pass.  The iterate at
// which the solve stops is kept, whichever buffer holds it.
ffvgpu_status ffvgpu_solve_rbgs(ffvgpu_pool* P, const ffvgpu_iter_params* prm,
                                ffvgpu_result* res) {
  if (!P || !prm) return bad("null argument");
  if (P->batch) return bad("a batch pool is used through the instance entry points");
  cudaSetDevice(P->device);
  ffvgpu_status s;
  if ((s = require_system(P))) return s;
  const int N = prm->count_max;
  ffvgpu_result R;
  std::memset(&R, 0, sizeof(R));
  if (N <= 0) {  // for(count=1; count<=countMax; ...) runs no pass
    R.count = 1;
    if (res) *res = R;
    return FFVGPU_OK;
  }
  if ((s = ensure_hist(P, N))) return s;
  if ((s = ensure_stream(P))) return s;
  if ((s = reset_state(P, prm->epsilon, N, P->hist_d))) return s;
  const KCtx C = P->ctx(P->bc_p);
  const int every = prm->check_every > 0 ? prm->check_every : 32;
  const bool poll = prm->epsilon > 0.0;
  CK(cudaEventRecord(P->ev0, P->stream));
  launch_dot(P->stream, C, P->b, P->b, P->partials, P->st, FIN_BB, 0);
  int launches = 1;
  int64_t bytes = interior_bytes(P, 2);
  const int c0 = P->xcur;
  launch_rbgs(P->stream, C, false, true, P->x[c0], P->x[1 - c0], P->coef, P->gx, prm->omega,
              P->partials, P->st, FIN_RBGS, 0);
  launches++;
  bytes += rbgs_pass_bytes(P, 10);
  CK(cudaEventRecord(P->ev2, P->stream));
  int swept = 0;
  // Each pass is a programmatic dependent of the pass before it (it
  // prefetches coefficients during that pass's tail), except where a host
  // poll or a timing event sits between them.
  bool polled_last = true;
  for (int n = 2; n <= N; ++n) {
    launch_rbgs(P->stream, C, true, true, P->x[(c0 + n - 1) & 1], P->x[(c0 + n) & 1], P->coef,
                nullptr, prm->omega, P->partials, P->st, FIN_RBGS, n - 1, !polled_last);
    polled_last = false;
    swept++;
    launches++;
    bytes += rbgs_pass_bytes(P, 10);
    if (poll && (n % every) == 0) {
      bool done = false;
      if ((s = poll_done(P, &done))) return s;
      polled_last = true;
      if (done) break;
    }
  }
  CK(cudaEventRecord(P->ev3, P->stream));
  launch_rbgs(P->stream, C, true, false, P->x[(c0 + N) & 1], nullptr, P->coef, nullptr,
              prm->omega, P->partials, P->st, FIN_RBGS, N, false);
  launches++;
  CK(cudaEventRecord(P->ev1, P->stream));
  CK(cudaGetLastError());
  SolveState h;
  if ((s = read_state(P, &h))) return s;
  const bool early = h.count >= 1 && h.count < N;  // stopped before the last pass
  // iterate kept: the stopping iteration's after an early stop; otherwise
  // (the solve ran to countMax, or converged on its last residual) iterate N
  const int m = early ? h.count : N;
  // passes that ran: sweeps 1..min(m+1, N), residual-only pass only at the end
  bytes = interior_bytes(P, 2) + rbgs_pass_bytes(P, 10) * (early ? (m + 1) : N) +
          (early ? 0 : rbgs_pass_bytes(P, 9));
  P->xcur = (c0 + m) & 1;
  launch_exchange(P->stream, C, P->x[P->xcur], P->gx);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(P->stream));
  float ms = 0.f, sms = 0.f;
  cudaEventElapsedTime(&ms, P->ev0, P->ev1);
  cudaEventElapsedTime(&sms, P->ev2, P->ev3);
  R.count = h.count;
  R.residual = h.residual;
  R.elapsed_ms = ms;
  R.sweep_ms = sms;
  R.sweep_launches = swept;
  R.bytes_moved = bytes;
  R.kernel_launches = launches + 1;
  R.uniform_blocks = P->ucount_h;
  if (prm->history) {
    const int nh = (h.count >= 1 && h.count <= N) ? h.count : N;
    CK(download_sync(P, prm->history, P->hist_d, sizeof(double) * nh));
  }
  if (res) *res = R;
  return solve_status(h, prm, N, R.count);
}

// FFVILS::RBGS_WithFixedAverage (src/FFV/FFVILS.h:596-659): each iteration an
// RB sweep (stored guides the first time, the in-kernel exchange after), the
// shift x += -sum(x)/ncells (CalcSum / ShiftByA, LocalScalar3D.h:130-178,
// then the exchange, made by the next kernel's gathers), and the residual of
// the shifted x.  The reference's xave argument is unused by the reference.
ffvgpu_status ffvgpu_solve_rbgs_fixed_average(ffvgpu_pool* P, const ffvgpu_iter_params* prm,
                                              int64_t ncells, ffvgpu_result* res) {
  if (!P || !prm) return bad("null argument");
  if (P->batch) return bad("a batch pool is used through the instance entry points");
  if (ncells <= 0) return bad("ncells must be positive");
  cudaSetDevice(P->device);
  ffvgpu_status s;
  if ((s = require_system(P))) return s;
  const int N = prm->count_max;
  ffvgpu_result R;
  std::memset(&R, 0, sizeof(R));
  if (N <= 0) {
    R.count = 1;
    if (res) *res = R;
    return FFVGPU_OK;
  }
  if ((s = ensure_hist(P, N)) || (s = ensure_stream(P))) return s;
  SolveState h0;
  std::memset(&h0, 0, sizeof(h0));
  h0.eps = prm->epsilon;
  h0.count_max = N;
  h0.rr0 = 1.0;
  h0.gamma = 1.0;
  h0.hist = P->hist_d;
  h0.scale = (double)ncells;
  CK(cudaMemcpyAsync(P->st, &h0, sizeof(h0), cudaMemcpyHostToDevice, P->stream));
  const KCtx C = P->ctx(P->bc_p);
  const int every = prm->check_every > 0 ? prm->check_every : 32;
  const bool poll = prm->epsilon > 0.0;
  CK(cudaEventRecord(P->ev0, P->stream));
  launch_dot(P->stream, C, P->b, P->b, P->partials, P->st, FIN_BB, 0);
  int launches = 1;
  int64_t bytes = interior_bytes(P, 2);
  const int c0 = P->xcur;
  int cur = c0;
  for (int n = 1; n <= N; ++n) {
    // once the solve has stopped these kernels return at entry: the iterate
    // kept is the one of the stopping iteration (below)
    launch_rbgs(P->stream, C, false, true, P->x[cur], P->x[1 - cur], P->coef,
                n == 1 ? P->gx : nullptr, prm->omega, P->partials, P->st, FIN_STORE, n);
    cur = 1 - cur;
    launch_sum(P->stream, C, P->x[cur], P->partials, P->st, FIN_FA_SHIFT);
    launch_shift(P->stream, C, P->x[cur], P->st);
    launch_rbgs(P->stream, C, true, false, P->x[cur], nullptr, P->coef, nullptr, prm->omega,
                P->partials, P->st, FIN_RBGS, n);
    launches += 4;
    bytes += rbgs_pass_bytes(P, 10) + interior_bytes(P, 1 + 2) + rbgs_pass_bytes(P, 9);
    if (poll && (n % every) == 0) {
      bool done = false;
      if ((s = poll_done(P, &done))) return s;
      if (done) break;
    }
  }
  CK(cudaEventRecord(P->ev1, P->stream));
  CK(cudaGetLastError());
  SolveState h;
  if ((s = read_state(P, &h))) return s;
  const int kept = (h.count >= 1 && h.count <= N) ? h.count : N;
  P->xcur = (c0 + kept) & 1;
  launch_exchange(P->stream, C, P->x[P->xcur], P->gx);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(P->stream));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, P->ev0, P->ev1);
  R.count = h.count;
  R.residual = h.residual;
  R.elapsed_ms = ms;
  R.bytes_moved = bytes;
  R.kernel_launches = launches + 1;
  if (prm->history) {
    const int nh = (h.count >= 1 && h.count <= N) ? h.count : N;
    CK(download_sync(P, prm->history, P->hist_d, sizeof(double) * nh));
  }
  if (res) *res = R;
  return solve_status(h, prm, N, R.count);
}

// FFVILS::CG (src/FFV/FFVILS.h:661-791) with Jacobi_PreConditioner
// (FFVILS.h:469-492).  Guide cells of r are never read by a stencil in the
// reference's CG, so its exchanges of r are value-neutral and not run; those
// of z and p are the in-kernel gathers of the Jacobi and A*p kernels.
ffvgpu_status ffvgpu_solve_cg(ffvgpu_pool* P, const ffvgpu_iter_params* prm,
                              ffvgpu_result* res) {
  if (!P || !prm) return bad("null argument");
  if (P->batch) return bad("a batch pool is used through the instance entry points");
  cudaSetDevice(P->device);
  ffvgpu_status s;
  if ((s = require_system(P))) return s;
  const size_t n = field_count(P);
  if ((s = dalloc_t(P, &P->r, n)) || (s = dalloc_t(P, &P->p, n)) || (s = dalloc_t(P, &P->q, n)) ||
      (s = dalloc_t(P, &P->z[0], n)) || (s = dalloc_t(P, &P->z[1], n)))
    return s;
  const int N = prm->count_max;
  ffvgpu_result R;
  std::memset(&R, 0, sizeof(R));
  if ((s = ensure_hist(P, N > 0 ? N : 1))) return s;
  if ((s = reset_state(P, prm->epsilon, N, P->hist_d))) return s;
  if ((s = ensure_kpipe(P))) return s;
  const KCtx C = P->ctx(P->bc_p);
  const int every = prm->check_every > 0 ? prm->check_every : 16;
  const bool poll = prm->epsilon > 0.0;
  double* x = P->x[P->xcur];
  CK(cudaEventRecord(P->ev0, P->stream));
  launch_dot(P->stream, C, P->b, P->b, P->partials, P->st, FIN_BB, 0);
  CK(cudaGetLastError());
  int launches = 1;
  int64_t words = 2, coef = 0;  // values moved per cell; coefficients uniform blocks skip
  SolveState h;
  if ((s = read_state(P, &h))) return s;
  if (std::fabs(h.bb) < (double)FLT_MIN) {  // FFVILS.h:686-690
    R.count = 0;
    R.residual = 0.0;
    if (res) *res = R;
    return FFVGPU_OK;
  }
  launch_calc_r(P->stream, C, x, P->gx, P->A, P->b, P->r, P->st);
  launches++;
  words += 10;
  const int K = prm->pre_count;
  int c = 1;
  if (N >= 1 && K <= 0) {
    // z stays the zero field, so r.z = 0 < FLT_MIN: count = 0 (FFVILS.h:720-724)
    R.count = 0;
    R.residual = 0.0;
    launch_exchange(P->stream, C, x, P->gx);
    CK(cudaStreamSynchronize(P->stream));
    if (res) *res = R;
    return FFVGPU_OK;
  }
  CK(cudaEventRecord(P->ev2, P->stream));
  const int launches_before = launches;
  for (c = 1; c <= N; ++c) {
    // z = Jacobi^K(0) with b = r; last pass also forms r.z
    launch_jacobi(P->stream, C, K == 1, P->z[0], P->A, P->r, prm->omega, P->partials, P->st);
    words += 9;
    coef += 7;
    launches++;
    for (int k = 2; k <= K; ++k) {
      krylov_jacobi(P, P->z[(k - 2) & 1], P->z[(k - 1) & 1], P->r, prm->omega, k == K);
      words += 10;
      coef += 7;
      launches++;
    }
    const double* z = P->z[(K - 1) & 1];
    launch_p_update(P->stream, C, z, P->p, c == 1 ? 1 : 0, P->st);
    words += c == 1 ? 2 : 3;
    krylov_matvec(P, P->p, P->q, P->p, FIN_CG_QP, false);  // x, A, w, y
    words += 10;
    coef += 7;
    launch_cg_update(P->stream, C, x, P->p, P->r, P->q, P->partials, P->st, c);
    words += 6;
    launches += 3;
    if (poll && (c % every) == 0) {
      bool done = false;
      if ((s = poll_done(P, &done))) return s;
      if (done) break;
    }
  }
  CK(cudaEventRecord(P->ev3, P->stream));
  CK(cudaEventRecord(P->ev1, P->stream));
  CK(cudaGetLastError());
  if ((s = read_state(P, &h))) return s;
  launch_exchange(P->stream, C, x, P->gx);  // FFVILS.h:790
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(P->stream));
  float ms = 0.f, sms = 0.f;
  cudaEventElapsedTime(&ms, P->ev0, P->ev1);
  cudaEventElapsedTime(&sms, P->ev2, P->ev3);
  R.sweep_ms = sms;
  R.sweep_launches = launches - launches_before;
  R.count = h.done ? h.count : (N + 1);
  R.residual = h.residual;
  R.elapsed_ms = ms;
  if ((s = krylov_bytes(P, words, coef, &R.bytes_moved))) return s;
  R.kernel_launches = launches + 1;
  if (prm->history && N > 0) {
    const int nh = (h.count >= 1 && h.count <= N) ? h.count : (h.count == 0 ? h.iter : N);
    if (nh > 0)
      CK(download_sync(P, prm->history, P->hist_d, sizeof(double) * nh));
  }
  if (res) *res = R;
  return solve_status(h, prm, N, R.count);
}


// Jacobi_PreConditioner (FFVILS.h:469-492) from z = 0 with right-hand side
// rhs: K passes through the two buffers zz; returns the buffer holding the
// result.  K = 0 leaves the zero field.
static double* jacobi_pre(ffvgpu_pool* P, const KCtx& C, double* const zz[2], const double* rhs,
                          int K, double omega, int64_t& words, int64_t& coef, int& launches) {
  if (K <= 0) {
    launch_fill(P->stream, P->nb, zz[0], BC, nullptr, 0.0);
    words += 1;
    launches++;
    return zz[0];
  }
  launch_jacobi(P->stream, C, false, zz[0], P->A, rhs, omega, P->partials, P->st);
  words += 9;
  coef += 7;
  launches++;
  for (int k = 2; k <= K; ++k) {
    krylov_jacobi(P, zz[(k - 2) & 1], zz[(k - 1) & 1], rhs, omega, false);
    words += 10;
    coef += 7;
    launches++;
  }
  return zz[(K - 1) & 1];
}

// FFVILS::BiCGSTAB (src/FFV/FFVILS.h:793-974), Jacobi-preconditioned: the
// reference's default pressure solver.  As in CG, guide cells of p and s are
// never read by a stencil (they are right-hand sides of the preconditioner
// and operands of dots), so their exchanges are value-neutral and not run;
// those of p_ and s_ are the gathers of the Jacobi and A*p kernels.
ffvgpu_status ffvgpu_solve_bicgstab(ffvgpu_pool* P, const ffvgpu_iter_params* prm,
                                    ffvgpu_result* res) {
  if (!P || !prm) return bad("null argument");
  if (P->batch) return bad("a batch pool is used through the instance entry points");
  cudaSetDevice(P->device);
  ffvgpu_status s;
  if ((s = require_system(P))) return s;
  const size_t n = field_count(P);
  if ((s = dalloc_t(P, &P->r, n)) || (s = dalloc_t(P, &P->r0, n)) || (s = dalloc_t(P, &P->p, n)) ||
      (s = dalloc_t(P, &P->q, n)) || (s = dalloc_t(P, &P->sv, n)) || (s = dalloc_t(P, &P->tv, n)) ||
      (s = dalloc_t(P, &P->z[0], n)) || (s = dalloc_t(P, &P->z[1], n)) ||
      (s = dalloc_t(P, &P->zb[0], n)) || (s = dalloc_t(P, &P->zb[1], n)))
    return s;
  const int N = prm->count_max;
  ffvgpu_result R;
  std::memset(&R, 0, sizeof(R));
  if ((s = ensure_hist(P, N > 0 ? N : 1))) return s;
  if (!(prm->restart_drop >= 0.0 && prm->restart_drop < 1.0))
    return bad("restart_drop must lie in [0, 1)");
  if ((s = reset_state(P, prm->epsilon, N, P->hist_d, prm->restart_drop))) return s;
  if ((s = ensure_kpipe(P))) return s;
  const KCtx C = P->ctx(P->bc_p);
  const int every = prm->check_every > 0 ? prm->check_every : 16;
  const bool poll = prm->epsilon > 0.0;
  double* x = P->x[P->xcur];
  CK(cudaEventRecord(P->ev0, P->stream));
  launch_dot(P->stream, C, P->b, P->b, P->partials, P->st, FIN_BB, 0);
  CK(cudaGetLastError());
  int launches = 1;
  int64_t words = 2, coef = 0;  // values moved per cell; coefficients uniform blocks skip
  SolveState h;
  if ((s = read_state(P, &h))) return s;
  if (std::fabs(h.bb) < (double)FLT_MIN) {  // FFVILS.h:822-826
    R.count = 0;
    R.residual = 0.0;
    if (res) *res = R;
    return FFVGPU_OK;
  }
  launch_calc_r(P->stream, C, x, P->gx, P->A, P->b, P->r, P->st);  // FFVILS.h:828
  // r0 = r (FFVILS.h:830-833) is made by the first DOT(r, r0) of the loop
  launches++;
  words += 10 + 2;
  const int K = prm->pre_count;
  CK(cudaEventRecord(P->ev2, P->stream));
  const int launches_before = launches;
  for (int c = 1; c <= N; ++c) {
    launch_dot_rr0(P->stream, C, P->r, P->r0, P->partials, P->st, FIN_BI_RR1, c);  // rr1
    launch_bicg_p(P->stream, C, P->r, P->p, P->q, P->st);
    const double* pz = jacobi_pre(P, C, P->z, P->p, K, prm->omega, words, coef, launches);
    krylov_matvec(P, pz, P->q, P->r0, FIN_BI_QR0, false);
    launch_axpyz(P->stream, C, P->sv, P->q, P->r, P->st);
    const double* sz = jacobi_pre(P, C, P->zb, P->sv, K, prm->omega, words, coef, launches);
    krylov_matvec(P, sz, P->tv, P->sv, FIN_BI_TS, true);  // t_.s and t_.t
    launch_bicg_update(P->stream, C, x, pz, sz, P->r, P->tv, P->sv, P->partials, P->st, c);
    launches += 6;
    // r.r0, p, two A*x (x, A, w, y), s, the update
    words += 2 + (c == 1 ? 2 : 4) + 10 + 3 + 10 + 9;
    coef += 14;
    if (poll && (c % every) == 0) {
      bool done = false;
      if ((s = poll_done(P, &done))) return s;
      if (done) break;
    }
  }
  CK(cudaEventRecord(P->ev3, P->stream));
  CK(cudaEventRecord(P->ev1, P->stream));
  CK(cudaGetLastError());
  if ((s = read_state(P, &h))) return s;
  launch_exchange(P->stream, C, x, P->gx);  // FFVILS.h:973
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(P->stream));
  float ms = 0.f, sms = 0.f;
  cudaEventElapsedTime(&ms, P->ev0, P->ev1);
  cudaEventElapsedTime(&sms, P->ev2, P->ev3);
  R.sweep_ms = sms;
  R.sweep_launches = launches - launches_before;
  R.count = h.done ? h.count : (N + 1);
  R.residual = h.residual;
  R.elapsed_ms = ms;
  if ((s = krylov_bytes(P, words, coef, &R.bytes_moved))) return s;
  R.kernel_launches = launches + 1;
  if (prm->history && N > 0) {
    const int nh = (h.count >= 1 && h.count <= N) ? h.count : (h.count == 0 ? h.iter : N);
    if (nh > 0)
      CK(download_sync(P, prm->history, P->hist_d, sizeof(double) * nh));
  }
  if (res) *res = R;
  return solve_status(h, prm, N, R.count);
}

}  // extern "C"

// ---- pieces of a sharded solve (ffvgpu_shard_*): one pass over a shard's
// own blocks, per-block partial sums, the device address of the iterate ----

ffvgpu_status ffvgpu_rbgs_pass(ffvgpu_pool* P, int32_t blocks, int32_t residual, int32_t sweep,
                               int32_t stored, double omega, double* partials) {
  if (!P) return bad("null pool");
  if (P->batch) return bad("a batch pool is used through the instance entry points");
  if (blocks < 1 || blocks > P->nb) return bad("blocks must lie in [1, pool blocks]");
  const bool res = residual != 0, swp = sweep != 0, st = stored != 0;
  if (!((!res && swp && st) || (res && swp && !st) || (res && !swp && !st)))
    return bad("pass kinds: first sweep (stored guides), residual + sweep, residual");
  if (res && !partials) return bad("null partials");
  cudaSetDevice(P->device);
  ffvgpu_status s;
  if ((s = require_system(P))) return s;
  if ((s = ensure_stream(P))) return s;
  if ((s = reset_state(P, 0.0, 0, nullptr))) return s;
  KCtx C = P->ctx(P->bc_p);
  C.nb = blocks;
  const int c = P->xcur;
  launch_rbgs(P->stream, C, res, swp, P->x[c], swp ? P->x[1 - c] : nullptr, P->coef,
              st ? P->gx : nullptr, omega, P->partials, P->st, FIN_STORE, 0);
  CK(cudaGetLastError());
  if (swp) P->xcur = 1 - c;
  SolveState h;
  if ((s = read_state(P, &h))) return s;
  if (h.status == 3) {
    g_last_error = timeout_message(h.timeout_where);
    return FFVGPU_TIMEOUT;
  }
  if (res) CK(download_sync(P, partials, P->partials, sizeof(double) * blocks));
  return FFVGPU_OK;
}

ffvgpu_status ffvgpu_block_dots(ffvgpu_pool* P, ffvgpu_field fx, ffvgpu_field fy, int32_t blocks,
                                double* partials) {
  if (!P || !partials) return bad("null argument");
  if (P->batch) return bad("a batch pool is used through the instance entry points");
  if (blocks < 1 || blocks > P->nb) return bad("blocks must lie in [1, pool blocks]");
  cudaSetDevice(P->device);
  double *x, *y, *g;
  size_t sx, sy;
  ffvgpu_status s;
  if ((s = field_ptr(P, fx, false, &x, &sx, &g)) || (s = field_ptr(P, fy, false, &y, &sy, &g)))
    return s;
  if (sx != BC || sy != BC) return bad("dot of matrix fields is not supported");
  if ((s = reset_state(P, 0.0, 0, nullptr))) return s;
  KCtx C = P->ctx(P->bc_p);
  C.nb = blocks;
  launch_dot(P->stream, C, x, y, P->partials, P->st, FIN_STORE, 0);
  CK(cudaGetLastError());
  return download_sync(P, partials, P->partials, sizeof(double) * blocks) == cudaSuccess
             ? FFVGPU_OK
             : cuda_fail(cudaGetLastError(), "block_dots");
}

ffvgpu_status ffvgpu_pool_field_device(ffvgpu_pool* P, ffvgpu_field f, void** ptr) {
  if (!P || !ptr) return bad("null argument");
  if (f != FFVGPU_FIELD_X && f != FFVGPU_FIELD_B) return bad("only X and B are exposed");
  double *x, *g;
  size_t stride;
  ffvgpu_status s;
  if ((s = field_ptr(P, f, false, &x, &stride, &g))) return s;
  if (!x) return bad("field not allocated");
  *ptr = x;
  return FFVGPU_OK;
}
