// pool_internal.h -- the device block pool shared by the host-side sources
// of the library (pool.cpp: fields and the FFVILS-form solves; instances.cpp:
// batches of independent problems and the mixed-precision form).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/ffvgpu.h"
#include "ffvgpu_kernels.h"
#include "ffvgpu_layout.h"

namespace ffvgpu {
namespace detail {

inline thread_local std::string g_last_error;

inline ffvgpu_status cuda_fail(cudaError_t e, const char* what) {
  g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
  return e == cudaErrorMemoryAllocation ? FFVGPU_OOM : FFVGPU_CUDA_ERROR;
}

inline ffvgpu_status bad(const char* why) {
  g_last_error = why;
  return FFVGPU_BAD_ARG;
}

// Message of a solve that a bounded device wait ended: which roles gave up
// (SolveState::timeout_where bits).
inline std::string timeout_message(int where) {
  std::string m = "a bounded device wait gave up (";
  const char* names[] = {"producer", "gatherer", "consumer", "sweep", "drain", "A*x"};
  bool any = false;
  for (int b = 0; b < 6; ++b)
    if (where & (1 << b)) {
      m += any ? ", " : "";
      m += names[b];
      any = true;
    }
  m += any ? ")" : "no role recorded)";
  if (where & 16) m += "; a copy into shared memory was still in flight when its CTA exited";
  return m;
}

constexpr size_t BC = BLOCK_CELLS;

}  // namespace detail
}  // namespace ffvgpu

#define CK(call)                                                        \
  do {                                                                  \
    cudaError_t e_ = (call);                                            \
    if (e_ != cudaSuccess) return ffvgpu::detail::cuda_fail(e_, #call); \
  } while (0)

// One admitted problem of a pool.
struct ffvgpu_instance {
  bool used = false;     // admitted
  bool running = false;  // a mixed solve has begun and its end is not yet reported
  int32_t first = 0, count = 0;
  int32_t count_max = 0;
  double epsilon = 0.0;
  int32_t status = 0;  // of the last solve: 0 ok, 2 NaN/Inf residual, 3 a device wait gave up
  int32_t timeout_where = 0;  // roles whose wait gave up (SolveState::timeout_where)
  int32_t last_iter = 0;  // iterations with a residual before an early exit
  int32_t ublocks = 0;    // blocks with the same coefficients in every cell (known after a poll)
  ffvgpu_result result{};
  ffvgpu_grid_desc desc{};  // level / block_index point into the vectors below
  std::vector<int32_t> level, index;
};

struct ffvgpu_pool {
  int device = 0;
  int nb = 0;  // blocks (a batch pool: its capacity)
  cudaStream_t stream = nullptr;      // where work is enqueued
  cudaStream_t own_stream = nullptr;  // the pool's own stream
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr, ev3 = nullptr;
  std::vector<int32_t> level, index;
  std::vector<ffvgpu::FaceNbr> nbr_h;
  std::vector<double> dx_h;
  ffvgpu::FaceNbr* nbr_d = nullptr;
  double* dx_d = nullptr;
  ffvgpu::BCSet bc_p;  // pressure BCs
  ffvgpu::BCSet bc_u[3];
  int64_t bytes = 0;
  uint64_t wait_ns = ffvgpu::DEFAULT_WAIT_NS;  // limit of every bounded device wait

  // fields (device, colour-split interiors)
  double* x[2] = {nullptr, nullptr};
  int xcur = 0;
  double* gx = nullptr;  // stored first guide layer of x
  double* A = nullptr;   // [nb][7][4096]
  double* coef = nullptr;         // sweep coefficient stream [nb][STREAM_BLOCK]
  double* urec = nullptr;         // [nb][8] uniform records of the stream (launch_pack_stream)
  int32_t* ucount_d = nullptr;    // uniform blocks of the stream
  int32_t ucount_h = 0;           // the same, read after each repack
  int64_t sys_version = 1;        // bumped whenever A or b change
  int64_t stream_version = 0;     // sys_version the stream was packed from
  int64_t urec_version = 0;       // sys_version the uniform records come from
  int64_t ucount_version = 0;     // sys_version ucount_h was read back for
  double* b = nullptr;
  double* u[3] = {nullptr, nullptr, nullptr};
  double* gu[3] = {nullptr, nullptr, nullptr};
  double* cut = nullptr;    // [6][nb*4096]
  double* vface = nullptr;  // [6][nb*4096]
  double* lapp = nullptr;   // Laplacian of p (bcut_corr_u)
  uint8_t* flags = nullptr; // bits 0..5 cut ids, bit 7 fluid
  double* r = nullptr;
  double* p = nullptr;
  double* q = nullptr;
  double* z[2] = {nullptr, nullptr};
  double* r0 = nullptr;            // BiCGSTAB shadow residual
  double* sv = nullptr;            // BiCGSTAB s
  double* tv = nullptr;            // BiCGSTAB t_
  double* zb[2] = {nullptr, nullptr};  // BiCGSTAB s_ (Jacobi iterates)
  double* partials = nullptr;
  ffvgpu::SolveState* st = nullptr;
  double* hist_d = nullptr;
  int hist_cap = 0;
  void* stage = nullptr;
  size_t stage_bytes = 0;
  int32_t* host_done = nullptr;  // pinned
  // the FP64 solvers' pipelined A*x: the pool as one instance.  kpipe:
  // [1 + nb] the block list (count, then the blocks that stream their
  // coefficients first), [nb] instance of each block (0), then first (0) and
  // count (nb); kraw: the list in block order; kpart: [2][nb] per-block sums
  int32_t* kpipe = nullptr;
  int32_t* kraw = nullptr;
  double* kpart = nullptr;
  int64_t kpipe_version = 0;  // sys_version the list was ordered for
  bool kpipe_ready = false;   // all three allocated and the tables uploaded

  // instances: a pool made from one grid is instance 0 over every block; a
  // batch pool admits and releases instances over its block capacity
  bool batch = false;
  std::vector<ffvgpu_instance> inst;
  std::vector<int32_t> blk_inst_h;  // [nb], -1 for a free block
  int32_t* blk_inst_d = nullptr;
  int32_t* inst_first_d = nullptr;
  int32_t* inst_count_d = nullptr;
  int32_t* blk_geo_d = nullptr;      // [nb][4]: level, index x, y, z (device generator)
  ffvgpu::SolveState* mst = nullptr;  // [instances]
  ffvgpu::SolveState* mst_h = nullptr;  // pinned copy for polls
  double* mpartials = nullptr;       // [2][nb]
  double* mhist = nullptr;           // [instances][mhist_cap]
  int mhist_cap = 0;
  bool inst_dirty = true;            // host tables changed since the last upload

  // mixed form
  uint32_t* mcoef = nullptr;  // [nb][7][4096] 32-bit sweep coefficients (FP64 high words)
  double* mguide = nullptr;   // [nb][6][256] guide layer of the sweep iterate between passes
  double* mucoef = nullptr;   // [nb][8] per-block coefficients of uniform blocks (MixCtx::ucoef)
  float* me[2] = {nullptr, nullptr};
  float* mph = nullptr;     // preconditioned p (p_)
  float* msh = nullptr;     // preconditioned s (s_)
  // the FP64-data variant (ffvgpu_mixed_params.fp64_data): FP64 coefficients
  // in the sweep's thread order, FP64 iterate and preconditioned vectors
  double* mcoef64 = nullptr;  // [nb][7][4096]
  double* me64[2] = {nullptr, nullptr};
  double* mph64 = nullptr;
  double* msh64 = nullptr;
  int64_t mcoef_version = 0;  // sys_version the sweep coefficients come from (one-grid pools)
  double m_omega = 0.0;
  int m_sweeps = 0, m_per_exchange = 0;
  int m_cf = 0;   // coarse-fine flux correction of the running solves
  int m_d64 = 0;  // the running solves use the FP64-data variant
  int m_depth = 1;  // sweep kernel staging depth (L2 prefetch distance in blocks)
  int m_threads = 256;  // CTA size of the update kernel (and of the A*x kernel in form 1)
  int m_sweep_threads = 256;  // CTA size of the sweep kernel
  int m_mvform = 0;           // A*x kernel: 0 pipelined, 1 a block per CTA
  cudaGraphExec_t mgraph = nullptr;
  int mgraph_iters = 0;
  double mgraph_omega = 0.0;
  int mgraph_sweeps = 0, mgraph_per = 0;
  uint64_t mgraph_wait_ns = 0;
  int mgraph_stall = 0;
  int mgraph_cap = 0;
  int mgraph_cf = 0;
  int mgraph_d64 = 0;
  int mgraph_depth = 0, mgraph_threads = 0, mgraph_sweep_threads = 0, mgraph_mvform = -1;
  int stall_sweep = 0;  // test hook: 1 sweep, 2 A*x (ffvgpu_pool_stall_next_solve / _matvec),
                        // cleared when a solve ends
  int64_t m_launches = 0;
  int64_t m_bytes = 0;
  // active-block list of the persistent kernels: device [1 + capacity]
  // (count, then block ids), refilled from two pinned staging buffers
  int32_t* act_d = nullptr;
  int32_t* act_raw_d = nullptr;  // the host list as uploaded, before mx_order_active
  int32_t* act_h[2] = {nullptr, nullptr};
  cudaEvent_t act_ev[2] = {nullptr, nullptr};
  int act_next = 0;
  int grid_sweep = 0, grid_matvec = 0, grid_update = 0, grid_guides = 0, grid_mvpipe = 0;
  int grid_cap = 0;  // test hook: at most this many CTAs per persistent grid (0: none)
  int grid_threads = 0;  // m_threads the grid sizes were computed for

  ffvgpu::KCtx ctx(const ffvgpu::BCSet& bc) const {
    ffvgpu::KCtx C;
    C.nbr = nbr_d;
    C.dx = dx_d;
    C.bc = bc;
    C.nb = nb;
    C.first = 0;
    C.wait_ns = wait_ns;
    C.urec = (urec && urec_version == sys_version) ? urec : nullptr;
    return C;
  }
};

namespace ffvgpu {
namespace detail {

ffvgpu_status dalloc(ffvgpu_pool* P, void** ptr, size_t bytes);
// Copies between host and device ordered on the pool's stream.  The pool's
// stream is non-blocking, so it does not wait for the legacy default stream:
// a plain cudaMemcpy from pageable memory may return before its data reaches
// the device, and a kernel enqueued next on the pool's stream could read the
// old contents.  Pageable sources are staged before upload() returns.
inline cudaError_t upload(ffvgpu_pool* P, void* dst, const void* src, size_t bytes) {
  return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, P->stream);
}
// Waits for the pool's stream, so the copy sees all work enqueued before it.
inline cudaError_t download_sync(ffvgpu_pool* P, void* dst, const void* src, size_t bytes) {
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, P->stream);
  return e != cudaSuccess ? e : cudaStreamSynchronize(P->stream);
}
template <class T>
ffvgpu_status dalloc_t(ffvgpu_pool* P, T** ptr, size_t count) {
  return dalloc(P, reinterpret_cast<void**>(ptr), count * sizeof(T));
}
ffvgpu_status ensure_stage(ffvgpu_pool* P, size_t bytes);
// The values of a host buffer (bytes long) as the pack kernel reads them: the
// buffer itself when it is pinned host memory the device can address (the
// kernel then reads across the link only what it packs), else a staging copy
// in device memory.
ffvgpu_status host_source(ffvgpu_pool* P, const void* host, size_t bytes, const double** src);
size_t field_count(const ffvgpu_pool* P);
ffvgpu_status field_ptr(ffvgpu_pool* P, int f, bool alloc, double** ptr, size_t* stride,
                        double** guides);
const BCSet& field_bc(const ffvgpu_pool* P, int f);
ffvgpu_status derive_neighbors(int nb, const int32_t* level, const int32_t* index,
                               const ffvgpu_grid_desc* d, std::vector<FaceNbr>& out);
ffvgpu_status pool_init_device(ffvgpu_pool* P);
void release_instances(ffvgpu_pool* P);

}  // namespace detail
}  // namespace ffvgpu
