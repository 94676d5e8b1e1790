// rbgs_pipelined.cu -- persistent, TMA-pipelined fused residual + red-black
// sweep for sm_100a (the hot kernel of FFVILS::RBGS).
//
// Per pass over the pool it computes, for every leaf block, the residual
// sum of x_in (calc_r2, src/CGMfuncs/bils.f90:256-304) and the red-black
// SOR sweep x_in -> x_out (rbgs_smoother, bils.f90:57-108, colour 0 then
// colour 1 against guide values from the previous exchange), with the same
// rounding as the reference (compiled with --fmad=false) and the same sum
// tree as the rest of the path.
//
// One CTA per SM walks blocks blockIdx.x, blockIdx.x + gridDim.x, ...  Its
// warps have fixed roles:
//   warp 0      producer: one lane issues cp.async.bulk copies (global ->
//               shared, completion on mbarriers): each block's x (32 KB, the
//               colour-split layout of HBM, copied as is) into one of two
//               tile buffers a block ahead, and the coefficient stream -- for
//               each colour and each four z planes, the 512 cells' Ap..At
//               and b, stored contiguously (32 KB) by pack_stream_kernel --
//               one copy per slot of a STAGES ring;
//   warps 1-8   gatherers: the guide layer of the block after the current
//               one (the in-kernel exchange, computed from the neighbours'
//               interiors of x_in) into one of two guide buffers;
//   warps 9-24  consumers (512 threads, one cell each per slot): the
//               colour-0 pass (residual, and
//               the update kept in a colour-0 buffer and streamed to x_out),
//               then the colour-1 pass (residual against the old colour-0
//               values, update against the new), and the residual sum.
// Stencil neighbours are read straight from the colour-split tile: every
// neighbour of a cell of one colour lies in the other colour's half, and
// cells on the block surface take the guide buffer instead.
// Every wait on an mbarrier is bounded in time (KCtx::wait_ns); a wait that
// gives up raises the CTA's abort flag, every role leaves its loop, the
// producer waits for the copies it has in flight to land (bounded by
// DRAIN_NS, independently of the wait limit; a drain that gives up is
// reported as ROLE_DRAIN), and the solver state reports TIMEOUT.
#include <cfloat>
#include <cstddef>
#include <cstdint>
#include <mutex>
#include <cuda_runtime.h>

#include "ffvgpu_async.cuh"
#include "ffvgpu_internal.cuh"
#include "ffvgpu_kernels.h"

namespace ffvgpu {

namespace pipe {

constexpr int CPT = 2;               // stream chunks per slot (512 cells)
constexpr int STAGES = 3;
constexpr int NARR = 8;              // Ap, Aw, Ae, As, An, Ab, At, b
constexpr int SUB_CELLS = 256;       // cells of one stream chunk (one colour, two z planes)
constexpr int SLOT_BYTES = CPT * NARR * SUB_CELLS * 8;
constexpr int SLOTS = 16 / CPT;      // slots per block (SLOTS / 2 per colour)
constexpr int X_ISSUE_AT = SLOTS / 2;  // slot of block m after which x(m+1) is issued
constexpr int PRODUCER_WARPS = 1, GATHER_WARPS = 8, CONSUMER_WARPS = 16;
constexpr int GATHER0 = 32 * PRODUCER_WARPS;
constexpr int CONS0 = GATHER0 + 32 * GATHER_WARPS;
constexpr int NTHREADS = CONS0 + 32 * CONSUMER_WARPS;  // 800
constexpr int NCONS = 32 * CONSUMER_WARPS;            // one cell per consumer per slot
constexpr int NGATHER = 32 * GATHER_WARPS;
enum { ROLE_PRODUCER = 1, ROLE_GATHER = 2, ROLE_CONSUMER = 4 };
// Uniform flags of a CTA's first 32 UMASK_WORDS blocks are kept in shared
// memory; later blocks (pools of more than 148 x 1024 blocks) stream all
// their coefficients, which gives the same results.
constexpr int UMASK_WORDS = 32;
constexpr uint32_t B_ROW_BYTES = SUB_CELLS * 8;  // b of one stream chunk

struct __align__(128) Smem {
  double ring[STAGES][CPT][NARR][SUB_CELLS];  // 96 KB
  double xt[2][BLOCK_CELLS];               // 64 KB: x_in of the current / next block
  double xnew0[HALF_CELLS];                // 16 KB: updated colour-0 values
  double gbuf[2][6 * FACE_CELLS];          // 24 KB: guide layers, [face][v][u]
  uint64_t full[STAGES], empty[STAGES];
  uint64_t xfull[2], xempty[2], gfull[2], gempty[2];
  double urec[2][8];                       // the uniform record of the block in xt[]
  uint32_t umask[UMASK_WORDS];             // uniform flags of this CTA's blocks
  double ws[CONSUMER_WARPS];
  int abort_flag;
  int last;
};

using namespace async;

// The coefficients of one cell, read from a ring slot.
struct Coef {
  double ap, aw, ae, as, an, ab, at, b;
};
__device__ __forceinline__ Coef load_coef(const double (*slot)[SUB_CELLS], int t) {
  Coef c;
  c.ap = slot[0][t]; c.aw = slot[1][t]; c.ae = slot[2][t]; c.as = slot[3][t];
  c.an = slot[4][t]; c.ab = slot[5][t]; c.at = slot[6][t]; c.b = slot[7][t];
  return c;
}
__device__ __forceinline__ void hold(const Coef& c) {
  asm volatile("" ::"d"(c.ap), "d"(c.aw), "d"(c.ae), "d"(c.as), "d"(c.an), "d"(c.ab), "d"(c.at),
               "d"(c.b));
}
// Hands a ring slot back to the producer: each thread has waited for its
// loads of the slot to land in registers (hold), fences them; one lane per
// warp arrives.
__device__ __forceinline__ void release_slot(uint64_t* bar, int lane, bool live) {
  fence_proxy_async();
  __syncwarp();
  if (lane == 0 && live) mbar_arrive(bar);
}
__device__ __forceinline__ void consumer_sync() {
  asm volatile("bar.sync 1, %0;" ::"n"(32 * CONSUMER_WARPS) : "memory");
}

}  // namespace pipe

template <bool DO_RES, bool DO_SWEEP>
__global__ void __launch_bounds__(pipe::NTHREADS, 1)
rbgs_pipelined_kernel(KCtx C, const double* __restrict__ xin, double* __restrict__ xout,
                      const double* __restrict__ stream, const double* __restrict__ gst,
                      double omega,
                      double* __restrict__ partials, SolveState* st, int fin, int iter) {
  using namespace pipe;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  Smem& S = *reinterpret_cast<Smem*>(smem_raw);
  const int tid = threadIdx.x;
  const int nb = C.nb;
  volatile int* abort_flag = &S.abort_flag;

  if (tid < UMASK_WORDS) S.umask[tid] = 0;
  __syncthreads();
  // uniform blocks (launch_pack_stream's records, written before this pass's
  // dependency): their slots bring b only and their seven coefficients come
  // with x
  if (C.urec) {
    const int mine = (blockIdx.x < nb) ? (nb - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
    for (int k = tid; k < mine && k < 32 * UMASK_WORDS; k += NTHREADS)
      if (C.urec[(size_t)(blockIdx.x + k * gridDim.x) * 8 + 7] != 0.0)
        atomicOr(&S.umask[k >> 5], 1u << (k & 31));
  }
  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&S.full[s], 1);
      mbar_init(&S.empty[s], CONSUMER_WARPS);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&S.xfull[b], 1);
      mbar_init(&S.xempty[b], 1);
      mbar_init(&S.gfull[b], NGATHER);
      mbar_init(&S.gempty[b], 1);
    }
    S.abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    fence_proxy_async();
    // the next pass may start its prologue as soon as SMs free up
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  }
  __syncthreads();
  const int myblocks = (blockIdx.x < nb) ? (nb - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  const int total_slots = myblocks * SLOTS;
  // is this CTA's m-th block uniform
  auto uniform = [&](int m) {
    return m < 32 * UMASK_WORDS && ((S.umask[m >> 5] >> (m & 31)) & 1u);
  };

  if (tid < GATHER0) {
    // ------------------------------------------------------------ producer
    if (tid == 0) {
      uint32_t g = 0;            // slots issued
      uint32_t nx[2] = {0, 0};   // x copies issued per tile buffer
      bool ok = true;
      // The coefficient stream does not depend on the previous pass: the
      // first STAGES slots are issued before waiting for it.
      auto issue_slot = [&](uint32_t gg) {
        const int s = gg % STAGES;
        const int m = (int)(gg / SLOTS);
        const int blk = blockIdx.x + m * gridDim.x;
        const int j = gg % SLOTS;
        // slot j: stream chunks CPT*j .. CPT*j+CPT-1 (colour = j / (SLOTS/2))
        const double* src = stream + (size_t)blk * STREAM_BLOCK + (size_t)j * CPT * STREAM_CHUNK;
        if (uniform(m)) {  // b of each chunk into its row of the slot
          mbar_expect_tx(&S.full[s], CPT * B_ROW_BYTES);
          for (int c = 0; c < CPT; ++c)
            bulk_g2s(S.ring[s][c][NARR - 1], src + (size_t)c * STREAM_CHUNK + 7 * SUB_CELLS,
                     B_ROW_BYTES, &S.full[s]);
        } else {
          mbar_expect_tx(&S.full[s], SLOT_BYTES);
          bulk_g2s(S.ring[s], src, SLOT_BYTES, &S.full[s]);
        }
      };
      // x of the CTA's m-th block into tile buffer xb, with its uniform
      // record when it has one
      auto issue_x = [&](int m, int xb) {
        const int blk = blockIdx.x + m * gridDim.x;
        const bool u = uniform(m);
        mbar_expect_tx(&S.xfull[xb], BLOCK_CELLS * 8 + (u ? 64u : 0u));
        bulk_g2s(S.xt[xb], xin + (size_t)blk * BLOCK_CELLS, BLOCK_CELLS * 8, &S.xfull[xb]);
        if (u) bulk_g2s(S.urec[xb], C.urec + (size_t)blk * 8, 64, &S.xfull[xb]);
      };
      for (; g < (uint32_t)STAGES && g < (uint32_t)total_slots; ++g) issue_slot(g);
      asm volatile("griddepcontrol.wait;" ::: "memory");
      const bool skip = *((volatile const int32_t*)&st->done) != 0;
      if (!skip && myblocks > 0) {
        ++nx[0];
        issue_x(0, 0);
      }
      for (; !skip && ok && g < (uint32_t)total_slots; ++g) {
        const int s = g % STAGES;
        const uint32_t u = g / STAGES;
        if (!(ok = mbar_wait(&S.empty[s], (u & 1) ^ 1, abort_flag, ROLE_PRODUCER, C.wait_ns)))
          break;
        issue_slot(g);
        const int m = g / SLOTS, j = g % SLOTS;
        const int blk = blockIdx.x + m * gridDim.x;
        if (j == X_ISSUE_AT && blk + (int)gridDim.x < nb) {
          // x of block m+1 into the buffer block m-1 used (released by now:
          // the consumers are in block m)
          const int xb = (m + 1) & 1;
          if (m >= 1 &&
              !(ok = mbar_wait(&S.xempty[xb], ((m - 1) >> 1) & 1, abort_flag, ROLE_PRODUCER,
                               C.wait_ns)))
            break;
          ++nx[xb];
          issue_x(m + 1, xb);
        }
      }
      // Drain: the last armed phase of every barrier a copy completes on must
      // complete before the CTA may exit (copies land in its shared memory).
      // Each barrier has at most one copy in flight (a slot or tile buffer is
      // refilled only after the consumers released it, which they do after
      // its copy landed), so the last armed phase completing means every
      // copy on it has landed.
      bool drained = true;
      for (int s = 0; s < STAGES; ++s) {
        const uint32_t issued = (g > (uint32_t)s) ? (g - 1 - s) / STAGES + 1 : 0;
        if (issued) drained = mbar_drain(&S.full[s], (issued - 1) & 1) && drained;
      }
      for (int b = 0; b < 2; ++b)
        if (nx[b]) drained = mbar_drain(&S.xfull[b], (nx[b] - 1) & 1) && drained;
      if (!drained) atomicOr((int*)abort_flag, ROLE_DRAIN);
    } else {
      asm volatile("griddepcontrol.wait;" ::: "memory");
    }
  } else if (tid < CONS0) {
    // ----------------------------------------------------------- gatherers
    asm volatile("griddepcontrol.wait;" ::: "memory");
    const int gt = tid - GATHER0;
    const int grp = gt >> 7, p0 = gt & 127, p1 = p0 + 128;
    int m = 0;
    const bool skip = *((volatile const int32_t*)&st->done) != 0;
    for (int blk = blockIdx.x; !skip && blk < nb; blk += gridDim.x, ++m) {
      const int gb = m & 1;
      if (m >= 2 &&
          !mbar_wait(&S.gempty[gb], ((m - 2) >> 1) & 1, abort_flag, ROLE_GATHER, C.wait_ns))
        break;
      const double dx = C.dx[blk];
      // two groups of 128 threads take alternate faces; each thread resolves
      // two positions of its face with all their loads in flight
      for (int r = 0; r < 3; ++r) {
        const int f = 2 * r + grp;
        double v0, v1;
        if (gst) {
          const double* gs = gst + ((size_t)blk * 6 + f) * FACE_CELLS;
          v0 = __ldg(gs + p0);
          v1 = __ldg(gs + p1);
        } else {
          const FaceNbr nbf = C.nbr[blk * 6 + f];
          guide_pair(xin, blk, f, p0, p1, nbf, C.bc, dx, v0, v1);
        }
        S.gbuf[gb][f * FACE_CELLS + p0] = v0;
        S.gbuf[gb][f * FACE_CELLS + p1] = v1;
      }
      mbar_arrive(&S.gfull[gb]);
    }
  } else {
    // ----------------------------------------------------------- consumers
    // Every consumer executes the same sequence of named barriers, warp
    // syncs and shuffles whatever happens; only the work is predicated on
    // 'live', which drops when a wait gives up.
    asm volatile("griddepcontrol.wait;" ::: "memory");
    const int ct = tid - CONS0;
    const int lane = ct & 31, warp = ct >> 5;
    uint32_t g = 0;
    int m = 0;
    bool live = true;
    const bool skip = *((volatile const int32_t*)&st->done) != 0;
    for (int blk = blockIdx.x; !skip && blk < nb; blk += gridDim.x, ++m) {
      const int xb = m & 1;
      const uint32_t par = (m >> 1) & 1;
      live = live && mbar_wait(&S.xfull[xb], par, abort_flag, ROLE_CONSUMER, C.wait_ns);
      live = live && mbar_wait(&S.gfull[xb], par, abort_flag, ROLE_CONSUMER, C.wait_ns);
      const double* T = S.xt[xb];
      const double* G = S.gbuf[xb];
      double* xo = xout + (size_t)blk * BLOCK_CELLS;
      double acc[2] = {0.0, 0.0};
      // a uniform block: the seven coefficients of every cell, from its record
      const bool uni = uniform(m);
      Coef cu;
      cu.ap = S.urec[xb][0]; cu.aw = S.urec[xb][1]; cu.ae = S.urec[xb][2]; cu.as = S.urec[xb][3];
      cu.an = S.urec[xb][4]; cu.ab = S.urec[xb][5]; cu.at = S.urec[xb][6]; cu.b = 0.0;
      // colour 0: neighbours are colour 1 (unchanged).  Consumer ct takes the
      // cell q = mm*512 + ct of every slot (stream chunk ct >> 8 of the slot).
      const int h = ct >> 8, t = ct & 255;
      for (int mm = 0; mm < SLOTS / 2; ++mm, ++g) {
        const int s = g % STAGES;
        live = live && mbar_wait(&S.full[s], (g / STAGES) & 1, abort_flag, ROLE_CONSUMER,
                                 C.wait_ns);
        Coef c = {1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        if (live && uni) {
          c = cu;
          c.b = S.ring[s][h][NARR - 1][t];
        } else if (live) {
          c = load_coef(S.ring[s][h], t);
        }
        hold(c);
        release_slot(&S.empty[s], lane, live);
        if (!live) continue;
        const int q = mm * NCONS + ct;
        const Nbrs v = split_neighbours(T + HALF_CELLS, G, q, 0);
        const double rs = c.b - c.aw * v.w - c.ae * v.e - c.as * v.s - c.an * v.n - c.ab * v.b -
                          c.at * v.t;
        const double xp = T[q];
        if (DO_RES) {
          const double r = rs - c.ap * xp;
          acc[0] += r * r;
        }
        if (DO_SWEEP) {
          const double xt = rs / c.ap;
          const double xn = xp - omega * (xp - xt);
          S.xnew0[q] = xn;
          xo[q] = xn;
        }
      }
      consumer_sync();
      // colour 1: residual against the old colour-0 values, update against the new
      for (int mm = 0; mm < SLOTS / 2; ++mm, ++g) {
        const int s = g % STAGES;
        live = live && mbar_wait(&S.full[s], (g / STAGES) & 1, abort_flag, ROLE_CONSUMER,
                                 C.wait_ns);
        Coef c = {1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        if (live && uni) {
          c = cu;
          c.b = S.ring[s][h][NARR - 1][t];
        } else if (live) {
          c = load_coef(S.ring[s][h], t);
        }
        hold(c);
        release_slot(&S.empty[s], lane, live);
        if (!live) continue;
        const int q = mm * NCONS + ct;
        const double xp = T[HALF_CELLS + q];
        if (DO_RES) {
          const Nbrs v = split_neighbours(T, G, q, 1);
          const double r = c.b - c.aw * v.w - c.ae * v.e - c.as * v.s - c.an * v.n - c.ab * v.b -
                           c.at * v.t - c.ap * xp;
          acc[1] += r * r;
        }
        if (DO_SWEEP) {
          const Nbrs v = split_neighbours(S.xnew0, G, q, 1);
          const double rs = c.b - c.aw * v.w - c.ae * v.e - c.as * v.s - c.an * v.n - c.ab * v.b -
                            c.at * v.t;
          const double xt = rs / c.ap;
          xo[HALF_CELLS + q] = xp - omega * (xp - xt);
        }
      }
      if (DO_RES) {
        // block tree: virtual thread ct (512 per block), butterfly per warp,
        // warp sums in order
        double v = acc[0] + acc[1];
#pragma unroll
        for (int off = 16; off >= 1; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
        if (lane == 0) S.ws[warp] = v;
        consumer_sync();
        if (ct == 0 && live) {
          double sum = 0.0;
#pragma unroll
          for (int w = 0; w < CONSUMER_WARPS; ++w) sum += S.ws[w];
          __stcg(partials + blk, sum);
        }
      }
      // the tile is refilled by TMA and the guide buffer by the gatherers
      fence_proxy_async();
      consumer_sync();
      if (ct == 0 && live) {
        mbar_arrive(&S.xempty[xb]);
        mbar_arrive(&S.gempty[xb]);
      }
    }
  }

  __syncthreads();
  if (*((volatile const int32_t*)&st->done) != 0 && !*abort_flag) return;
  if (*abort_flag) {
    if (tid == 0) {
      atomicOr(&st->timeout_where, *abort_flag);
      atomicExch(&st->status, 3);
      atomicExch(&st->done, 1);
    }
    return;
  }
  if (!DO_RES) return;
  if (tid == CONS0) {
    __threadfence();
    const unsigned t = atomicAdd(&st->ticket, 1u);
    S.last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!S.last || tid < CONS0) return;
  __threadfence();
  // cross-block tree: 256 threads over the partials, butterfly, 8 warp sums
  const int ct = tid - CONS0;
  double Ssum = 0.0;
  if (ct < 256)
    for (int b = ct; b < nb; b += 256) Ssum += __ldcg(partials + b);
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1) Ssum += __shfl_xor_sync(0xffffffffu, Ssum, off);
  if ((ct & 31) == 0 && ct < 256) S.ws[ct >> 5] = Ssum;
  consumer_sync();
  if (ct == 0) {
    double total = 0.0;
#pragma unroll
    for (int w = 0; w < 8; ++w) total += S.ws[w];
    finalize(st, total, fin, iter);
    st->ticket = 0;
    __threadfence();
  }
}

namespace {
// Per-device launch data: SM count (grid size) and whether the dynamic
// shared-memory limit of each instantiation has been raised on that device
// (cudaFuncSetAttribute applies to the current device only).
constexpr int MAX_DEVICES = 64;
struct DeviceCache {
  int sm_count = 0;
  bool attr_set[3] = {false, false, false};
};
std::mutex g_cache_mu;
DeviceCache g_cache[MAX_DEVICES];

template <bool R, bool W>
void launch_one(cudaStream_t s, const KCtx& C, const double* xin, double* xout,
                const double* stream, const double* gst, double omega, double* partials,
                SolveState* st, int fin, int iter, int slot, bool pdl) {
  const size_t smem = sizeof(pipe::Smem);
  int dev = 0;
  cudaGetDevice(&dev);
  int sms = 0;
  {
    std::lock_guard<std::mutex> lock(g_cache_mu);
    DeviceCache local;
    DeviceCache& D = (dev >= 0 && dev < MAX_DEVICES) ? g_cache[dev] : local;
    if (D.sm_count == 0) {
      cudaDeviceGetAttribute(&D.sm_count, cudaDevAttrMultiProcessorCount, dev);
      if (D.sm_count <= 0) D.sm_count = 1;
    }
    if (!D.attr_set[slot]) {
      cudaFuncSetAttribute(rbgs_pipelined_kernel<R, W>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      D.attr_set[slot] = true;
    }
    sms = D.sm_count;
  }
  const int grid = C.nb < sms ? C.nb : sms;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(pipe::NTHREADS);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = pdl ? 1 : 0;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, rbgs_pipelined_kernel<R, W>, C, xin, xout, stream, gst, omega, partials,
                     st, fin, iter);
}
}  // namespace

void launch_rbgs(cudaStream_t s, const KCtx& C, bool res, bool sweep, const double* xin,
                 double* xout, const double* stream, const double* gst, double omega,
                 double* partials, SolveState* st, int fin, int iter, bool pdl) {
  if (res && sweep)
    launch_one<true, true>(s, C, xin, xout, stream, gst, omega, partials, st, fin, iter, 0, pdl);
  else if (sweep)
    launch_one<false, true>(s, C, xin, xout, stream, gst, omega, partials, st, fin, iter, 1, pdl);
  else
    launch_one<true, false>(s, C, xin, xout, stream, gst, omega, partials, st, fin, iter, 2, pdl);
}

size_t rbgs_pipelined_smem_bytes() { return sizeof(pipe::Smem); }
// bulk copies land in ring rows, xt[] and urec[]: 16-byte aligned
static_assert(offsetof(pipe::Smem, urec) % 16 == 0, "urec must be 16-byte aligned");
static_assert(offsetof(pipe::Smem, xt) % 16 == 0, "xt must be 16-byte aligned");

}  // namespace ffvgpu
