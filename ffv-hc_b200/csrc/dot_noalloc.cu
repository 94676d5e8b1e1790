// dot_noalloc.cu -- the dot product of two block-pool vectors without any
// device allocation.
//
// Some callers cannot call cudaMalloc: an application that hands all of the
// GPU's memory to its own allocator when it starts (a coupled multi-physics
// code, for instance) has nothing left for a library to allocate, and a
// time-stepping loop that must not stall cannot afford cudaMalloc/cudaFree,
// which synchronise the device.  This entry point serves them: the caller
// passes the two input vectors and the output location, all on the device,
// and the per-block partial sums live in a fixed array compiled into this
// library, FFVGPU_NOALLOC_MAX_BLOCKS doubles (512 KB) plus a completion
// counter, which every GPU that loads the library holds until the process
// exits.
//
// The array is shared by every call on a device and keeps the last call's
// partial sums; calls that overlap on the GPU (two streams at once) race on
// it and must be serialised by the caller.  The counter is cleared by each
// call before its reduction starts.
//
// The array's device address is looked up once per device and kept for the
// life of the process: it assumes that device's primary context lives as
// long as the process does (after cudaDeviceReset the module may load
// elsewhere, so the cached address would be stale).  The stream passed must
// belong to the device that is current at the call.
//
// The sum uses the same fixed tree as ffvgpu_dot, so the result is bit for
// bit the one the pool-based entry point returns for the same vectors.
#include <cstdio>
#include <mutex>
#include <string>

#include <cuda_runtime.h>

#include "../../include/ffvgpu.h"
#include "ffvgpu_kernels.h"
#include "ffvgpu_layout.h"

namespace ffvgpu {
namespace {

constexpr int MAX_DEVICES = 64;

static __device__ __align__(256) double g_noalloc_partials[FFVGPU_NOALLOC_MAX_BLOCKS];
static __device__ __align__(256) unsigned int g_noalloc_ticket;

// g_noalloc_partials / g_noalloc_ticket are host-side stand-ins in host
// code; their device addresses are looked up once per device.
struct DeviceScratch {
  double* partials = nullptr;
  unsigned int* ticket = nullptr;
};
DeviceScratch g_scratch[MAX_DEVICES];
std::mutex g_scratch_mutex;

__global__ void clear_ticket_kernel(unsigned int* ticket) { *ticket = 0u; }

// One CTA of 256 threads per leaf block; thread r carries virtual threads r
// and r + 256 of the block tree (cells c*2048 + r + 256*m, m even / odd).
__global__ void __launch_bounds__(THREADS)
dot_noalloc_kernel(const double* __restrict__ x, const double* __restrict__ y,
                   double* __restrict__ partials, unsigned int* __restrict__ ticket,
                   double* __restrict__ result) {
  __shared__ double ws[16];
  __shared__ int amlast;
  const int tid = threadIdx.x;
  const size_t base = (size_t)blockIdx.x * BLOCK_CELLS;
  double acc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
#pragma unroll
  for (int c = 0; c < 2; ++c) {
#pragma unroll 4
    for (int m = 0; m < 8; ++m) {
      const size_t s = base + c * HALF_CELLS + tid + THREADS * m;
      acc[c][m & 1] += __ldg(x + s) * __ldg(y + s);
    }
  }
  double v0 = acc[0][0] + acc[1][0], v1 = acc[0][1] + acc[1][1];
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1) {
    v0 += __shfl_xor_sync(0xffffffffu, v0, off);
    v1 += __shfl_xor_sync(0xffffffffu, v1, off);
  }
  if ((tid & 31) == 0) {
    ws[tid >> 5] = v0;
    ws[8 + (tid >> 5)] = v1;
  }
  __syncthreads();
  if (tid == 0) {
    double sum = 0.0;
#pragma unroll
    for (int w = 0; w < 16; ++w) sum += ws[w];
    __stcg(partials + blockIdx.x, sum);
    __threadfence();
    amlast = (atomicAdd(ticket, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (!amlast) return;
  __threadfence();
  double S = 0.0;
  for (int b = tid; b < (int)gridDim.x; b += THREADS) S += __ldcg(partials + b);
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1) S += __shfl_xor_sync(0xffffffffu, S, off);
  __syncthreads();
  if ((tid & 31) == 0) ws[tid >> 5] = S;
  __syncthreads();
  if (tid == 0) {
    double total = 0.0;
#pragma unroll
    for (int w = 0; w < 8; ++w) total += ws[w];
    *result = total;
  }
}

// First call on a device (with that device current): look up the scratch's
// device addresses.  Lookups take no allocation.
ffvgpu_status device_scratch(int dev, DeviceScratch** out) {
  if (dev < 0 || dev >= MAX_DEVICES) {
    set_last_error("device ordinal beyond the scratch table");
    return FFVGPU_BAD_ARG;
  }
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  DeviceScratch& d = g_scratch[dev];
  if (!d.partials) {
    double* p = nullptr;
    unsigned int* t = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void**)&p, g_noalloc_partials);
    if (e == cudaSuccess) e = cudaGetSymbolAddress((void**)&t, g_noalloc_ticket);
    if (e != cudaSuccess) {
      set_last_error(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      return FFVGPU_CUDA_ERROR;
    }
    d.partials = p;
    d.ticket = t;
  }
  *out = &d;
  return FFVGPU_OK;
}

}  // namespace
}  // namespace ffvgpu

extern "C" ffvgpu_status ffvgpu_dot_noalloc(const double* x, const double* y, int32_t num_blocks,
                                            double* result, void* stream) {
  using namespace ffvgpu;
  if (!x || !y || !result) {
    set_last_error("null pointer");
    return FFVGPU_BAD_ARG;
  }
  if (num_blocks <= 0 || num_blocks > FFVGPU_NOALLOC_MAX_BLOCKS) {
    set_last_error("num_blocks must be in [1, " + std::to_string(FFVGPU_NOALLOC_MAX_BLOCKS) +
                   "] for ffvgpu_dot_noalloc (its scratch is a fixed array)");
    return FFVGPU_BAD_ARG;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    set_last_error(std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    return FFVGPU_NO_DEVICE;
  }
  DeviceScratch* d = nullptr;
  ffvgpu_status s = device_scratch(dev, &d);
  if (s != FFVGPU_OK) return s;
  cudaStream_t st = (cudaStream_t)stream;
  clear_ticket_kernel<<<1, 1, 0, st>>>(d->ticket);
  dot_noalloc_kernel<<<num_blocks, THREADS, 0, st>>>(x, y, d->partials, d->ticket, result);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_last_error(std::string("launch: ") + cudaGetErrorString(e));
    return FFVGPU_CUDA_ERROR;
  }
  return FFVGPU_OK;
}
