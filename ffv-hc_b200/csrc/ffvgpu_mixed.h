// ffvgpu_mixed.h -- host-side launchers of the mixed-precision kernels
// (kernels_mixed.cu) and the per-instance context they take.
#pragma once
#include <cuda_runtime.h>

#include "ffvgpu_layout.h"

namespace ffvgpu {

// What every mixed-form kernel needs.  The iteration kernels are persistent:
// their CTAs walk the device list active[0, *n_active) of blocks of running
// instances (a CUDA graph replays them while the list changes between
// replays); the start-of-solve kernel covers blocks [first, first + count).
// Blocks of an instance whose solve has stopped are skipped.
struct MixCtx {
  const int32_t* active;    // [capacity] block ids
  const int32_t* n_active;  // device count of active entries
  const FaceNbr* nbr;  // [capacity][6]
  const double* dx;    // [capacity]
  BCSet bc;            // pressure BCs (outer guide cells of the FP64 stencils)
  InstTable inst;
  double* partials;    // [2][capacity] per-block sums
  // [capacity][8]: ap, aw, ae, as, an, ab, at of cell 0 and a flag (1.0) when
  // every cell of the block has those seven coefficients; the sweep and A*x
  // kernels then take them from here instead of streaming the per-cell arrays
  const double* ucoef;
  int capacity;
  int first;
  uint64_t wait_ns;    // limit of every bounded device wait (ffvgpu_pool_set_wait_limit)
  int stall;           // test hook: the sweep issues no copy, so its first wait runs out
};

// CTAs of the persistent grids: SMs x resident CTAs per SM of each kernel.
void mx_grid_sizes(int* sweep, int* matvec, int* update, int* guides);
// 32-bit sweep coefficients of blocks [first, first + count): [blk][7][8][512]
// words (FP64 high words, rounded), MIXED_COEF_WORDS per block.
constexpr int MIXED_COEF_WORDS = 7 * 8 * 512;
// Also writes each block's ucoef record and adds the instance's uniform
// blocks to st->ublocks.
void launch_mx_pack(cudaStream_t s, int first, int count, const double* A, uint32_t* coef,
                    double* ucoef, SolveState* st);
void launch_mx_init(cudaStream_t s, const MixCtx& C, int count, const double* x,
                    const double* gx, const double* A, const double* b, double* r, double* r0);
// The iteration launchers take 'count' = CTAs of the persistent grid.
// One pass of sweeps; a later pass (first false) takes ein and its guide
// layer, written by launch_mx_guides.
void launch_mx_sweep(cudaStream_t s, const MixCtx& C, int count, int mode, bool first,
                     float omega, int nsweep, const double* r, double* r0, double* pv,
                     const double* q, const uint32_t* coef, const float* ein,
                     const double* guides, float* eout);
// Guide layer [blk][6][256] (FP64) of the FP32 iterate e for the next pass.
void launch_mx_guides(cudaStream_t s, const MixCtx& C, int count, const float* e,
                      double* guides);
void launch_mx_matvec(cudaStream_t s, const MixCtx& C, int count, int ndot, const float* x,
                      const double* A, double* y, const double* w0);
void launch_mx_update(cudaStream_t s, const MixCtx& C, int count, double* x, const float* ph,
                      const float* sh, double* r, const double* t, const double* sv,
                      const double* r0);

}  // namespace ffvgpu
