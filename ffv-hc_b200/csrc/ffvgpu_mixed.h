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
  int stall;           // test hook: 1 the sweep kernel, 2 the pipelined A*x issues no copy,
                       // so its first wait runs out
  int cf;              // coarse-fine flux correction in the FP64 residual and A*x
  int depth;           // sweep kernel: L2 prefetch distance in blocks (staging depth, >= 1)
  int sweep_threads;   // sweep kernel: 256 (two rows per thread, the default) or 512 (one row)
  // pipelined A*x only: 0 the mixed form's finalisers, else the FP64
  // solver's (one instance): FIN_BI_QR0 or FIN_CG_QP on the one sum, or
  // FIN_BI_TS on the first of two sums and FIN_BI_TT on the second
  int fin = 0;
};

// CTAs of the persistent grids: SMs x resident CTAs per SM of each kernel,
// with 'threads' (128, 256 or 512) per CTA of the A*x (form 1) and update
// kernels; mvpipe: the pipelined A*x (one CTA per SM).
void mx_grid_sizes(int threads, int* sweep, int* matvec, int* update, int* guides, int* mvpipe);
// Sweep coefficients of blocks [first, first + count), MIXED_COEF_WORDS per
// block, in the thread order of a sweep kernel of sweep_threads threads:
// 32-bit words (FP64 high words, rounded) into coef, or with d64 (the
// FP64-data variant) the FP64 values into coef64.  Also writes each block's ucoef record and adds the instance's
// uniform blocks to st->ublocks.
constexpr int MIXED_COEF_WORDS = 7 * 4096;
void launch_mx_pack(cudaStream_t s, int first, int count, const double* A, uint32_t* coef,
                    double* coef64, double* ucoef, SolveState* st, bool d64, int sweep_threads);
void launch_mx_init(cudaStream_t s, const MixCtx& C, int count, const double* x,
                    const double* gx, const double* A, const double* b, double* r, double* r0);
// The iteration launchers take 'count' = CTAs of the persistent grid.  The
// iterate between passes and the preconditioned vectors (void* below) are
// float, or double with d64.
// One pass of sweeps; a later pass (first false) takes ein and its guide
// layer, written by launch_mx_guides.
void launch_mx_sweep(cudaStream_t s, const MixCtx& C, int count, int mode, bool first,
                     float omega, int nsweep, const double* r, double* r0, double* pv,
                     const double* q, const uint32_t* coef, const double* coef64,
                     const void* ein, const double* guides, void* eout, bool d64);
// Guide layer [blk][6][256] (FP64) of the iterate e for the next pass.
void launch_mx_guides(cudaStream_t s, const MixCtx& C, int count, const void* e, double* guides,
                      bool d64);
// The active list raw ([0] = n, then block ids) reordered into act: the
// blocks that stream their coefficients (ucoef flag 0) first, then the
// uniform ones, each in list order.  The persistent grids walk items
// c, c + grid, ..., so the expensive blocks are dealt out evenly; results do
// not depend on the order (every sum runs over blocks in block order).
void launch_mx_order_active(cudaStream_t s, const int32_t* raw, const double* ucoef,
                            int32_t* act);
// y = A x with its dot products; form 0: the pipelined kernel ('count' CTAs,
// one per SM), form 1: a block per CTA of 'threads' threads (C.fin 0 only).
void launch_mx_matvec(cudaStream_t s, const MixCtx& C, int count, int ndot, int threads, int form,
                      const void* x, const double* A, double* y, const double* w0, bool d64);
// An FP64 Jacobi sweep y = J(x; A, b) (bils.f90:5-55) on the pipelined
// kernel (its tile, guide layer and coefficient slots, with b in the dot
// partner's place); with dot also b.y, finalised by C.fin (FIN_CG_RR1).
void launch_jacobi_pipe(cudaStream_t s, const MixCtx& C, int count, bool dot, const double* x,
                        const double* A, const double* b, double* y, double omega);
// Coarse-fine flux mismatch per face cell of the (block, face) pairs
// [npairs][2] of kind NB_FINE: out [npairs][256][2] = (delta, F).
void launch_cf_mismatch(cudaStream_t s, int npairs, const double* x, const double* gx,
                        const double* A, const FaceNbr* nbr, const double* dx, const BCSet& bc,
                        const int32_t* pairs, double* out);
void launch_mx_update(cudaStream_t s, const MixCtx& C, int count, int threads, double* x,
                      const void* ph, const void* sh, double* r, const double* t,
                      const double* sv, const double* r0, bool d64);

}  // namespace ffvgpu
