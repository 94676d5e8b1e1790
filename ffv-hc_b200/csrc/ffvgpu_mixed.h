// ffvgpu_mixed.h -- host-side launchers of the mixed-precision kernels
// (kernels_mixed.cu) and the per-instance context they take.
#pragma once
#include <cuda_runtime.h>

#include "ffvgpu_layout.h"

namespace ffvgpu {

// What every mixed-form kernel needs.  A launch covers the blocks
// [first, first + count) of the pool; blocks of no instance, or of an
// instance whose solve has stopped, return at entry.
struct MixCtx {
  const FaceNbr* nbr;  // [capacity][6]
  const double* dx;    // [capacity]
  BCSet bc;            // pressure BCs (outer guide cells of the FP64 stencils)
  InstTable inst;
  double* partials;    // [2][capacity] per-block sums
  int capacity;
  int first;
};

void launch_mx_pack(cudaStream_t s, int first, int count, const double* A, float* coef);
void launch_mx_init(cudaStream_t s, const MixCtx& C, int count, const double* x,
                    const double* gx, const double* A, const double* b, double* r, double* r0);
void launch_mx_sweep(cudaStream_t s, const MixCtx& C, int count, int mode, bool first, bool last,
                     float omega, int nsweep, const double* r, double* pv, const double* q,
                     const float* coef, float* v32, const float* ein, float* eout);
void launch_mx_matvec(cudaStream_t s, const MixCtx& C, int count, int ndot, const float* x,
                      const double* A, double* y, const double* w0);
void launch_mx_update(cudaStream_t s, const MixCtx& C, int count, double* x, const float* ph,
                      const float* sh, double* r, const double* t, const double* sv,
                      const double* r0);

}  // namespace ffvgpu
