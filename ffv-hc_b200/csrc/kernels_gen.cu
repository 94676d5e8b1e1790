// kernels_gen.cu -- device generator of the synthetic sphere-flow inputs of
// an instance (u*, cut positions, cut and fluid flags), bit-identical to the
// host generator (sphere_gen.h holds the shared per-cell definitions).
// Compiled with --fmad=false.
#include <cuda_runtime.h>

#include "ffvgpu_gen.h"
#include "sphere_gen.h"

namespace ffvgpu {

constexpr int GT = 256;

// One CTA per block of [first, first + count); cell (i, j, k) of the
// instance's local block b = blk - first draws from counter
// b*4096 + i + 16*(j + 16*k), as the host generator does for its block b.
__global__ void __launch_bounds__(GT)
gen_sphere_kernel(int first, const int32_t* __restrict__ geo, SphereGenParams G,
                  double* __restrict__ ux, double* __restrict__ uy, double* __restrict__ uz,
                  double* __restrict__ cut, size_t field_stride, uint8_t* __restrict__ flags) {
  const int blk = first + blockIdx.x;
  const int32_t L = geo[4 * blk];
  const int32_t idx[3] = {geo[4 * blk + 1], geo[4 * blk + 2], geo[4 * blk + 3]};
  double org[3];
  const double dx = block_geometry(G.domain_origin, G.root_length, L, idx, org);
  const uint64_t lb = (uint64_t)blockIdx.x;
  for (int m = 0; m < BLOCK_CELLS / GT; ++m) {
    const int s = threadIdx.x + GT * m;
    int i, j, k;
    cell_of(s, i, j, k);
    const size_t gs = (size_t)blk * BLOCK_CELLS + s;
    const uint64_t cell = lb * 4096u + (uint64_t)(i + 16 * (j + 16 * k));
    ux[gs] = 1.0 + G.sigma * normal_draw(G.seed, cell, 0);
    uy[gs] = G.sigma * normal_draw(G.seed, cell, 1);
    uz[gs] = G.sigma * normal_draw(G.seed, cell, 2);
    const CellCut cc = sphere_cell(org, dx, i, j, k, G.center, G.radius);
    for (int f = 0; f < 6; ++f) cut[f * field_stride + gs] = cc.c[f];
    flags[gs] = (uint8_t)(cc.cid | (cc.fluid ? 128 : 0));
  }
}

void launch_gen_sphere(cudaStream_t s, int first, int count, const int32_t* geo,
                       const SphereGenParams& G, double* ux, double* uy, double* uz, double* cut,
                       size_t field_stride, uint8_t* flags) {
  gen_sphere_kernel<<<count, GT, 0, s>>>(first, geo, G, ux, uy, uz, cut, field_stride, flags);
}

}  // namespace ffvgpu
