// ffvgpu_gen.h -- launcher of the device generator of sphere-flow inputs.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace ffvgpu {

struct SphereGenParams {
  double domain_origin[3];
  double root_length;
  double center[3];
  double radius;
  uint64_t seed;
  double sigma;
};

// Blocks [first, first + count); geo[4*blk] = level, then the block index.
void launch_gen_sphere(cudaStream_t s, int first, int count, const int32_t* geo,
                       const SphereGenParams& G, double* ux, double* uy, double* uz, double* cut,
                       size_t field_stride, uint8_t* flags);

}  // namespace ffvgpu
