// restart.cpp -- the reference's per-rank restart files for pool fields:
// LocalScalar3D::Dump2 / Load2 (src/FFV/LocalScalar3D.cpp:216-354).
//
// File: six native ints -- cells per block along x, y, z, guide width vc,
// element count 1, number of blocks -- then every block's (n+2vc)^3 doubles
// in block order, i fastest, guide cells included (after the exchange).
// Load2 also takes a file at half the resolution (8^3 blocks): each coarse
// cell fills its 2x2x2 fine cells (sf3d_copy_x2, src/CGMfuncs/bsf3d.f90:5-33).
// Both finish with the field's exchange, as the reference's do.
#include <cstdio>
#include <cstring>
#include <fstream>
#include <vector>

#include "../../include/ffvgpu.h"
#include "pool_internal.h"

using namespace ffvgpu;
using namespace ffvgpu::detail;

namespace {

bool real_vector_field(ffvgpu_field f) {
  return f == FFVGPU_FIELD_X || (f >= FFVGPU_FIELD_UX && f <= FFVGPU_FIELD_UZ);
}

}  // namespace

extern "C" {

int32_t ffvgpu_restart_filename(char* out, int32_t cap, const char* path, const char* prefix,
                                const char* label, int32_t rank, int32_t step) {
  if (!out || cap <= 0 || !path || !prefix || !label) return -1;
  // LocalScalar3D.cpp:224-243: path/prefix label-rank(5 digits)-step(10 digits).bin
  const int n = std::snprintf(out, (size_t)cap, "%s/%s%s-%05d-%010d.bin", path, prefix, label,
                              (int)rank, (int)step);
  return (n < 0 || n >= cap) ? -1 : n;
}

ffvgpu_status ffvgpu_dump2(ffvgpu_pool* P, ffvgpu_field f, int32_t vc, const char* filename) {
  if (!P || !filename) return bad("null argument");
  if (P->batch) return bad("a batch pool is used through the instance entry points");
  if (!real_vector_field(f)) return bad("Dump2 writes X, UX, UY or UZ");
  if (vc < 1 || vc > 2) return bad("vc must be 1 or 2");
  ffvgpu_status s;
  if ((s = ffvgpu_exchange(P, f, nullptr, nullptr))) return s;  // LocalScalar3D.cpp:217
  const size_t w = 16 + 2 * (size_t)vc, per = w * w * w;
  std::vector<double> data(per * (size_t)P->nb);
  if ((s = ffvgpu_pool_download(P, f, data.data(), vc))) return s;
  std::ofstream ofs(filename, std::ios::out | std::ios::binary);
  if (!ofs) return bad("Dump2: cannot open the file for writing");
  const int32_t head[6] = {16, 16, 16, vc, 1, P->nb};
  ofs.write(reinterpret_cast<const char*>(head), sizeof(head));
  ofs.write(reinterpret_cast<const char*>(data.data()), (std::streamsize)(sizeof(double) * data.size()));
  if (!ofs) return bad("Dump2: write failed");
  return FFVGPU_OK;
}

ffvgpu_status ffvgpu_load2(ffvgpu_pool* P, ffvgpu_field f, int32_t vc, const char* filename) {
  if (!P || !filename) return bad("null argument");
  if (P->batch) return bad("a batch pool is used through the instance entry points");
  if (!real_vector_field(f)) return bad("Load2 reads X, UX, UY or UZ");
  if (vc < 1 || vc > 4) return bad("vc must be in [1,4]");
  std::ifstream ifs(filename, std::ios::in | std::ios::binary);
  if (!ifs) return bad("Load2: cannot open the file");
  int32_t h[6] = {0, 0, 0, 0, 0, 0};
  ifs.read(reinterpret_cast<char*>(h), sizeof(h));
  if (!ifs) return bad("Load2: short header");
  const int nx = h[0], ny = h[1], nz = h[2], nv = h[3], ne = h[4], nb = h[5];
  const size_t w = 16 + 2 * (size_t)vc, per = w * w * w;
  std::vector<double> data(per * (size_t)P->nb, 0.0);
  // LocalScalar3D.cpp:320-349: the same shape, or half the cells per edge
  if (nx == 16 && ny == 16 && nz == 16 && nv == vc && ne == 1 && nb == P->nb) {
    ifs.read(reinterpret_cast<char*>(data.data()), (std::streamsize)(sizeof(double) * data.size()));
    if (!ifs) return bad("Load2: short data");
  } else if (2 * nx == 16 && 2 * ny == 16 && 2 * nz == 16 && nv == vc && ne == 1 &&
             nb == P->nb) {
    const size_t wc = 8 + 2 * (size_t)vc, perc = wc * wc * wc;
    std::vector<double> coarse(perc);
    for (int b = 0; b < nb; ++b) {
      ifs.read(reinterpret_cast<char*>(coarse.data()), (std::streamsize)(sizeof(double) * perc));
      if (!ifs) return bad("Load2: short data");
      double* x = data.data() + (size_t)b * per;
      // sf3d_copy_x2: x(i,j,k) = xc((i+1)/2, (j+1)/2, (k+1)/2), 1-based interiors
      for (int k = 1; k <= 16; ++k)
        for (int j = 1; j <= 16; ++j)
          for (int i = 1; i <= 16; ++i) {
            const size_t m = (size_t)(i - 1 + vc) + w * ((size_t)(j - 1 + vc) + w * (k - 1 + vc));
            const size_t mc = (size_t)((i + 1) / 2 - 1 + vc) +
                              wc * ((size_t)((j + 1) / 2 - 1 + vc) + wc * ((k + 1) / 2 - 1 + vc));
            x[m] = coarse[mc];
          }
    }
  } else {
    return bad("Load2: the file's block shape, guide width or block count does not match");
  }
  ffvgpu_status s;
  if ((s = ffvgpu_pool_upload(P, f, data.data(), vc))) return s;
  return ffvgpu_exchange(P, f, nullptr, nullptr);  // LocalScalar3D.cpp:353
}

}  // extern "C"
