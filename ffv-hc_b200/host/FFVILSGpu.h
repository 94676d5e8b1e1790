// FFVILSGpu.h -- C++ host-side mirror of FFV-HC's FFVILS solve interface
// (src/FFV/FFVILS.h) over the device block pool of include/ffvgpu.h.
//
// FFVILS takes a BCMTools BlockManager and LocalScalar3D field objects; the
// GPU path keeps those fields in a device pool instead, so each method here
// takes the pool in place of (blockManager, plsx, plsAp..plsAt, plsb) and
// keeps the rest of the reference's signature: the same names, the same
// argument meanings (omega, countMax, epsilon, countPreConditioner) and the
// same out-parameters (count, residual).  Error behaviour follows the
// reference by default: a NaN/Inf residual prints "bb rr" and exits
// (FFVILS.h:36-43); set exit_on_nan = false to get the status back instead.
// Work vectors the reference's CG takes as arguments (r, p, q, z, x0) are
// owned by the pool.
#ifndef FFVILS_GPU_H
#define FFVILS_GPU_H

#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <string>

#include "../../include/ffvgpu.h"

class FFVILSGpu {
 public:
  explicit FFVILSGpu(bool exit_on_nan = true) : exit_on_nan_(exit_on_nan) {}

  // FFVILS::RBGS (FFVILS.h:547-594).
  ffvgpu_status RBGS(ffvgpu_pool* pool, double omega, int countMax, double epsilon, int& count,
                     double& residual, double* history = nullptr) {
    ffvgpu_iter_params prm = {omega, countMax, epsilon, 0, 0, history};
    ffvgpu_result res;
    const ffvgpu_status s = ffvgpu_solve_rbgs(pool, &prm, &res);
    return finish(s, res, count, residual);
  }

  // FFVILS::CG (FFVILS.h:661-791).
  ffvgpu_status CG(ffvgpu_pool* pool, double omega, int countPreConditioner, int countMax,
                   double epsilon, int& count, double& residual, double* history = nullptr) {
    ffvgpu_iter_params prm = {omega, countMax, epsilon, countPreConditioner, 0, history};
    ffvgpu_result res;
    const ffvgpu_status s = ffvgpu_solve_cg(pool, &prm, &res);
    return finish(s, res, count, residual);
  }

  // FFVILS::BiCGSTAB (FFVILS.h:793-974).
  ffvgpu_status BiCGSTAB(ffvgpu_pool* pool, double omega, int countPreConditioner, int countMax,
                         double epsilon, int& count, double& residual,
                         double* history = nullptr) {
    ffvgpu_iter_params prm = {omega, countMax, epsilon, countPreConditioner, 0, history};
    ffvgpu_result res;
    const ffvgpu_status s = ffvgpu_solve_bicgstab(pool, &prm, &res);
    return finish(s, res, count, residual);
  }

  // FFVILS::Fill (FFVILS.h:425-445).
  ffvgpu_status Fill(ffvgpu_pool* pool, ffvgpu_field field, double value) {
    return check(ffvgpu_fill(pool, field, value), "Fill");
  }

  const ffvgpu_result& last_result() const { return last_; }

 private:
  ffvgpu_status finish(ffvgpu_status s, const ffvgpu_result& res, int& count, double& residual) {
    last_ = res;
    if (s == FFVGPU_OK || s == FFVGPU_NOT_CONVERGED) {
      // the reference is silent when countMax is reached (FFVILS.h:44-45)
      count = res.count;
      residual = res.residual;
      return s;
    }
    if (s == FFVGPU_NAN_DETECTED) {
      count = res.count;
      residual = res.residual;
      if (exit_on_nan_) {
        std::printf("%s\n", ffvgpu_last_error());
        std::exit(0);  // the reference's Exit(0)
      }
      return s;
    }
    return check(s, "solve");
  }

  ffvgpu_status check(ffvgpu_status s, const char* what) {
    if (s != FFVGPU_OK)
      throw std::runtime_error(std::string("FFVILSGpu::") + what + ": " + ffvgpu_last_error());
    return s;
  }

  bool exit_on_nan_;
  ffvgpu_result last_{};
};

#endif  // FFVILS_GPU_H
