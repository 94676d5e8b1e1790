// ffvgpu_kernels.h -- host-side launchers of the FP64 kernels.
#pragma once
#include <cstddef>
#include <cstdint>
#include <string>
#include <cuda_runtime.h>

#include "ffvgpu_layout.h"

namespace ffvgpu {


// Parameters every block kernel needs: neighbour table, cell sizes and the
// outer BCs of the field being staged.
// Kernels that take a block range (exchange, unpack, assembly, BC folding)
// cover blocks [first, first + nb); the solver kernels run with first = 0.
struct KCtx {
  const FaceNbr* nbr;  // [blocks][6]
  const double* dx;    // [blocks]
  BCSet bc;
  int nb;
  int first;
  uint64_t wait_ns;    // limit of every bounded device wait (ffvgpu_pool_set_wait_limit)
  // [blocks][8] uniform records of A (launch_pack_stream, launch_urec), or
  // null: every block streams all its coefficients
  const double* urec;
};

// Fused residual + red-black sweep over the coefficient stream (rbgs_pipelined.cu).
// pdl: launched as a programmatic dependent of the previous kernel on the
// stream, which must then be a pass of this kernel (it overlaps that pass's
// tail: its coefficient prefetch runs before the dependency wait).
void launch_rbgs(cudaStream_t s, const KCtx& C, bool res, bool sweep, const double* xin,
                 double* xout, const double* stream, const double* gst, double omega,
                 double* partials, SolveState* st, int fin, int iter, bool pdl = false);
// Packs A and b into the sweep's coefficient stream and writes each block's
// uniform record urec[blk][8] (Ap..At of cell 0, then 1.0 when every cell has
// those seven coefficients, else 0.0), adding the uniform blocks to *ucount.
void launch_pack_stream(cudaStream_t s, int nb, const double* A, const double* b, double* stream,
                        double* urec, int32_t* ucount);
// The uniform records alone (the record format of launch_pack_stream).
void launch_urec(cudaStream_t s, int nb, const double* A, double* urec, int32_t* ucount);
// Jacobi sweep from the zero field (the preconditioner's first pass); a
// block with a set uniform record (C.urec) reads its seven coefficients from
// it.  dot: also b.x1 (FIN_CG_RR1).
void launch_jacobi(cudaStream_t s, const KCtx& C, bool dot, double* xout, const double* A,
                   const double* b, double omega, double* partials, SolveState* st);
void launch_calc_r(cudaStream_t s, const KCtx& C, const double* x, const double* gst,
                   const double* A, const double* b, double* r, SolveState* st);
void launch_p_update(cudaStream_t s, const KCtx& C, const double* z, double* p, int first,
                     SolveState* st);
// p = r on the first iteration of a cycle (st->cycle == 1), else the update.
void launch_bicg_p(cudaStream_t s, const KCtx& C, const double* r, double* p, const double* q,
                   SolveState* st);
// Sum of x over the interior (finaliser fin); x += st->alpha.
void launch_sum(cudaStream_t s, const KCtx& C, const double* x, double* partials, SolveState* st,
                int fin);
void launch_shift(cudaStream_t s, const KCtx& C, double* x, SolveState* st);
// r.r0 (setting r0 = r first on the first iteration of a cycle).
void launch_dot_rr0(cudaStream_t s, const KCtx& C, const double* r, double* r0, double* partials,
                    SolveState* st, int fin, int iter);
void launch_axpyz(cudaStream_t s, const KCtx& C, double* z, const double* x, const double* y,
                  SolveState* st);
void launch_bicg_update(cudaStream_t s, const KCtx& C, double* x, const double* pz,
                        const double* sz, double* r, const double* t, const double* sv,
                        double* partials, SolveState* st, int iter);
void launch_cg_update(cudaStream_t s, const KCtx& C, double* x, const double* p, double* r,
                      const double* q, double* partials, SolveState* st, int iter);
void launch_dot(cudaStream_t s, const KCtx& C, const double* x, const double* y,
                double* partials, SolveState* st, int fin, int iter);
void launch_exchange(cudaStream_t s, const KCtx& C, const double* x, double* g);
void launch_pack(cudaStream_t s, int nb, const double* stage, int vc, double* dst, size_t stride,
                 double* gdst);
void launch_pack_flag(cudaStream_t s, int nb, const int32_t* stage, int vc, uint8_t* flags,
                      int bit, int mode);
void launch_unpack_flag(cudaStream_t s, int nb, const uint8_t* flags, int vc, int32_t* stage,
                        int bit);
void launch_unpack(cudaStream_t s, const KCtx& C, const double* src, size_t stride, int vc,
                   int with_guides, double* stage);
void launch_assemble(cudaStream_t s, const KCtx& C, const double* ux, const double* uy,
                     const double* uz, const double* gux, const double* guy, const double* guz,
                     const double* cut, const uint8_t* flags, double* A, double* b,
                     double* vface, double rhof, double dt, size_t field_stride);
void launch_fold_bc(cudaStream_t s, const KCtx& C, double* A, double* b);
// bcut_remove_p (corr false) or bcut_corr_u (corr true) on every block.
void launch_projection(cudaStream_t s, const KCtx& C, bool corr, const double* p,
                       const double* gp, const double* cut, const uint8_t* flags, double* ux,
                       double* uy, double* uz, double* vface, double* lapp, double rhof,
                       double dt, size_t field_stride);
void launch_fill(cudaStream_t s, int nb, double* x, size_t stride, double* g, double value);

// Sets the message ffvgpu_last_error() returns on this thread.
void set_last_error(const std::string& msg);

}  // namespace ffvgpu
