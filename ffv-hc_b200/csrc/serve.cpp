// serve.cpp -- a request loop over a batch pool: continuous batching of
// pressure solves (no counterpart in the reference).
//
// Requests arrive at given times.  Each pass of the loop admits waiting
// requests in arrival order while a block range and an instance slot are
// free (a request that does not fit waits; later, smaller ones may pass
// it), starts their solves, advances every running solve by a fixed number
// of iterations (one graph replay), and retires the solves that ended:
// their pressure (interior, the device layout) is copied to the host and
// their blocks are released.  Latency = completion - arrival, both on the
// host's steady clock from the start of the run.
#include <chrono>
#include <cstring>
#include <deque>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/ffvgpu.h"
#include "pool_internal.h"

using namespace ffvgpu;
using namespace ffvgpu::detail;

extern "C" {

ffvgpu_status ffvgpu_serve(ffvgpu_pool* P, const ffvgpu_mixed_params* prm, int32_t n,
                           const ffvgpu_request* req, int32_t iterations_per_step,
                           ffvgpu_request_result* out) {
  if (!P || !prm || (n > 0 && (!req || !out))) return bad("null argument");
  if (!P->batch) return bad("ffvgpu_serve runs on a batch pool");
  if (iterations_per_step <= 0) return bad("iterations_per_step must be positive");
  for (int i = 1; i < n; ++i)
    if (req[i].arrival_s < req[i - 1].arrival_s) return bad("requests must be sorted by arrival");
  for (const ffvgpu_instance& I : P->inst)
    if (I.running) return bad("a solve is already running on this pool");
  cudaSetDevice(P->device);
  std::memset(out, 0, sizeof(ffvgpu_request_result) * (size_t)(n > 0 ? n : 0));
  // pinned staging for the returned pressure, grown to the largest request
  double* host_x = nullptr;
  size_t host_cap = 0;
  std::vector<int> slot_req(P->inst.size(), -1);
  std::deque<int> waiting;
  int next = 0, finished = 0, running = 0;
  ffvgpu_status status = FFVGPU_OK;
  const auto t0 = std::chrono::steady_clock::now();
  auto now = [&]() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  };
  std::vector<int32_t> done(P->inst.size());
  auto cancelled = [&](int k, double t) { return req[k].cancel_s > 0.0 && req[k].cancel_s <= t; };
  while (finished < n && status == FFVGPU_OK) {
    const double t = now();
    while (next < n && req[next].arrival_s <= t) waiting.push_back(next++);
    // withdraw what has passed its cancel time: waiting requests are dropped,
    // running solves stopped and their blocks released
    for (auto it = waiting.begin(); it != waiting.end();) {
      if (!cancelled(*it, t)) {
        ++it;
        continue;
      }
      out[*it].finish_s = now();
      out[*it].status = FFVGPU_CANCELLED;
      ++finished;
      it = waiting.erase(it);
    }
    for (int inst = 0; inst < (int)slot_req.size() && status == FFVGPU_OK; ++inst) {
      const int k = slot_req[inst];
      if (k < 0 || !cancelled(k, t)) continue;
      if ((status = ffvgpu_mixed_cancel(P, inst)) != FFVGPU_OK) break;
      ffvgpu_result r;
      ffvgpu_instance_result(P, inst, &r, nullptr);
      out[k].finish_s = now();
      out[k].count = r.count;
      out[k].residual = r.residual;
      out[k].status = FFVGPU_CANCELLED;
      slot_req[inst] = -1;
      --running;
      ++finished;
      status = ffvgpu_instance_release(P, inst);
    }
    if (status != FFVGPU_OK) break;
    if (finished >= n) break;
    // admit in arrival order; a request that does not fit waits
    for (auto it = waiting.begin(); it != waiting.end();) {
      const int k = *it;
      int32_t inst = -1;
      ffvgpu_status s = ffvgpu_instance_admit_sphere(P, &req[k].problem, &inst);
      if (s == FFVGPU_OOM) {
        ++it;
        continue;
      }
      if (s != FFVGPU_OK) {
        status = s;
        break;
      }
      if ((s = ffvgpu_mixed_begin(P, inst, prm)) != FFVGPU_OK) {
        status = s;
        break;
      }
      out[k].admit_s = now();
      out[k].blocks = ffvgpu_instance_blocks(P, inst);
      slot_req[inst] = k;
      ++running;
      it = waiting.erase(it);
    }
    if (status != FFVGPU_OK) break;
    if (running == 0) {
      if (!waiting.empty()) {
        status = bad("a waiting request does not fit in the pool");
        break;
      }
      if (next < n) {  // idle until the next arrival
        const double dt = req[next].arrival_s - now();
        if (dt > 0) std::this_thread::sleep_for(std::chrono::duration<double>(dt));
      }
      continue;
    }
    if ((status = ffvgpu_mixed_advance(P, iterations_per_step)) != FFVGPU_OK) break;
    int32_t nf = 0;
    if ((status = ffvgpu_mixed_poll(P, done.data(), (int32_t)done.size(), &nf)) != FFVGPU_OK)
      break;
    for (int f = 0; f < nf; ++f) {
      const int inst = done[f];
      const int k = slot_req[inst];
      ffvgpu_result r;
      const ffvgpu_status rs = ffvgpu_instance_result(P, inst, &r, nullptr);
      const ffvgpu_instance& I = P->inst[inst];
      // the response: the instance's pressure, copied back
      const size_t need = (size_t)I.count * BC;
      cudaError_t e = cudaSuccess;
      if (need > host_cap) {
        if (host_x) cudaFreeHost(host_x);
        host_x = nullptr;
        host_cap = 0;
        e = cudaMallocHost(&host_x, sizeof(double) * need);
        if (e == cudaSuccess) host_cap = need;
      }
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(host_x, P->x[P->xcur] + (size_t)I.first * BC, sizeof(double) * need,
                            cudaMemcpyDeviceToHost, P->stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(P->stream);
      if (e != cudaSuccess) {
        status = cuda_fail(e, "returning a pressure field");
        break;
      }
      out[k].finish_s = now();
      out[k].count = r.count;
      out[k].residual = r.residual;
      out[k].status = rs;
      slot_req[inst] = -1;
      --running;
      ++finished;
      if ((status = ffvgpu_instance_release(P, inst)) != FFVGPU_OK) break;
    }
  }
  if (host_x) cudaFreeHost(host_x);
  return status;
}

}  // extern "C"
