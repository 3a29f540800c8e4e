// pd_critical_time_step_static: the critical time step computed with no device
// allocation at all. The block minima of the critical-dt kernel go to a
// file-scope static device array instead of the context's scratch buffer, and
// the result goes through the array's last slot to the caller's host double.
//
// Who needs it: pd_critical_time_step allocates and frees a one-double device
// buffer on every call (and may grow the context's scratch). A host whose own
// pool allocator has reserved the device's memory up front sees cudaMalloc
// fail there, and cudaFree synchronises the whole device, stalling every other
// stream of a host that re-checks the stable step inside its time loop. This
// entry point does neither.
//
// Limits and rules (also in include/pd_b200.h):
//   * kStaticPartials block minima at most: ceil(n * lanes_per_point / 256)
//     blocks, so 1,048,576 points at the default 16 lanes per point. Larger
//     problems are rejected with PD_ERR_ARG; use pd_critical_time_step.
//   * Nothing in the array needs to start at zero: every call writes each
//     partial slot it reduces before reading it, and overwrites the result slot.
//   * One array per device, shared by every context on it: overlapping calls
//     on the same device (two threads, or two streams in flight) race on it.
//   * The first call on a device resolves the array's address
//     (cudaGetSymbolAddress, which may load this module on that device); make
//     that first call before any stream capture begins.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "pd_internal.cuh"

namespace {

constexpr int64_t kStaticPartials = 65536;  // 512 KiB of block minima
constexpr int kMaxDevices = 64;

// Block minima [0, kStaticPartials) and the result slot [kStaticPartials].
static __device__ __align__(256) double g_dt_scratch[kStaticPartials + 1];

std::mutex g_mu;
double* g_scratch_ptr[kMaxDevices] = {};

// Address of g_dt_scratch on the context's device, resolved once per device
// with that device current.
int static_scratch(pd_ctx* c, double** out) {
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_ptr[c->device]) {
    PD_CUDA_TRY(c, cudaSetDevice(c->device));
    void* p = nullptr;
    PD_CUDA_TRY(c, cudaGetSymbolAddress(&p, g_dt_scratch));
    g_scratch_ptr[c->device] = static_cast<double*>(p);
  }
  *out = g_scratch_ptr[c->device];
  return PD_OK;
}

}  // namespace

extern "C" int pd_critical_time_step_static(pd_ctx* c, double* dt_out) {
  if (!c) return PD_ERR_ARG;
  if (!dt_out) {
    c->err = "pd_critical_time_step_static: null output";
    return PD_ERR_ARG;
  }
  if (c->device < 0 || c->device >= kMaxDevices) {
    c->err = "pd_critical_time_step_static: device ordinal " + std::to_string(c->device) + " out of range [0, " +
             std::to_string(kMaxDevices) + ")";
    return PD_ERR_ARG;
  }
  const int64_t blocks = pdb::critical_dt_partials(c);
  if (blocks > kStaticPartials) {
    c->err = "pd_critical_time_step_static: " + std::to_string(c->n) + " points need " + std::to_string(blocks) +
             " block minima, more than the " + std::to_string(kStaticPartials) +
             " its static scratch holds; use pd_critical_time_step";
    return PD_ERR_ARG;
  }
  // Everything below runs on buffers the context already holds; the set-up
  // that allocates them is left to the allocating entry points.
  if (c->n == 0 || !c->row.p || !c->wv_done) {
    c->err =
        "pd_critical_time_step_static: the context is not set up (points, bonds, material and a first "
        "pd_weighted_volume or evaluation are needed); this entry point allocates nothing, so it does no set-up";
    return PD_ERR_STATE;
  }
  double* scratch = nullptr;
  TRY_RC(static_scratch(c, &scratch));
  PD_CUDA_TRY(c, cudaSetDevice(c->device));
  PD_CUDA_TRY(c, pdb::launch_critical_dt_into(c, scratch, scratch + kStaticPartials));
  PD_CUDA_TRY(c, cudaMemcpyAsync(dt_out, scratch + kStaticPartials, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  PD_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  return PD_OK;
}
