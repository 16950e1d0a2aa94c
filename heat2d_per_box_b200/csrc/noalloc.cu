// Allocation-free execution of a planned transform.
//
// Some callers cannot call cudaMalloc while they run the transform.  A solver
// whose memory manager owns all device memory (a caching allocator, or pools
// reserved at start-up and handed out by the solver itself) must not have a
// library allocate behind its back, and cudaMalloc/cudaFree can also stall
// the device, which a time-stepping loop that keeps the GPU busy cannot
// afford.  bfgt_plan_execute_noalloc runs the same kernels as
// bfgt_plan_execute, but takes the plane-wave scratch it needs (the partial
// expansions of every chunk of leaves, their group sums and the expansions of
// the cutoff boxes) from one file-scope device array of fixed size instead of
// the plan's own buffers.  It calls no allocating routine.
//
// The array holds kNoallocScratchBytes on every GPU that loads this library,
// until the process exits.  On the first call on a device this file resolves
// the array's device address with cudaGetSymbolAddress (with that device
// current); make that first call before any stream capture.  The address is
// kept per device ordinal for the life of the process: after cudaDeviceReset
// it no longer names the array of the new context, so do not use this entry
// point in a process that resets its device.  Every call shares the array:
// calls that overlap on the GPU (other streams, other threads) race on it.
// Each call writes every partial and group expansion it reads, and the
// expansion of every cutoff box that holds plane-wave leaves.  The cutoff
// translation also reads the expansion of a cutoff box without plane-wave
// leaves (its own term), which then holds whatever an earlier call left there;
// the local expansion computed from it is never read, so no result depends on
// it and nothing has to be cleared between calls.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/bfgt.h"
#include "plan_internal.hpp"

namespace {

constexpr size_t kNoallocScratchBytes = (size_t)32 << 20;  // 32 MiB
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

std::mutex g_mu;
void *g_scratch_addr[128] = {};

int scratch_for_device(int dev, void **out, std::string &msg) {
  if (dev < 0 || dev >= 128) {
    msg = "device ordinal out of range";
    return BFGT_ERR_ARG;
  }
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch_addr[dev]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
      cudaGetLastError();
      msg = std::string("cudaGetSymbolAddress of the static scratch failed: ") + cudaGetErrorString(e);
      return BFGT_ERR_CUDA;
    }
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  return BFGT_OK;
}

}  // namespace

extern "C" int bfgt_noalloc_scratch_bytes(size_t *bytes) {
  if (!bytes) return BFGT_ERR_ARG;
  *bytes = kNoallocScratchBytes;
  return BFGT_OK;
}

extern "C" int bfgt_plan_noalloc_need(bfgt_plan plan, size_t *bytes) {
  if (!plan || !bytes) return BFGT_ERR_ARG;
  const bfgt::DevicePlan &dp = plan->dp;
  *bytes = sizeof(double2) * (size_t)dp.nd * dp.nexp *
           ((size_t)dp.nchunks + 2 * (size_t)dp.ncut + (dp.multi_group ? (size_t)dp.ngroups : 0));
  return BFGT_OK;
}

// defined in capi.cpp: records the message for bfgt_last_error
int bfgt_record_error(int code, const char *msg);

extern "C" int bfgt_plan_execute_noalloc(bfgt_plan plan, const double *d_fvals, double *d_pot, void *stream) {
  if (!plan) return bfgt_record_error(BFGT_ERR_ARG, "plan is NULL");
  if (!d_fvals || !d_pot) return bfgt_record_error(BFGT_ERR_ARG, "fvals/pot device pointers are NULL");
  bfgt::DevicePlan &dp = plan->dp;
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return bfgt_record_error(BFGT_ERR_NODEVICE, "no current CUDA device");
  }
  if (dev != dp.device) return bfgt_record_error(BFGT_ERR_ARG, "the current device is not the plan's device");
  size_t need = 0;
  bfgt_plan_noalloc_need(plan, &need);
  if (need > kNoallocScratchBytes) {
    const std::string m = "plan needs " + std::to_string(need) + " bytes of plane-wave scratch; the static scratch of "
                          "bfgt_plan_execute_noalloc holds " + std::to_string(kNoallocScratchBytes) +
                          " bytes (use bfgt_plan_execute)";
    return bfgt_record_error(BFGT_ERR_CAPACITY, m.c_str());
  }
  std::string msg;
  void *base = nullptr;
  int rc = scratch_for_device(dev, &base, msg);
  if (rc != BFGT_OK) return bfgt_record_error(rc, msg.c_str());
  // same launch sequence as bfgt_plan_execute, with the scratch pointers moved
  // into the static array and no stage events recorded
  bfgt::DevicePlan view = dp;
  view.events = false;
  double2 *sc = static_cast<double2 *>(base);
  const size_t ex = (size_t)dp.nd * dp.nexp;
  view.Mpart = sc;
  view.M = sc + ex * (size_t)dp.nchunks;
  view.L = view.M + ex * (size_t)dp.ncut;
  view.G = dp.multi_group ? view.L + ex * (size_t)dp.ncut : nullptr;
  rc = bfgt::device_plan_execute(view, d_fvals, d_pot, (cudaStream_t)stream, msg);
  if (rc != BFGT_OK) return bfgt_record_error(rc, msg.c_str());
  bfgt_record_error(BFGT_OK, "");
  return BFGT_OK;
}
