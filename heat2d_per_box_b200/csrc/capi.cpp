// C ABI of libbfgt_b200.so (declared in include/bfgt.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cstdint>
#include <initializer_list>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/bfgt.h"
#include "batch.hpp"
#include "device_plan.hpp"
#include "host_plan.hpp"
#include "split_kernels.cuh"
#include "plan_internal.hpp"


struct bfgt_tree_s {
  std::unique_ptr<bfgt::TreeData> t;
};

struct bfgt_batch_s {
  std::vector<bfgt_plan> plans;  // not owned; must outlive the batch
  bfgt::DeviceBatch db;
  std::unique_ptr<bfgt::DeviceBatch> adj;  // the plans' transposed transforms, built on first use
  int device = 0;
};

namespace {

thread_local std::string g_err;

int fail(int code, const std::string &m) {
  g_err = m;
  if (std::getenv("BFGT_ABORT_ON_ERROR")) {
    std::fprintf(stderr, "bfgt: %s\n", m.c_str());
    std::abort();
  }
  return code;
}

bfgt::TreeView make_view(int nboxes, int nlevels, int ltree, int *itree, const int *iptr, const double *centers,
                         const double *boxsize) {
  if (!itree || !iptr || !centers || !boxsize) throw std::runtime_error("null tree array");
  if (iptr[0] != 1 || iptr[1] != 2 * (nlevels + 1) + 1) throw std::runtime_error("iptr(1:2) inconsistent with nlevels");
  const long need = (long)iptr[6] - 1 + 9L * nboxes;
  if (need > ltree) throw std::runtime_error("ltree too small for nboxes");
  if (iptr[2] != iptr[1] + nboxes || iptr[3] != iptr[2] + nboxes || iptr[4] != iptr[3] + nboxes ||
      iptr[5] != iptr[4] + 4 * nboxes || iptr[6] != iptr[5] + nboxes)
    throw std::runtime_error("iptr(3:7) inconsistent with nboxes (expected the vol_tree_build layout)");
  bfgt::TreeView t;
  t.nboxes = nboxes;
  t.nlevels = nlevels;
  t.itree = itree;
  t.iptr = iptr;
  t.centers = centers;
  t.boxsize = boxsize;
  return t;
}

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace

// used by noalloc.cu to report through bfgt_last_error
int bfgt_record_error(int code, const char *msg) {
  if (code == BFGT_OK) {
    g_err.clear();
    return BFGT_OK;
  }
  return fail(code, msg ? msg : "");
}

extern "C" {

const char *bfgt_last_error(void) { return g_err.c_str(); }

int bfgt_plan_create(bfgt_plan *plan, int nd, double delta, double eps, int ipoly, int iperiod, int norder,
                     int nboxes, int nlevels, int ltree, int *itree, const int *iptr, const double *centers,
                     const double *boxsize, int precision) {
  g_err.clear();
  if (!plan) return fail(BFGT_ERR_ARG, "plan pointer is NULL");
  *plan = nullptr;
  if (precision != BFGT_PREC_FP64 && precision != BFGT_PREC_SPLIT) return fail(BFGT_ERR_ARG, "unknown precision mode");
  std::unique_ptr<bfgt_plan_s> p(new bfgt_plan_s());
  bfgt::TreeView t;
  try {
    t = make_view(nboxes, nlevels, ltree, itree, iptr, centers, boxsize);
    bfgt::build_host_plan(p->hp, t, nd, delta, eps, ipoly, iperiod, norder, precision);
    constexpr int kMaxGap = 64;  // non-leaf boxes copied rather than starting a new run
    for (int b = 1; b <= nboxes; b++) {
      if (t.nchild(b) != 0) continue;
      if (!p->leaf_runs.empty() && b - 1 - p->leaf_runs.back().second <= kMaxGap)
        p->leaf_runs.back().second = b;
      else
        p->leaf_runs.emplace_back(b - 1, b);
    }
  } catch (const std::exception &e) {
    return fail(BFGT_ERR_TREE, e.what());
  }
  std::string msg;
  int rc = bfgt::device_plan_create(p->dp, p->hp, msg);
  if (rc == BFGT_OK) rc = bfgt::device_plan_prepare_targets(p->dp, p->hp, t, msg);
  if (rc != BFGT_OK) {
    bfgt::device_plan_destroy(p->dp);
    return fail(rc, msg);
  }
  *plan = p.release();
  return BFGT_OK;
}

}  // extern "C"

namespace {

// Device arrays must live on the plan's device: a kernel reading another
// device's memory (without peer access) or a host array would fault.  With
// one process per GPU this catches a plan made before the caller selected
// its device.  Null pointers are the callers' checks.
int check_device_array(const void *p, int dev, const char *what) {
  if (!p) return BFGT_OK;
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return fail(BFGT_ERR_ARG, std::string(what) + ": not a CUDA allocation");
  }
  if ((at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged) && at.device == dev) return BFGT_OK;
  return fail(BFGT_ERR_ARG, std::string(what) + ": not device memory of the plan's device " + std::to_string(dev));
}

int check_device_arrays(int dev, std::initializer_list<std::pair<const void *, const char *>> arrays) {
  for (const auto &a : arrays) {
    const int rc = check_device_array(a.first, dev, a.second);
    if (rc != BFGT_OK) return rc;
  }
  return BFGT_OK;
}

}  // namespace

extern "C" {

int bfgt_plan_execute(bfgt_plan plan, const double *d_fvals, double *d_pot, void *stream) {
  g_err.clear();
  if (!plan) return fail(BFGT_ERR_ARG, "plan is NULL");
  if (!d_fvals || !d_pot) return fail(BFGT_ERR_ARG, "fvals/pot device pointers are NULL");
  if (check_device_arrays(plan->dp.device, {{d_fvals, "fvals"}, {d_pot, "pot"}}) != BFGT_OK) return BFGT_ERR_ARG;
  std::string msg;
  int rc = bfgt::device_plan_execute(plan->dp, d_fvals, d_pot, (cudaStream_t)stream, msg);
  if (rc != BFGT_OK) return fail(rc, msg);
  return BFGT_OK;
}

}  // extern "C"

namespace {

// True when the n doubles at p are all +0.0 (every bit clear), tested in
// blocks on the host threads.  Only +0.0 counts: -0.0 + x and +0.0 + x differ
// when x is -0.0, so a run holding -0.0 is uploaded like any other.
bool all_zero_bits(const double *p, size_t n) {
  constexpr size_t kBlock = 1 << 16;
  const long nb = (long)((n + kBlock - 1) / kBlock);
  std::atomic<bool> nonzero{false};
#pragma omp parallel for schedule(dynamic, 4) if (nb > 4)
  for (long b = 0; b < nb; b++) {
    if (nonzero.load(std::memory_order_relaxed)) continue;
    const uint64_t *w = reinterpret_cast<const uint64_t *>(p) + (size_t)b * kBlock;
    const size_t m = std::min(kBlock, n - (size_t)b * kBlock);
    uint64_t acc = 0;
    for (size_t i = 0; i < m; i++) acc |= w[i];
    if (acc) nonzero.store(true, std::memory_order_relaxed);
  }
  return !nonzero.load();
}

// Copies between a caller's host arrays and the device.  Page-locked arrays
// are copied directly.  Pageable ones (a Fortran caller's ordinary arrays;
// cudaMemcpyAsync stages those through the driver's own buffers at a fraction
// of the link rate) go through two pinned 8 MB chunks of the plan: the host
// threads fill or drain one chunk while the DMA engine moves the other.
constexpr size_t kStageChunk = 8u << 20;

bool page_locked(const void *p) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeHost;
}

void par_copy(void *dst, const void *src, size_t bytes) {
  constexpr size_t kPart = 1u << 20;
  const long np = (long)((bytes + kPart - 1) / kPart);
#pragma omp parallel for schedule(static) if (np > 1)
  for (long i = 0; i < np; i++) {
    const size_t o = (size_t)i * kPart;
    std::memcpy(static_cast<char *>(dst) + o, static_cast<const char *>(src) + o, std::min(kPart, bytes - o));
  }
}

class Stager {
 public:
  Stager(bfgt::DevicePlan &dp, cudaStream_t s) : dp_(dp), s_(s) {}
  ~Stager() {
    for (cudaEvent_t e : ev_)
      if (e) cudaEventDestroy(e);
  }
  // host -> device (queued on the stream; a pageable source is read before return)
  bool up(double *d, const double *h, size_t bytes) {
    if (page_locked(h)) return cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, s_) == cudaSuccess;
    for (size_t off = 0; off < bytes; off += kStageChunk) {
      const size_t len = std::min(kStageChunk, bytes - off);
      char *b = chunk();
      if (!b) return false;
      par_copy(b, reinterpret_cast<const char *>(h) + off, len);
      if (cudaMemcpyAsync(reinterpret_cast<char *>(d) + off, b, len, cudaMemcpyHostToDevice, s_) != cudaSuccess ||
          cudaEventRecord(ev_[k_ & 1], s_) != cudaSuccess)
        return false;
      used_[k_ & 1] = true;
      k_++;
    }
    return true;
  }
  // device -> host (a pageable destination is written by finish() at the latest)
  bool down(double *h, const double *d, size_t bytes) {
    if (page_locked(h)) return cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, s_) == cudaSuccess;
    for (size_t off = 0; off < bytes; off += kStageChunk) {
      const size_t len = std::min(kStageChunk, bytes - off);
      char *b = chunk();
      if (!b) return false;
      if (cudaMemcpyAsync(b, reinterpret_cast<const char *>(d) + off, len, cudaMemcpyDeviceToHost, s_) != cudaSuccess ||
          cudaEventRecord(ev_[k_ & 1], s_) != cudaSuccess)
        return false;
      used_[k_ & 1] = true;
      // the previous chunk's data, if any, to its host array while this one moves
      if (!drain()) return false;
      pend_ = {reinterpret_cast<char *>(h) + off, b, len, k_ & 1};
      k_++;
    }
    return true;
  }
  bool finish() { return drain(); }

 private:
  struct Pending {
    char *dst = nullptr;
    const char *src = nullptr;
    size_t len = 0;
    int slot = 0;
  };
  // the next free chunk: allocated on first use, reused once its last copy is done
  char *chunk() {
    if (!dp_.h_stage_f) {
      if (cudaHostAlloc(reinterpret_cast<void **>(&dp_.h_stage_f), 2 * kStageChunk, cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        dp_.h_stage_f = nullptr;
        return nullptr;
      }
    }
    const int b = k_ & 1;
    if (!ev_[b] && cudaEventCreateWithFlags(&ev_[b], cudaEventDisableTiming) != cudaSuccess) return nullptr;
    if (used_[b]) {
      if (pend_.dst && pend_.slot == b && !drain()) return nullptr;
      if (cudaEventSynchronize(ev_[b]) != cudaSuccess) return nullptr;
    }
    return reinterpret_cast<char *>(dp_.h_stage_f) + (size_t)b * kStageChunk;
  }
  bool drain() {
    if (!pend_.dst) return true;
    if (cudaEventSynchronize(ev_[pend_.slot]) != cudaSuccess) return false;
    par_copy(pend_.dst, pend_.src, pend_.len);
    pend_ = Pending();
    return true;
  }
  bfgt::DevicePlan &dp_;
  cudaStream_t s_;
  cudaEvent_t ev_[2] = {nullptr, nullptr};
  bool used_[2] = {false, false};
  int k_ = 0;
  Pending pend_;
};

// Device staging arrays of a host-array execute (input, pot; grad and hess
// for ifpgh >= 2), allocated on first use.
int ensure_staging(bfgt::DevicePlan &dp, int ifpgh) {
  const size_t elems = (size_t)dp.nd * dp.n * dp.n * dp.nboxes;
  if (dp.stage_elems < elems) {
    if (dp.d_stage_f) cudaFree(dp.d_stage_f);
    if (dp.d_stage_p) cudaFree(dp.d_stage_p);
    dp.d_stage_f = dp.d_stage_p = nullptr;
    dp.stage_elems = 0;
    if (cudaMalloc(&dp.d_stage_f, elems * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&dp.d_stage_p, elems * sizeof(double)) != cudaSuccess) {
      cudaGetLastError();
      return fail(BFGT_ERR_OOM, "cannot allocate device staging buffers");
    }
    dp.stage_elems = elems;
  }
  if (ifpgh >= 2 && dp.stage_gh_elems < elems) {
    if (dp.d_stage_gh) cudaFree(dp.d_stage_gh);
    dp.d_stage_gh = nullptr;
    dp.stage_gh_elems = 0;
    if (cudaMalloc(&dp.d_stage_gh, 5 * elems * sizeof(double)) != cudaSuccess) {
      cudaGetLastError();
      return fail(BFGT_ERR_OOM, "cannot allocate device staging buffers (grad/hess)");
    }
    dp.stage_gh_elems = elems;
  }
  return BFGT_OK;
}

// The input's leaf runs of a page-locked host array queued for upload into
// dp's staging array (the drop-in entry's speculation on its cached plan).
int stage_input(bfgt_plan plan, bfgt::DevicePlan &dp, const double *in, cudaStream_t s) {
  int rc = ensure_staging(dp, 1);
  if (rc != BFGT_OK) return rc;
  const size_t per = (size_t)dp.nd * dp.n * dp.n;
  for (const auto &r : plan->leaf_runs) {
    const size_t o = per * r.first, c = per * (r.second - r.first) * sizeof(double);
    if (cudaMemcpyAsync(dp.d_stage_f + o, in + o, c, cudaMemcpyHostToDevice, s) != cudaSuccess)
      return fail(BFGT_ERR_CUDA, "host-to-device copy failed");
  }
  return BFGT_OK;
}

// Host-array form of one transform on dp: uploads the leaf runs of the input
// and of the accumulators, runs, and copies the accumulators' leaf runs back.
// With ifpgh >= 2 grad(nd,2,..) and, for 3, hess(nd,3,..) are accumulated too.
// The reference's callers zero pot before every call (hpots2dadap.f:97-101,
// 321-325): an accumulator run that is all +0.0 on the host is cleared on the
// device instead of uploaded, which gives the same sums bit for bit.  The
// zero test runs on the host while the input's upload is in flight (pinned
// input; a pageable one is staged by the copy call first).  input_staged:
// the input's leaf runs are already on their way (stage_input on this plan).
int execute_host_on(bfgt_plan plan, bfgt::DevicePlan &dp, const double *in, double *acc, cudaStream_t s,
                    int ifpgh = 1, double *grad = nullptr, double *hess = nullptr, bool input_staged = false) {
  const size_t elems = (size_t)dp.nd * dp.n * dp.n * dp.nboxes;
  int rs = ensure_staging(dp, ifpgh);
  if (rs != BFGT_OK) return rs;
  double *dg = ifpgh >= 2 ? dp.d_stage_gh : nullptr;
  double *dh = ifpgh == 3 ? dp.d_stage_gh + 2 * elems : nullptr;
  // only the leaf boxes are read (input) and accumulated into
  const size_t per = (size_t)dp.nd * dp.n * dp.n;
  struct Acc {
    double *h, *d;
    size_t k;  // components per point
  };
  std::vector<Acc> accs = {{acc, dp.d_stage_p, 1}};
  if (dg) accs.push_back({grad, dg, 2});
  if (dh) accs.push_back({hess, dh, 3});
  Stager st(dp, s);
  double up = 0;
  for (const auto &r : plan->leaf_runs) {
    const size_t o = per * r.first, c = per * (r.second - r.first) * sizeof(double);
    if (!input_staged && !st.up(dp.d_stage_f + o, in + o, c)) return fail(BFGT_ERR_CUDA, "host-to-device copy failed");
    up += (double)c;
  }
  for (const auto &r : plan->leaf_runs) {
    const size_t o = per * r.first, c = per * (r.second - r.first) * sizeof(double);
    for (const Acc &a : accs) {
      if (all_zero_bits(a.h + a.k * o, a.k * c / sizeof(double))) {
        if (cudaMemsetAsync(a.d + a.k * o, 0, a.k * c, s) != cudaSuccess)
          return fail(BFGT_ERR_CUDA, "device clear failed");
      } else {
        if (!st.up(a.d + a.k * o, a.h + a.k * o, a.k * c)) return fail(BFGT_ERR_CUDA, "host-to-device copy failed");
        up += (double)(a.k * c);
      }
    }
  }
  plan->last_h2d_bytes = up;
  std::string msg;
  int rc = ifpgh >= 2 ? bfgt::device_plan_execute_pgh(dp, ifpgh, dp.d_stage_f, dp.d_stage_p, dg, dh, s, msg)
                      : bfgt::device_plan_execute(dp, dp.d_stage_f, dp.d_stage_p, s, msg);
  if (rc != BFGT_OK) return fail(rc, msg);
  double down = 0;
  for (const auto &r : plan->leaf_runs) {
    const size_t o = per * r.first, c = per * (r.second - r.first) * sizeof(double);
    for (const Acc &a : accs) {
      if (!st.down(a.h + a.k * o, a.d + a.k * o, a.k * c)) return fail(BFGT_ERR_CUDA, "device-to-host copy failed");
      down += (double)(a.k * c);
    }
  }
  if (!st.finish()) return fail(BFGT_ERR_CUDA, "device-to-host copy failed");
  plan->last_d2h_bytes = down;
  if (cudaStreamSynchronize(s) != cudaSuccess) return fail(BFGT_ERR_CUDA, std::string("transform failed: ") + cudaGetErrorString(cudaGetLastError()));
  return BFGT_OK;
}

// Step 11 on the values a host execute left in dp's staging buffers (pot and,
// as ifpghtarg asks, grad and hess): pote/grade/hesse are overwritten.
int targets_host_on(bfgt::DevicePlan &dp, int ifpghtarg, int ntarg, const double *targs, double *pote,
                    double *grade, double *hesse, cudaStream_t s) {
  if (ntarg <= 0) return BFGT_OK;
  const size_t elems = (size_t)dp.nd * dp.n * dp.n * dp.nboxes;
  double *d_t = nullptr, *d_o = nullptr;
  if (cudaMalloc(&d_t, sizeof(double) * 2 * (size_t)ntarg) != cudaSuccess ||
      cudaMalloc(&d_o, sizeof(double) * 3 * (size_t)dp.nd * ntarg) != cudaSuccess) {
    cudaGetLastError();
    if (d_t) cudaFree(d_t);
    return fail(BFGT_ERR_OOM, "cannot allocate target buffers");
  }
  int rc = BFGT_OK;
  std::string msg;
  struct Part {
    int ncomp;
    const double *vals;
    double *out;
  };
  const Part parts[3] = {{1, dp.d_stage_p, pote}, {2, dp.d_stage_gh, grade}, {3, dp.d_stage_gh + 2 * elems, hesse}};
  if (cudaMemcpyAsync(d_t, targs, sizeof(double) * 2 * (size_t)ntarg, cudaMemcpyHostToDevice, s) != cudaSuccess)
    rc = fail(BFGT_ERR_CUDA, "target upload failed");
  for (int p = 0; p < ifpghtarg && rc == BFGT_OK; p++) {
    const Part &pt = parts[p];
    int r = bfgt::device_plan_eval_targets(dp, pt.ncomp, pt.vals, ntarg, d_t, d_o, s, msg);
    if (r != BFGT_OK) rc = fail(r, msg);
    else if (cudaMemcpyAsync(pt.out, d_o, sizeof(double) * pt.ncomp * dp.nd * (size_t)ntarg, cudaMemcpyDeviceToHost,
                             s) != cudaSuccess)
      rc = fail(BFGT_ERR_CUDA, "target download failed");
    else if (cudaStreamSynchronize(s) != cudaSuccess)
      rc = fail(BFGT_ERR_CUDA, std::string("target evaluation failed: ") + cudaGetErrorString(cudaGetLastError()));
  }
  cudaFree(d_t);
  cudaFree(d_o);
  return rc;
}

// Uploads the derivative tables on first use.
int ensure_pgh(bfgt_plan plan) {
  if (plan->dp.pgh_ready) return BFGT_OK;
  std::string msg;
  int rc = bfgt::device_plan_prepare_pgh(plan->dp, plan->hp, msg);
  if (rc != BFGT_OK) return fail(rc, msg);
  return BFGT_OK;
}

// Builds the plan's transposed twin on first use (host tables, then upload).
int ensure_adjoint(bfgt_plan plan) {
  if (plan->adj_dp) return BFGT_OK;
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev != plan->dp.device) {
    cudaGetLastError();
    return fail(BFGT_ERR_ARG, "the current device is not the plan's device");
  }
  std::unique_ptr<bfgt::HostPlan> h(new bfgt::HostPlan());
  try {
    bfgt::build_adjoint_host_plan(*h, plan->hp);
  } catch (const std::exception &e) {
    return fail(BFGT_ERR_TREE, e.what());
  }
  std::unique_ptr<bfgt::DevicePlan> d(new bfgt::DevicePlan());
  std::string msg;
  int rc = bfgt::device_plan_create(*d, *h, msg);
  if (rc != BFGT_OK) {
    bfgt::device_plan_destroy(*d);
    return fail(rc, msg);
  }
  plan->adj_hp = std::move(h);
  plan->adj_dp = std::move(d);
  return BFGT_OK;
}

}  // namespace

extern "C" {

int bfgt_plan_execute_host(bfgt_plan plan, const double *fvals, double *pot, void *stream) {
  g_err.clear();
  if (!plan) return fail(BFGT_ERR_ARG, "plan is NULL");
  if (!fvals || !pot) return fail(BFGT_ERR_ARG, "fvals/pot are NULL");
  return execute_host_on(plan, plan->dp, fvals, pot, (cudaStream_t)stream);
}

int bfgt_plan_execute_pgh(bfgt_plan plan, int ifpgh, const double *d_fvals, double *d_pot, double *d_grad,
                          double *d_hess, void *stream) {
  g_err.clear();
  if (!plan) return fail(BFGT_ERR_ARG, "plan is NULL");
  if (ifpgh < 1 || ifpgh > 3) return fail(BFGT_ERR_ARG, "ifpgh must be 1, 2 or 3");
  if (!d_fvals || !d_pot || (ifpgh >= 2 && !d_grad) || (ifpgh == 3 && !d_hess))
    return fail(BFGT_ERR_ARG, "a device array that ifpgh asks for is NULL");
  if (check_device_arrays(plan->dp.device, {{d_fvals, "fvals"}, {d_pot, "pot"}, {ifpgh >= 2 ? d_grad : nullptr, "grad"},
                                            {ifpgh == 3 ? d_hess : nullptr, "hess"}}) != BFGT_OK)
    return BFGT_ERR_ARG;
  if (ifpgh >= 2) {
    int rc = ensure_pgh(plan);
    if (rc != BFGT_OK) return rc;
  }
  std::string msg;
  int rc = bfgt::device_plan_execute_pgh(plan->dp, ifpgh, d_fvals, d_pot, d_grad, d_hess, (cudaStream_t)stream, msg);
  if (rc != BFGT_OK) return fail(rc, msg);
  return BFGT_OK;
}

int bfgt_plan_execute_pgh_host(bfgt_plan plan, int ifpgh, const double *fvals, double *pot, double *grad,
                               double *hess, void *stream) {
  g_err.clear();
  if (!plan) return fail(BFGT_ERR_ARG, "plan is NULL");
  if (ifpgh < 1 || ifpgh > 3) return fail(BFGT_ERR_ARG, "ifpgh must be 1, 2 or 3");
  if (!fvals || !pot || (ifpgh >= 2 && !grad) || (ifpgh == 3 && !hess))
    return fail(BFGT_ERR_ARG, "an array that ifpgh asks for is NULL");
  if (ifpgh >= 2) {
    int rc = ensure_pgh(plan);
    if (rc != BFGT_OK) return rc;
  }
  return execute_host_on(plan, plan->dp, fvals, pot, (cudaStream_t)stream, ifpgh, grad, hess);
}

int bfgt_plan_eval_targets(bfgt_plan plan, int ncomp, const double *d_vals, int ntarg, const double *d_targs,
                           double *d_out, void *stream) {
  g_err.clear();
  if (!plan) return fail(BFGT_ERR_ARG, "plan is NULL");
  if (ncomp < 1 || ncomp > 3) return fail(BFGT_ERR_ARG, "ncomp must be 1, 2 or 3");
  if (ntarg < 0) return fail(BFGT_ERR_ARG, "ntarg is negative");
  if (ntarg > 0 && (!d_vals || !d_targs || !d_out)) return fail(BFGT_ERR_ARG, "vals/targs/out device pointers are NULL");
  if (ntarg > 0 && check_device_arrays(plan->dp.device, {{d_vals, "vals"}, {d_targs, "targs"}, {d_out, "out"}}) != BFGT_OK)
    return BFGT_ERR_ARG;
  std::string msg;
  int rc = bfgt::device_plan_eval_targets(plan->dp, ncomp, d_vals, ntarg, d_targs, d_out, (cudaStream_t)stream, msg);
  if (rc != BFGT_OK) return fail(rc, msg);
  return BFGT_OK;
}

int bfgt_plan_execute_adjoint(bfgt_plan plan, const double *d_potbar, double *d_fbar, void *stream) {
  g_err.clear();
  if (!plan) return fail(BFGT_ERR_ARG, "plan is NULL");
  if (!d_potbar || !d_fbar) return fail(BFGT_ERR_ARG, "potbar/fbar device pointers are NULL");
  if (check_device_arrays(plan->dp.device, {{d_potbar, "potbar"}, {d_fbar, "fbar"}}) != BFGT_OK) return BFGT_ERR_ARG;
  int rc = ensure_adjoint(plan);
  if (rc != BFGT_OK) return rc;
  std::string msg;
  rc = bfgt::device_plan_execute(*plan->adj_dp, d_potbar, d_fbar, (cudaStream_t)stream, msg);
  if (rc != BFGT_OK) return fail(rc, msg);
  return BFGT_OK;
}

int bfgt_plan_execute_adjoint_host(bfgt_plan plan, const double *potbar, double *fbar, void *stream) {
  g_err.clear();
  if (!plan) return fail(BFGT_ERR_ARG, "plan is NULL");
  if (!potbar || !fbar) return fail(BFGT_ERR_ARG, "potbar/fbar are NULL");
  int rc = ensure_adjoint(plan);
  if (rc != BFGT_OK) return rc;
  return execute_host_on(plan, *plan->adj_dp, potbar, fbar, (cudaStream_t)stream);
}

int bfgt_plan_graph_capture(bfgt_plan plan, const double *d_fvals, double *d_pot, void *stream) {
  g_err.clear();
  if (!plan) return fail(BFGT_ERR_ARG, "plan is NULL");
  if (!d_fvals || !d_pot) return fail(BFGT_ERR_ARG, "fvals/pot device pointers are NULL");
  if (check_device_arrays(plan->dp.device, {{d_fvals, "fvals"}, {d_pot, "pot"}}) != BFGT_OK) return BFGT_ERR_ARG;
  bfgt::DevicePlan &dp = plan->dp;
  cudaStream_t s = (cudaStream_t)stream;
  cudaStream_t cs = s;
  bool own = false;
  if (!cs) {
    if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) return fail(BFGT_ERR_CUDA, "stream create failed");
    own = true;
  }
  if (dp.graph_exec) cudaGraphExecDestroy(dp.graph_exec);
  if (dp.graph) cudaGraphDestroy(dp.graph);
  dp.graph_exec = nullptr;
  dp.graph = nullptr;
  bool ev = dp.events;
  dp.events = false;  // no event records inside the graph
  std::string msg;
  int rc = BFGT_OK;
  if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) != cudaSuccess) rc = BFGT_ERR_CUDA, msg = "begin capture failed";
  if (rc == BFGT_OK) rc = bfgt::device_plan_execute(dp, d_fvals, d_pot, cs, msg);
  cudaGraph_t g = nullptr;
  if (cudaStreamEndCapture(cs, &g) != cudaSuccess && rc == BFGT_OK) rc = BFGT_ERR_CUDA, msg = "end capture failed";
  dp.events = ev;
  if (rc == BFGT_OK && cudaGraphInstantiate(&dp.graph_exec, g, 0) != cudaSuccess) rc = BFGT_ERR_CUDA, msg = "graph instantiate failed";
  dp.graph = g;
  if (own) cudaStreamDestroy(cs);
  if (rc != BFGT_OK) {
    cudaGetLastError();
    return fail(rc, msg);
  }
  return BFGT_OK;
}

int bfgt_plan_graph_launch(bfgt_plan plan, void *stream) {
  g_err.clear();
  if (!plan || !plan->dp.graph_exec) return fail(BFGT_ERR_ARG, "no captured graph on this plan");
  if (cudaGraphLaunch(plan->dp.graph_exec, (cudaStream_t)stream) != cudaSuccess) return fail(BFGT_ERR_CUDA, "graph launch failed");
  return BFGT_OK;
}

int bfgt_plan_stage_ms(bfgt_plan plan, double *out) {
  g_err.clear();
  if (!plan || !out) return fail(BFGT_ERR_ARG, "NULL argument");
  if (bfgt::device_plan_stage_ms(plan->dp, out) != BFGT_OK) return fail(BFGT_ERR_CUDA, "event read-out failed");
  return BFGT_OK;
}

int bfgt_plan_reserve_events(bfgt_plan plan, int n) {
  g_err.clear();
  if (!plan) return fail(BFGT_ERR_ARG, "plan is NULL");
  if (bfgt::device_plan_reserve_events(plan->dp, n) != BFGT_OK) return fail(BFGT_ERR_CUDA, "event creation failed");
  return BFGT_OK;
}

int bfgt_plan_info(bfgt_plan plan, int *out) {
  g_err.clear();
  if (!plan || !out) return fail(BFGT_ERR_ARG, "NULL argument");
  const bfgt::HostPlan &h = plan->hp;
  for (int i = 0; i < 16; i++) out[i] = 0;
  out[0] = h.npwlevel;
  out[1] = h.npw;
  out[2] = h.nlevstart;
  out[3] = h.nlevend;
  out[4] = h.regime;
  out[5] = h.nleafbox;
  out[6] = (int)h.leaves.size();
  out[7] = (int)h.nf_target.size();
  out[8] = (int)h.nf_src.size();
  out[9] = h.mnlist1;
  out[10] = h.iperiod_int;
  out[11] = plan->dp.nchunks;
  // FP64 tile shapes in use (100 tm + 10 tn + tiles per lane), 0 for split plans
  const bool f64 = plan->dp.precision == BFGT_PREC_FP64;
  out[13] = f64 ? 100 * plan->dp.form_tile[0] + 10 * plan->dp.form_tile[1] + plan->dp.form_tile[2] : 0;
  out[14] = f64 ? 100 * plan->dp.eval_tile[0] + 10 * plan->dp.eval_tile[1] + plan->dp.eval_tile[2] : 0;
  out[12] = (!plan->dp.direct_only && plan->dp.nchunks > 0 ? 3 : 0) + (plan->dp.nnf > 0 ? 1 : 0);
  // split kernels' shapes in use (100 eval step group + 10 x tiles per form
  // thread + 1 if the form kernel stages Y as float2), 0 for FP64 plans
  const bfgt::SplitPlan &sp = plan->dp.split;
  out[15] = f64 ? 0 : 1000 * (sp.ehalf ? 1 : 0) + 100 * sp.ebatch + 10 * sp.nt + (sp.yfloat ? 1 : 0);
  return BFGT_OK;
}

int bfgt_plan_work(bfgt_plan plan, double *out) {
  g_err.clear();
  if (!plan || !out) return fail(BFGT_ERR_ARG, "NULL argument");
  out[0] = plan->hp.flops;
  out[1] = plan->hp.bytes;
  out[2] = plan->hp.tc_flops;
  out[3] = plan->hp.points;
  out[4] = plan->hp.flops_form;
  out[5] = plan->hp.flops_eval;
  out[6] = plan->hp.flops_near;
  out[7] = plan->hp.flops_translate;
  out[8] = plan->hp.bytes_form;
  out[9] = plan->hp.bytes_eval;
  out[10] = plan->hp.bytes_near;
  out[11] = plan->dp.split.tc_flops_form;
  out[12] = plan->dp.split.tc_flops_eval;
  out[2] = out[11] + out[12];
  double run_bytes = 0;
  for (const auto &r : plan->leaf_runs) run_bytes += 8.0 * plan->dp.nd * plan->dp.n * plan->dp.n * (r.second - r.first);
  out[13] = 2 * run_bytes;  // bfgt_plan_execute_host: fvals and pot up
  out[14] = run_bytes;      // and pot down
  out[15] = plan->last_h2d_bytes;  // bytes the last host execute uploaded
  return BFGT_OK;
}

int bfgt_plan_autotune(bfgt_plan plan, void *stream, double *report) {
  g_err.clear();
  if (!plan) return fail(BFGT_ERR_ARG, "plan is NULL");
  double rep[4];
  std::string msg;
  int rc = bfgt::device_plan_autotune(plan->dp, (cudaStream_t)stream, report ? report : rep, msg);
  if (rc != BFGT_OK) return fail(rc, msg);
  return BFGT_OK;
}

int bfgt_plan_check(bfgt_plan plan) {
  g_err.clear();
  if (!plan) return fail(BFGT_ERR_ARG, "plan is NULL");
  if (cudaDeviceSynchronize() != cudaSuccess) return fail(BFGT_ERR_CUDA, std::string("device error: ") + cudaGetErrorString(cudaGetLastError()));
  int rc = bfgt::split_check(plan->dp);
  if (rc == BFGT_OK && plan->adj_dp) rc = bfgt::split_check(*plan->adj_dp);
  if (rc == BFGT_ERR_TIMEOUT) return fail(rc, "a bounded device-side wait gave up (tensor-core pipeline)");
  if (rc != BFGT_OK) return fail(rc, "error flag read-out failed");
  return BFGT_OK;
}

int bfgt_plan_set_wait_limit(bfgt_plan plan, unsigned int polls) {
  g_err.clear();
  if (!plan) return fail(BFGT_ERR_ARG, "plan is NULL");
  plan->dp.split.wait_iters = polls == 0xFFFFFFFFu ? bfgt::split_default_wait_iters() : polls;
  if (plan->adj_dp) plan->adj_dp->split.wait_iters = plan->dp.split.wait_iters;
  return BFGT_OK;
}

int bfgt_plan_destroy(bfgt_plan plan) {
  g_err.clear();
  if (!plan) return BFGT_OK;
  bfgt::device_plan_destroy(plan->dp);
  if (plan->adj_dp) bfgt::device_plan_destroy(*plan->adj_dp);
  delete plan;
  return BFGT_OK;
}

}  // extern "C"

namespace {

// ---- plan cache behind boxfgt_ / bfgt_boxfgt ---------------------------------
// The reference's solvers call boxfgt several times per time step on an
// unchanged tree (hpots/hpots2dadap.f:103, 343), each call paying the step-0
// precomputation (boxfgt.f:472-703).  The drop-in entry points keep the plans
// of the last few (tree, delta, eps, order, nd, precision) combinations.  The
// key is the scalar arguments and a copy of the tree arrays that define the
// lists and tables (itree up to its colleague arrays, iptr, centers,
// boxsize), compared exactly; the colleague arrays are left out because every
// call rewrites them (boxfgt.f:516-528) and a hit writes back what a fresh
// plan would.
struct CacheKey {
  int ints[8] = {0};  // nd, ipoly, iperiod, norder, nboxes, nlevels, ltree, precision
  double delta = 0, eps = 0;
  int device = 0;
  std::vector<int> iptr, itree;
  std::vector<double> centers, boxsize;
};

struct CacheEntry {
  CacheKey key;
  std::vector<int> coll;  // itree's colleague arrays as the plan left them
  bfgt_plan plan = nullptr;
  uint64_t last = 0;
  bool hit_last = false;  // its last use was a hit
};

std::mutex g_cache_mu;
std::vector<CacheEntry> g_cache;
uint64_t g_cache_clock = 0, g_cache_hits = 0, g_cache_misses = 0;
double g_last_bytes[2] = {0, 0};  // host<->device bytes of the last drop-in call
int g_default_precision = -1;  // -1: from BFGT_PRECISION at first use

// 16 by default: a solver step calls boxfgt once per delta (an initial-value
// transform and one per Gauss node, per species: hpots2dadap.f:79, 329-346),
// and an LRU cache smaller than that cycle would miss on every call
int cache_capacity() {
  const char *e = std::getenv("BFGT_PLAN_CACHE");
  if (!e || !*e) return 16;
  return std::max(0, std::atoi(e));
}

int default_precision() {
  if (g_default_precision < 0) {
    const char *e = std::getenv("BFGT_PRECISION");
    g_default_precision = (e && std::strcmp(e, "split") == 0) ? BFGT_PREC_SPLIT : BFGT_PREC_FP64;
  }
  return g_default_precision;
}

// Byte-wise equality of two arrays, compared in 256 KB blocks on the host
// threads (the tree arrays of a large tree are several MB).
bool same_bytes(const void *a, const void *b, size_t bytes) {
  constexpr size_t kBlock = 256 * 1024;
  const long nb = (long)((bytes + kBlock - 1) / kBlock);
  if (nb <= 1) return std::memcmp(a, b, bytes) == 0;
  const unsigned char *x = static_cast<const unsigned char *>(a), *y = static_cast<const unsigned char *>(b);
  std::atomic<bool> differ{false};
#pragma omp parallel for schedule(static)
  for (long k = 0; k < nb; k++) {
    if (differ.load(std::memory_order_relaxed)) continue;
    const size_t o = (size_t)k * kBlock;
    if (std::memcmp(x + o, y + o, std::min(kBlock, bytes - o)) != 0) differ.store(true, std::memory_order_relaxed);
  }
  return !differ.load();
}

template <class T>
bool same_array(const std::vector<T> &v, const T *p, size_t n) {
  return v.size() == n && same_bytes(v.data(), p, n * sizeof(T));
}

CacheKey make_key(int nd, double delta, double eps, int ipoly, int iperiod, int norder, int nboxes, int nlevels,
                  int ltree, const int *itree, const int *iptr, const double *centers, const double *boxsize,
                  int precision, int device) {
  CacheKey k;
  const int ints[8] = {nd, ipoly, iperiod, norder, nboxes, nlevels, ltree, precision};
  std::memcpy(k.ints, ints, sizeof(ints));
  k.delta = delta;
  k.eps = eps;
  k.device = device;
  k.iptr.assign(iptr, iptr + 8);
  k.itree.assign(itree, itree + (iptr[5] - 1));  // laddr, ilevel, iparent, nchild, ichild
  k.centers.assign(centers, centers + 2 * (size_t)nboxes);
  k.boxsize.assign(boxsize, boxsize + nlevels + 1);
  return k;
}

// The cheap scalar comparison first, then the arrays.
bool key_matches(const CacheKey &k, int nd, double delta, double eps, int ipoly, int iperiod, int norder, int nboxes,
                 int nlevels, int ltree, const int *itree, const int *iptr, const double *centers,
                 const double *boxsize, int precision, int device) {
  const int ints[8] = {nd, ipoly, iperiod, norder, nboxes, nlevels, ltree, precision};
  if (std::memcmp(k.ints, ints, sizeof(ints)) != 0 || device != k.device) return false;
  if (std::memcmp(&k.delta, &delta, sizeof(double)) != 0 || std::memcmp(&k.eps, &eps, sizeof(double)) != 0)
    return false;
  return same_array(k.iptr, iptr, 8) && same_array(k.boxsize, boxsize, (size_t)nlevels + 1) &&
         same_array(k.itree, itree, (size_t)(iptr[5] - 1)) && same_array(k.centers, centers, 2 * (size_t)nboxes);
}

// The cached plan a call with these scalar arguments will most likely find:
// the only entry with the same scalars, and only if its last use was a hit
// (a solver's steady state).  The drop-in entry starts the input's upload on
// it while the arrays are compared; if the comparison then picks another
// plan, that upload was wasted but harmless (the plan uploads into its own
// staging array, in stream order).
bfgt_plan speculative_plan(int nd, double delta, double eps, int ipoly, int iperiod, int norder, int nboxes,
                           int nlevels, int ltree, int precision) {
  if (cache_capacity() <= 0) return nullptr;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  const int ints[8] = {nd, ipoly, iperiod, norder, nboxes, nlevels, ltree, precision};
  bfgt_plan found = nullptr;
  int n = 0;
  for (const CacheEntry &e : g_cache) {
    if (std::memcmp(e.key.ints, ints, sizeof(ints)) != 0 || e.key.device != dev) continue;
    if (std::memcmp(&e.key.delta, &delta, sizeof(double)) != 0 || std::memcmp(&e.key.eps, &eps, sizeof(double)) != 0)
      continue;
    n++;
    if (e.hit_last) found = e.plan;
  }
  return n == 1 ? found : nullptr;
}

// A plan for these arguments: from the cache (writing the colleague arrays
// back into itree) or newly created (and cached).  *cached tells the caller
// not to destroy it.  Called with g_cache_mu held when caching is on.
int get_plan(bfgt_plan *out, bool *cached, double *precompute_s, int nd, double delta, double eps, int ipoly,
             int iperiod, int norder, int nboxes, int nlevels, int ltree, int *itree, const int *iptr,
             const double *centers, const double *boxsize, int precision) {
  const double t0 = now_s();
  *cached = false;
  const int cap = cache_capacity();
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) cudaGetLastError();
  const bool arrays_ok = itree && iptr && centers && boxsize && iptr[5] >= 1 && iptr[6] >= iptr[5] &&
                         (long)iptr[6] - 1 + 9L * nboxes <= ltree;
  if (cap > 0 && arrays_ok) {
    for (CacheEntry &e : g_cache)
      if (key_matches(e.key, nd, delta, eps, ipoly, iperiod, norder, nboxes, nlevels, ltree, itree, iptr, centers,
                      boxsize, precision, dev)) {
        std::memcpy(itree + iptr[5] - 1, e.coll.data(), sizeof(int) * e.coll.size());
        e.last = ++g_cache_clock;
        e.hit_last = true;
        g_cache_hits++;
        *out = e.plan;
        *cached = true;
        *precompute_s = now_s() - t0;
        return BFGT_OK;
      }
  }
  int rc = bfgt_plan_create(out, nd, delta, eps, ipoly, iperiod, norder, nboxes, nlevels, ltree, itree, iptr, centers,
                            boxsize, precision);
  if (rc != BFGT_OK) return rc;
  *precompute_s = now_s() - t0;
  if (cap > 0 && arrays_ok) {
    g_cache_misses++;
    if ((int)g_cache.size() >= cap) {
      auto victim = std::min_element(g_cache.begin(), g_cache.end(),
                                     [](const CacheEntry &a, const CacheEntry &b) { return a.last < b.last; });
      bfgt_plan_destroy(victim->plan);
      g_cache.erase(victim);
    }
    CacheEntry e;
    e.key = make_key(nd, delta, eps, ipoly, iperiod, norder, nboxes, nlevels, ltree, itree, iptr, centers, boxsize,
                     precision, dev);
    e.coll.assign(itree + iptr[5] - 1, itree + iptr[6] - 1 + 9 * (size_t)nboxes);
    e.plan = *out;
    e.last = ++g_cache_clock;
    g_cache.push_back(std::move(e));
    *cached = true;
  }
  return BFGT_OK;
}

int boxfgt_impl(int nd, double delta, double eps, int ipoly, int iperiod, int norder, int nboxes, int nlevels,
                int ltree, int *itree, const int *iptr, const double *centers, const double *boxsize,
                const double *fvals, int ifpgh, double *pot, double *grad, double *hess, double *timeinfo,
                int precision, int ntarg = 0, const double *targs = nullptr, int ifpghtarg = 0,
                double *pote = nullptr, double *grade = nullptr, double *hesse = nullptr) {
  std::unique_lock<std::mutex> lk(g_cache_mu, std::defer_lock);
  if (cache_capacity() > 0) lk.lock();  // cached plans are shared: one drop-in call at a time
  // the input's upload starts on the plan the call will most likely find, so
  // that it overlaps the comparison of the tree arrays (page-locked input)
  bfgt_plan spec = nullptr;
  if (lk.owns_lock() && fvals && page_locked(fvals)) {
    spec = speculative_plan(nd, delta, eps, ipoly, iperiod, norder, nboxes, nlevels, ltree, precision);
    if (spec && stage_input(spec, spec->dp, fvals, nullptr) != BFGT_OK) {
      spec = nullptr;
      g_err.clear();
    }
  }
  bfgt_plan plan = nullptr;
  bool cached = false;
  double t_pre = 0;
  int rc = get_plan(&plan, &cached, &t_pre, nd, delta, eps, ipoly, iperiod, norder, nboxes, nlevels, ltree, itree,
                    iptr, centers, boxsize, precision);
  if (rc != BFGT_OK) return rc;
  const bool staged = spec != nullptr && plan == spec;
  {
    double drop[8];
    bfgt::device_plan_stage_ms(plan->dp, drop);  // stage times of earlier calls on a cached plan
  }
  // as boxfgt.f:207-276: when the targets ask for more derivatives than the
  // boxes, the transform computes them into zeroed internal arrays
  const int ifpgh2 = std::max(ifpgh, ifpghtarg);
  const size_t elems = (size_t)nd * norder * norder * nboxes;
  std::vector<double> g2, h2;
  double *gp = grad, *hp = hess;
  if (ifpgh2 >= 2 && ifpgh < 2) {
    g2.assign(2 * elems, 0.0);
    gp = g2.data();
  }
  if (ifpgh2 == 3 && ifpgh < 3) {
    h2.assign(3 * elems, 0.0);
    hp = h2.data();
  }
  if (!fvals || !pot || (ifpgh2 >= 2 && !gp) || (ifpgh2 == 3 && !hp))
    rc = fail(BFGT_ERR_ARG, "an array that ifpgh asks for is NULL");
  if (rc == BFGT_OK && ifpgh2 >= 2) rc = ensure_pgh(plan);
  if (rc == BFGT_OK) rc = execute_host_on(plan, plan->dp, fvals, pot, nullptr, ifpgh2, gp, hp, staged);
  {
    std::unique_lock<std::mutex> lb(g_cache_mu, std::defer_lock);
    if (!lk.owns_lock()) lb.lock();
    g_last_bytes[0] = plan->last_h2d_bytes;
    g_last_bytes[1] = plan->last_d2h_bytes;
  }
  const double t2 = now_s();
  if (rc == BFGT_OK && ifpghtarg > 0) rc = targets_host_on(plan->dp, ifpghtarg, ntarg, targs, pote, grade, hesse, nullptr);
  const double t_targ = now_s() - t2;
  if (rc == BFGT_OK) rc = bfgt_plan_check(plan);
  if (rc == BFGT_OK && timeinfo) {
    double st[8];
    bfgt::device_plan_stage_ms(plan->dp, st);
    for (int i = 0; i < 20; i++) timeinfo[i] = 0;
    timeinfo[0] = t_pre;             // step 0: precomputation (near zero on a cached plan)
    timeinfo[1] = st[0] * 1e-3;      // steps 1+2: leaf -> cutoff expansions
    timeinfo[2] = st[1] * 1e-3;      // fixed-order partial-sum reduction
    timeinfo[3] = st[2] * 1e-3;      // step 3: cutoff translations
    timeinfo[4] = 0;                 // step 4 is fused into step 5
    timeinfo[5] = st[3] * 1e-3;      // steps 4+5: cutoff expansions -> leaf values
    timeinfo[6] = st[4] * 1e-3;      // step 6: near field
    timeinfo[11] = ifpghtarg > 0 ? t_targ : 0;  // step 11: extra targets
  }
  if (!cached) {
    std::string keep = g_err;
    bfgt_plan_destroy(plan);
    g_err = keep;
  }
  return rc;
}

}  // namespace

extern "C" {

int bfgt_boxfgt(int nd, double delta, double eps, int ipoly, int iperiod, int norder, int nboxes, int nlevels,
                int ltree, int *itree, const int *iptr, const double *centers, const double *boxsize,
                const double *fvals, double *pot, double *timeinfo, int precision) {
  return boxfgt_impl(nd, delta, eps, ipoly, iperiod, norder, nboxes, nlevels, ltree, itree, iptr, centers, boxsize,
                     fvals, 1, pot, nullptr, nullptr, timeinfo, precision);
}

void boxfgt_(const int *nd, const int *ndim, const double *delta, const double *eps, const int *ipoly, int *iperiod,
             const int *norder, const int *npbox, int *nboxes, int *nlevels, int *ltree, int *itree, int *iptr,
             double *centers, double *boxsize, const double *fvals, const int *ifpgh, double *pot, double *grad,
             double *hess, const int *ifnewtree, const int *ntarg, const double *targs, const int *ifpghtarg,
             double *pote, double *grade, double *hesse, double *timeinfo) {
  g_err.clear();
  if (!nd || !ndim || !delta || !eps || !ipoly || !iperiod || !norder || !npbox || !nboxes || !nlevels || !ltree ||
      !ifpgh || !ifnewtree || !ntarg || !ifpghtarg) {
    fail(BFGT_ERR_ARG, "boxfgt_: NULL scalar argument");
    return;
  }
  if (*ndim != 2) {
    fail(BFGT_ERR_ARG, "boxfgt_: only ndim=2 is supported");
    return;
  }
  if (*ifpgh < 1 || *ifpgh > 3 || *ifpghtarg < 0 || *ifpghtarg > 3 || *ifnewtree != 0) {
    fail(BFGT_ERR_ARG, "boxfgt_: only ifpgh=1,2,3, ifpghtarg=0..3 with ifnewtree=0 are supported");
    return;
  }
  if ((*ifpgh >= 2 && !grad) || (*ifpgh == 3 && !hess)) {
    fail(BFGT_ERR_ARG, "boxfgt_: grad/hess arrays are NULL");
    return;
  }
  if (*ifpghtarg > 0 && *ntarg > 0 &&
      (!targs || !pote || (*ifpghtarg >= 2 && !grade) || (*ifpghtarg == 3 && !hesse))) {
    fail(BFGT_ERR_ARG, "boxfgt_: targs/pote/grade/hesse arrays are NULL");
    return;
  }
  if (*npbox != (*norder) * (*norder)) {
    fail(BFGT_ERR_ARG, "boxfgt_: npbox must equal norder**2");
    return;
  }
  double ti[20];
  int prec = BFGT_PREC_FP64;
  {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    prec = default_precision();
  }
  int rc = boxfgt_impl(*nd, *delta, *eps, *ipoly, *iperiod, *norder, *nboxes, *nlevels, *ltree, itree, iptr, centers,
                       boxsize, fvals, *ifpgh, pot, grad, hess, timeinfo ? timeinfo : ti, prec, *ntarg, targs,
                       *ifpghtarg, pote, grade, hesse);
  // split precision serves norder 8 and 16, npw <= 64 and eps >= 1e-11; other
  // calls run in FP64, which meets every eps
  if (rc == BFGT_ERR_CAPACITY && prec == BFGT_PREC_SPLIT)
    boxfgt_impl(*nd, *delta, *eps, *ipoly, *iperiod, *norder, *nboxes, *nlevels, *ltree, itree, iptr, centers, boxsize,
                fvals, *ifpgh, pot, grad, hess, timeinfo ? timeinfo : ti, BFGT_PREC_FP64, *ntarg, targs, *ifpghtarg,
                pote, grade, hesse);
}

int bfgt_set_default_precision(int precision) {
  g_err.clear();
  if (precision != BFGT_PREC_FP64 && precision != BFGT_PREC_SPLIT) return fail(BFGT_ERR_ARG, "unknown precision mode");
  std::lock_guard<std::mutex> lk(g_cache_mu);
  g_default_precision = precision;
  return BFGT_OK;
}

int bfgt_plan_cache_clear(void) {
  g_err.clear();
  std::lock_guard<std::mutex> lk(g_cache_mu);
  for (CacheEntry &e : g_cache) bfgt_plan_destroy(e.plan);
  g_cache.clear();
  return BFGT_OK;
}

int bfgt_boxfgt_last_bytes(double *out) {
  g_err.clear();
  if (!out) return fail(BFGT_ERR_ARG, "NULL argument");
  std::lock_guard<std::mutex> lk(g_cache_mu);
  out[0] = g_last_bytes[0];
  out[1] = g_last_bytes[1];
  return BFGT_OK;
}

int bfgt_plan_cache_info(int64_t *out) {
  g_err.clear();
  if (!out) return fail(BFGT_ERR_ARG, "NULL argument");
  std::lock_guard<std::mutex> lk(g_cache_mu);
  out[0] = (int64_t)g_cache.size();
  out[1] = (int64_t)cache_capacity();
  out[2] = (int64_t)g_cache_hits;
  out[3] = (int64_t)g_cache_misses;
  return BFGT_OK;
}

int bfgt_host_plan_dump(int nd, double delta, double eps, int ipoly, int iperiod, int norder, int nboxes,
                        int nlevels, int ltree, int *itree, const int *iptr, const double *centers,
                        const double *boxsize, int *info, int *ifpwexp, int *nlist1, int *list1, int mnlist1_cap,
                        int *nlistpw, int *listpw, int *ind_loc, double *tab_loc, double *ts, double *ws) {
  g_err.clear();
  bfgt::HostPlan hp;
  try {
    bfgt::TreeView t = make_view(nboxes, nlevels, ltree, itree, iptr, centers, boxsize);
    bfgt::build_host_plan(hp, t, nd, delta, eps, ipoly, iperiod, norder, BFGT_PREC_FP64);
  } catch (const std::exception &e) {
    return fail(BFGT_ERR_TREE, e.what());
  }
  if (info) {
    for (int i = 0; i < 16; i++) info[i] = 0;
    info[0] = hp.npwlevel;
    info[1] = hp.npw;
    info[2] = hp.nlevstart;
    info[3] = hp.nlevend;
    info[4] = hp.regime;
    info[5] = hp.nleafbox;
    info[6] = (int)hp.leaves.size();
    info[7] = (int)hp.nf_target.size();
    info[8] = (int)hp.nf_src.size();
    info[9] = hp.mnlist1;
    info[10] = hp.iperiod_int;
    info[11] = (int)hp.chunks.size();
  }
  if (ifpwexp) std::memcpy(ifpwexp, hp.ifpwexp.data(), sizeof(int) * nboxes);
  if (nlist1) std::memcpy(nlist1, hp.nlist1.data(), sizeof(int) * nboxes);
  if (list1) {
    if (mnlist1_cap < hp.mnlist1) return fail(BFGT_ERR_ARG, "mnlist1_cap smaller than mnlist1");
    for (int b = 0; b < nboxes; b++)
      for (int j = 0; j < hp.nlist1[b]; j++) list1[(size_t)mnlist1_cap * b + j] = hp.list1[(size_t)hp.mnlist1 * b + j];
  }
  if (nlistpw) {
    if (hp.nlistpw.empty()) std::memset(nlistpw, 0, sizeof(int) * nboxes);
    else std::memcpy(nlistpw, hp.nlistpw.data(), sizeof(int) * nboxes);
  }
  if (listpw && !hp.listpw.empty()) std::memcpy(listpw, hp.listpw.data(), sizeof(int) * 8 * (size_t)nboxes);
  if (ind_loc) std::memcpy(ind_loc, hp.ind_loc.data(), sizeof(int) * hp.ind_loc.size());
  if (tab_loc) std::memcpy(tab_loc, hp.tab_loc.data(), sizeof(double) * hp.tab_loc.size());
  if (ts && !hp.ts.empty()) std::memcpy(ts, hp.ts.data(), sizeof(double) * hp.ts.size());
  if (ws && !hp.ws.empty()) std::memcpy(ws, hp.ws.data(), sizeof(double) * hp.ws.size());
  return BFGT_OK;
}

int bfgt_tree_build_gauss(bfgt_tree *tree, int ipoly, int iperiod, double eps, double boxlen, int norder, double eta,
                          int ng, const double *gauss, int minlev, int maxlev) {
  g_err.clear();
  if (!tree) return fail(BFGT_ERR_ARG, "tree pointer is NULL");
  *tree = nullptr;
  try {
    auto *h = new bfgt_tree_s();
    h->t.reset(bfgt::tree_build(ipoly, iperiod, eps, boxlen, norder, eta, ng, gauss, minlev, maxlev, false));
    *tree = h;
  } catch (const std::exception &e) {
    return fail(BFGT_ERR_ARG, e.what());
  }
  return BFGT_OK;
}

int bfgt_tree_build_uniform(bfgt_tree *tree, int ipoly, int iperiod, double boxlen, int norder, int nlev, int ng,
                            const double *gauss) {
  g_err.clear();
  if (!tree) return fail(BFGT_ERR_ARG, "tree pointer is NULL");
  *tree = nullptr;
  try {
    auto *h = new bfgt_tree_s();
    h->t.reset(bfgt::tree_build(ipoly, iperiod, 1.0, boxlen, norder, 0.0, ng, gauss, nlev, nlev, true));
    *tree = h;
  } catch (const std::exception &e) {
    return fail(BFGT_ERR_ARG, e.what());
  }
  return BFGT_OK;
}

int bfgt_tree_sizes(bfgt_tree tree, int *nboxes, int *nlevels, int *ltree) {
  g_err.clear();
  if (!tree) return fail(BFGT_ERR_ARG, "tree is NULL");
  if (nboxes) *nboxes = tree->t->nboxes;
  if (nlevels) *nlevels = tree->t->nlevels;
  if (ltree) *ltree = (int)tree->t->itree.size();
  return BFGT_OK;
}

int bfgt_tree_export(bfgt_tree tree, int *itree, int *iptr, double *centers, double *boxsize, double *fvals) {
  g_err.clear();
  if (!tree) return fail(BFGT_ERR_ARG, "tree is NULL");
  const bfgt::TreeData &t = *tree->t;
  if (itree) std::memcpy(itree, t.itree.data(), sizeof(int) * t.itree.size());
  if (iptr) std::memcpy(iptr, t.iptr, sizeof(int) * 8);
  if (centers) std::memcpy(centers, t.centers.data(), sizeof(double) * t.centers.size());
  if (boxsize) std::memcpy(boxsize, t.boxsize.data(), sizeof(double) * t.boxsize.size());
  if (fvals) std::memcpy(fvals, t.fvals.data(), sizeof(double) * t.fvals.size());
  return BFGT_OK;
}

int bfgt_tree_free(bfgt_tree tree) {
  delete tree;
  return BFGT_OK;
}

int bfgt_batch_create(bfgt_batch *batch, int nplans, const bfgt_plan *plans) {
  g_err.clear();
  if (!batch) return fail(BFGT_ERR_ARG, "batch pointer is NULL");
  *batch = nullptr;
  if (nplans <= 0 || !plans) return fail(BFGT_ERR_ARG, "a batch needs at least one plan");
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return fail(BFGT_ERR_NODEVICE, "no current CUDA device");
  }
  std::unique_ptr<bfgt_batch_s> b(new bfgt_batch_s());
  std::vector<bfgt::DevicePlan *> dps;
  for (int i = 0; i < nplans; i++) {
    if (!plans[i]) return fail(BFGT_ERR_ARG, "plan " + std::to_string(i) + " is NULL");
    if (plans[i]->dp.device != dev) return fail(BFGT_ERR_ARG, "plan " + std::to_string(i) + " is on another device");
    // a plan owns its expansion scratch and arrival counters: two entries of
    // one plan in a launch would mix their partial sums
    for (int j = 0; j < i; j++)
      if (plans[j] == plans[i])
        return fail(BFGT_ERR_ARG, "plan " + std::to_string(i) + " repeats plan " + std::to_string(j) +
                                      " (each entry of a batch needs its own plan)");
    b->plans.push_back(plans[i]);
    dps.push_back(&plans[i]->dp);
  }
  b->device = dev;
  std::string msg;
  int rc = bfgt::device_batch_create(b->db, dps, msg);
  if (rc != BFGT_OK) {
    bfgt::device_batch_destroy(b->db);
    return fail(rc, msg);
  }
  *batch = b.release();
  return BFGT_OK;
}

int bfgt_batch_layout(bfgt_batch batch, int64_t *offsets) {
  g_err.clear();
  if (!batch || !offsets) return fail(BFGT_ERR_ARG, "NULL argument");
  for (size_t i = 0; i < batch->db.offs.size(); i++) offsets[i] = batch->db.offs[i];
  return BFGT_OK;
}

int bfgt_batch_execute(bfgt_batch batch, const double *d_fvals, double *d_pot, void *stream) {
  g_err.clear();
  if (!batch) return fail(BFGT_ERR_ARG, "batch is NULL");
  if (!d_fvals || !d_pot) return fail(BFGT_ERR_ARG, "fvals/pot device pointers are NULL");
  if (check_device_arrays(batch->device, {{d_fvals, "fvals"}, {d_pot, "pot"}}) != BFGT_OK)
    return BFGT_ERR_ARG;
  std::string msg;
  int rc = bfgt::device_batch_execute(batch->db, d_fvals, d_pot, (cudaStream_t)stream, msg);
  if (rc != BFGT_OK) return fail(rc, msg);
  return BFGT_OK;
}

int bfgt_batch_execute_adjoint(bfgt_batch batch, const double *d_potbar, double *d_fbar, void *stream) {
  g_err.clear();
  if (!batch) return fail(BFGT_ERR_ARG, "batch is NULL");
  if (!d_potbar || !d_fbar) return fail(BFGT_ERR_ARG, "potbar/fbar device pointers are NULL");
  if (check_device_arrays(batch->device, {{d_potbar, "potbar"}, {d_fbar, "fbar"}}) != BFGT_OK)
    return BFGT_ERR_ARG;
  if (!batch->adj) {
    std::vector<bfgt::DevicePlan *> dps;
    for (bfgt_plan p : batch->plans) {
      int rc = ensure_adjoint(p);
      if (rc != BFGT_OK) return rc;
      dps.push_back(p->adj_dp.get());
    }
    std::unique_ptr<bfgt::DeviceBatch> b(new bfgt::DeviceBatch());
    std::string msg;
    int rc = bfgt::device_batch_create(*b, dps, msg);
    if (rc != BFGT_OK) {
      bfgt::device_batch_destroy(*b);
      return fail(rc, msg);
    }
    batch->adj = std::move(b);
  }
  std::string msg;
  int rc = bfgt::device_batch_execute(*batch->adj, d_potbar, d_fbar, (cudaStream_t)stream, msg);
  if (rc != BFGT_OK) return fail(rc, msg);
  return BFGT_OK;
}

int bfgt_batch_graph_capture(bfgt_batch batch, const double *d_fvals, double *d_pot, void *stream) {
  g_err.clear();
  if (!batch) return fail(BFGT_ERR_ARG, "batch is NULL");
  if (!d_fvals || !d_pot) return fail(BFGT_ERR_ARG, "fvals/pot device pointers are NULL");
  if (check_device_arrays(batch->device, {{d_fvals, "fvals"}, {d_pot, "pot"}}) != BFGT_OK)
    return BFGT_ERR_ARG;
  bfgt::DeviceBatch &db = batch->db;
  cudaStream_t cs = (cudaStream_t)stream;
  bool own = false;
  if (!cs) {
    if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) return fail(BFGT_ERR_CUDA, "stream create failed");
    own = true;
  }
  if (db.graph_exec) cudaGraphExecDestroy(db.graph_exec);
  if (db.graph) cudaGraphDestroy(db.graph);
  db.graph_exec = nullptr;
  db.graph = nullptr;
  const bool ev = db.events;
  db.events = false;  // no event records inside the graph
  std::string msg;
  int rc = BFGT_OK;
  if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) != cudaSuccess) rc = BFGT_ERR_CUDA, msg = "begin capture failed";
  if (rc == BFGT_OK) rc = bfgt::device_batch_execute(db, d_fvals, d_pot, cs, msg);
  cudaGraph_t g = nullptr;
  if (cudaStreamEndCapture(cs, &g) != cudaSuccess && rc == BFGT_OK) rc = BFGT_ERR_CUDA, msg = "end capture failed";
  db.events = ev;
  if (rc == BFGT_OK && cudaGraphInstantiate(&db.graph_exec, g, 0) != cudaSuccess) rc = BFGT_ERR_CUDA, msg = "graph instantiate failed";
  db.graph = g;
  if (own) cudaStreamDestroy(cs);
  if (rc != BFGT_OK) {
    cudaGetLastError();
    return fail(rc, msg);
  }
  return BFGT_OK;
}

int bfgt_batch_graph_launch(bfgt_batch batch, void *stream) {
  g_err.clear();
  if (!batch || !batch->db.graph_exec) return fail(BFGT_ERR_ARG, "no captured graph on this batch");
  if (cudaGraphLaunch(batch->db.graph_exec, (cudaStream_t)stream) != cudaSuccess) return fail(BFGT_ERR_CUDA, "graph launch failed");
  return BFGT_OK;
}

int bfgt_batch_stage_ms(bfgt_batch batch, double *out) {
  g_err.clear();
  if (!batch || !out) return fail(BFGT_ERR_ARG, "NULL argument");
  if (bfgt::device_batch_stage_ms(batch->db, out) != BFGT_OK) return fail(BFGT_ERR_CUDA, "event read-out failed");
  return BFGT_OK;
}

int bfgt_batch_info(bfgt_batch batch, int *out) {
  g_err.clear();
  if (!batch || !out) return fail(BFGT_ERR_ARG, "NULL argument");
  for (int i = 0; i < 8; i++) out[i] = 0;
  const bfgt::DeviceBatch &db = batch->db;
  out[0] = (int)batch->plans.size();
  out[1] = bfgt::device_batch_launches(db);
  for (const auto &g : db.split.form_groups) out[2] += g.count;
  for (const auto &g : db.split.eval_groups) out[3] += g.count;
  out[4] = db.tr_blocks;
  out[5] = db.nf_blocks;
  return BFGT_OK;
}

int bfgt_batch_check(bfgt_batch batch) {
  g_err.clear();
  if (!batch) return fail(BFGT_ERR_ARG, "batch is NULL");
  for (bfgt_plan p : batch->plans) {
    int rc = bfgt_plan_check(p);
    if (rc != BFGT_OK) return rc;
  }
  return BFGT_OK;
}

int bfgt_batch_destroy(bfgt_batch batch) {
  g_err.clear();
  if (!batch) return BFGT_OK;
  bfgt::device_batch_destroy(batch->db);
  if (batch->adj) bfgt::device_batch_destroy(*batch->adj);
  delete batch;
  return BFGT_OK;
}

}  // extern "C"
