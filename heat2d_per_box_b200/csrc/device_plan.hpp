// Device half of a box-FGT plan: the uploaded tables and work lists, and the
// launch sequence of one transform.
#pragma once
#include <cuda_runtime.h>

#include <array>
#include <cstdint>
#include <vector>

#include "host_plan.hpp"

namespace bfgt {

// Tensor-core (split precision) part of a plan.
struct SplitPlan {
  int cpc = 0, KA = 0, NP = 0, KH = 0, KE = 0, NB = 0, nt = 0, nchunks = 0;
  int lslots = 1;  // densities whose L the eval kernel holds in shared memory at once
  int ebatch = 8;  // steps per tensor-core group of the eval kernel (8, or 4)
  bool yfloat = false;  // the form kernel stages Y as float2 (exact: an FP32 sum)
  // operand slices: three floating ones, or S fixed-point digits (eps < 1e-7)
  bool fixed = false;
  int S = 3;
  double *csc = nullptr, *esc = nullptr;  // fixed-point column scales of Ty, Ey per level
  // work items {chunk, pass} when densities are packed (nd > 1): one CTA per
  // pass of a chunk; null: one CTA per chunk running all its passes
  int2 *items = nullptr;
  int nitems = 0, items_nd = 0;  // items_nd: the density count the passes were cut for
  int4 *chunks = nullptr;
  int *step_begin = nullptr, *steps = nullptr;
  // the eval kernel's alternative work: every column group of the chunks cut
  // into two halves (twice the CTAs, each with half the rows); used when
  // ehalf is set (the autotuner's choice), else the eval runs the chunks
  int4 *echunks = nullptr;
  int *estep_begin = nullptr, *esteps = nullptr;
  int2 *eitems = nullptr;
  int nechunks = 0, neitems = 0;
  bool ehalf = false;
  uint16_t *TyB = nullptr, *EyB = nullptr;
  long long *tyb_off = nullptr, *eyb_off = nullptr;
  long long tyb_tile = 0, eyb_tile = 0;
  int *err = nullptr;
  uint32_t wait_iters = 0;
  size_t smem_form = 0, smem_eval = 0;
  double tc_flops_form = 0, tc_flops_eval = 0;
};

// Tensor-core near field of a split plan (near_tc.cuh); empty when the FP64
// near-field kernel serves the plan.
struct NearTcPlan {
  int4 *ctas = nullptr, *tiles = nullptr, *blocks = nullptr;
  int *targets = nullptr, *slot_q = nullptr;
  uint16_t *tabB = nullptr;  // split plans: BF16 slices of the tables
  double *tabD = nullptr;    // FP64 plans (and fixed-point split plans): the tables in FP64
  bool fp64 = false;         // which of the two kernels runs the lists
  int nctas = 0, maxslot = 0;
  size_t smem = 0;
};

struct DevicePlan {
  int device = 0;
  int nd = 1, n = 0, npw = 0, hh = 0, nexp = 0, nlevels = 0, nboxes = 0, precision = 0;
  int ncut = 0, nchunks = 0, nleaves = 0, nnf = 0, nnf_entries = 0;
  bool direct_only = false;
  // plane-wave part
  double2 *T = nullptr;         // tab_poly2pw, per level (n, npw)
  double2 *E = nullptr;         // tab_pw2pot, per level (npw, n)
  double2 *PH = nullptr;        // phase tables
  long long *ph_off = nullptr;  // per level offsets into PH
  int4 *leaves = nullptr;       // {box, ox, oy, level}
  int4 *chunks = nullptr;       // {column begin, column end, icut, level}
  int4 *columns = nullptr;      // {leaf begin, leaf end, ox, -}
  // the FP64 kernels' columns: the same, with a column of more than 64 leaves
  // cut into sub-columns of up to 64 (dp.chunks index into these)
  int4 *columns64 = nullptr;
  int ncolumns = 0;
  int form_tile[3] = {0, 0, 0}, eval_tile[3] = {0, 0, 0};
  int *cut_chunk_begin = nullptr, *cut_pw_begin = nullptr, *cut_pw_src = nullptr, *cut_pw_ind = nullptr;
  double2 *W = nullptr;         // cutoff shifts (nexp, 9)
  double *pw_weight = nullptr;  // (hh)
  double *kscale = nullptr;     // (hh) translation factor per k2, or null
  // gradient / hessian outputs (built on first use): per-element derivative
  // factors (5, nexp) for x, y, xx, xy, yy; scratch for the derivative local
  // expansions (ncut, 3 nd, nexp); the near tables with their first and
  // second derivatives appended
  double2 *dfac = nullptr, *Ld = nullptr;
  double *tab3_loc = nullptr;
  bool pgh_ready = false;
  // extra targets (built on first use): the tree on the device (0-based box
  // ids), the values->coefficients matrix, and scratch
  int *t_nchild = nullptr, *t_ichild = nullptr, *t_level = nullptr, *t_has = nullptr, *t_leaf = nullptr;
  double *t_centers = nullptr, *t_boxsize = nullptr, *t_umat = nullptr, *t_coefs = nullptr;
  size_t t_coef_elems = 0;
  int t_leaf_cap = 0, ipoly = 0;
  bool targ_ready = false;
  NearTcPlan ntc;
  double2 *Mpart = nullptr;     // (nchunks, nd, nexp) partial expansions per chunk
  double2 *M = nullptr;         // (ncut, nd, nexp) cutoff-box expansions
  double2 *L = nullptr;         // (ncut, nd, nexp) cutoff-box local expansions
  double2 *G = nullptr;         // (ngroups, nd, nexp) group sums (boxes with > 32 chunks)
  int *gcnt = nullptr, *bcnt = nullptr, *chunk_group = nullptr, *box_groups = nullptr;
  int4 *groups = nullptr;
  int ngroups = 0;
  bool multi_group = false;
  SplitPlan split;
  // near field
  int *nf_target = nullptr, *nf_begin = nullptr, *nf_src = nullptr;
  int2 *nf_ixy = nullptr;
  double *tab_loc = nullptr;
  int *ind_loc = nullptr;
  // staging for host-buffer execution
  // pinned host chunks (2 x 8 MB) through which the host-array entry points
  // copy pageable caller arrays; allocated on first use
  double *h_stage_f = nullptr;
  double *d_stage_f = nullptr, *d_stage_p = nullptr;
  size_t stage_elems = 0;
  double *d_stage_gh = nullptr;  // grad (2 x) and hess (3 x) staging, 5 * stage_gh_elems
  size_t stage_gh_elems = 0;
  // timing: one set of stage events per execute since the last read-out
  std::vector<std::array<cudaEvent_t, 6>> evsets;
  int nrec = 0;
  bool events = false;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  size_t smem_form = 0, smem_eval = 0, smem_near = 0;
};

struct ReduceArgs;
// (Re)builds the reduction groups for a chunk list sorted by cutoff box.
// arrivals: CTAs that write each chunk's partials (empty: one per chunk)
int build_reduce_groups(DevicePlan &dp, const std::vector<int> &cut_of_chunk, std::string &msg,
                        const std::vector<int> &arrivals = {});

// Allocates and uploads; returns a BFGT_* status and fills msg on failure.
int device_plan_create(DevicePlan &dp, const HostPlan &hp, std::string &msg);
void device_plan_destroy(DevicePlan &dp);
// Times every compiled FP64 tile shape of the form and eval kernels on this
// plan's work (scratch inputs; the caller's arrays are not touched), keeps the
// fastest and remembers it for later plans of the same (norder, npw, nd).
// report: best form ms, best eval ms, form and eval candidates timed.
// Split-precision plans go to split_autotune (the form kernel's Y staging and
// x tiles, the eval kernel's step groups and column halves; same bits).
int device_plan_autotune(DevicePlan &dp, cudaStream_t s, double *report, std::string &msg);
// Uploads the derivative tables used by device_plan_execute_pgh.
int device_plan_prepare_pgh(DevicePlan &dp, const HostPlan &hp, std::string &msg);
// pot += K f and, for ifpgh >= 2, grad(nd,2,npbox,nboxes) += grad K f, for
// ifpgh = 3 also hess(nd,3,npbox,nboxes) (xx, xy, yy).
int device_plan_execute_pgh(DevicePlan &dp, int ifpgh, const double *d_fvals, double *d_pot, double *d_grad,
                            double *d_hess, cudaStream_t stream, std::string &msg);
// Uploads the tree arrays used by device_plan_eval_targets.
int device_plan_prepare_targets(DevicePlan &dp, const HostPlan &hp, const TreeView &t, std::string &msg);
// out(nd*ncomp, nt) = the leaf interpolant of vals(nd*ncomp, n*n, nboxes) at
// targs(2, nt) (boxfgt.f step 11).  Grows its scratch when needed.
int device_plan_eval_targets(DevicePlan &dp, int ncomp, const double *d_vals, int nt, const double *d_targs,
                             double *d_out, cudaStream_t s, std::string &msg);
// Queues the transform on stream; returns BFGT_* status.
int device_plan_execute(DevicePlan &dp, const double *d_fvals, double *d_pot, cudaStream_t stream,
                        std::string &msg);
// Makes sure at least n event sets exist (no event creation inside timed loops).
int device_plan_reserve_events(DevicePlan &dp, int n);
// Sums the stage times of every execute since the last call; out[0..4] stage
// ms, out[5] total ms, out[6] number of executes summed.
int device_plan_stage_ms(DevicePlan &dp, double *out);

}  // namespace bfgt
