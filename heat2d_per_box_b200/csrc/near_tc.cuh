// Near field (step 6) of split-precision plans on the tensor cores.
//
// For a target leaf t and each entry p of its list1 the reference adds
// (g2d_tens_prod_to_potloc, bfgt/bfgt_local.f:315-375; loop boxfgt.f:915-1071)
//   pot_t(k1,k2) += sum_{j1,j2} tx_p(j1,k1) ty_p(j2,k2) F_p(j1,j2)
// with the banded 1D tables tx_p = tab_loc(:,:,ix_p), ty_p = tab_loc(:,:,iy_p)
// of the target's level.  Here the tables are dense n x n operands with the
// entries outside the band pattern set to zero (so exactly the reference's
// banded sums), and the two contractions are tcgen05 MMAs (BF16 x 3 slices,
// FP32 accumulators in TMEM), M = 128 rows:
//   stage A (y):  G_{s,iy}(j1,k2) = sum_j2 F_s(j1,j2) ty_iy(j2,k2), once per
//                 (source, iy) of the CTA's pairs ("block"), rows (block, j1),
//                 a tile of 128/n blocks that share iy (one B operand);
//   each block row is added to Q_{t,ix}(j1,k2) of each pair (t, s) it serves
//                 (FP32, shared memory): neighbouring targets share sources,
//                 so a CTA has about a third as many blocks as pairs;
//   stage B (x):  pot_t(k1,k2) += sum_ix sum_j1 tx_ix(j1,k1) Q_{t,ix}(j1,k2),
//                 rows (target, k2), one K block of 16 per distinct ix ("slot")
//                 of the CTA's 128/n targets.
// n = 8 pads K and N to 16 with zeros.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "device_plan.hpp"

namespace bfgt {

constexpr int kNearTcSlots = 16;  // distinct x tables (slots) per CTA at most

struct NearTcArgs {
  const int4 *ctas;      // {tile begin, tile end, target begin, ntarget | nslot << 8}
  const int *targets;    // target leaf boxes (0-based), CTA after CTA
  const int4 *tiles;     // {table slot of ty, block begin, block count, 0}
  const int4 *blocks;    // {source box, consumers 0 | 1 << 16, 2 | 3 << 16, count};
                         // a consumer is target (CTA-local) | x slot << 8
  const int *slot_q;     // kNearTcSlots per CTA: table slot of each x slot
  const uint16_t *tabB;  // per table slot: 3 BF16 slices of a 16 x 16 K-major B operand;
                         // three sets (values, first, second derivatives in the
                         // target coordinate), nslot_tab slots each
  const double *tabD;    // the FP64 kernel's tables: per slot n x n, tab(j, k) at j + n k,
                         // zero outside the band pattern; the same three sets
  int *err;
  int nd, n, nctas;
  uint32_t wait_iters;
  long long elem_off;  // start of this plan's leaf arrays in the (packed) fvals/pot
  // out(out_nd, npbox, nboxes) += component out_off / nd of the transform
  // (out_nd = nd ncomp); the x and y tables are read at slot + xoff / yoff
  // (0: values, nslot_tab: first derivatives, 2 nslot_tab: second)
  int out_nd, out_off, xoff, yoff;
};

// a single plan (descs null: CTA b is the plan's CTA b) or a batch (CTA b is
// CTA work[b].y of plan work[b].x)
struct NearTcLaunch {
  NearTcArgs one;
  const NearTcArgs *descs;
  const int2 *work;
  const double *fbase;
  double *pbase;
};

// Builds the CTA, tile and block lists and the tables of a plan with norder 8
// or 16: BF16 table operands for the tensor-core kernel (split plans with
// floating slices, fp64 false), or FP64 tables for k_near_f64, the same
// decomposition on the FP64 pipes (FP64 plans and fixed-point split plans,
// fp64 true).  Leaves dp.ntc empty (the per-target FP64 kernel runs) when the
// plan has no near field or cannot use it.
int near_tc_create(DevicePlan &dp, const HostPlan &hp, std::string &msg, bool fp64 = false);
void near_tc_destroy(DevicePlan &dp);
NearTcArgs near_tc_args(const DevicePlan &dp, long long elem_off);
// table slots per derivative set (13 offsets per level)
inline int near_tc_nslot(const DevicePlan &dp) { return 13 * (dp.nlevels + 1); }
// one plan's near field, or (lp.descs set) grid CTAs of a batch
void near_tc_launch(int n, int grid, size_t smem, cudaStream_t s, const NearTcLaunch &lp);
void near_f64_launch(int n, int grid, size_t smem, cudaStream_t s, const NearTcLaunch &lp);

}  // namespace bfgt
