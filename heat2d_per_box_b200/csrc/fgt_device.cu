// Device kernels of the 2D box FGT and the plan's launch sequence.
//
// The reference's steps (bfgt/boxfgt.f) map onto the kernels as follows:
//   step 1 (leaf values -> multipole PW, boxfgt.f:728-744, g2d_tens_prod_to_pw
//   bfgt_pwrouts.f:98-147) and step 2 (merge to parents, boxfgt.f:764-783,
//   gnd_shiftpw bfgt_pwrouts.f:1798-1844) are fused in k_form: the merge shifts
//   are diagonal, so the product of the shifts from a leaf up to its cutoff
//   ancestor is one phase exp(-i ts.(c_leaf - c_anc)/sqrt(delta0)), taken from
//   a precomputed FP64 phase table, and each leaf's expansion is added
//   straight into its ancestor's expansion.  Partial sums per chunk of leaves
//   are summed in a fixed chunk order by the last CTA of each cutoff box, so
//   the result is deterministic.
//   step 3 (mp -> loc at the cutoff level, boxfgt.f:805-822) is k_translate.
//   step 4 (split, boxfgt.f:845-863, gnd_shiftpw_loc bfgt_pwrouts.f:1905-1941)
//   and step 5 (loc PW -> values, boxfgt.f:884-900, g2d_pw2pot
//   bfgt_pwrouts.f:549-602) are fused in k_eval by the conjugate phases.
//   step 6 (near field, boxfgt.f:915-1071, g2d_tens_prod_to_potloc
//   bfgt_local.f:315-375) is k_near over a host-built list of
//   (target, source, table x, table y) entries that already contains the
//   periodic level-1 images of boxfgt.f:938-1053.
#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/bfgt.h"
#include "batch.hpp"
#include "device_plan.hpp"
#include "fgt_common.cuh"
#include "near_tc.cuh"
#include "split_kernels.cuh"

namespace bfgt {

namespace {

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ void cfma(double2 &acc, double2 a, double2 b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(a.y, b.x, acc.y);
}

constexpr int kWarps = 4;
// leaves of an FP64 chunk made of sub-columns (kFp64ColumnLeaves / kWarps each)
constexpr int kFp64ColumnLeaves = 64;

struct FormArgs {
  const double *fvals;
  const int4 *leaves;   // {box, ox, oy, level}, sorted by (icut, level, ox, oy)
  const int4 *columns;  // {leaf begin, leaf end, ox, -}
  const int4 *chunks;   // {column begin, column end, icut, level}
  const double2 *T;
  const double2 *PH;
  const long long *ph_off;
  double2 *Mpart;
  ReduceArgs red;
  int nd, n, npw, hh, nexp;
};

// Leaf values -> cutoff expansions, sum-factorised over a column of leaves.
// One CTA per chunk (columns of one cutoff ancestor and level), one warp per
// column.  With Ty(m2,k2) = T(m2,k2) conj(ph_oy(k2)) and
// Tx(m1,k1) = T(m1,k1) conj(ph_ox(k1)) (ph = exp(i ts.(c_leaf-c_anc)/sqrt(delta0))),
//   Y(m1,k2)   = sum_{leaves of the column} sum_m2 F(m1,m2) Ty(m2,k2)
//   M(k1,k2)  += sum_m1 Tx(m1,k1) Y(m1,k2)
// which equals sum over the column's leaves of the reference's step-1
// expansion shifted to the ancestor (steps 1+2, boxfgt.f:728-783).  The M
// accumulators of a warp stay in registers (NT tiles of TM x TN per lane)
// across its columns; warps are then summed in a fixed order.
// L(icut) = M(icut) + sum over its plane-wave list of M(src) * W(shift)
// (mp -> loc at the cutoff level, boxfgt.f:805-822), one thread per element and group of densities.
// kscale (hh entries, may be null) multiplies element (k1,k2) by kscale[k2];
// the transposed transform uses it for the half-spectrum weight.
struct TrArgs {
  const double2 *M;
  const int *pw_begin, *pw_src, *pw_ind;
  const double2 *W;
  const double *kscale;
  double2 *L;
  int ncut, nd, npw, nexp;
};
// a single plan (descs null, block b of `one`) or a batch (block b = block
// work[b].y of plan work[b].x)
struct TrLaunch {
  TrArgs one;
  const TrArgs *descs;
  const int2 *work;
};

constexpr int kTrThreads = 256;

// One thread per (cutoff box, group of kTrDens densities, element e): the
// shift W of each plane-wave-list neighbour is loaded once for the group's
// densities, and the group's M loads of a neighbour are independent.
constexpr int kTrDens = 4;
__host__ __device__ inline size_t tr_threads(int ncut, int nd, int nexp) {
  return (size_t)ncut * ((nd + kTrDens - 1) / kTrDens) * nexp;
}

__global__ void __launch_bounds__(kTrThreads) k_translate(const __grid_constant__ TrLaunch lp) {
  const TrArgs &a = lp.descs ? lp.descs[lp.work[blockIdx.x].x] : lp.one;
  const int blk = lp.descs ? lp.work[blockIdx.x].y : (int)blockIdx.x;
  const int nexp = a.nexp, nd = a.nd, ng = (nd + kTrDens - 1) / kTrDens;
  const size_t per = (size_t)nd * nexp;
  const size_t idx = (size_t)blk * blockDim.x + threadIdx.x;
  if (idx >= (size_t)a.ncut * ng * nexp) return;
  if (nd == 1) {
    // one density: one element per thread, neighbour loop unrolled by 4 (the
    // group loop below measured slower here)
    const int icut = (int)(idx / nexp), e = (int)(idx - (size_t)icut * nexp);
    double2 s = __ldg(&a.M[idx]);
    const int j0 = a.pw_begin[icut], j1 = a.pw_begin[icut + 1];
#pragma unroll 4
    for (int j = j0; j < j1; j++) {
      const double2 m = __ldg(&a.M[(size_t)a.pw_src[j] * nexp + e]);
      const double2 w = __ldg(&a.W[(size_t)a.pw_ind[j] * nexp + e]);
      s.x += m.x * w.x - m.y * w.y;
      s.y += m.x * w.y + m.y * w.x;
    }
    if (a.kscale) {
      const double f = a.kscale[e / a.npw];
      s.x *= f;
      s.y *= f;
    }
    a.L[idx] = s;
    return;
  }
  const int icut = (int)(idx / ((size_t)ng * nexp));
  const int rem = (int)(idx - (size_t)icut * ng * nexp);
  const int g = rem / nexp, e = rem - g * nexp;
  const int d0 = g * kTrDens, dn = min(kTrDens, nd - d0);
  const size_t r = (size_t)d0 * nexp + e;  // element (d0, e) within a box's expansions
  double2 s[kTrDens];
#pragma unroll
  for (int u = 0; u < kTrDens; u++)
    s[u] = u < dn ? __ldg(&a.M[(size_t)icut * per + r + (size_t)u * nexp]) : make_double2(0, 0);
  const int j0 = a.pw_begin[icut], j1 = a.pw_begin[icut + 1];
#pragma unroll 2
  for (int j = j0; j < j1; j++) {
    const double2 w = __ldg(&a.W[(size_t)a.pw_ind[j] * nexp + e]);
    const double2 *Ms = a.M + (size_t)a.pw_src[j] * per + r;
#pragma unroll
    for (int u = 0; u < kTrDens; u++) {
      if (u >= dn) break;
      const double2 m = __ldg(&Ms[(size_t)u * nexp]);
      s[u].x += m.x * w.x - m.y * w.y;
      s[u].y += m.x * w.y + m.y * w.x;
    }
  }
  const double f = a.kscale ? a.kscale[e / a.npw] : 1.0;
#pragma unroll
  for (int u = 0; u < kTrDens; u++) {
    if (u >= dn) break;
    a.L[(size_t)icut * per + r + (size_t)u * nexp] = a.kscale ? make_double2(s[u].x * f, s[u].y * f) : s[u];
  }
}

// Ld(icut, c*nd + ind, e) = L(icut, ind, e) * fac(c, e) for nc components:
// the local expansions of derivatives of the potential (fac = (i ts/sqrt(delta0))
// to the derivative orders in x (first index of e) and y (second)).
__global__ void k_deriv_expand(const double2 *__restrict__ L, const double2 *__restrict__ fac,
                               double2 *__restrict__ Ld, int ncut, int nd, int nc, int nexp) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t tot = (size_t)ncut * nd * nc * nexp;
  if (idx >= tot) return;
  const int e = (int)(idx % nexp);
  const size_t r = idx / nexp;
  const int q = (int)(r % ((size_t)nd * nc));
  const size_t icut = r / ((size_t)nd * nc);
  const int c = q / nd, ind = q - c * nd;
  const double2 l = L[(icut * nd + ind) * nexp + e];
  const double2 f = fac[(size_t)c * nexp + e];
  Ld[idx] = make_double2(l.x * f.x - l.y * f.y, l.x * f.y + l.y * f.x);
}

template <int TM, int TN, int NT>
__global__ void __launch_bounds__(kWarps * 32, 3) k_form_fp64(FormArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int4 ch = a.chunks[blockIdx.x];
  const int n = a.n, npw = a.npw, hh = a.hh, nd = a.nd, npb = n * n;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double2 *sT = reinterpret_cast<double2 *>(smem_raw);  // [m][k], n x npw
  double2 *sRed = sT + (size_t)n * npw;                  // npw x hh, [k2][k1]
  const size_t per_warp = (size_t)n * hh + npw + hh + (npb + 1) / 2;
  double2 *wb = sRed + (size_t)npw * hh + per_warp * warp;
  double2 *sY = wb;                    // [m1][k2]
  double2 *sphx = sY + (size_t)n * hh;
  double2 *sphy = sphx + npw;
  double *sF = reinterpret_cast<double *>(sphy + hh);  // [m2][m1]

  const double2 *Tg = a.T + (size_t)n * npw * ch.w;
  for (int i = threadIdx.x; i < n * npw; i += blockDim.x) {
    const int m = i % n, k = i / n;
    sT[m * npw + k] = Tg[i];
  }
  __syncthreads();
  const long long phoff = a.ph_off[ch.w];
  const int ntm = (npw + TM - 1) / TM, ntn = (hh + TN - 1) / TN, ntiles = ntm * ntn;
  for (int ind = 0; ind < nd; ind++) {
    double2 M[NT][TM][TN];
#pragma unroll
    for (int t = 0; t < NT; t++)
#pragma unroll
      for (int i = 0; i < TM; i++)
#pragma unroll
        for (int j = 0; j < TN; j++) M[t][i][j] = make_double2(0, 0);
    for (int c = ch.x + warp; c < ch.y; c += kWarps) {
      const int4 col = a.columns[c];
      for (int e = lane; e < n * hh; e += 32) sY[e] = make_double2(0, 0);
      const double2 *phx = a.PH + phoff + (size_t)col.z * npw;
      for (int k = lane; k < npw; k += 32) {
        const double2 p = phx[k];
        sphx[k] = make_double2(p.x, -p.y);
      }
      for (int li = col.x; li < col.y; li++) {
        const int4 lf = a.leaves[li];
        const double *fv = a.fvals + (size_t)lf.x * nd * npb;
        __syncwarp();
        for (int j = lane; j < npb; j += 32) sF[j] = fv[ind + (size_t)nd * j];
        const double2 *phy = a.PH + phoff + (size_t)lf.z * npw;
        for (int k = lane; k < hh; k += 32) {
          const double2 p = phy[k];
          sphy[k] = make_double2(p.x, -p.y);
        }
        __syncwarp();
        for (int o = lane; o < n * hh; o += 32) {
          const int m1 = o / hh, k2 = o - m1 * hh;
          double2 acc = make_double2(0, 0);
#pragma unroll 4
          for (int m2 = 0; m2 < n; m2++) {
            const double f = sF[m1 + n * m2];
            const double2 t = sT[m2 * npw + k2];
            acc.x = fma(f, t.x, acc.x);
            acc.y = fma(f, t.y, acc.y);
          }
          const double2 v = cmul(acc, sphy[k2]);
          sY[o].x += v.x;
          sY[o].y += v.y;
        }
      }
      __syncwarp();
#pragma unroll
      for (int t = 0; t < NT; t++) {
        const int tile = lane + 32 * t;
        if (tile >= ntiles) continue;
        const int k1b = (tile % ntm) * TM, k2b = (tile / ntm) * TN;
        double2 ph[TM];
#pragma unroll
        for (int i = 0; i < TM; i++) ph[i] = (k1b + i < npw) ? sphx[k1b + i] : make_double2(0, 0);
#pragma unroll 2
        for (int m1 = 0; m1 < n; m1++) {
          double2 av[TM], bv[TN];
#pragma unroll
          for (int i = 0; i < TM; i++) av[i] = cmul((k1b + i < npw) ? sT[m1 * npw + k1b + i] : make_double2(0, 0), ph[i]);
#pragma unroll
          for (int j = 0; j < TN; j++) bv[j] = (k2b + j < hh) ? sY[m1 * hh + k2b + j] : make_double2(0, 0);
#pragma unroll
          for (int i = 0; i < TM; i++)
#pragma unroll
            for (int j = 0; j < TN; j++) cfma(M[t][i][j], av[i], bv[j]);
        }
      }
      __syncwarp();
    }
    // fixed-order sum of the warps' accumulators: warp 0 stores, 1..3 add
    for (int w = 0; w < kWarps; w++) {
      if (warp == w) {
#pragma unroll
        for (int t = 0; t < NT; t++) {
          const int tile = lane + 32 * t;
          if (tile >= ntiles) continue;
          const int k1b = (tile % ntm) * TM, k2b = (tile / ntm) * TN;
#pragma unroll
          for (int i = 0; i < TM; i++)
#pragma unroll
            for (int j = 0; j < TN; j++) {
              if (k1b + i >= npw || k2b + j >= hh) continue;
              double2 &r = sRed[(k2b + j) * npw + k1b + i];
              if (w == 0) {
                r = M[t][i][j];
              } else {
                r.x += M[t][i][j].x;
                r.y += M[t][i][j].y;
              }
            }
        }
      }
      __syncthreads();
    }
    double2 *out = a.Mpart + ((size_t)blockIdx.x * nd + ind) * a.nexp;
    for (int e = threadIdx.x; e < a.nexp; e += blockDim.x) out[e] = sRed[e];
    __syncthreads();
  }
  __shared__ int s_last;
  finish_cutoff_box(a.red, blockIdx.x, nd, a.nexp, &s_last);
}

struct EvalArgs {
  double *pot;
  const int4 *leaves;
  const int4 *columns;
  const int4 *chunks;
  const double2 *E;
  const double2 *PH;
  const long long *ph_off;
  const double2 *L;
  const double *pw_weight;
  int nd, n, npw, hh, nexp;
};

// Cutoff expansions -> leaf values (steps 4+5, boxfgt.f:845-900), sum-factorised
// over a column: one warp per column computes
//   H(k1,m2) = sum_m1 E(m1,k1) ph_ox(m1) L(m1,m2)          (once per column)
// and for each leaf of the column
//   pot(k1,k2) += 2 Re sum_m2 H(k1,m2) w(m2) ph_oy(m2) E(m2,k2)
// with w = 1/2 on the zero frequency of an odd npw (g2d_pw2pot).
template <int GM, int GN, int NG>
__global__ void __launch_bounds__(kWarps * 32) k_eval_fp64(EvalArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int4 ch = a.chunks[blockIdx.x];
  const int n = a.n, npw = a.npw, hh = a.hh, nd = a.nd, npb = n * n;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double2 *sE = reinterpret_cast<double2 *>(smem_raw);  // [m][k] (npw x n, k fastest)
  double2 *sL = sE + (size_t)npw * n;                    // [m1][m2]
  const size_t per_warp = (size_t)n * hh + npw + hh;
  double2 *wb = sL + (size_t)npw * hh + per_warp * warp;
  double2 *sHp = wb;                    // [m2][k1]
  double2 *sphx = sHp + (size_t)n * hh;
  double2 *sphy = sphx + npw;
  const double2 *Eg = a.E + (size_t)n * npw * ch.w;  // Fortran (npw, n)
  for (int i = threadIdx.x; i < n * npw; i += blockDim.x) {
    const int m = i % npw, k = i / npw;
    sE[m * n + k] = Eg[i];
  }
  const long long phoff = a.ph_off[ch.w];
  const int ntm = (n + GM - 1) / GM, ntn = (hh + GN - 1) / GN, ntiles = ntm * ntn;
  for (int ind = 0; ind < nd; ind++) {
    const double2 *Lg = a.L + ((size_t)ch.z * nd + ind) * a.nexp;
    for (int e = threadIdx.x; e < a.nexp; e += blockDim.x) {
      const int m2 = e / npw, m1 = e - m2 * npw;
      sL[m1 * hh + m2] = Lg[e];
    }
    __syncthreads();
    for (int c = ch.x + warp; c < ch.y; c += kWarps) {
      const int4 col = a.columns[c];
      const double2 *phx = a.PH + phoff + (size_t)col.z * npw;
      for (int k = lane; k < npw; k += 32) sphx[k] = phx[k];
      __syncwarp();
      double2 H[NG][GM][GN];
#pragma unroll
      for (int t = 0; t < NG; t++) {
#pragma unroll
        for (int i = 0; i < GM; i++)
#pragma unroll
          for (int j = 0; j < GN; j++) H[t][i][j] = make_double2(0, 0);
        const int tile = lane + 32 * t;
        if (tile >= ntiles) continue;
        const int k1b = (tile % ntm) * GM, m2b = (tile / ntm) * GN;
#pragma unroll 2
        for (int m1 = 0; m1 < npw; m1++) {
          const double2 p = sphx[m1];
          double2 av[GM], bv[GN];
#pragma unroll
          for (int i = 0; i < GM; i++) av[i] = cmul((k1b + i < n) ? sE[m1 * n + k1b + i] : make_double2(0, 0), p);
#pragma unroll
          for (int j = 0; j < GN; j++) bv[j] = (m2b + j < hh) ? sL[m1 * hh + m2b + j] : make_double2(0, 0);
#pragma unroll
          for (int i = 0; i < GM; i++)
#pragma unroll
            for (int j = 0; j < GN; j++) cfma(H[t][i][j], av[i], bv[j]);
        }
      }
      for (int li = col.x; li < col.y; li++) {
        const int4 lf = a.leaves[li];
        const double2 *phy = a.PH + phoff + (size_t)lf.z * npw;
        __syncwarp();
        for (int k = lane; k < hh; k += 32) {
          const double2 p = phy[k];
          const double w = a.pw_weight[k];
          sphy[k] = make_double2(p.x * w, p.y * w);
        }
        __syncwarp();
#pragma unroll
        for (int t = 0; t < NG; t++) {
          const int tile = lane + 32 * t;
          if (tile >= ntiles) continue;
          const int k1b = (tile % ntm) * GM, m2b = (tile / ntm) * GN;
#pragma unroll
          for (int j = 0; j < GN; j++) {
            if (m2b + j >= hh) continue;
            const double2 p = sphy[m2b + j];
#pragma unroll
            for (int i = 0; i < GM; i++)
              if (k1b + i < n) sHp[(m2b + j) * n + k1b + i] = cmul(H[t][i][j], p);
          }
        }
        __syncwarp();
        double *pb = a.pot + (size_t)lf.x * nd * npb;
        for (int o = lane; o < npb; o += 32) {
          const int k1 = o % n, k2 = o / n;
          double acc = 0;
#pragma unroll 4
          for (int m2 = 0; m2 < hh; m2++) {
            const double2 e = sE[m2 * n + k2];
            const double2 g = sHp[m2 * n + k1];
            acc = fma(e.x, g.x, acc);
            acc = fma(-e.y, g.y, acc);
          }
          pb[ind + (size_t)nd * o] += 2 * acc;
        }
      }
      __syncwarp();
    }
    __syncthreads();
  }
}

// tile shape (and tiles per lane) with the fewest wasted lane-slots for an
// a x b output, at most maxnt tiles per lane
struct TileChoice {
  int tm, tn, nt;
};
inline TileChoice best_tile(int a, int b, const TileChoice *cands, int nc) {
  TileChoice best{0, 0, 0};
  double beff = -1;
  for (int i = 0; i < nc; i++) {
    const int tm = cands[i].tm, tn = cands[i].tn;
    const int tiles = ((a + tm - 1) / tm) * ((b + tn - 1) / tn);
    const int nt = (tiles + 31) / 32;
    if (nt != cands[i].nt) continue;
    const double eff = (double)a * b / (32.0 * nt * tm * tn);
    if (eff > beff + 1e-9) {
      beff = eff;
      best = cands[i];
    }
  }
  return best;
}

const TileChoice kFormTiles[] = {{4, 4, 1}, {5, 4, 1}, {4, 5, 1}, {5, 5, 1}, {4, 4, 2}, {5, 5, 2}, {6, 4, 2},
                                 {4, 6, 2}, {6, 6, 2}, {8, 4, 2}, {6, 6, 3}, {8, 8, 2}};
const TileChoice kEvalTiles[] = {{1, 5, 1}, {2, 5, 1}, {2, 4, 1}, {4, 4, 1}, {2, 8, 1}, {4, 5, 1}, {2, 5, 2},
                                 {4, 4, 2}, {4, 5, 2}, {4, 8, 2}, {4, 8, 3}, {8, 8, 2}};
constexpr int kNFormTiles = sizeof(kFormTiles) / sizeof(kFormTiles[0]);
constexpr int kNEvalTiles = sizeof(kEvalTiles) / sizeof(kEvalTiles[0]);

#define FORM_LIST(X) X(4, 4, 1) X(5, 4, 1) X(4, 5, 1) X(5, 5, 1) X(4, 4, 2) X(5, 5, 2) X(6, 4, 2) X(4, 6, 2) X(6, 6, 2) X(8, 4, 2) X(6, 6, 3) X(8, 8, 2)
#define EVAL_LIST(X) X(1, 5, 1) X(2, 5, 1) X(2, 4, 1) X(4, 4, 1) X(2, 8, 1) X(4, 5, 1) X(2, 5, 2) X(4, 4, 2) X(4, 5, 2) X(4, 8, 2) X(4, 8, 3) X(8, 8, 2)

bool launch_form_fp64(const TileChoice &t, int grid, size_t smem, cudaStream_t s, const FormArgs &a) {
#define FORM_CASE(M_, N_, T_)                                      \
  if (t.tm == M_ && t.tn == N_ && t.nt == T_) {                    \
    k_form_fp64<M_, N_, T_><<<grid, kWarps * 32, smem, s>>>(a);    \
    return true;                                                   \
  }
  FORM_LIST(FORM_CASE)
#undef FORM_CASE
  return false;
}

bool launch_eval_fp64(const TileChoice &t, int grid, size_t smem, cudaStream_t s, const EvalArgs &a) {
#define EVAL_CASE(M_, N_, T_)                                      \
  if (t.tm == M_ && t.tn == N_ && t.nt == T_) {                    \
    k_eval_fp64<M_, N_, T_><<<grid, kWarps * 32, smem, s>>>(a);    \
    return true;                                                   \
  }
  EVAL_LIST(EVAL_CASE)
#undef EVAL_CASE
  return false;
}

void set_smem_attrs(int bytes) {
#define FORM_ATTR(M_, N_, T_) cudaFuncSetAttribute(k_form_fp64<M_, N_, T_>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
#define EVAL_ATTR(M_, N_, T_) cudaFuncSetAttribute(k_eval_fp64<M_, N_, T_>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  FORM_LIST(FORM_ATTR)
  EVAL_LIST(EVAL_ATTR)
#undef FORM_ATTR
#undef EVAL_ATTR
}

struct NearArgs {
  const int *target, *begin, *src;
  const int2 *ixy;  // per entry: table slots (level * 13 + offset + 6) in x and y
  const double *tab_loc;
  const int *ind_loc;
  int ntarget, nd, n;
  long long elem_off;  // start of this plan's leaf arrays in the (packed) fvals/pot
  // output out(nd, ncomp, npbox, nboxes) += component (out_off / nd) of the
  // transform (out_nd = nd * ncomp); the x and y tables are read at slot +
  // xoff / yoff (0: values, one table set further: first derivatives, two:
  // second derivatives), the band pattern always at the slot itself
  int out_nd, out_off, xoff, yoff;
};
// a single plan (descs null, block b takes targets kWarps b..) or a batch
// (block b takes targets work[b].y.. of plan work[b].x)
struct NearLaunch {
  NearArgs one;
  const NearArgs *descs;
  const int2 *work;
  const double *fbase;
  double *pbase;
};

// One warp per near-field target leaf; pot(k1,k2) += sum over its list1
// entries of Ty^T (Tx^T F) on the banded 1D tables of each entry's slots
// (the forward pass uses the target's level, the transposed pass the level
// of the forward target).
__global__ void __launch_bounds__(kWarps * 32) k_near_fp64(const __grid_constant__ NearLaunch lp) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const NearArgs &a = lp.descs ? lp.descs[lp.work[blockIdx.x].x] : lp.one;
  const int first = lp.descs ? lp.work[blockIdx.x].y : (int)blockIdx.x * kWarps;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int t = first + warp;
  if (t >= a.ntarget) return;
  const int n = a.n, npb = n * n, nd = a.nd;
  const double *fvals = lp.fbase + a.elem_off;
  double *pot = lp.pbase + a.elem_off;
  double *wb = reinterpret_cast<double *>(smem_raw) + (size_t)warp * 3 * npb;
  double *sF = wb, *sff = wb + npb, *sP = wb + 2 * npb;
  const int tb = a.target[t];
  const double *tl = a.tab_loc;
  const int *il = a.ind_loc;
  for (int ind = 0; ind < nd; ind++) {
    for (int o = lane; o < npb; o += 32) sP[o] = 0;
    for (int e = a.begin[t]; e < a.begin[t + 1]; e++) {
      const int sb = a.src[e];
      const int ix = a.ixy[e].x, iy = a.ixy[e].y;
      const int *bx = il + (size_t)2 * (n + 1) * ix;
      const int *by = il + (size_t)2 * (n + 1) * iy;
      const int kx0 = bx[2 * n], kx1 = bx[2 * n + 1], ky0 = by[2 * n], ky1 = by[2 * n + 1];
      if (kx1 - kx0 + 1 == 0 || ky1 - ky0 + 1 == 0) continue;
      const double *tx = tl + (size_t)npb * (ix + a.xoff);
      const double *ty = tl + (size_t)npb * (iy + a.yoff);
      const double *fv = fvals + (size_t)sb * nd * npb;
      __syncwarp();
      for (int o = lane; o < npb; o += 32) sF[o] = fv[ind + (size_t)nd * o];
      __syncwarp();
      // ff(k1, j2) for k1 in [kx0, kx1] (1-based)
      const int nkx = kx1 - kx0 + 1;
      for (int o = lane; o < nkx * n; o += 32) {
        const int k1 = kx0 + o % nkx, j2 = o / nkx;
        const int lo = bx[2 * (k1 - 1)], hi = bx[2 * (k1 - 1) + 1];
        double cd = 0;
        for (int j1 = lo; j1 <= hi; j1++) cd = fma(tx[(j1 - 1) + (size_t)n * (k1 - 1)], sF[(j1 - 1) + (size_t)n * j2], cd);
        sff[(k1 - 1) + (size_t)n * j2] = cd;
      }
      __syncwarp();
      const int nky = ky1 - ky0 + 1;
      for (int o = lane; o < nkx * nky; o += 32) {
        const int k1 = kx0 + o % nkx, k2 = ky0 + o / nkx;
        const int lo = by[2 * (k2 - 1)], hi = by[2 * (k2 - 1) + 1];
        double cd = 0;
        for (int j2 = lo; j2 <= hi; j2++) cd = fma(ty[(j2 - 1) + (size_t)n * (k2 - 1)], sff[(k1 - 1) + (size_t)n * (j2 - 1)], cd);
        sP[(k1 - 1) + (size_t)n * (k2 - 1)] += cd;
      }
    }
    __syncwarp();
    double *pb = pot + (size_t)tb * a.out_nd * npb + a.out_off;
    for (int o = lane; o < npb; o += 32) pb[ind + (size_t)a.out_nd * o] += sP[o];
    __syncwarp();
  }
}

template <typename T>
int upload(T *&dptr, const std::vector<T> &v, std::string &msg) {
  dptr = nullptr;
  if (v.empty()) return BFGT_OK;
  if (cudaMalloc(&dptr, sizeof(T) * v.size()) != cudaSuccess) {
    msg = "cudaMalloc failed (" + std::to_string(sizeof(T) * v.size()) + " bytes)";
    return BFGT_ERR_OOM;
  }
  if (cudaMemcpy(dptr, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
    msg = "cudaMemcpy to device failed";
    return BFGT_ERR_CUDA;
  }
  return BFGT_OK;
}

int alloc_bytes(void **p, size_t bytes, std::string &msg) {
  *p = nullptr;
  if (bytes == 0) return BFGT_OK;
  if (cudaMalloc(p, bytes) != cudaSuccess) {
    msg = "cudaMalloc failed (" + std::to_string(bytes) + " bytes)";
    return BFGT_ERR_OOM;
  }
  return BFGT_OK;
}

}  // namespace

// Groups of at most 32 chunks per cutoff box for the fixed-order reduction
// done at the end of the form kernels (fgt_common.cuh).
int build_reduce_groups(DevicePlan &dp, const std::vector<int> &cut_of_chunk, std::string &msg,
                        const std::vector<int> &arrivals) {
  const void *old[] = {dp.G, dp.gcnt, dp.bcnt, dp.chunk_group, dp.groups, dp.box_groups};
  for (const void *p : old)
    if (p) cudaFree(const_cast<void *>(p));
  dp.G = nullptr;
  dp.gcnt = dp.bcnt = dp.chunk_group = dp.box_groups = nullptr;
  dp.groups = nullptr;
  const int nch = (int)cut_of_chunk.size();
  std::vector<int> chunk_group(std::max(nch, 1), 0), box_groups(dp.ncut + 1, 0);
  std::vector<int4> groups;
  int c = 0;
  for (int ic = 0; ic < dp.ncut; ic++) {
    box_groups[ic] = (int)groups.size();
    int c1 = c;
    while (c1 < nch && cut_of_chunk[c1] == ic) c1++;
    for (int g0 = c; g0 < c1; g0 += 32) {
      const int g1 = std::min(g0 + 32, c1);
      int arr = 0;
      for (int q = g0; q < g1; q++) {
        chunk_group[q] = (int)groups.size();
        arr += arrivals.empty() ? 1 : arrivals[q];
      }
      groups.push_back(make_int4(g0, g1, ic, arr));
    }
    c = c1;
  }
  box_groups[dp.ncut] = (int)groups.size();
  if (c != nch) {
    msg = "chunks are not sorted by cutoff box";
    return BFGT_ERR_TREE;
  }
  bool multi = false;
  for (int ic = 0; ic < dp.ncut; ic++) multi = multi || (box_groups[ic + 1] - box_groups[ic] > 1);
  dp.ngroups = (int)groups.size();
  dp.multi_group = multi;
  int rc = BFGT_OK;
  auto chk = [&](int r) {
    if (rc == BFGT_OK && r != BFGT_OK) rc = r;
  };
  std::vector<int> zg(std::max(dp.ngroups, 1), 0), zb(std::max(dp.ncut, 1), 0);
  chk(upload(dp.chunk_group, chunk_group, msg));
  chk(upload(dp.groups, groups, msg));
  chk(upload(dp.box_groups, box_groups, msg));
  chk(upload(dp.gcnt, zg, msg));
  chk(upload(dp.bcnt, zb, msg));
  if (multi) chk(alloc_bytes((void **)&dp.G, sizeof(double2) * (size_t)dp.nd * dp.nexp * dp.ngroups, msg));
  return rc;
}

ReduceArgs reduce_args(const DevicePlan &dp) {
  return ReduceArgs{dp.Mpart, dp.G, dp.M, dp.gcnt, dp.bcnt, dp.chunk_group, dp.groups, dp.box_groups};
}

// ---- autotuner of the FP64 tile shapes ---------------------------------------

namespace {

std::mutex g_tune_mu;
std::map<std::array<int, 3>, std::pair<TileChoice, TileChoice>> g_tuned;  // (n, npw, nd) -> (form, eval)

// every compiled tile shape whose lanes cover an a x b output
std::vector<TileChoice> valid_tiles(int a, int b, const TileChoice *cands, int nc) {
  std::vector<TileChoice> v;
  for (int i = 0; i < nc; i++) {
    const int tiles = ((a + cands[i].tm - 1) / cands[i].tm) * ((b + cands[i].tn - 1) / cands[i].tn);
    if (32 * cands[i].nt >= tiles) v.push_back(cands[i]);
  }
  return v;
}

}  // namespace

void tuned_tiles(int n, int npw, int nd, TileChoice &form, TileChoice &eval) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto it = g_tuned.find({n, npw, nd});
  if (it == g_tuned.end()) return;
  form = it->second.first;
  eval = it->second.second;
}

int device_plan_autotune(DevicePlan &dp, cudaStream_t s, double *report, std::string &msg) {
  for (int i = 0; i < 4; i++) report[i] = 0;
  if (dp.precision == BFGT_PREC_SPLIT) return split_autotune(dp, s, report, msg);
  if (dp.direct_only || dp.nchunks == 0) return BFGT_OK;  // no tile choice to make
  const size_t elems = (size_t)dp.nd * dp.n * dp.n * dp.nboxes;
  double *f = nullptr, *p = nullptr;
  if (alloc_bytes((void **)&f, sizeof(double) * elems, msg) != BFGT_OK) return BFGT_ERR_OOM;
  if (alloc_bytes((void **)&p, sizeof(double) * elems, msg) != BFGT_OK) {
    cudaFree(f);
    return BFGT_ERR_OOM;
  }
  cudaMemsetAsync(f, 0, sizeof(double) * elems, s);
  cudaMemsetAsync(p, 0, sizeof(double) * elems, s);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const TileChoice f0{dp.form_tile[0], dp.form_tile[1], dp.form_tile[2]};
  const TileChoice v0{dp.eval_tile[0], dp.eval_tile[1], dp.eval_tile[2]};
  auto time_ms = [&](auto &&launch) {
    launch();  // warm-up
    cudaEventRecord(e0, s);
    for (int r = 0; r < 3; r++) launch();
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    return ms / 3.0;
  };
  TileChoice bf = f0, be = v0;
  double tf = 1e30, te = 1e30;
  const std::vector<TileChoice> fc = valid_tiles(dp.npw, dp.hh, kFormTiles, kNFormTiles);
  const std::vector<TileChoice> ec = valid_tiles(dp.n, dp.hh, kEvalTiles, kNEvalTiles);
  for (const TileChoice &t : fc) {
    FormArgs fa{f, dp.leaves, dp.columns64, dp.chunks, dp.T, dp.PH, dp.ph_off, dp.Mpart, reduce_args(dp), dp.nd, dp.n,
                dp.npw, dp.hh, dp.nexp};
    const double ms = time_ms([&] { launch_form_fp64(t, dp.nchunks, dp.smem_form, s, fa); });
    if (ms < tf) tf = ms, bf = t;
  }
  for (const TileChoice &t : ec) {
    EvalArgs ea{p, dp.leaves, dp.columns64, dp.chunks, dp.E, dp.PH, dp.ph_off, dp.L, dp.pw_weight, dp.nd, dp.n,
                dp.npw, dp.hh, dp.nexp};
    const double ms = time_ms([&] { launch_eval_fp64(t, dp.nchunks, dp.smem_eval, s, ea); });
    if (ms < te) te = ms, be = t;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(f);
  cudaFree(p);
  if (cudaGetLastError() != cudaSuccess) {
    msg = "CUDA error while autotuning";
    return BFGT_ERR_CUDA;
  }
  dp.form_tile[0] = bf.tm, dp.form_tile[1] = bf.tn, dp.form_tile[2] = bf.nt;
  dp.eval_tile[0] = be.tm, dp.eval_tile[1] = be.tn, dp.eval_tile[2] = be.nt;
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tuned[{dp.n, dp.npw, dp.nd}] = {bf, be};
  }
  report[0] = tf;
  report[1] = te;
  report[2] = (double)fc.size();
  report[3] = (double)ec.size();
  return BFGT_OK;
}

int device_plan_create(DevicePlan &dp, const HostPlan &hp, std::string &msg) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    msg = "no CUDA device visible";
    return BFGT_ERR_NODEVICE;
  }
  cudaGetDevice(&dp.device);
  dp.nd = hp.nd;
  dp.n = hp.norder;
  dp.npw = hp.npw;
  dp.hh = hp.hh;
  dp.nexp = hp.nexp;
  dp.nlevels = hp.nlevels;
  dp.nboxes = hp.nboxes;
  dp.precision = hp.precision;
  dp.direct_only = hp.direct_only;
  int rc = BFGT_OK;
  auto chk = [&](int r) {
    if (rc == BFGT_OK && r != BFGT_OK) rc = r;
  };
  const int n = dp.n;
  if (!hp.direct_only) {
    dp.ncut = (int)hp.cut_box.size();
    dp.nchunks = (int)hp.chunks.size();
    dp.nleaves = (int)hp.leaves.size();
    std::vector<double2> T(hp.tab_poly2pw.size()), E(hp.tab_pw2pot.size()), PH(hp.phase.size()), W(hp.wshift.size());
    for (size_t i = 0; i < T.size(); i++) T[i] = make_double2(hp.tab_poly2pw[i].re, hp.tab_poly2pw[i].im);
    for (size_t i = 0; i < E.size(); i++) E[i] = make_double2(hp.tab_pw2pot[i].re, hp.tab_pw2pot[i].im);
    for (size_t i = 0; i < PH.size(); i++) PH[i] = make_double2(hp.phase[i].re, hp.phase[i].im);
    for (size_t i = 0; i < W.size(); i++) W[i] = make_double2(hp.wshift[i].re, hp.wshift[i].im);
    chk(upload(dp.T, T, msg));
    chk(upload(dp.E, E, msg));
    chk(upload(dp.PH, PH, msg));
    chk(upload(dp.W, W, msg));
    std::vector<long long> po(hp.phase_off.begin(), hp.phase_off.end());
    chk(upload(dp.ph_off, po, msg));
    std::vector<int4> lv(hp.leaves.size()), colv(hp.columns.size());
    for (size_t i = 0; i < lv.size(); i++) lv[i] = make_int4(hp.leaves[i].box, hp.leaves[i].ox, hp.leaves[i].oy, hp.leaves[i].level);
    for (size_t i = 0; i < colv.size(); i++) colv[i] = make_int4(hp.columns[i].begin, hp.columns[i].end, hp.columns[i].ox, 0);
    // FP64 chunks: the host's chunks, except that a chunk with fewer columns
    // than warps (the kernels give each warp a column) has its columns cut
    // into sub-columns of at most kFp64ColumnLeaves / kWarps leaves, regrouped
    // kWarps to a chunk.  A coarse cutoff level gives such chunks: two columns
    // of 32 leaves, or one of 64 or 256; cut, they keep every warp and SM busy.
    // The kernels treat a sub-column like a column; the partial sums meet in
    // the warp and chunk reductions.
    std::vector<int4> cv, colv64;
    std::vector<int> cut_of_chunk;
    const int sub = kFp64ColumnLeaves / kWarps;
    for (const Chunk &ch : hp.chunks) {
      bool cut = ch.end - ch.begin < kWarps;
      if (cut) {
        cut = false;
        for (int c = ch.begin; c < ch.end; c++) cut = cut || hp.columns[c].end - hp.columns[c].begin > sub;
      }
      if (cut) {
        std::vector<int4> subs;
        for (int c = ch.begin; c < ch.end; c++)
          for (int q = hp.columns[c].begin; q < hp.columns[c].end; q += sub)
            subs.push_back(make_int4(q, std::min(q + sub, hp.columns[c].end), hp.columns[c].ox, 0));
        for (size_t i = 0; i < subs.size(); i += kWarps) {
          const int first = (int)colv64.size();
          for (size_t j = i; j < std::min(i + kWarps, subs.size()); j++) colv64.push_back(subs[j]);
          cv.push_back(make_int4(first, (int)colv64.size(), ch.icut, ch.level));
          cut_of_chunk.push_back(ch.icut);
        }
      } else {
        cv.push_back(make_int4((int)colv64.size(), (int)colv64.size() + (ch.end - ch.begin), ch.icut, ch.level));
        for (int c = ch.begin; c < ch.end; c++)
          colv64.push_back(make_int4(hp.columns[c].begin, hp.columns[c].end, hp.columns[c].ox, 0));
        cut_of_chunk.push_back(ch.icut);
      }
    }
    dp.nchunks = (int)cv.size();
    chk(upload(dp.leaves, lv, msg));
    chk(upload(dp.chunks, cv, msg));
    chk(upload(dp.columns, colv, msg));
    chk(upload(dp.columns64, colv64, msg));
    dp.ncolumns = (int)colv.size();
    chk(upload(dp.cut_chunk_begin, hp.cut_chunk_begin, msg));
    chk(upload(dp.cut_pw_begin, hp.cut_pw_begin, msg));
    chk(upload(dp.cut_pw_src, hp.cut_pw_src, msg));
    chk(upload(dp.cut_pw_ind, hp.cut_pw_ind, msg));
    chk(upload(dp.pw_weight, hp.pw_weight, msg));
    chk(upload(dp.kscale, hp.kscale, msg));
    const size_t ex = (size_t)dp.nd * dp.nexp * sizeof(double2);
    chk(alloc_bytes((void **)&dp.Mpart, ex * dp.nchunks, msg));
    chk(alloc_bytes((void **)&dp.M, ex * dp.ncut, msg));
    chk(alloc_bytes((void **)&dp.L, ex * dp.ncut, msg));
    if (rc == BFGT_OK) cudaMemset(dp.M, 0, ex * dp.ncut);  // boxes without PW leaves keep zero
    chk(build_reduce_groups(dp, cut_of_chunk, msg));
    const int npb = n * n;
    dp.smem_form = sizeof(double2) * ((size_t)n * dp.npw + (size_t)dp.npw * dp.hh +
                                      (size_t)kWarps * ((size_t)n * dp.hh + dp.npw + dp.hh + (npb + 1) / 2));
    dp.smem_eval = sizeof(double2) * ((size_t)n * dp.npw + (size_t)dp.npw * dp.hh +
                                      (size_t)kWarps * ((size_t)n * dp.hh + dp.npw + dp.hh));
    TileChoice ft = best_tile(dp.npw, dp.hh, kFormTiles, kNFormTiles);
    TileChoice et = best_tile(n, dp.hh, kEvalTiles, kNEvalTiles);
    tuned_tiles(n, dp.npw, dp.nd, ft, et);  // an earlier autotune of this shape wins
    dp.form_tile[0] = ft.tm, dp.form_tile[1] = ft.tn, dp.form_tile[2] = ft.nt;
    dp.eval_tile[0] = et.tm, dp.eval_tile[1] = et.tn, dp.eval_tile[2] = et.nt;
    if (rc == BFGT_OK && (ft.nt == 0 || et.nt == 0)) {
      msg = "npw=" + std::to_string(dp.npw) + " with norder=" + std::to_string(n) + " exceeds the built FP64 tile shapes";
      rc = BFGT_ERR_CAPACITY;
    }
    if (rc == BFGT_OK && dp.precision == BFGT_PREC_SPLIT) rc = split_plan_create(dp, hp, msg);
  }
  dp.nnf = (int)hp.nf_target.size();
  dp.nnf_entries = (int)hp.nf_src.size();
  if (dp.nnf > 0) {
    std::vector<int2> ixy(hp.nf_src.size());
    for (size_t i = 0; i < ixy.size(); i++)
      ixy[i] = make_int2(hp.nf_elev[i] * 13 + hp.nf_ix[i] + 6, hp.nf_elev[i] * 13 + hp.nf_iy[i] + 6);
    chk(upload(dp.nf_target, hp.nf_target, msg));
    chk(upload(dp.nf_begin, hp.nf_begin, msg));
    chk(upload(dp.nf_src, hp.nf_src, msg));
    chk(upload(dp.nf_ixy, ixy, msg));
    chk(upload(dp.tab_loc, hp.tab_loc, msg));
    chk(upload(dp.ind_loc, hp.ind_loc, msg));
    dp.smem_near = sizeof(double) * (size_t)kWarps * 3 * n * n;
    // split plans with floating slices: the near field on the tensor cores
    // (fixed-point plans keep the FP64 kernel, which meets their smaller eps)
    if (rc == BFGT_OK && dp.precision == BFGT_PREC_SPLIT && hp.eps >= 1e-7 && !dp.split.fixed) {
      if (!dp.split.err) {
        std::vector<int> zero(4, 0);
        chk(upload(dp.split.err, zero, msg));
      }
      chk(near_tc_create(dp, hp, msg));
    } else if (rc == BFGT_OK) {
      // FP64 plans and fixed-point split plans: the same work lists on the FP64 pipes
      chk(near_tc_create(dp, hp, msg, true));
    }
  }
  // the 227 KB per-block limit minus room for the kernels' static shared variables
  const size_t smax = 227 * 1024 - 1024;
  if (rc == BFGT_OK && (dp.smem_form > smax || dp.smem_eval > smax || dp.smem_near > smax)) {
    msg = "npw/norder need more than 227 KB of shared memory per block";
    rc = BFGT_ERR_CAPACITY;
  }
  if (rc == BFGT_OK) {
    set_smem_attrs((int)smax);
    cudaFuncSetAttribute(k_near_fp64, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smax);
    dp.events = true;
    device_plan_reserve_events(dp, 8);
    if (cudaGetLastError() != cudaSuccess) {
      msg = "CUDA error while creating the plan";
      rc = BFGT_ERR_CUDA;
    }
  }
  return rc;
}

void device_plan_destroy(DevicePlan &dp) {
  if (dp.graph_exec) cudaGraphExecDestroy(dp.graph_exec);
  if (dp.graph) cudaGraphDestroy(dp.graph);
  near_tc_destroy(dp);
  split_plan_destroy(dp);
  void *ptrs[] = {dp.T, dp.E, dp.PH, dp.ph_off, dp.leaves, dp.chunks, dp.columns, dp.columns64, dp.cut_chunk_begin, dp.cut_pw_begin,
                  dp.cut_pw_src, dp.cut_pw_ind, dp.W, dp.pw_weight, dp.kscale, dp.dfac, dp.Ld, dp.tab3_loc, dp.t_nchild, dp.t_ichild, dp.t_level, dp.t_centers, dp.t_boxsize, dp.t_umat, dp.t_has, dp.t_coefs, dp.t_leaf, dp.Mpart, dp.M, dp.L, dp.G, dp.gcnt, dp.bcnt, dp.chunk_group, dp.groups, dp.box_groups, dp.nf_target,
                  dp.nf_begin, dp.nf_src, dp.nf_ixy, dp.tab_loc, dp.ind_loc, dp.d_stage_f, dp.d_stage_p, dp.d_stage_gh};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  if (dp.h_stage_f) cudaFreeHost(dp.h_stage_f);
  for (auto &es : dp.evsets)
    for (cudaEvent_t e : es) cudaEventDestroy(e);
  dp = DevicePlan();
}

int reserve_event_sets(std::vector<std::array<cudaEvent_t, 6>> &evsets, int n) {
  while ((int)evsets.size() < n) {
    std::array<cudaEvent_t, 6> es;
    for (auto &e : es)
      if (cudaEventCreate(&e) != cudaSuccess) return BFGT_ERR_CUDA;
    evsets.push_back(es);
  }
  return BFGT_OK;
}

int read_stage_ms(std::vector<std::array<cudaEvent_t, 6>> &evsets, int &nrec, double *out) {
  for (int i = 0; i < 8; i++) out[i] = 0;
  if (nrec == 0) return BFGT_OK;
  const int nr = std::min<int>(nrec, (int)evsets.size());
  if (cudaEventSynchronize(evsets[nr - 1][5]) != cudaSuccess) return BFGT_ERR_CUDA;
  for (int r = 0; r < nr; r++) {
    float ms;
    for (int i = 0; i < 5; i++)
      if (cudaEventElapsedTime(&ms, evsets[r][i], evsets[r][i + 1]) == cudaSuccess) out[i] += ms;
    if (cudaEventElapsedTime(&ms, evsets[r][0], evsets[r][5]) == cudaSuccess) out[5] += ms;
  }
  out[6] = nr;
  nrec = 0;
  cudaGetLastError();
  return BFGT_OK;
}

int device_plan_reserve_events(DevicePlan &dp, int n) { return reserve_event_sets(dp.evsets, n); }

int device_plan_stage_ms(DevicePlan &dp, double *out) { return read_stage_ms(dp.evsets, dp.nrec, out); }

namespace {

TrArgs tr_args(const DevicePlan &dp) {
  return TrArgs{dp.M, dp.cut_pw_begin, dp.cut_pw_src, dp.cut_pw_ind, dp.W, dp.kscale, dp.L, dp.ncut, dp.nd, dp.npw,
                dp.nexp};
}

NearArgs near_args(const DevicePlan &dp, long long elem_off) {
  return NearArgs{dp.nf_target, dp.nf_begin, dp.nf_src, dp.nf_ixy, dp.tab_loc, dp.ind_loc, dp.nnf, dp.nd, dp.n,
                  elem_off, dp.nd, 0, 0, 0};
}

bool has_pw(const DevicePlan &dp) { return !dp.direct_only && dp.nchunks > 0; }

// steps 1+2 (leaf values -> cutoff expansions, merge fused) of one plan
void plan_form(DevicePlan &dp, const double *d_fvals, cudaStream_t s) {
  if (dp.precision == BFGT_PREC_SPLIT) {
    split_form(dp, d_fvals, s);
  } else {
    FormArgs fa{d_fvals, dp.leaves, dp.columns64, dp.chunks, dp.T, dp.PH, dp.ph_off, dp.Mpart, reduce_args(dp),
                dp.nd, dp.n, dp.npw, dp.hh, dp.nexp};
    launch_form_fp64(TileChoice{dp.form_tile[0], dp.form_tile[1], dp.form_tile[2]}, dp.nchunks, dp.smem_form, s, fa);
  }
}

// steps 4+5 (cutoff expansions -> leaf values, split fused) of one plan
void plan_eval(DevicePlan &dp, double *d_pot, cudaStream_t s) {
  if (dp.precision == BFGT_PREC_SPLIT) {
    split_eval(dp, d_pot, s);
  } else {
    EvalArgs ea{d_pot, dp.leaves, dp.columns64, dp.chunks, dp.E, dp.PH, dp.ph_off, dp.L, dp.pw_weight, dp.nd, dp.n,
                dp.npw, dp.hh, dp.nexp};
    launch_eval_fp64(TileChoice{dp.eval_tile[0], dp.eval_tile[1], dp.eval_tile[2]}, dp.nchunks, dp.smem_eval, s, ea);
  }
}

cudaEvent_t *next_events(std::vector<std::array<cudaEvent_t, 6>> &evsets, int &nrec, bool on) {
  if (!on) return nullptr;
  if (nrec >= (int)evsets.size() && evsets.size() < 65536) reserve_event_sets(evsets, nrec + 1);
  cudaEvent_t *ev = evsets[nrec % evsets.size()].data();
  nrec++;
  return ev;
}

}  // namespace

// NVTX range around the host-side queuing of one transform (visible to
// profilers that record NVTX; no cost without one)
struct NvtxRange {
  explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
};

int device_plan_execute(DevicePlan &dp, const double *d_fvals, double *d_pot, cudaStream_t s, std::string &msg) {
  NvtxRange range(dp.precision == BFGT_PREC_SPLIT ? "bfgt execute (split)" : "bfgt execute (fp64)");
  cudaEvent_t *ev = next_events(dp.evsets, dp.nrec, dp.events);
  if (ev) cudaEventRecord(ev[0], s);
  if (has_pw(dp)) {
    plan_form(dp, d_fvals, s);
    // the merge to the cutoff level finishes inside the form kernels
    if (ev) cudaEventRecord(ev[1], s);
    if (ev) cudaEventRecord(ev[2], s);
    const size_t tot = tr_threads(dp.ncut, dp.nd, dp.nexp);
    k_translate<<<(unsigned)((tot + kTrThreads - 1) / kTrThreads), kTrThreads, 0, s>>>(
        TrLaunch{tr_args(dp), nullptr, nullptr});
    if (ev) cudaEventRecord(ev[3], s);
    plan_eval(dp, d_pot, s);
    if (ev) cudaEventRecord(ev[4], s);
  } else if (ev) {
    for (int i = 1; i <= 4; i++) cudaEventRecord(ev[i], s);
  }
  if (dp.ntc.nctas > 0)
    (dp.ntc.fp64 ? near_f64_launch : near_tc_launch)(dp.n, dp.ntc.nctas, dp.ntc.smem, s,
                                                      NearTcLaunch{near_tc_args(dp, 0), nullptr, nullptr, d_fvals, d_pot});
  else if (dp.nnf > 0)
    k_near_fp64<<<(dp.nnf + kWarps - 1) / kWarps, kWarps * 32, dp.smem_near, s>>>(
        NearLaunch{near_args(dp, 0), nullptr, nullptr, d_fvals, d_pot});
  if (ev) cudaEventRecord(ev[5], s);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    msg = std::string("kernel launch failed: ") + cudaGetErrorString(e);
    return BFGT_ERR_CUDA;
  }
  return BFGT_OK;
}

int device_plan_prepare_pgh(DevicePlan &dp, const HostPlan &hp, std::string &msg) {
  if (dp.pgh_ready) return BFGT_OK;
  int rc = BFGT_OK;
  auto chk = [&](int r) {
    if (rc == BFGT_OK && r != BFGT_OK) rc = r;
  };
  if (has_pw(dp)) {
    // derivative factor of PW index m (1-based), as mk_pw2pgh_tables builds
    // tab_pw2der = tab_pw2pot * ts * dfac for m > npw/2 and its conjugate
    // mirror below (bfgt_volrouts.f:339-401; dfac = i / sqrt(delta0))
    const int npw = hp.npw, hh = hp.hh, npw2 = npw / 2;
    const double s0 = 1.0 / std::sqrt(hp.delta0);
    std::vector<double2> f(npw);
    for (int m = 1; m <= npw; m++) {
      if (m > npw2) f[m - 1] = make_double2(0.0, hp.ts[m - 1] * s0);
      else f[m - 1] = make_double2(0.0, -hp.ts[npw - m] * s0);
    }
    auto mul = [](double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); };
    std::vector<double2> fac((size_t)5 * hp.nexp);
    for (int k2 = 0; k2 < hh; k2++)
      for (int k1 = 0; k1 < npw; k1++) {
        const size_t e = (size_t)k1 + (size_t)npw * k2;
        const double2 fx = f[k1], fy = f[k2];
        fac[e] = fx;                                  // d/dx
        fac[hp.nexp + e] = fy;                        // d/dy
        fac[2 * (size_t)hp.nexp + e] = mul(fx, fx);   // d2/dx2
        fac[3 * (size_t)hp.nexp + e] = mul(fx, fy);   // d2/dxdy
        fac[4 * (size_t)hp.nexp + e] = mul(fy, fy);   // d2/dy2
      }
    chk(upload(dp.dfac, fac, msg));
    chk(alloc_bytes((void **)&dp.Ld, sizeof(double2) * (size_t)dp.ncut * dp.nd * 3 * dp.nexp, msg));
  }
  if (dp.nnf > 0) {
    std::vector<double> t3(hp.tab_loc);
    t3.insert(t3.end(), hp.tabx_loc.begin(), hp.tabx_loc.end());
    t3.insert(t3.end(), hp.tabxx_loc.begin(), hp.tabxx_loc.end());
    chk(upload(dp.tab3_loc, t3, msg));
  }
  if (rc == BFGT_OK) dp.pgh_ready = true;
  return rc;
}

int device_plan_execute_pgh(DevicePlan &dp, int ifpgh, const double *d_fvals, double *d_pot, double *d_grad,
                            double *d_hess, cudaStream_t s, std::string &msg) {
  NvtxRange range("bfgt execute pgh");
  int rc = device_plan_execute(dp, d_fvals, d_pot, s, msg);
  if (rc != BFGT_OK || ifpgh < 2) return rc;
  if (!dp.pgh_ready) {
    msg = "derivative tables are not prepared";
    return BFGT_ERR_ARG;
  }
  struct Part {
    int nc, c0;
    double *out;
  };
  const Part parts[2] = {{2, 0, d_grad}, {3, 2, d_hess}};
  for (int p = 0; p < (ifpgh == 3 ? 2 : 1); p++) {
    const Part &pt = parts[p];
    if (has_pw(dp)) {
      const size_t tot = (size_t)dp.ncut * dp.nd * pt.nc * dp.nexp;
      k_deriv_expand<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(dp.L, dp.dfac + (size_t)pt.c0 * dp.nexp, dp.Ld,
                                                                    dp.ncut, dp.nd, pt.nc, dp.nexp);
      DevicePlan view = dp;
      view.events = false;
      view.nd = dp.nd * pt.nc;
      view.L = dp.Ld;
      plan_eval(view, pt.out, s);
    }
    if (dp.nnf > 0) {
      // derivative orders of the components: grad x, y; hess xx, xy, yy
      static const int ox[5] = {1, 0, 2, 1, 0}, oy[5] = {0, 1, 0, 1, 2};
      const int nslot = 13 * (dp.nlevels + 1);
      for (int c = 0; c < pt.nc; c++) {
        if (dp.ntc.nctas > 0) {
          // the block kernels (tensor cores or FP64) on the derivative tables
          NearTcArgs ta = near_tc_args(dp, 0);
          ta.out_nd = dp.nd * pt.nc;
          ta.out_off = c * dp.nd;
          ta.xoff = ox[pt.c0 + c] * nslot;
          ta.yoff = oy[pt.c0 + c] * nslot;
          (dp.ntc.fp64 ? near_f64_launch : near_tc_launch)(dp.n, dp.ntc.nctas, dp.ntc.smem, s,
                                                            NearTcLaunch{ta, nullptr, nullptr, d_fvals, pt.out});
          continue;
        }
        NearArgs na = near_args(dp, 0);
        na.tab_loc = dp.tab3_loc;
        na.out_nd = dp.nd * pt.nc;
        na.out_off = c * dp.nd;
        na.xoff = ox[pt.c0 + c] * nslot;
        na.yoff = oy[pt.c0 + c] * nslot;
        k_near_fp64<<<(dp.nnf + kWarps - 1) / kWarps, kWarps * 32, dp.smem_near, s>>>(
            NearLaunch{na, nullptr, nullptr, d_fvals, pt.out});
      }
    }
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    msg = std::string("kernel launch failed: ") + cudaGetErrorString(e);
    return BFGT_ERR_CUDA;
  }
  return BFGT_OK;
}

// ---- extra targets (boxfgt.f step 11) ---------------------------------------

namespace {

struct TargArgs {
  const int *nchild, *ichild, *level;  // per box (0-based ids); ichild(4, nboxes), 0-based, -1 none
  const double *centers, *boxsize;     // (2, nboxes), (0:nlevels)
  const double *umat;                  // values -> coefficients (n, n), column-major
  int n, ipoly;
};

// Leaf box of each target, by the descent of pts_tree_sort
// (common/pts_tree_nd.f:1226-1260, find_childbox_ind 713-740): child
// 1 + (x - cx >= 0) + 2 (y - cy >= 0) from the root until a leaf.  Marks the
// leaves that hold targets.
__global__ void k_target_leaf(TargArgs a, const double *__restrict__ targs, int nt, int *__restrict__ leaf_of,
                              int *__restrict__ has_targ) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  const double x = targs[2 * (size_t)t], y = targs[2 * (size_t)t + 1];
  int b = 0;
  while (a.nchild[b] > 0) {
    const int k = (x - a.centers[2 * (size_t)b] >= 0 ? 1 : 0) + (y - a.centers[2 * (size_t)b + 1] >= 0 ? 2 : 0);
    b = a.ichild[4 * (size_t)b + k];
  }
  leaf_of[t] = b;
  has_targ[b] = 1;
}

// Coefficients of the leaves that hold targets: ortho_trans_2d with itype 0
// (common/tensor_prod_routs_nd.f:103-170), one warp per box, ndc components.
__global__ void __launch_bounds__(128) k_leaf_coefs(TargArgs a, const double *__restrict__ vals,
                                                    double *__restrict__ coefs, const int *__restrict__ has_targ,
                                                    int nboxes, int ndc) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int b = blockIdx.x * 4 + warp;
  if (b >= nboxes || !has_targ[b]) return;
  const int n = a.n, npb = n * n;
  double *sw = reinterpret_cast<double *>(smem_raw) + (size_t)warp * npb;
  const double *fin = vals + (size_t)b * ndc * npb;
  double *fout = coefs + (size_t)b * ndc * npb;
  for (int ind = 0; ind < ndc; ind++) {
    // work(k, j) = sum_k1 umat(k, k1) fin(k1, j)
    for (int o = lane; o < npb; o += 32) {
      const int k = o % n, j = o / n;
      double dd = 0;
      for (int k1 = 0; k1 < n; k1++) dd = fma(a.umat[k + n * k1], fin[ind + (size_t)ndc * (k1 + n * j)], dd);
      sw[o] = dd;
    }
    __syncwarp();
    // fout(k, i) = sum_i1 umat(i, i1) work(k, i1)
    for (int o = lane; o < npb; o += 32) {
      const int k = o % n, i = o / n;
      double dd = 0;
      for (int i1 = 0; i1 < n; i1++) dd = fma(a.umat[i + n * i1], sw[k + n * i1], dd);
      fout[ind + (size_t)ndc * o] = dd;
    }
    __syncwarp();
  }
}

// out(ndc, t) = sum_j py(j) sum_k coefs(k, j) px(k) at the target's local
// coordinates (t - c) 2 / boxsize (ortho_evalt_2d, tensor_prod_routs_nd.f:
// 2030-2066; legepols / chebpols recurrences), one thread per target.
__global__ void __launch_bounds__(128) k_eval_targets(TargArgs a, const double *__restrict__ coefs,
                                                      const double *__restrict__ targs, const int *__restrict__ leaf_of,
                                                      int nt, int ndc, double *__restrict__ out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  const int n = a.n, npb = n * n;
  const int b = leaf_of[t];
  const double sc = 2.0 / a.boxsize[a.level[b]];
  const double x = (targs[2 * (size_t)t] - a.centers[2 * (size_t)b]) * sc;
  const double y = (targs[2 * (size_t)t + 1] - a.centers[2 * (size_t)b + 1]) * sc;
  double px[16];
  px[0] = 1.0;
  px[1] = x;
#pragma unroll
  for (int k = 1; k < 15; k++) {
    if (k + 1 < n) {
      if (a.ipoly == 0) px[k + 1] = ((2 * k + 1) * x * px[k] - k * px[k - 1]) / (k + 1);
      else px[k + 1] = 2 * x * px[k] - px[k - 1];
    }
  }
  const double *c = coefs + (size_t)b * ndc * npb;
  for (int ind = 0; ind < ndc; ind++) {
    double pot = 0;
    double pym = 1.0, py = 1.0;  // P_{j-1}(y), P_j(y) by the same recurrence
#pragma unroll 1
    for (int j = 0; j < n; j++) {
      if (j == 1) py = y;
      else if (j > 1) {
        const double pn = a.ipoly == 0 ? ((2 * (j - 1) + 1) * y * py - (j - 1) * pym) / j : 2 * y * py - pym;
        pym = py;
        py = pn;
      }
      if (j == 1) pym = 1.0;
      double pp = 0;
      const double *cj = c + ind + (size_t)ndc * n * j;
#pragma unroll
      for (int k = 0; k < 16; k++)
        if (k < n) pp = pp + cj[(size_t)ndc * k] * px[k];
      pot = pot + pp * py;
    }
    out[ind + (size_t)ndc * t] = pot;
  }
}

}  // namespace

int device_plan_prepare_targets(DevicePlan &dp, const HostPlan &hp, const TreeView &t, std::string &msg) {
  if (dp.targ_ready) return BFGT_OK;
  const int nb = t.nboxes;
  std::vector<int> nchild(nb), ichild(4 * (size_t)nb), level(nb);
  std::vector<double> cen(2 * (size_t)nb), bs(t.boxsize, t.boxsize + t.nlevels + 1);
  for (int b = 1; b <= nb; b++) {
    nchild[b - 1] = t.nchild(b);
    level[b - 1] = t.ilevel(b);
    for (int j = 1; j <= 4; j++) ichild[4 * (size_t)(b - 1) + j - 1] = t.nchild(b) > 0 ? t.ichild(j, b) - 1 : -1;
    cen[2 * (size_t)(b - 1)] = t.cen(1, b);
    cen[2 * (size_t)(b - 1) + 1] = t.cen(2, b);
  }
  std::vector<double> x, u, v, w;
  leaf_nodes(hp.ipoly, hp.norder, x, u, v, w);
  int rc = BFGT_OK;
  auto chk = [&](int r) {
    if (rc == BFGT_OK && r != BFGT_OK) rc = r;
  };
  chk(upload(dp.t_nchild, nchild, msg));
  chk(upload(dp.t_ichild, ichild, msg));
  chk(upload(dp.t_level, level, msg));
  chk(upload(dp.t_centers, cen, msg));
  chk(upload(dp.t_boxsize, bs, msg));
  chk(upload(dp.t_umat, u, msg));
  chk(alloc_bytes((void **)&dp.t_has, sizeof(int) * (size_t)nb, msg));
  if (rc == BFGT_OK) {
    dp.targ_ready = true;
    dp.ipoly = hp.ipoly;
  }
  return rc;
}

int device_plan_eval_targets(DevicePlan &dp, int ncomp, const double *d_vals, int nt, const double *d_targs,
                             double *d_out, cudaStream_t s, std::string &msg) {
  if (!dp.targ_ready) {
    msg = "target tables are not prepared";
    return BFGT_ERR_ARG;
  }
  if (nt <= 0) return BFGT_OK;
  const int ndc = dp.nd * ncomp, npb = dp.n * dp.n;
  const size_t celems = (size_t)ndc * npb * dp.nboxes;
  if (dp.t_coef_elems < celems) {
    if (dp.t_coefs) cudaFree(dp.t_coefs);
    dp.t_coefs = nullptr;
    dp.t_coef_elems = 0;
    if (alloc_bytes((void **)&dp.t_coefs, sizeof(double) * celems, msg) != BFGT_OK) return BFGT_ERR_OOM;
    dp.t_coef_elems = celems;
  }
  if (dp.t_leaf_cap < nt) {
    if (dp.t_leaf) cudaFree(dp.t_leaf);
    dp.t_leaf = nullptr;
    dp.t_leaf_cap = 0;
    if (alloc_bytes((void **)&dp.t_leaf, sizeof(int) * (size_t)nt, msg) != BFGT_OK) return BFGT_ERR_OOM;
    dp.t_leaf_cap = nt;
  }
  TargArgs a{dp.t_nchild, dp.t_ichild, dp.t_level, dp.t_centers, dp.t_boxsize, dp.t_umat, dp.n, dp.ipoly};
  cudaMemsetAsync(dp.t_has, 0, sizeof(int) * (size_t)dp.nboxes, s);
  k_target_leaf<<<(nt + 127) / 128, 128, 0, s>>>(a, d_targs, nt, dp.t_leaf, dp.t_has);
  k_leaf_coefs<<<(dp.nboxes + 3) / 4, 128, sizeof(double) * 4 * npb, s>>>(a, d_vals, dp.t_coefs, dp.t_has, dp.nboxes,
                                                                           ndc);
  k_eval_targets<<<(nt + 127) / 128, 128, 0, s>>>(a, dp.t_coefs, d_targs, dp.t_leaf, nt, ndc, d_out);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    msg = std::string("kernel launch failed: ") + cudaGetErrorString(e);
    return BFGT_ERR_CUDA;
  }
  return BFGT_OK;
}

int device_batch_create(DeviceBatch &b, const std::vector<DevicePlan *> &plans, std::string &msg) {
  device_batch_destroy(b);
  b.plans = plans;
  b.offs.assign(plans.size() + 1, 0);
  for (size_t i = 0; i < plans.size(); i++)
    b.offs[i + 1] = b.offs[i] + (long long)plans[i]->nd * plans[i]->n * plans[i]->n * plans[i]->nboxes;
  int rc = split_batch_create(b.split, plans, b.offs, msg);
  if (rc != BFGT_OK) return rc;
  std::vector<TrArgs> tr;
  std::vector<NearArgs> nf;
  std::vector<NearTcArgs> ntc;
  std::vector<int2> trw, nfw, ntw[4];
  for (size_t i = 0; i < plans.size(); i++) {
    const DevicePlan &dp = *plans[i];
    tr.push_back(tr_args(dp));
    nf.push_back(near_args(dp, b.offs[i]));
    if (has_pw(dp)) {
      const size_t tot = tr_threads(dp.ncut, dp.nd, dp.nexp);
      for (size_t k = 0; k < (tot + kTrThreads - 1) / kTrThreads; k++) trw.push_back(make_int2((int)i, (int)k));
    }
    ntc.push_back(near_tc_args(dp, b.offs[i]));
    if (dp.ntc.nctas > 0) {
      // the block near-field kernels: one launch per kind (tensor cores,
      // FP64) and order (8, 16)
      const int v = (dp.n == 16 ? 1 : 0) + (dp.ntc.fp64 ? 2 : 0);
      for (int c = 0; c < dp.ntc.nctas; c++) ntw[v].push_back(make_int2((int)i, c));
      b.smem_ntc[v] = std::max(b.smem_ntc[v], dp.ntc.smem);
    } else {
      for (int t = 0; t < dp.nnf; t += kWarps) nfw.push_back(make_int2((int)i, t));
      b.smem_near = std::max(b.smem_near, dp.smem_near);
    }
  }
  b.tr_blocks = (int)trw.size();
  b.nf_blocks = (int)nfw.size();
  for (int v = 0; v < 4; v++) b.ntc_blocks[v] = (int)ntw[v].size();
  TrArgs *dtr = nullptr;
  NearArgs *dnf = nullptr;
  NearTcArgs *dnt = nullptr;
  auto chk = [&](int r) {
    if (rc == BFGT_OK && r != BFGT_OK) rc = r;
  };
  chk(upload(dtr, tr, msg));
  chk(upload(dnf, nf, msg));
  chk(upload(b.tr_work, trw, msg));
  chk(upload(b.nf_work, nfw, msg));
  if (b.ntc_blocks[0] + b.ntc_blocks[1] + b.ntc_blocks[2] + b.ntc_blocks[3] > 0) {
    chk(upload(dnt, ntc, msg));
    for (int v = 0; v < 4; v++) chk(upload(b.ntc_work[v], ntw[v], msg));
  }
  b.tr_descs = dtr;
  b.nf_descs = dnf;
  b.ntc_descs = dnt;
  if (rc == BFGT_OK) {
    b.events = true;
    reserve_event_sets(b.evsets, 8);
  }
  return rc;
}

int device_batch_launches(const DeviceBatch &b) {
  int n = split_batch_launches(b.split) + (b.tr_blocks > 0) + (b.nf_blocks > 0);
  for (int v = 0; v < 4; v++) n += b.ntc_blocks[v] > 0;
  for (const DevicePlan *dp : b.plans)
    if (dp->precision != BFGT_PREC_SPLIT && has_pw(*dp)) n += 2;
  return n;
}

int device_batch_execute(DeviceBatch &b, const double *d_fvals, double *d_pot, cudaStream_t s, std::string &msg) {
  NvtxRange range("bfgt batch execute");
  cudaEvent_t *ev = next_events(b.evsets, b.nrec, b.events);
  if (ev) cudaEventRecord(ev[0], s);
  split_batch_form(b.split, d_fvals, s);
  for (size_t i = 0; i < b.plans.size(); i++)
    if (b.plans[i]->precision != BFGT_PREC_SPLIT && has_pw(*b.plans[i])) plan_form(*b.plans[i], d_fvals + b.offs[i], s);
  if (ev) cudaEventRecord(ev[1], s);
  if (ev) cudaEventRecord(ev[2], s);
  if (b.tr_blocks > 0)
    k_translate<<<b.tr_blocks, kTrThreads, 0, s>>>(TrLaunch{TrArgs{}, static_cast<const TrArgs *>(b.tr_descs), b.tr_work});
  if (ev) cudaEventRecord(ev[3], s);
  split_batch_eval(b.split, d_pot, s);
  for (size_t i = 0; i < b.plans.size(); i++)
    if (b.plans[i]->precision != BFGT_PREC_SPLIT && has_pw(*b.plans[i])) plan_eval(*b.plans[i], d_pot + b.offs[i], s);
  if (ev) cudaEventRecord(ev[4], s);
  if (b.nf_blocks > 0)
    k_near_fp64<<<b.nf_blocks, kWarps * 32, b.smem_near, s>>>(
        NearLaunch{NearArgs{}, static_cast<const NearArgs *>(b.nf_descs), b.nf_work, d_fvals, d_pot});
  for (int v = 0; v < 4; v++)
    if (b.ntc_blocks[v] > 0)
      ((v & 2) ? near_f64_launch : near_tc_launch)((v & 1) ? 16 : 8, b.ntc_blocks[v], b.smem_ntc[v], s,
                                                   NearTcLaunch{NearTcArgs{}, static_cast<const NearTcArgs *>(b.ntc_descs),
                                                                b.ntc_work[v], d_fvals, d_pot});
  if (ev) cudaEventRecord(ev[5], s);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    msg = std::string("kernel launch failed: ") + cudaGetErrorString(e);
    return BFGT_ERR_CUDA;
  }
  return BFGT_OK;
}

int device_batch_stage_ms(DeviceBatch &b, double *out) { return read_stage_ms(b.evsets, b.nrec, out); }

void device_batch_destroy(DeviceBatch &b) {
  if (b.graph_exec) cudaGraphExecDestroy(b.graph_exec);
  if (b.graph) cudaGraphDestroy(b.graph);
  split_batch_destroy(b.split);
  void *ptrs[] = {b.tr_descs,      b.nf_descs,      b.tr_work,       b.nf_work,      b.ntc_descs,
                  b.ntc_work[0], b.ntc_work[1], b.ntc_work[2], b.ntc_work[3]};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  for (auto &es : b.evsets)
    for (cudaEvent_t e : es) cudaEventDestroy(e);
  b = DeviceBatch();
}

}  // namespace bfgt
