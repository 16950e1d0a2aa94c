// Split-precision plane-wave kernels on the sm_100a tensor cores (tcgen05):
// the kernel templates, shared by the two translation units that instantiate
// them (split_kernels.cu: floating slices; split_fix.cu: fixed-point slices).
//
// Same sum-factorised scheme as the FP64 kernels (fgt_device.cu): a CTA takes
// up to 128/n columns of one cutoff ancestor and level and walks the
// y-offsets oy present in them.  The per-leaf contractions are tensor-core
// GEMMs with M = 128 rows = (column slot, leaf grid index):
//   form:  D[(slot,m1), (re/im,k2)] += F_{slot,oy}(m1,m2) * Ty_oy(m2,(re/im,k2))
//   eval:  D[(slot,k1), k2] = [Hr|Hi](k1,(re/im,m2)) * [Eyr;-Eyi]((re/im,m2),k2)
// where Ty_oy = T conj(phase_oy) and Ey_oy = w E phase_oy are per-offset tables
// precomputed in FP64 on the host.  The once-per-column contractions (x
// direction) and all cross-leaf sums run in FP64 on the CUDA cores; the
// plane-wave phases stay FP64 throughout.
//
// Every operand is cut into BF16 slices, in one of two ways (a plan property,
// chosen from eps):
// * floating (eps >= 1e-7): x = s0 + s1 + s2, each slice relative to x itself
//   (the tables exactly to ~2^-27 relative, the leaf values and H through
//   FP32, to 2^-24).  The six slice products with i+j <= 2 are accumulated in
//   FP32 in tensor memory, the leading product s0*s0 in its own accumulator
//   and the five corrections in a second one.  The FP32 accumulation rounds
//   at 2^-24 relative: about 1e-6 relative L2 in all.
// * fixed-point (Ozaki, eps < 1e-7): a row of A (one leaf grid row over all
//   steps of a chunk, or one row of H) and a column of B share one power-of-two
//   scale; x / scale is cut into S digits d_c in [-128, 128], slice
//   c = d_c 2^-(7+8c), each exact in BF16.  A product of slices i and j is then
//   an integer multiple of 2^-(14+8(i+j)) of at most 2^14 such units, so the
//   FP32 sums of the level-0 products (i+j = 0) and of the level-1 products
//   are exact as long as they stay below 2^24 units: at most 512 K-terms per
//   accumulation (chunks are cut to respect that).  Levels >= 2 share a third
//   accumulator whose rounding is 2^-40 of the leading term.  The error is then
//   set by the S-digit truncation, 2^-(8S) of the row and column scales.
#pragma once
#include <cuda_bf16.h>

#include <algorithm>
#include <type_traits>

#include "fgt_common.cuh"
#include "tc_sm100.cuh"

namespace bfgt {
namespace splitk {

constexpr int kThreads = 128;
constexpr int kRows = 128;                // MMA M
constexpr uint32_t kWaitIters = 1u << 26;  // bounded spin on an mbarrier
constexpr int kMaxSlices = 6;             // fixed-point digits per operand, at most
// dynamic shared memory opt-in: the 227 KB per-block limit minus room for the
// kernels' static shared variables
constexpr int kMaxDynSmem = 227 * 1024 - 2048;

__device__ __forceinline__ double2 zmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// x (|x| < 1) -> S fixed-point digits: v[c] = d_c 2^-(7+8c), d_c integer in
// [-128, 128], x - sum v[c] at most half the last digit's unit, 2^-(8S), in
// magnitude.  X = rint(x 2^(7 + 8 (S - 1))) is exact for S <= 6 (at most 47
// bits; the scaling is by a power of two), the balanced base-256 digits are
// cut from the least significant one up with integer operations (each
// X - d is a multiple of 256), and the top digit keeps the rest.  Each v[c]
// has at most 8 significant bits, so the conversions to FP32 and BF16 are
// exact.
__device__ __forceinline__ void fix_digits(double x, int S, float (&v)[kMaxSlices]) {
  const int sh = 7 + 8 * (S - 1);
  long long X = __double2ll_rn(x * __longlong_as_double((long long)(1023 + sh) << 52));
#pragma unroll
  for (int c = kMaxSlices - 1; c >= 1; c--) {
    if (c < S) {
      const int d = (int)((X + 128) & 255) - 128;
      X = (X - d) >> 8;
      v[c] = (float)d * __int_as_float((127 - 7 - 8 * c) << 23);
    } else {
      v[c] = 0.0f;
    }
  }
  v[0] = (float)(int)X * (1.0f / 128.0f);
}

// power of two 2^e >= |mx| with mx / 2^e < 1, and its inverse.  Rows whose
// largest value is below 2^-1000 (zero, or the subnormal tail of a Gaussian)
// keep the scale 1: their inverse scale would overflow, and their digits are
// then zero, an absolute error below 2^-1000.
__device__ __forceinline__ void pow2_scale(double mx, double &sc, double &inv) {
  sc = inv = 1.0;
  if (mx > 0x1p-1000) {
    int e;
    frexp(mx, &e);
    sc = ldexp(1.0, e);
    inv = ldexp(1.0, -e);
  }
}

struct FormTcArgs {
  const int4 *chunks;      // {column begin, column end, icut, level}
  const int *step_begin;   // nchunks + 1
  const int *steps;        // stride 1 + cpc: oy, then box per slot (-1: no leaf)
  const int4 *columns;     // {leaf begin, leaf end, ox, -}
  const uint16_t *TyB;     // per (level, oy): S slices x NP rows x KA, K-major core layout
  const long long *tyb_off;
  long long tyb_tile;      // uint16 elements per (level, oy) tile
  const double2 *T;        // tab_poly2pw, per level (n, npw)
  const double2 *PH;
  const long long *ph_off;
  double2 *Mpart;
  ReduceArgs red;
  int *err;
  int nd, n, npw, hh, nexp, cpc, NP, KA;
  uint32_t wait_iters;
  long long elem_off;      // start of this plan's leaf arrays in the (packed) fvals
  const int2 *items;       // {chunk, pass} per CTA; null: CTA b = chunk b, all passes
  const double *csc;       // fixed-point slices: scale of each Ty column, NP per level
  int S;                   // slices per operand
  int pad_;
};

// One launch of the form kernel: a single plan (descs null, CTA b = work item b
// of `one`), or a batch of plans (CTA b = work item work[b].y of plan
// work[b].x).  A plan's work item is a chunk (all its density passes), or
// one pass of a chunk when the plan lists items.
struct FormTcLaunch {
  FormTcArgs one;
  const FormTcArgs *descs;
  const int2 *work;
  const double *fbase;
};

struct EvalTcArgs {
  const int4 *chunks;
  const int *step_begin;
  const int *steps;
  const int4 *columns;
  const uint16_t *EyB;     // per (level, oy): S slices x NB rows x KE, K-major core layout
  const long long *eyb_off;
  long long eyb_tile;
  const double2 *E;        // tab_pw2pot, per level (npw, n)
  const double2 *PH;
  const long long *ph_off;
  const double2 *L;
  int *err;
  int nd, n, npw, hh, nexp, cpc, NB, KE, KH;
  int lslots;              // densities whose L the shared memory holds at once
  int ebatch;              // steps per tensor-core group
  uint32_t wait_iters;
  long long elem_off;      // start of this plan's leaf arrays in the (packed) pot
  const int2 *items;       // {chunk, pass} per CTA; null: CTA b = chunk b, all passes
  const double *esc;       // fixed-point slices: scale of each Ey column (leaf grid index), 16 per level
  int S;                   // slices per operand
  int pad_;
};

struct EvalTcLaunch {
  EvalTcArgs one;
  const EvalTcArgs *descs;
  const int2 *work;
  double *pbase;
};

// Copies this CTA's plan descriptor into shared memory and returns its work item.
template <typename Args, typename Launch>
__device__ __forceinline__ int load_desc(const Launch &lp, Args &dst, int *s_item) {
  const Args *src = lp.descs ? lp.descs + lp.work[blockIdx.x].x : &lp.one;
  for (int i = threadIdx.x; i < (int)(sizeof(Args) / 4); i += blockDim.x)
    reinterpret_cast<int *>(&dst)[i] = reinterpret_cast<const int *>(src)[i];
  if (threadIdx.x == 0) *s_item = lp.descs ? lp.work[blockIdx.x].y : (int)blockIdx.x;
  __syncthreads();
  return *s_item;
}

// Densities packed into the MMA rows.  A chunk of ncol columns fills
// rpd = ncol n rows per density, so dpc = min(nd, 128 / rpd) densities share
// one pass through the chunk's steps.  MMA row (and TMEM lane)
// R = (slot n + m) dpc + dl holds density dl of the pass, the density index
// fastest: the lanes of a warp then cover consecutive densities of a leaf
// point, which are adjacent in the (nd, n, n) leaf layout, so their loads and
// stores of fvals and pot are coalesced.  The passes are balanced:
// npass = ceil(nd / dpc) passes of ceil(nd / npass) densities (the last one
// possibly fewer, never none).
struct DensityPass {
  int rpd, dpc, npass;
};
__device__ __forceinline__ DensityPass density_pass(int ncol, int n, int nd) {
  DensityPass d;
  d.rpd = ncol * n;
  const int dpc = max(min(nd, kRows / d.rpd), 1);
  d.npass = (nd + dpc - 1) / dpc;
  d.dpc = (nd + d.npass - 1) / d.npass;
  return d;
}

// MMAs of one K-block: floating slices, the six products with i+j <= 2 (s0 s0
// into D0, the rest into D1); fixed-point slices, every product with
// i+j <= S-1, level 0 into D0, level 1 into D1, levels >= 2 into D2.
// first: the block starts the accumulation (no accumulate into D0..D2).
template <bool kFix>
__device__ __forceinline__ void issue_slice_mmas(uint32_t tD0, uint32_t tD1, uint32_t tD2, const uint64_t (&ad)[kMaxSlices],
                                                 const uint64_t (&bd)[kMaxSlices], uint32_t idesc, bool first, int S) {
  const uint32_t acc = first ? 0u : 1u;
  tc::mma_bf16(tD0, ad[0], bd[0], idesc, acc);
  tc::mma_bf16(tD1, ad[0], bd[1], idesc, acc);
  tc::mma_bf16(tD1, ad[1], bd[0], idesc, 1u);
  if constexpr (!kFix) {
    tc::mma_bf16(tD1, ad[0], bd[2], idesc, 1u);
    tc::mma_bf16(tD1, ad[1], bd[1], idesc, 1u);
    tc::mma_bf16(tD1, ad[2], bd[0], idesc, 1u);
  } else {
    bool f2 = first;
#pragma unroll
    for (int t = 2; t < kMaxSlices; t++) {
      if (t >= S) break;
#pragma unroll
      for (int i = 0; i <= t; i++) {
        tc::mma_bf16(tD2, ad[i], bd[t - i], idesc, f2 ? 0u : 1u);
        f2 = false;
      }
    }
  }
}

// kBatch: the arguments come from the per-plan descriptors (copied to shared
// memory) instead of the launch's own parameter block.  kPack: densities are
// packed into the rows (plans with nd > 1); without it one density per pass,
// with the row arithmetic folded at compile time, and NT x-contraction tiles
// per thread (1 or 2; unused when packed).  kYF: Y staged as float2 (see sY).
// kN: the leaf order n (8 or 16), so that per-thread arrays hold n values.
// kFix: fixed-point slices (a.S of them); otherwise three floating slices.
template <bool kBatch, bool kPack, int NT, bool kYF, int kN, bool kFix>
__global__ void __launch_bounds__(kThreads) k_form_tc(const __grid_constant__ FormTcLaunch lp) {
  static_assert(!(kFix && kYF), "fixed-point slices need Y in FP64");
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ FormTcArgs s_desc;
  __shared__ int s_item;
  const int item = kBatch ? load_desc(lp, s_desc, &s_item) : (int)blockIdx.x;
  const FormTcArgs &a = kBatch ? s_desc : lp.one;
  const int chunk = (kPack && a.items) ? a.items[item].x : item;  // items exist for nd > 1 only
  const double *fvals = lp.fbase + a.elem_off;
  uint64_t *mbar = reinterpret_cast<uint64_t *>(smem);  // [0],[1] operand buffers, [2] drain
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(smem + 64);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int4 ch = a.chunks[chunk];
  const int n = a.n, npw = a.npw, hh = a.hh, nd = a.nd, npb = n * n, cpc = a.cpc, NP = a.NP, KA = a.KA;
  const int S = kFix ? a.S : 3;
  const int ncol = ch.y - ch.x;
  const DensityPass pk = kPack ? density_pass(ncol, n, nd) : DensityPass{ncol * n, 1, nd};
  // this CTA's density passes: one of an item, or all of the chunk
  const int pitem = (kPack && a.items) ? a.items[item].y : -1;
  const int pbeg = pitem < 0 ? 0 : pitem, pend = pitem < 0 ? pk.npass : pitem + 1;
  const int abytes = S * kRows * KA * 2, bbytes = S * NP * KA * 2, bufbytes = abytes + bbytes;
  // Y = D0 + D1 (+ D2) held as (re, im) in YT.  Floating slices: an FP32 sum,
  // exact as float2 where a double2 Y would be the largest user of this shared
  // area (large npw, unpacked: less shared memory and traffic, measured
  // faster), else double2 (no conversions in the x contraction, measured
  // faster).  Fixed-point slices: an FP64 sum, double2.  Rows padded to an odd
  // number of elements so that the readout's per-row stores spread over the
  // banks.
  using YT = typename std::conditional<kYF, float2, double2>::type;
  const int ys = hh | 1;
  const int ybytes = kRows * ys * (int)sizeof(YT);
  const int ubytes = ((max(2 * bufbytes, ybytes) + 127) / 128) * 128;
  unsigned char *U = smem + 128;
  YT *sY = reinterpret_cast<YT *>(U);  // after the tensor-core loop: [row][k2], row stride ys
  double2 *sT = reinterpret_cast<double2 *>(U + ubytes);  // [m][k] n x npw
  constexpr uint32_t kTmemCols = kFix ? 256 : 128;

  if (warp == 0) tc::tmem_alloc(tmem_slot, kTmemCols);
  if (tid == 0) {
    tc::mbar_init(&mbar[0], 1);
    tc::mbar_init(&mbar[1], 1);
    tc::mbar_init(&mbar[2], 1);
    tc::fence_mbar_init();
  }
  const double2 *Tg = a.T + (size_t)n * npw * ch.w;
  for (int i = tid; i < n * npw; i += kThreads) {
    const int m = i % n, k = i / n;
    sT[m * npw + k] = Tg[i];
  }
  const long long phoff = a.ph_off[ch.w];
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tmem_slot;
  const uint32_t tD0 = tmem, tD1 = tmem + (uint32_t)NP, tD2 = tmem + 2u * (uint32_t)NP;
  const uint32_t idesc = tc::idesc_bf16_f32(kRows, NP);
  const int sb = a.step_begin[chunk], se = a.step_begin[chunk + 1], nsteps = se - sb;
  const int stride = 1 + cpc;
  const uint16_t *tyb = a.TyB + a.tyb_off[ch.w];
  bool ok = true;
  // this thread's A row R = (rslot n + rm1) dpc + rdl
  const int r = tid, rdl = r % pk.dpc, rsk = r / pk.dpc, rslot = rsk / n, rm1 = rsk - rslot * n;

  // per-thread share of a B tile (16-byte pieces)
  const int bpieces = bbytes / 16;
  constexpr int kMaxPieces = kFix ? 1 : 4;  // floating: bbytes <= 3*64*16*2 = 6 KB -> 3 per thread
  for (int pass = pbeg; pass < pend; pass++) {
    const int d0 = pass * pk.dpc, dcnt = kPack ? min(pk.dpc, nd - d0) : 1;
    const bool rowok = rdl < dcnt && rsk < pk.rpd;
    auto leaf_row = [&](int s2) -> const double * {
      const int *st2 = a.steps + (size_t)(sb + s2) * stride;
      const int box = rowok ? st2[1 + rslot] : -1;
      return box < 0 ? nullptr : fvals + (size_t)box * nd * npb + (d0 + rdl) + (size_t)nd * rm1;
    };
    // fixed-point slices: one power-of-two scale per row for the whole pass
    // (every step accumulates into the same TMEM row)
    double rsc = 1.0, rinv = 1.0;
    if constexpr (kFix) {
      double mx = 0.0;
#pragma unroll 4
      for (int s2 = 0; s2 < nsteps; s2++) {
        const double *fv = leaf_row(s2);
        if (!fv) continue;
#pragma unroll
        for (int k = 0; k < kN; k++)
          if (kN == 8 || k < n) mx = fmax(mx, fabs(fv[(size_t)nd * (kN == 8 ? kN : n) * k]));
      }
      pow2_scale(mx, rsc, rinv);
    }
    // software pipeline: the leaf values (and, floating, the B tile) of step
    // s+1 are loaded into registers while step s is converted and multiplied
    double fnext[kN];
    uint4 bnext[kMaxPieces];
    auto load_step = [&](int s2) {
      const double *fv = leaf_row(s2);
#pragma unroll
      for (int k = 0; k < kN; k++)
        // read once: evict-first loads (the leaf values do not displace the
        // expansions and pot lines in L2; A/B on the bench tree: the step
        // 219.8 -> 212.4 us together with the eval kernel's streaming pot)
        fnext[k] = (fv && (kN == 8 || k < n)) ? __ldcs(fv + (size_t)nd * (kN == 8 ? kN : n) * k) : 0.0;
      if constexpr (!kFix) {
        const int *st2 = a.steps + (size_t)(sb + s2) * stride;
        const uint4 *src = reinterpret_cast<const uint4 *>(tyb + (size_t)st2[0] * a.tyb_tile);
#pragma unroll
        for (int q = 0; q < kMaxPieces; q++) {
          const int i = tid + kThreads * q;
          if (i < bpieces) bnext[q] = src[i];
        }
      }
    };
    if (nsteps > 0) load_step(0);
    for (int s = 0; s < nsteps; s++) {
      const int g = (pass - pbeg) * nsteps + s, b = g & 1;  // operand buffer uses so far
      double fcur[kN];
      uint4 bcur[kMaxPieces];
#pragma unroll
      for (int k = 0; k < kN; k++) fcur[k] = fnext[k];
#pragma unroll
      for (int q = 0; q < kMaxPieces; q++) bcur[q] = bnext[q];
      if (s + 1 < nsteps) load_step(s + 1);
      if (g >= 2 && ok && !tc::mbar_wait(&mbar[b], ((g >> 1) - 1) & 1, a.wait_iters)) {
        ok = false;
        atomicExch(a.err, 1);
      }
      unsigned char *Ab = U + b * bufbytes, *Bb = Ab + abytes;
      if constexpr (kFix) {
        // the step's B tile straight into the free buffer (the digit split
        // below covers the copy's latency)
        const int oy = a.steps[(size_t)(sb + s) * stride];
        const unsigned char *src = reinterpret_cast<const unsigned char *>(tyb + (size_t)oy * a.tyb_tile);
        for (int i = tid; i < bpieces; i += kThreads) tc::cp_async16(Bb + 16 * i, src + 16 * i);
        tc::cp_async_commit();
      }
      // A row r = (slot, m1, dl): F(m1, m2) for m2 = 0..n-1, zero-padded to KA
#pragma unroll
      for (int h = 0; h < 2; h++) {
        if (h >= KA / 8) break;
        const uint32_t off = tc::kmajor_off(r, 8 * h, kRows);
        if constexpr (kFix) {
          uint32_t p[kMaxSlices][4];
#pragma unroll
          for (int q = 0; q < 4; q++) {
            const int k = 8 * h + 2 * q;  // K columns past n are zero
            float v0[kMaxSlices], v1[kMaxSlices];
            fix_digits(k < kN ? fcur[k < kN ? k : 0] * rinv : 0.0, S, v0);
            fix_digits(k + 1 < kN ? fcur[k + 1 < kN ? k + 1 : 0] * rinv : 0.0, S, v1);
#pragma unroll
            for (int c = 0; c < kMaxSlices; c++)  // (exact BF16 values: their top 16 bits)
              p[c][q] = __byte_perm(__float_as_uint(v0[c]), __float_as_uint(v1[c]), 0x7632);
          }
#pragma unroll
          for (int c = 0; c < kMaxSlices; c++)
            if (c < S) *reinterpret_cast<uint4 *>(Ab + c * kRows * KA * 2 + off) = *reinterpret_cast<uint4 *>(p[c]);
        } else {
          uint32_t s0[4], s1[4], s2[4];
#pragma unroll
          for (int q = 0; q < 4; q++) {
            const int k = 8 * h + 2 * q;  // K columns past n are zero
            tc::split3_bf16x2(k < kN ? fcur[k < kN ? k : 0] : 0.0, k + 1 < kN ? fcur[k + 1 < kN ? k + 1 : 0] : 0.0,
                              s0[q], s1[q], s2[q]);
          }
          *reinterpret_cast<uint4 *>(Ab + off) = *reinterpret_cast<uint4 *>(s0);
          *reinterpret_cast<uint4 *>(Ab + kRows * KA * 2 + off) = *reinterpret_cast<uint4 *>(s1);
          *reinterpret_cast<uint4 *>(Ab + 2 * kRows * KA * 2 + off) = *reinterpret_cast<uint4 *>(s2);
        }
      }
      if constexpr (kFix) {
        tc::cp_async_wait_all();
      } else {
#pragma unroll
        for (int q = 0; q < kMaxPieces; q++) {
          const int i = tid + kThreads * q;
          if (i < bpieces) reinterpret_cast<uint4 *>(Bb)[i] = bcur[q];
        }
      }
      tc::fence_async_smem();
      tc::fence_before_sync();
      __syncthreads();
      if (tid == 0 && ok) {
        tc::fence_after_sync();
        const uint32_t aA = tc::smem_u32(Ab), aB = tc::smem_u32(Bb);
        const uint32_t lboA = (kRows / 8) * 128, lboB = (NP / 8) * 128;
        for (int kk = 0; kk < KA / 16; kk++) {
          uint64_t ad[kMaxSlices], bd[kMaxSlices];
#pragma unroll
          for (int c = 0; c < kMaxSlices; c++) {
            const int cc = c < S ? c : 0;
            ad[c] = tc::smem_desc(aA + cc * kRows * KA * 2 + kk * 2 * lboA, lboA, 128);
            bd[c] = tc::smem_desc(aB + cc * NP * KA * 2 + kk * 2 * lboB, lboB, 128);
          }
          issue_slice_mmas<kFix>(tD0, tD1, tD2, ad, bd, idesc, s == 0 && kk == 0, S);
        }
        tc::commit(&mbar[b]);
      }
    }
    if (nsteps > 0) {
      const int gl = (pass - pbeg) * nsteps + nsteps - 1;
      if (ok && !tc::mbar_wait(&mbar[gl & 1], (gl >> 1) & 1, a.wait_iters)) {
        ok = false;
        atomicExch(a.err, 1);
      }
    }
    tc::fence_after_sync();
    // read the accumulators of this thread's row and sum them
    {
      const uint32_t lanebase = (uint32_t)(32 * warp) << 16;
      const double *csc = kFix ? a.csc + (size_t)ch.w * NP : nullptr;
      for (int j0 = 0; j0 < NP; j0 += 16) {
        float v0[16], v1[16];
        tc::tmem_ld16(tD0 + lanebase + j0, v0);
        tc::tmem_ld16(tD1 + lanebase + j0, v1);
        tc::tmem_ld_wait();
        if constexpr (kFix) {
          double y[16];
#pragma unroll
          for (int i = 0; i < 16; i++) y[i] = (double)v0[i] + (double)v1[i];
          tc::tmem_ld16(tD2 + lanebase + j0, v0);
          tc::tmem_ld_wait();
#pragma unroll
          for (int i = 0; i < 16; i++) {
            const int j = j0 + i;
            const double yv = ok ? (y[i] + (double)v0[i]) * rsc * __ldg(&csc[j]) : 0.0;
            if (j < hh) sY[r * ys + j].x = yv;
            else if (j < 2 * hh) sY[r * ys + (j - hh)].y = yv;
          }
        } else {
#pragma unroll
          for (int i = 0; i < 16; i++) {
            const int j = j0 + i;
            // D0 + D1 in FP32 (one more rounding of 2^-24, below the accumulated
            // error); the x contraction converts it to FP64 exactly
            const float y = ok ? v0[i] + v1[i] : 0.0f;  // stored exactly in YT
            if (j < hh) sY[r * ys + j].x = y;
            else if (j < 2 * hh) sY[r * ys + (j - hh)].y = y;
          }
        }
      }
    }
    tc::fence_before_sync();
    __syncthreads();
    // x contraction (FP64) of each density dl of the pass:
    // M(k1,k2) = sum_{slot,m1} T(m1,k1) conj(ph_ox(k1)) Y((slot n + m1) dpc + dl, k2),
    // in 2 x 4 tiles (k1 pair, k2 quad): NT per thread unpacked, (dl, tile)
    // pairs over the block packed
    {
      const int ntm = (npw + 1) / 2, ntd = ntm * ((hh + 3) / 4), ntiles = dcnt * ntd;
      const int yst = pk.dpc * ys;  // row stride between grid points of one density
      for (int it = 0; kPack || it < NT; it++) {
        const int tile = tid + kThreads * it;
        if (tile >= ntiles) break;
        const int dl = kPack ? tile / ntd : 0, tt = tile - dl * ntd;
        const int k1b = (tt % ntm) * 2, k2b = (tt / ntm) * 4;
        const YT *Yd = sY + (size_t)dl * ys;
        double2 acc[2][4];
#pragma unroll
        for (int i = 0; i < 2; i++)
#pragma unroll
          for (int j = 0; j < 4; j++) acc[i][j] = make_double2(0, 0);
        for (int slot = 0; slot < ncol; slot++) {
          double2 ph[2];
          const double2 *phs = a.PH + phoff + (size_t)a.columns[ch.x + slot].z * npw;
#pragma unroll
          for (int i = 0; i < 2; i++) {
            const double2 p = (k1b + i < npw) ? phs[k1b + i] : make_double2(0, 0);
            ph[i] = make_double2(p.x, -p.y);
          }
          for (int m1 = 0; m1 < n; m1++) {
            double2 av[2], bv[4];
#pragma unroll
            for (int i = 0; i < 2; i++) av[i] = zmul((k1b + i < npw) ? sT[m1 * npw + k1b + i] : make_double2(0, 0), ph[i]);
#pragma unroll
            for (int j = 0; j < 4; j++) {
              const YT y = (k2b + j < hh) ? Yd[(slot * n + m1) * yst + k2b + j] : YT{0, 0};
              bv[j] = make_double2(y.x, y.y);
            }
#pragma unroll
            for (int i = 0; i < 2; i++)
#pragma unroll
              for (int j = 0; j < 4; j++) {
                acc[i][j].x = fma(av[i].x, bv[j].x, acc[i][j].x);
                acc[i][j].x = fma(-av[i].y, bv[j].y, acc[i][j].x);
                acc[i][j].y = fma(av[i].x, bv[j].y, acc[i][j].y);
                acc[i][j].y = fma(av[i].y, bv[j].x, acc[i][j].y);
              }
          }
        }
        double2 *out = a.Mpart + ((size_t)chunk * nd + d0 + dl) * a.nexp;
#pragma unroll
        for (int i = 0; i < 2; i++)
#pragma unroll
          for (int j = 0; j < 4; j++)
            if (k1b + i < npw && k2b + j < hh) out[(size_t)(k2b + j) * npw + k1b + i] = acc[i][j];
      }
    }
    __syncthreads();
  }
  // drain: no tensor-core operation of this CTA may be in flight when TMEM is freed
  if (tid == 0) tc::commit(&mbar[2]);
  if (!tc::mbar_wait(&mbar[2], 0, kWaitIters)) atomicExch(a.err, 2);
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, kTmemCols);
  finish_cutoff_box(a.red, chunk, nd, a.nexp, reinterpret_cast<int *>(smem + 68));
}

// Steps of a chunk per tensor-core group in the eval kernel: the group's B
// operand is the step tiles side by side, N = 16 x steps (the TMEM
// accumulators hold 128 columns each with floating slices, 64 with
// fixed-point ones, which use three accumulators).  A plan uses fewer where
// that is what keeps two CTAs per SM (large npw).
constexpr int kEvalBatchMax = 8;
constexpr int kEvalBatchFix = 4;
constexpr int kEvalThreads = 256;

// H rows of kT 8-row tiles that share one density's L, on the FP64 tensor
// cores: the real GEMM [Hr Hi] = [Er Ei] [[Lr Li], [-Li Lr]] with K = (m1,
// re/im) and N = (m2, re/im) interleaved, E(m1,k1) phase_ox(m1) formed on the
// fly.  Lane (g8, t4) of tile mt has row slot rs[mt] and grid index rk[mt].
template <int NNT, int kT>
__device__ __forceinline__ void h_tiles(double (&c)[kT][NNT][2], const double2 *sE, const double2 *sph,
                                        const double2 *Lt, const int (&rs)[kT], const int (&rk)[kT], int n, int npw,
                                        int hh, int g8, int t4) {
#pragma unroll
  for (int mt = 0; mt < kT; mt++)
#pragma unroll
    for (int i = 0; i < NNT; i++) c[mt][i][0] = c[mt][i][1] = 0.0;
  const int p = t4 & 1, q = g8 & 1;
  for (int j = 0; j < (npw + 1) / 2; j++) {
    const int m1 = 2 * j + (t4 >> 1);
    const bool mok = m1 < npw;
    double av[kT];
#pragma unroll
    for (int mt = 0; mt < kT; mt++) {
      double v = 0.0;
      if (mok) {
        const double2 e = zmul(sE[m1 * n + rk[mt]], sph[rs[mt] * npw + m1]);
        v = p ? e.y : e.x;
      }
      av[mt] = v;
    }
#pragma unroll
    for (int i = 0; i < NNT; i++) {
      const int m2 = 4 * i + (g8 >> 1);
      double bv = 0.0;
      if (mok && m2 < hh) {
        const double2 l = Lt[m1 * hh + m2];
        bv = p == 0 ? (q == 0 ? l.x : l.y) : (q == 0 ? -l.y : l.x);
      }
#pragma unroll
      for (int mt = 0; mt < kT; mt++) tc::dmma_8x8x4(c[mt][i], av[mt], bv);
    }
  }
}

// Lane (g8, t4) holds (Hr, Hi) of row r at m2 = 4i + t4: cut into the slices
// of the A operand (K = re/im x m2).  Fixed-point slices: the 4 lanes of the
// row (t4 = 0..3, a quad) agree on the row's power-of-two scale, stored in
// s_rsc[r] for the readout; every lane of the warp must call this.
template <int NNT, bool kFix>
__device__ __forceinline__ void h_to_operand(unsigned char *sA, int r, const double (&c)[NNT][2], int t4, int hh,
                                             int KH, int KE, int S, double *s_rsc) {
  if constexpr (kFix) {
    double mx = 0.0;
#pragma unroll
    for (int i = 0; i < NNT; i++)
      if (4 * i + t4 < hh) mx = fmax(mx, fmax(fabs(c[i][0]), fabs(c[i][1])));
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, 1));
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, 2));
    double sc, inv;
    pow2_scale(mx, sc, inv);
    if (t4 == 0) s_rsc[r] = sc;
#pragma unroll
    for (int i = 0; i < NNT; i++) {
      const int m2 = 4 * i + t4;
      if (m2 >= hh) continue;
      const uint32_t ore = tc::kmajor_off(r, m2, kRows), oim = tc::kmajor_off(r, KH + m2, kRows);
      float vr[kMaxSlices], vi[kMaxSlices];
      fix_digits(c[i][0] * inv, S, vr);
      fix_digits(c[i][1] * inv, S, vi);
#pragma unroll
      for (int cc = 0; cc < kMaxSlices; cc++) {
        if (cc >= S) break;
        // (exact BF16 values: their top 16 bits)
        *reinterpret_cast<uint16_t *>(sA + cc * kRows * KE * 2 + ore) = (uint16_t)(__float_as_uint(vr[cc]) >> 16);
        *reinterpret_cast<uint16_t *>(sA + cc * kRows * KE * 2 + oim) = (uint16_t)(__float_as_uint(vi[cc]) >> 16);
      }
    }
  } else {
#pragma unroll
    for (int i = 0; i < NNT; i++) {
      const int m2 = 4 * i + t4;
      if (m2 >= hh) continue;
      uint16_t s0, s1, s2;
      const uint32_t ore = tc::kmajor_off(r, m2, kRows), oim = tc::kmajor_off(r, KH + m2, kRows);
      tc::split3_bf16x1(c[i][0], s0, s1, s2);
      *reinterpret_cast<uint16_t *>(sA + ore) = s0;
      *reinterpret_cast<uint16_t *>(sA + kRows * KE * 2 + ore) = s1;
      *reinterpret_cast<uint16_t *>(sA + 2 * kRows * KE * 2 + ore) = s2;
      tc::split3_bf16x1(c[i][1], s0, s1, s2);
      *reinterpret_cast<uint16_t *>(sA + oim) = s0;
      *reinterpret_cast<uint16_t *>(sA + kRows * KE * 2 + oim) = s1;
      *reinterpret_cast<uint16_t *>(sA + 2 * kRows * KE * 2 + oim) = s2;
    }
  }
}

// Cutoff expansions -> leaf values (steps 4+5).  One CTA of 8 warps per chunk,
// two CTAs per SM.  H(k1,m2) = sum_m1 E(m1,k1) phase_ox(m1) L(m1,m2) is formed
// in FP64 once per chunk and density, on 8-row tiles of one density each, and
// cut into the A operand (row (slot n + k1) dpc + dl, K = re/im x m2).  The
// steps are then taken a.ebatch at a time: their Ey tiles are copied side by
// side into one B operand (cp.async, issued while the previous group is read
// out), the slice MMAs with N = 16 x steps produce the values of every leaf of
// the group, and the readout adds 2 (D0 + D1 (+ D2)) into pot.  Warps w and w+4
// share TMEM lanes 32 (w%4).. and split the group's steps.  H is formed for
// a.lslots densities at a time (their L in shared memory), so the packing of
// densities into rows does not depend on the shared-memory size.
// Shared memory: [A][B][E (npw x n)][phases (cpc x npw)][L (lslots x npw x hh)].
template <int NNT, bool kBatch, bool kPack, int kN, bool kFix>
__global__ void __launch_bounds__(kEvalThreads, 2) k_eval_tc(const __grid_constant__ EvalTcLaunch lp) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ EvalTcArgs s_desc;
  __shared__ int s_item;
  __shared__ double s_rsc[kFix ? kRows : 1];  // fixed-point slices: scale of each H row
  __shared__ double s_esc[kFix ? 16 : 1];     // and of each Ey column
  const int item = kBatch ? load_desc(lp, s_desc, &s_item) : (int)blockIdx.x;
  const EvalTcArgs &a = kBatch ? s_desc : lp.one;
  const int chunk = (kPack && a.items) ? a.items[item].x : item;  // items exist for nd > 1 only
  double *pot = lp.pbase + a.elem_off;
  uint64_t *mbar = reinterpret_cast<uint64_t *>(smem);  // [0] MMA group done, [1] drain
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(smem + 64);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int4 ch = a.chunks[chunk];
  const int n = a.n, npw = a.npw, hh = a.hh, nd = a.nd, npb = n * n, cpc = a.cpc, KE = a.KE, KH = a.KH;
  const int S = kFix ? a.S : 3;
  const int ncol = ch.y - ch.x;
  const DensityPass pk = kPack ? density_pass(ncol, n, nd) : DensityPass{ncol * n, 1, nd};
  // this CTA's density passes: one of an item, or all of the chunk
  const int pitem = (kPack && a.items) ? a.items[item].y : -1;
  const int pbeg = pitem < 0 ? 0 : pitem, pend = pitem < 0 ? pk.npass : pitem + 1;
  const int nl = npw * hh;  // L entries per density
  const int eb = a.ebatch;
  const int abytes = S * kRows * KE * 2, bbytes = S * (16 * eb) * KE * 2;
  unsigned char *sA = smem + 128;
  unsigned char *sB = sA + ((abytes + 127) / 128) * 128;
  double2 *sE = reinterpret_cast<double2 *>(sB + ((bbytes + 127) / 128) * 128);  // [m1][k1]
  double2 *sph = sE + (size_t)npw * n;                                            // [slot][m1]
  double2 *sL = sph + (size_t)cpc * npw;                                          // [dl][m1][m2]
  // accumulator column stride: D0, D1 (and D2) side by side in 256 columns
  constexpr uint32_t kAS = kFix ? 16 * kEvalBatchFix : 16 * kEvalBatchMax;

  if (warp == 0) tc::tmem_alloc(tmem_slot, 256);
  if (tid == 0) {
    tc::mbar_init(&mbar[0], 1);
    tc::mbar_init(&mbar[1], 1);
    tc::fence_mbar_init();
  }
  const int sb = a.step_begin[chunk], se = a.step_begin[chunk + 1], nsteps = se - sb;
  const int stride = 1 + cpc;
  const uint16_t *eyb = a.EyB + a.eyb_off[ch.w];
  const int nbatch = (nsteps + eb - 1) / eb;
  // Ey tiles of steps [s0, s0+Sg) -> B rows 16 s .. 16 s + 15 (K-major core layout, N = 16 Sg)
  auto load_batch = [&](int s0, int Sg) {
    const int N = 16 * Sg, KG = KE / 8, U = S * KG * 16;
    for (int u = tid; u < U * Sg; u += kEvalThreads) {
      const int st = u / U, rem = u - st * U;
      const int c = rem / (KG * 16), kg = (rem >> 4) % KG, w = rem & 15;
      const int oy = a.steps[(size_t)(sb + s0 + st) * stride];
      const unsigned char *src =
          reinterpret_cast<const unsigned char *>(eyb + (size_t)oy * a.eyb_tile) + c * (16 * KE * 2) + kg * 256 + w * 16;
      tc::cp_async16(sB + c * (N * KE * 2) + (kg * (N / 8) + 2 * st) * 128 + w * 16, src);
    }
    tc::cp_async_commit();
  };
  if (nbatch > 0) load_batch(0, min(eb, nsteps));
  // E(m1,k1) of this level and the x phases of the chunk's columns (FP64)
  for (int i = tid; i < npw * n; i += kEvalThreads) {
    const int m = i % npw, k = i / npw;
    sE[m * n + k] = a.E[(size_t)n * npw * ch.w + i];
  }
  for (int i = tid; i < ncol * npw; i += kEvalThreads) {
    const int slot = i / npw, m = i - slot * npw;
    sph[i] = a.PH[a.ph_off[ch.w] + (size_t)a.columns[ch.x + slot].z * npw + m];
  }
  if constexpr (kFix) {
    if (tid < 16) s_esc[tid] = tid < n ? a.esc[(size_t)ch.w * 16 + tid] : 0.0;
  }
  // A columns that H never writes: m2 in [hh, KH) of both parts, and K in [2 KH, KE)
  {
    const int padr = KH - hh, padk = KE - 2 * KH, per = 2 * padr + padk;
    for (int i = tid; i < kRows * per; i += kEvalThreads) {
      const int r = i / per, e = i - r * per;
      const int k = e < padr ? hh + e : (e < 2 * padr ? KH + hh + (e - padr) : 2 * KH + (e - 2 * padr));
      const uint32_t o = tc::kmajor_off(r, k, kRows);
      for (int c = 0; c < S; c++) *reinterpret_cast<uint16_t *>(sA + c * kRows * KE * 2 + o) = 0;
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tmem_slot;
  bool ok = true;
  int g = 0;  // MMA groups issued so far (mbarrier phase)

  for (int pass = pbeg; pass < pend; pass++) {
    const int d0 = pass * pk.dpc, dcnt = kPack ? min(pk.dpc, nd - d0) : 1;
    // H for logical rows r = (dl, slot, k1) (h_tiles).  Warp w owns logical
    // rows 16w..16w+15 (two 8-row tiles, each of one density dl) and all NNT
    // column tiles.  Densities [dg, dg + lslots) are formed together; a tile
    // whose density is outside that range waits for its own group.
    for (int dg = 0; dg < dcnt; dg += a.lslots) {
      const int gcnt = min(a.lslots, dcnt - dg);
      if (dg > 0) __syncthreads();  // every warp is done with the previous group's L
      for (int e = tid; e < gcnt * nl; e += kEvalThreads) {
        const int dl = e / nl, el = e - dl * nl;
        const int m2 = el / npw, m1 = el - m2 * npw;
        sL[(size_t)dl * nl + m1 * hh + m2] = a.L[((size_t)ch.z * nd + d0 + dg + dl) * a.nexp + el];
      }
      __syncthreads();
      const int g8 = lane >> 2, t4 = lane & 3;
      // the warp's two 8-row tiles of logical rows (dl, slot, k1): slot and
      // grid index of this lane's row, its MMA row (slot n + k1) dpc + dl,
      // offset of the tile density's L in sL, and whether that density is in
      // the group
      int rs[2], rk[2], lo[2], prow[2];
      bool tv[2];
#pragma unroll
      for (int mt = 0; mt < 2; mt++) {
        const int r0 = 16 * warp + 8 * mt;
        const int dl = r0 / pk.rpd;
        tv[mt] = dl >= dg && dl < dg + gcnt;
        lo[mt] = (dl - dg) * nl;
        const int rr = r0 + g8 - dl * pk.rpd;
        rs[mt] = rr / n;
        rk[mt] = rr - rs[mt] * n;
        prow[mt] = rr * pk.dpc + dl;
      }
      if (tv[0] && tv[1] && lo[0] == lo[1]) {
        // both tiles, one density (every full-width chunk)
        double c[2][NNT][2];
        h_tiles<NNT, 2>(c, sE, sph, sL + lo[0], rs, rk, n, npw, hh, g8, t4);
        h_to_operand<NNT, kFix>(sA, prow[0], c[0], t4, hh, KH, KE, S, s_rsc);
        h_to_operand<NNT, kFix>(sA, prow[1], c[1], t4, hh, KH, KE, S, s_rsc);
      } else {
        // tiles of two densities, or one tile in the group: one tile at a time
#pragma unroll 1
        for (int mt = 0; mt < 2; mt++) {
          if (!(mt ? tv[1] : tv[0])) continue;
          const int rs1[1] = {mt ? rs[1] : rs[0]}, rk1[1] = {mt ? rk[1] : rk[0]};
          double c[1][NNT][2];
          h_tiles<NNT, 1>(c, sE, sph, sL + (mt ? lo[1] : lo[0]), rs1, rk1, n, npw, hh, g8, t4);
          h_to_operand<NNT, kFix>(sA, mt ? prow[1] : prow[0], c[0], t4, hh, KH, KE, S, s_rsc);
        }
      }
    }
    for (int j = 0; j < nbatch; j++, g++) {
      const int s0 = j * eb, Sg = min(eb, nsteps - s0), N = 16 * Sg;
      tc::cp_async_wait_all();
      tc::fence_async_smem();
      tc::fence_before_sync();
      __syncthreads();
      if (tid == 0 && ok) {
        tc::fence_after_sync();
        const uint32_t aA = tc::smem_u32(sA), aB = tc::smem_u32(sB);
        const uint32_t lboA = (kRows / 8) * 128, lboB = (uint32_t)(N / 8) * 128;
        const uint32_t idesc = tc::idesc_bf16_f32(kRows, N);
        for (int kk = 0; kk < KE / 16; kk++) {
          uint64_t ad[kMaxSlices], bd[kMaxSlices];
#pragma unroll
          for (int c = 0; c < kMaxSlices; c++) {
            const int cc = c < S ? c : 0;
            ad[c] = tc::smem_desc(aA + cc * kRows * KE * 2 + kk * 2 * lboA, lboA, 128);
            bd[c] = tc::smem_desc(aB + cc * N * KE * 2 + kk * 2 * lboB, lboB, 128);
          }
          issue_slice_mmas<kFix>(tmem, tmem + kAS, tmem + 2 * kAS, ad, bd, idesc, kk == 0, S);
        }
        tc::commit(&mbar[0]);
      }
      // readout: warp w covers TMEM lanes 32 (w%4)..; warps 0-3 take even steps, 4-7 odd steps
      {
        const int qw = warp & 3, r = 32 * qw + lane, rdl = r % pk.dpc, rsk = r / pk.dpc;
        const int rslot = rsk / n, rk1 = rsk - rslot * n;
        const bool rowok = rdl < dcnt && rsk < pk.rpd;
        const uint32_t lb = (uint32_t)(32 * qw) << 16;
        double pv[kN];
        double *pb = nullptr;
        auto load_pot = [&](int st) {
          const int box = (rowok && st < Sg) ? a.steps[(size_t)(sb + s0 + st) * stride + 1 + rslot] : -1;
          pb = box >= 0 ? pot + (size_t)box * nd * npb + (d0 + rdl) + (size_t)nd * rk1 : nullptr;
#pragma unroll
          for (int k2 = 0; k2 < kN; k2++)  // (n = 16: the same code as before kN existed)
            // pot is read and written once per launch: streaming (evict-first) accesses
            pv[k2] = (pb && (kN == 8 || k2 < n)) ? __ldcs(pb + (size_t)nd * (kN == 8 ? kN : n) * k2) : 0.0;
        };
        // the group's first pot lines do not depend on the MMAs: in flight while they run
        load_pot(warp >> 2);
        if (ok && !tc::mbar_wait(&mbar[0], g & 1, a.wait_iters)) {
          ok = false;
          atomicExch(a.err, 1);
        }
        tc::fence_after_sync();
        // the B buffer is free again: fetch the next group's tiles during the readout
        if (j + 1 < nbatch) load_batch(s0 + eb, min(eb, nsteps - s0 - eb));
        else if (pass + 1 < pend) load_batch(0, min(eb, nsteps));
        const double f2 = kFix && rowok ? 2.0 * s_rsc[r] : 2.0;
        for (int st = warp >> 2; st < Sg; st += 2) {
          double pc[kN];
#pragma unroll
          for (int k2 = 0; k2 < kN; k2++) pc[k2] = pv[k2];
          double *pbc = pb;
          if (st + 2 < Sg) load_pot(st + 2);
          // L2 prefetch of this lane's line (k2 = rk1) of its step st + 4 box
          if (rowok && st + 4 < Sg) {
            const int box4 = a.steps[(size_t)(sb + s0 + st + 4) * stride + 1 + rslot];
            if (box4 >= 0)
              asm volatile("prefetch.global.L2 [%0];" ::"l"(pot + (size_t)box4 * nd * npb + (d0 + rdl) +
                                                             (size_t)nd * rk1 * (n + 1)));
          }
          float v0[kN], v1[kN];  // columns 16 st .. 16 st + n - 1 of the step
          const uint32_t col = lb + (uint32_t)(16 * st);
          if constexpr (kN == 16) {
            tc::tmem_ld16(tmem + col, v0);
            tc::tmem_ld16(tmem + kAS + col, v1);
          } else {
            tc::tmem_ld8(tmem + col, v0);
            tc::tmem_ld8(tmem + kAS + col, v1);
          }
          tc::tmem_ld_wait();
          if constexpr (kFix) {
#pragma unroll
            for (int k2 = 0; k2 < kN; k2++) pc[k2] = fma(f2 * s_esc[k2], (double)v0[k2] + (double)v1[k2], pc[k2]);
            if constexpr (kN == 16) tc::tmem_ld16(tmem + 2 * kAS + col, v0);
            else tc::tmem_ld8(tmem + 2 * kAS + col, v0);
            tc::tmem_ld_wait();
            if (ok && pbc) {
              // streaming store, as in the floating-slice readout
#pragma unroll
              for (int k2 = 0; k2 < kN; k2++)
                if (kN == 8 || k2 < n)
                  __stcs(pbc + (size_t)nd * (kN == 8 ? kN : n) * k2, fma(f2 * s_esc[k2], (double)v0[k2], pc[k2]));
            }
          } else {
            if (ok && pbc) {
#pragma unroll
              for (int k2 = 0; k2 < kN; k2++)
                if (kN == 8 || k2 < n) __stcs(pbc + (size_t)nd * (kN == 8 ? kN : n) * k2, pc[k2] + 2.0 * (double)(v0[k2] + v1[k2]));
            }
          }
        }
      }
      tc::fence_before_sync();
      __syncthreads();
    }
  }
  tc::cp_async_wait_all();
  if (tid == 0) tc::commit(&mbar[1]);
  if (!tc::mbar_wait(&mbar[1], 0, kWaitIters)) atomicExch(a.err, 2);
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, 256);
}

// Launches of the compiled variants (split_kernels.cu instantiates the
// floating-slice ones, split_fix.cu the fixed-point ones).
// form variant: 0, 1 = unpacked with 1, 2 x-contraction tiles per thread (+2
// with Y as float2; floating slices only); 4 = packed; +5 for n = 16.
template <bool kFix>
void launch_form(int variant, int grid, size_t smem, cudaStream_t s, const FormTcLaunch &lp);
// eval variant: nnt (column tiles of H, 1..8), packed or not, n = 16 or 8
template <bool kFix>
void launch_eval(int nnt, bool pack, bool n16, int grid, size_t smem, cudaStream_t s, const EvalTcLaunch &lp);
// Opts every kernel variant into the full dynamic shared memory.
template <bool kFix>
void set_smem_attrs();

extern template void launch_form<false>(int, int, size_t, cudaStream_t, const FormTcLaunch &);
extern template void launch_form<true>(int, int, size_t, cudaStream_t, const FormTcLaunch &);
extern template void launch_eval<false>(int, bool, bool, int, size_t, cudaStream_t, const EvalTcLaunch &);
extern template void launch_eval<true>(int, bool, bool, int, size_t, cudaStream_t, const EvalTcLaunch &);
extern template void set_smem_attrs<false>();
extern template void set_smem_attrs<true>();

}  // namespace splitk
}  // namespace bfgt
