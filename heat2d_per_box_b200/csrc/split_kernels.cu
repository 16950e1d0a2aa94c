// Split-precision plane-wave kernels on the sm_100a tensor cores (tcgen05).
//
// Same sum-factorised scheme as the FP64 kernels (fgt_device.cu): a CTA takes
// up to 128/n columns of one cutoff ancestor and level and walks the
// y-offsets oy present in them.  The per-leaf contractions are tensor-core
// GEMMs with M = 128 rows = (column slot, leaf grid index):
//   form:  D[(slot,m1), (re/im,k2)] += F_{slot,oy}(m1,m2) * Ty_oy(m2,(re/im,k2))
//   eval:  D[(slot,k1), k2] = [Hr|Hi](k1,(re/im,m2)) * [Eyr;-Eyi]((re/im,m2),k2)
// where Ty_oy = T conj(phase_oy) and Ey_oy = w E phase_oy are per-offset tables
// precomputed in FP64 on the host.  Every operand is split into three BF16
// slices (x = s0 + s1 + s2: the tables exactly to ~2^-27 relative, the leaf
// values and H through FP32, to 2^-24); the six slice products with
// i+j <= 2 are accumulated in FP32 in tensor memory, the leading product s0*s0
// in its own accumulator and the five correction products in a second one,
// and the two are summed in FP64.  The once-per-column contractions (x
// direction) and all cross-leaf sums run in FP64 on the CUDA cores; the
// plane-wave phases stay FP64 throughout.
#include <cuda_bf16.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/bfgt.h"
#include "fgt_common.cuh"
#include "split_kernels.cuh"
#include "tc_sm100.cuh"

namespace bfgt {

namespace {

constexpr int kThreads = 128;
constexpr int kRows = 128;                // MMA M
constexpr uint32_t kWaitIters = 1u << 26;  // bounded spin on an mbarrier
// dynamic shared memory opt-in: the 227 KB per-block limit minus room for the
// kernels' static shared variables
constexpr int kMaxDynSmem = 227 * 1024 - 1024;
// resident form CTAs per SM (registers and TMEM of the unpacked variants), and
// the shortest step range a long chunk is cut into
constexpr int kFormCtasPerSm = 4;
constexpr int kLongChunkSteps = 32;
constexpr int kPieceCols = 4;  // columns of a group split off a short, wide group
constexpr int kMinPieceSteps = 16;
// dynamic shared memory of an eval CTA that still lets two CTAs share an SM
// (228 KB per SM, 1 KB reserved per CTA, the kernel's static variables)
constexpr int kEvalSmemTwoPerSm = 112 * 1024;

__device__ __forceinline__ double2 zmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

struct FormTcArgs {
  const int4 *chunks;      // {column begin, column end, icut, level}
  const int *step_begin;   // nchunks + 1
  const int *steps;        // stride 1 + cpc: oy, then box per slot (-1: no leaf)
  const int4 *columns;     // {leaf begin, leaf end, ox, -}
  const uint16_t *TyB;     // per (level, oy): 3 slices x NP rows x KA, K-major core layout
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

// kBatch: the arguments come from the per-plan descriptors (copied to shared
// memory) instead of the launch's own parameter block.  kPack: densities are
// packed into the rows (plans with nd > 1); without it one density per pass,
// with the row arithmetic folded at compile time, and NT x-contraction tiles
// per thread (1 or 2; unused when packed).  kYF: Y staged as float2 (see sY).
// kN: the leaf order n (8 or 16), so that per-thread arrays hold n values.
template <bool kBatch, bool kPack, int NT, bool kYF, int kN>
__global__ void __launch_bounds__(kThreads) k_form_tc(const __grid_constant__ FormTcLaunch lp) {
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
  const int ncol = ch.y - ch.x;
  const DensityPass pk = kPack ? density_pass(ncol, n, nd) : DensityPass{ncol * n, 1, nd};
  // this CTA's density passes: one of an item, or all of the chunk
  const int pitem = (kPack && a.items) ? a.items[item].y : -1;
  const int pbeg = pitem < 0 ? 0 : pitem, pend = pitem < 0 ? pk.npass : pitem + 1;
  const int abytes = 3 * kRows * KA * 2, bbytes = 3 * NP * KA * 2, bufbytes = abytes + bbytes;
  // Y = D0 + D1 is an FP32 sum, held exactly as (re, im) in YT: float2 where
  // a double2 Y would be the largest user of this shared area (large npw,
  // unpacked: less shared memory and traffic, measured faster), else double2
  // (no conversions in the x contraction, measured faster).  Rows padded to
  // an odd number of elements so that the readout's per-row stores spread
  // over the banks.
  using YT = typename std::conditional<kYF, float2, double2>::type;
  const int ys = hh | 1;
  const int ybytes = kRows * ys * (int)sizeof(YT);
  const int ubytes = ((std::max(2 * bufbytes, ybytes) + 127) / 128) * 128;
  unsigned char *U = smem + 128;
  YT *sY = reinterpret_cast<YT *>(U);  // after the tensor-core loop: [row][k2], row stride ys
  double2 *sT = reinterpret_cast<double2 *>(U + ubytes);  // [m][k] n x npw

  if (warp == 0) tc::tmem_alloc(tmem_slot, 128);
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
  const uint32_t tD0 = tmem, tD1 = tmem + (uint32_t)NP;
  const uint32_t idesc = tc::idesc_bf16_f32(kRows, NP);
  const int sb = a.step_begin[chunk], se = a.step_begin[chunk + 1], nsteps = se - sb;
  const int stride = 1 + cpc;
  const uint16_t *tyb = a.TyB + a.tyb_off[ch.w];
  bool ok = true;
  // this thread's A row R = (rslot n + rm1) dpc + rdl
  const int r = tid, rdl = r % pk.dpc, rsk = r / pk.dpc, rslot = rsk / n, rm1 = rsk - rslot * n;

  // per-thread share of a B tile (16-byte pieces)
  const int bpieces = bbytes / 16;
  constexpr int kMaxPieces = 4;  // bbytes <= 3*64*16*2 = 6 KB -> 384 pieces / 128 threads = 3
  for (int pass = pbeg; pass < pend; pass++) {
    const int d0 = pass * pk.dpc, dcnt = kPack ? min(pk.dpc, nd - d0) : 1;
    const bool rowok = rdl < dcnt && rsk < pk.rpd;
    // software pipeline: the leaf values and the B tile of step s+1 are
    // loaded into registers while step s is converted and multiplied
    double fnext[kN];
    uint4 bnext[kMaxPieces];
    auto load_step = [&](int s2) {
      const int *st2 = a.steps + (size_t)(sb + s2) * stride;
      const int box = rowok ? st2[1 + rslot] : -1;
      const double *fv = fvals + (size_t)(box < 0 ? 0 : box) * nd * npb + (d0 + rdl) + (size_t)nd * rm1;
#pragma unroll
      for (int k = 0; k < kN; k++)
        fnext[k] = (box >= 0 && (kN == 8 || k < n)) ? fv[(size_t)nd * (kN == 8 ? kN : n) * k] : 0.0;
      const uint4 *src = reinterpret_cast<const uint4 *>(tyb + (size_t)st2[0] * a.tyb_tile);
#pragma unroll
      for (int q = 0; q < kMaxPieces; q++) {
        const int i = tid + kThreads * q;
        if (i < bpieces) bnext[q] = src[i];
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
      // A row r = (slot, m1, dl): F(m1, m2) for m2 = 0..n-1, zero-padded to KA
#pragma unroll
      for (int h = 0; h < 2; h++) {
        if (h >= KA / 8) break;
        uint32_t s0[4], s1[4], s2[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
          const int k = 8 * h + 2 * q;  // K columns past n are zero
          tc::split3_bf16x2(k < kN ? fcur[k < kN ? k : 0] : 0.0, k + 1 < kN ? fcur[k + 1 < kN ? k + 1 : 0] : 0.0, s0[q],
                            s1[q], s2[q]);
        }
        const uint32_t off = tc::kmajor_off(r, 8 * h, kRows);
        *reinterpret_cast<uint4 *>(Ab + off) = *reinterpret_cast<uint4 *>(s0);
        *reinterpret_cast<uint4 *>(Ab + kRows * KA * 2 + off) = *reinterpret_cast<uint4 *>(s1);
        *reinterpret_cast<uint4 *>(Ab + 2 * kRows * KA * 2 + off) = *reinterpret_cast<uint4 *>(s2);
      }
#pragma unroll
      for (int q = 0; q < kMaxPieces; q++) {
        const int i = tid + kThreads * q;
        if (i < bpieces) reinterpret_cast<uint4 *>(Bb)[i] = bcur[q];
      }
      tc::fence_async_smem();
      tc::fence_before_sync();
      __syncthreads();
      if (tid == 0 && ok) {
        tc::fence_after_sync();
        const uint32_t aA = tc::smem_u32(Ab), aB = tc::smem_u32(Bb);
        const uint32_t lboA = (kRows / 8) * 128, lboB = (NP / 8) * 128;
        for (int kk = 0; kk < KA / 16; kk++) {
          uint64_t ad[3], bd[3];
#pragma unroll
          for (int c = 0; c < 3; c++) {
            ad[c] = tc::smem_desc(aA + c * kRows * KA * 2 + kk * 2 * lboA, lboA, 128);
            bd[c] = tc::smem_desc(aB + c * NP * KA * 2 + kk * 2 * lboB, lboB, 128);
          }
          const uint32_t acc = (s > 0 || kk > 0) ? 1u : 0u;
          tc::mma_bf16(tD0, ad[0], bd[0], idesc, acc);
          tc::mma_bf16(tD1, ad[0], bd[1], idesc, acc);
          tc::mma_bf16(tD1, ad[1], bd[0], idesc, 1u);
          tc::mma_bf16(tD1, ad[0], bd[2], idesc, 1u);
          tc::mma_bf16(tD1, ad[1], bd[1], idesc, 1u);
          tc::mma_bf16(tD1, ad[2], bd[0], idesc, 1u);
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
    // read the two accumulators of this thread's row and sum them
    {
      const uint32_t lanebase = (uint32_t)(32 * warp) << 16;
      for (int j0 = 0; j0 < NP; j0 += 16) {
        float v0[16], v1[16];
        tc::tmem_ld16(tD0 + lanebase + j0, v0);
        tc::tmem_ld16(tD1 + lanebase + j0, v1);
        tc::tmem_ld_wait();
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
  if (warp == 0) tc::tmem_dealloc(tmem, 128);
  finish_cutoff_box(a.red, chunk, nd, a.nexp, reinterpret_cast<int *>(smem + 68));
}

struct EvalTcArgs {
  const int4 *chunks;
  const int *step_begin;
  const int *steps;
  const int4 *columns;
  const uint16_t *EyB;     // per (level, oy): 3 slices x NB rows x KE, K-major core layout
  const long long *eyb_off;
  long long eyb_tile;
  const double2 *E;        // tab_pw2pot, per level (npw, n)
  const double2 *PH;
  const long long *ph_off;
  const double2 *L;
  int *err;
  int nd, n, npw, hh, nexp, cpc, NB, KE, KH;
  int lslots;              // densities whose L the shared memory holds at once
  int ebatch;              // steps per tensor-core group (8, or 4 when shared memory is short)
  uint32_t wait_iters;
  long long elem_off;      // start of this plan's leaf arrays in the (packed) pot
  const int2 *items;       // {chunk, pass} per CTA; null: CTA b = chunk b, all passes
};

struct EvalTcLaunch {
  EvalTcArgs one;
  const EvalTcArgs *descs;
  const int2 *work;
  double *pbase;
};

// Steps of a chunk per tensor-core group in the eval kernel: the group's B
// operand is the step tiles side by side, N = 16 x steps <= 128 (the TMEM
// accumulators hold 128 columns each).  A plan uses 4 instead where that is
// what keeps two CTAs per SM (large npw).
constexpr int kEvalBatchMax = 8;
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

// Lane (g8, t4) holds (Hr, Hi) of row r at m2 = 4i + t4: split into the three
// BF16 slices of the A operand (K = re/im x m2).
template <int NNT>
__device__ __forceinline__ void h_to_operand(unsigned char *sA, int r, const double (&c)[NNT][2], int t4, int hh,
                                             int KH, int KE) {
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

// Cutoff expansions -> leaf values (steps 4+5).  One CTA of 8 warps per chunk,
// two CTAs per SM.  H(k1,m2) = sum_m1 E(m1,k1) phase_ox(m1) L(m1,m2) is formed
// in FP64 once per chunk and density, on 8-row tiles of one density each, and
// split into the A operand (row (slot n + k1) dpc + dl, K = re/im x m2).  The
// steps are then taken a.ebatch at a time: their Ey tiles are copied side by
// side into one B operand (cp.async, issued while the previous group is read
// out), 18 MMAs with N = 16 x steps produce the values of every leaf of the
// group, and the readout adds 2 (D0 + D1) into pot.  Warps w and w+4 share
// TMEM lanes 32 (w%4).. and split the group's steps.  H is formed for
// a.lslots densities at a time (their L in shared memory), so the packing of
// densities into rows does not depend on the shared-memory size.
// Shared memory: [A][B][E (npw x n)][phases (cpc x npw)][L (lslots x npw x hh)].
template <int NNT, bool kBatch, bool kPack, int kN>
__global__ void __launch_bounds__(kEvalThreads, 2) k_eval_tc(const __grid_constant__ EvalTcLaunch lp) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ EvalTcArgs s_desc;
  __shared__ int s_item;
  const int item = kBatch ? load_desc(lp, s_desc, &s_item) : (int)blockIdx.x;
  const EvalTcArgs &a = kBatch ? s_desc : lp.one;
  const int chunk = (kPack && a.items) ? a.items[item].x : item;  // items exist for nd > 1 only
  double *pot = lp.pbase + a.elem_off;
  uint64_t *mbar = reinterpret_cast<uint64_t *>(smem);  // [0] MMA group done, [1] drain
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(smem + 64);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int4 ch = a.chunks[chunk];
  const int n = a.n, npw = a.npw, hh = a.hh, nd = a.nd, npb = n * n, cpc = a.cpc, KE = a.KE, KH = a.KH;
  const int ncol = ch.y - ch.x;
  const DensityPass pk = kPack ? density_pass(ncol, n, nd) : DensityPass{ncol * n, 1, nd};
  // this CTA's density passes: one of an item, or all of the chunk
  const int pitem = (kPack && a.items) ? a.items[item].y : -1;
  const int pbeg = pitem < 0 ? 0 : pitem, pend = pitem < 0 ? pk.npass : pitem + 1;
  const int nl = npw * hh;  // L entries per density
  const int eb = a.ebatch;
  const int abytes = 3 * kRows * KE * 2, bbytes = 3 * (16 * eb) * KE * 2;
  unsigned char *sA = smem + 128;
  unsigned char *sB = sA + ((abytes + 127) / 128) * 128;
  double2 *sE = reinterpret_cast<double2 *>(sB + ((bbytes + 127) / 128) * 128);  // [m1][k1]
  double2 *sph = sE + (size_t)npw * n;                                            // [slot][m1]
  double2 *sL = sph + (size_t)cpc * npw;                                          // [dl][m1][m2]

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
  // Ey tiles of steps [s0, s0+S) -> B rows 16 s .. 16 s + 15 (K-major core layout, N = 16 S)
  auto load_batch = [&](int s0, int S) {
    const int N = 16 * S, KG = KE / 8, U = 3 * KG * 16;
    for (int u = tid; u < U * S; u += kEvalThreads) {
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
  // A columns that H never writes: m2 in [hh, KH) of both parts, and K in [2 KH, KE)
  {
    const int padr = KH - hh, padk = KE - 2 * KH, per = 2 * padr + padk;
    for (int i = tid; i < kRows * per; i += kEvalThreads) {
      const int r = i / per, e = i - r * per;
      const int k = e < padr ? hh + e : (e < 2 * padr ? KH + hh + (e - padr) : 2 * KH + (e - 2 * padr));
      const uint32_t o = tc::kmajor_off(r, k, kRows);
#pragma unroll
      for (int c = 0; c < 3; c++) *reinterpret_cast<uint16_t *>(sA + c * kRows * KE * 2 + o) = 0;
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
        h_to_operand<NNT>(sA, prow[0], c[0], t4, hh, KH, KE);
        h_to_operand<NNT>(sA, prow[1], c[1], t4, hh, KH, KE);
      } else {
        // tiles of two densities, or one tile in the group: one tile at a time
#pragma unroll 1
        for (int mt = 0; mt < 2; mt++) {
          if (!(mt ? tv[1] : tv[0])) continue;
          const int rs1[1] = {mt ? rs[1] : rs[0]}, rk1[1] = {mt ? rk[1] : rk[0]};
          double c[1][NNT][2];
          h_tiles<NNT, 1>(c, sE, sph, sL + (mt ? lo[1] : lo[0]), rs1, rk1, n, npw, hh, g8, t4);
          h_to_operand<NNT>(sA, mt ? prow[1] : prow[0], c[0], t4, hh, KH, KE);
        }
      }
    }
    for (int j = 0; j < nbatch; j++, g++) {
      const int s0 = j * eb, S = min(eb, nsteps - s0), N = 16 * S;
      tc::cp_async_wait_all();
      tc::fence_async_smem();
      tc::fence_before_sync();
      __syncthreads();
      if (tid == 0 && ok) {
        tc::fence_after_sync();
        const uint32_t aA = tc::smem_u32(sA), aB = tc::smem_u32(sB);
        const uint32_t lboA = (kRows / 8) * 128, lboB = (uint32_t)(N / 8) * 128;
        const uint32_t idesc = tc::idesc_bf16_f32(kRows, N);
        const uint32_t d0t = tmem, d1t = tmem + 128;
        for (int kk = 0; kk < KE / 16; kk++) {
          uint64_t ad[3], bd[3];
#pragma unroll
          for (int c = 0; c < 3; c++) {
            ad[c] = tc::smem_desc(aA + c * kRows * KE * 2 + kk * 2 * lboA, lboA, 128);
            bd[c] = tc::smem_desc(aB + c * N * KE * 2 + kk * 2 * lboB, lboB, 128);
          }
          const uint32_t acc = kk > 0 ? 1u : 0u;
          tc::mma_bf16(d0t, ad[0], bd[0], idesc, acc);
          tc::mma_bf16(d1t, ad[0], bd[1], idesc, acc);
          tc::mma_bf16(d1t, ad[1], bd[0], idesc, 1u);
          tc::mma_bf16(d1t, ad[0], bd[2], idesc, 1u);
          tc::mma_bf16(d1t, ad[1], bd[1], idesc, 1u);
          tc::mma_bf16(d1t, ad[2], bd[0], idesc, 1u);
        }
        tc::commit(&mbar[0]);
      }
      if (ok && !tc::mbar_wait(&mbar[0], g & 1, a.wait_iters)) {
        ok = false;
        atomicExch(a.err, 1);
      }
      tc::fence_after_sync();
      // the B buffer is free again: fetch the next group's tiles during the readout
      if (j + 1 < nbatch) load_batch(s0 + eb, min(eb, nsteps - s0 - eb));
      else if (pass + 1 < pend) load_batch(0, min(eb, nsteps));
      // readout: warp w covers TMEM lanes 32 (w%4)..; warps 0-3 take even steps, 4-7 odd steps
      {
        const int qw = warp & 3, r = 32 * qw + lane, rdl = r % pk.dpc, rsk = r / pk.dpc;
        const int rslot = rsk / n, rk1 = rsk - rslot * n;
        const bool rowok = rdl < dcnt && rsk < pk.rpd;
        const uint32_t lb = (uint32_t)(32 * qw) << 16;
        double pv[kN];
        double *pb = nullptr;
        auto load_pot = [&](int st) {
          const int box = (rowok && st < S) ? a.steps[(size_t)(sb + s0 + st) * stride + 1 + rslot] : -1;
          pb = box >= 0 ? pot + (size_t)box * nd * npb + (d0 + rdl) + (size_t)nd * rk1 : nullptr;
#pragma unroll
          for (int k2 = 0; k2 < kN; k2++)  // (n = 16: the same code as before kN existed)
            pv[k2] = (pb && (kN == 8 || k2 < n)) ? pb[(size_t)nd * (kN == 8 ? kN : n) * k2] : 0.0;
        };
        load_pot(warp >> 2);
        for (int st = warp >> 2; st < S; st += 2) {
          double pc[kN];
#pragma unroll
          for (int k2 = 0; k2 < kN; k2++) pc[k2] = pv[k2];
          double *pbc = pb;
          if (st + 2 < S) load_pot(st + 2);
          float v0[kN], v1[kN];  // columns 16 st .. 16 st + n - 1 of the step
          if constexpr (kN == 16) {
            tc::tmem_ld16(tmem + lb + (uint32_t)(16 * st), v0);
            tc::tmem_ld16(tmem + lb + 128u + (uint32_t)(16 * st), v1);
          } else {
            tc::tmem_ld8(tmem + lb + (uint32_t)(16 * st), v0);
            tc::tmem_ld8(tmem + lb + 128u + (uint32_t)(16 * st), v1);
          }
          tc::tmem_ld_wait();
          if (ok && pbc) {
#pragma unroll
            for (int k2 = 0; k2 < kN; k2++)
              if (kN == 8 || k2 < n) pbc[(size_t)nd * (kN == 8 ? kN : n) * k2] = pc[k2] + 2.0 * (double)(v0[k2] + v1[k2]);
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

// Opts every kernel variant into the full dynamic shared memory (per device;
// cheap to repeat).
void set_split_smem_attrs() {
#define SMEM_ATTR(K) cudaFuncSetAttribute(K, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
#define SMEM_FORM(N)                                                                         \
  SMEM_ATTR((k_form_tc<false, false, 1, false, N>)) SMEM_ATTR((k_form_tc<true, false, 1, false, N>)) \
  SMEM_ATTR((k_form_tc<false, false, 2, false, N>)) SMEM_ATTR((k_form_tc<true, false, 2, false, N>)) \
  SMEM_ATTR((k_form_tc<false, false, 1, true, N>)) SMEM_ATTR((k_form_tc<true, false, 1, true, N>))   \
  SMEM_ATTR((k_form_tc<false, false, 2, true, N>)) SMEM_ATTR((k_form_tc<true, false, 2, true, N>))   \
  SMEM_ATTR((k_form_tc<false, true, 1, false, N>)) SMEM_ATTR((k_form_tc<true, true, 1, false, N>))
  SMEM_FORM(8) SMEM_FORM(16)
#undef SMEM_FORM
#define SMEM_EVAL(X, N)                                                                    \
  SMEM_ATTR((k_eval_tc<X, false, false, N>)) SMEM_ATTR((k_eval_tc<X, true, false, N>)) \
  SMEM_ATTR((k_eval_tc<X, false, true, N>)) SMEM_ATTR((k_eval_tc<X, true, true, N>))
#define SMEM_EVAL_N(N)                                                                                 \
  SMEM_EVAL(1, N) SMEM_EVAL(2, N) SMEM_EVAL(3, N) SMEM_EVAL(4, N) SMEM_EVAL(5, N) SMEM_EVAL(6, N) \
  SMEM_EVAL(7, N) SMEM_EVAL(8, N)
  SMEM_EVAL_N(8) SMEM_EVAL_N(16)
#undef SMEM_EVAL_N
#undef SMEM_EVAL
#undef SMEM_ATTR
}

// ---- host-side table preparation -----------------------------------------

uint16_t bf16_bits(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  if ((u & 0x7f800000u) == 0x7f800000u) return (uint16_t)(u >> 16);  // inf / nan
  u += 0x7fffu + ((u >> 16) & 1u);
  return (uint16_t)(u >> 16);
}
float bf16_to_float(uint16_t b) {
  uint32_t u = (uint32_t)b << 16;
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}
void split3_host(double v, uint16_t *s) {
  s[0] = bf16_bits((float)v);
  const double r1 = v - (double)bf16_to_float(s[0]);
  s[1] = bf16_bits((float)r1);
  const double r2 = r1 - (double)bf16_to_float(s[1]);
  s[2] = bf16_bits((float)r2);
}
size_t kmajor_off_host(int r, int k, int R) {
  return (size_t)((((k >> 3) * (R >> 3) + (r >> 3)) << 7) + ((r & 7) << 4) + ((k & 7) << 1));
}

template <typename T>
int upload_vec(T *&d, const std::vector<T> &v, std::string &msg) {
  d = nullptr;
  if (v.empty()) return BFGT_OK;
  if (cudaMalloc(&d, sizeof(T) * v.size()) != cudaSuccess) {
    msg = "cudaMalloc failed (split tables)";
    return BFGT_ERR_OOM;
  }
  if (cudaMemcpy(d, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
    msg = "cudaMemcpy failed (split tables)";
    return BFGT_ERR_CUDA;
  }
  return BFGT_OK;
}

inline cplx cmulh(cplx a, cplx b) { return cplx{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }

}  // namespace

int split_plan_create(DevicePlan &dp, const HostPlan &hp, std::string &msg) {
  const int n = hp.norder, npw = hp.npw, hh = hp.hh, nl = hp.nlevels, ls = hp.nlevstart;
  if (n != 8 && n != 16) {
    msg = "split precision supports norder 8 and 16";
    return BFGT_ERR_CAPACITY;
  }
  if (hh > 32) {
    msg = "split precision supports npw <= 64";
    return BFGT_ERR_CAPACITY;
  }
  SplitPlan &sp = dp.split;
  sp.cpc = kRows / n;
  sp.KA = 16;
  sp.NP = ((2 * hh + 15) / 16) * 16;
  sp.KH = ((hh + 7) / 8) * 8;
  sp.KE = ((2 * sp.KH + 15) / 16) * 16;
  sp.NB = 16;
  int nsm = 0;
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dp.device) != cudaSuccess || nsm <= 0) {
    cudaGetLastError();
    nsm = 148;
  }
  const int slots = kFormCtasPerSm * nsm;  // resident form CTAs on the GPU
  // column groups: up to cpc columns of one (icut, level)
  const std::vector<Column> &cols = hp.columns;
  std::vector<std::pair<size_t, size_t>> groups;
  for (size_t c = 0; c < cols.size();) {
    size_t e = c;
    while (e < cols.size() && cols[e].icut == cols[c].icut && cols[e].level == cols[c].level && (int)(e - c) < sp.cpc) e++;
    groups.emplace_back(c, e);
    c = e;
  }
  // A plan whose groups fill less than a quarter of the form kernel's CTA
  // slots (a small tree, or a coarse cutoff level) splits its short, wide
  // groups (at most kLongChunkSteps steps, more than kPieceCols columns) into
  // groups of kPieceCols columns: each column is still contracted once, the
  // work spreads over more SMs.  Long groups are cut into step ranges below.
  if (!groups.empty() && 4 * (int)groups.size() <= slots) {
    std::vector<std::pair<size_t, size_t>> g2;
    for (const auto &gr : groups) {
      std::vector<int> oys;
      for (size_t q = gr.first; q < gr.second; q++)
        for (int i = cols[q].begin; i < cols[q].end; i++) oys.push_back(hp.leaves[i].oy);
      std::sort(oys.begin(), oys.end());
      const int nsteps = (int)(std::unique(oys.begin(), oys.end()) - oys.begin());
      if ((int)(gr.second - gr.first) > kPieceCols && nsteps <= kLongChunkSteps) {
        for (size_t q = gr.first; q < gr.second; q += kPieceCols) g2.emplace_back(q, std::min(q + kPieceCols, gr.second));
      } else {
        g2.push_back(gr);
      }
    }
    groups.swap(g2);
  }
  // chunks (one per group) and their oy steps
  std::vector<int4> chunks;
  std::vector<int> step_begin(1, 0), steps;
  for (const auto &gr : groups) {
    const size_t c = gr.first, e = gr.second;
    chunks.push_back(make_int4((int)c, (int)e, cols[c].icut, cols[c].level));
    std::vector<size_t> ptr(e - c);
    for (size_t q = c; q < e; q++) ptr[q - c] = cols[q].begin;
    for (;;) {
      int oy = INT32_MAX;
      for (size_t q = c; q < e; q++)
        if (ptr[q - c] < (size_t)cols[q].end) oy = std::min(oy, hp.leaves[ptr[q - c]].oy);
      if (oy == INT32_MAX) break;
      steps.push_back(oy);
      for (int slot = 0; slot < sp.cpc; slot++) {
        size_t q = c + slot;
        if (q < e && ptr[slot] < (size_t)cols[q].end && hp.leaves[ptr[slot]].oy == oy) {
          steps.push_back(hp.leaves[ptr[slot]].box);
          ptr[slot]++;
        } else {
          steps.push_back(-1);
        }
      }
    }
    step_begin.push_back((int)(steps.size() / (1 + sp.cpc)));
  }
  // A plan with few, long chunks (a coarse cutoff level: one cutoff box at
  // delta = 1e-2 on an order-16 tree gives 35 chunks of up to 256 steps)
  // would leave most SMs idle.  When the chunks fill less than a quarter of
  // the form kernel's CTA slots, chunks of more than kLongChunkSteps steps
  // are cut into step ranges of about (total steps) / (slots), at least
  // kMinPieceSteps: each piece is a chunk of the same columns.  The form kernel's x contraction and the eval
  // kernel's H are then done once per piece; the partial expansions of the
  // pieces are summed by the same reduction as those of separate chunks.
  {
    const int nch = (int)chunks.size(), total = step_begin.back();
    if (nch > 0 && 4 * nch <= slots) {
      const int smax = std::max(kMinPieceSteps, (total + slots - 1) / slots);
      std::vector<int4> pc;
      std::vector<int> pb(1, 0);
      for (int c = 0; c < nch; c++) {
        const int s0 = step_begin[c], ns = step_begin[c + 1] - s0;
        const int pieces = ns > kLongChunkSteps ? (ns + smax - 1) / smax : 1, per = (ns + pieces - 1) / pieces;
        for (int q = s0; q < s0 + ns; q += per) {
          pc.push_back(chunks[c]);
          pb.push_back(std::min(q + per, s0 + ns));
        }
      }
      chunks.swap(pc);
      step_begin.swap(pb);
    }
  }
  // per (level, offset) operand tables
  const long long tyt = 3LL * sp.NP * sp.KA, eyt = 3LL * sp.NB * sp.KE;
  std::vector<long long> tyoff(nl + 1, 0), eyoff(nl + 1, 0);
  long long nty = 0, ney = 0;
  for (int l = ls; l <= nl; l++) {
    const long long S = 1LL << (l - ls);
    tyoff[l] = nty;
    eyoff[l] = ney;
    nty += S * tyt;
    ney += S * eyt;
  }
  std::vector<uint16_t> TyB((size_t)nty, 0), EyB((size_t)ney, 0);
  for (int l = ls; l <= nl; l++) {
    const long long S = 1LL << (l - ls);
    const cplx *T = &hp.tab_poly2pw[(size_t)n * npw * l];
    const cplx *E = &hp.tab_pw2pot[(size_t)n * npw * l];
    for (long long o = 0; o < S; o++) {
      const cplx *ph = &hp.phase[(size_t)hp.phase_off[l] + (size_t)o * npw];
      uint16_t *ty = &TyB[(size_t)(tyoff[l] + o * tyt)];
      const size_t ts = (size_t)sp.NP * sp.KA;  // elements per slice
      for (int k2 = 0; k2 < hh; k2++)
        for (int m2 = 0; m2 < n; m2++) {
          const cplx t = cmulh(T[m2 + (size_t)n * k2], cplx{ph[k2].re, -ph[k2].im});
          uint16_t sr[3], si[3];
          split3_host(t.re, sr);
          split3_host(t.im, si);
          for (int c = 0; c < 3; c++) {
            *(uint16_t *)((char *)(ty + c * ts) + kmajor_off_host(k2, m2, sp.NP)) = sr[c];
            *(uint16_t *)((char *)(ty + c * ts) + kmajor_off_host(hh + k2, m2, sp.NP)) = si[c];
          }
        }
      uint16_t *ey = &EyB[(size_t)(eyoff[l] + o * eyt)];
      const size_t es = (size_t)sp.NB * sp.KE;
      for (int k2 = 0; k2 < n; k2++)
        for (int m2 = 0; m2 < hh; m2++) {
          const cplx e0 = cmulh(E[m2 + (size_t)npw * k2], ph[m2]);
          const double w = hp.pw_weight[m2];
          uint16_t sr[3], si[3];
          split3_host(w * e0.re, sr);
          split3_host(-w * e0.im, si);
          for (int c = 0; c < 3; c++) {
            *(uint16_t *)((char *)(ey + c * es) + kmajor_off_host(k2, m2, sp.NB)) = sr[c];
            *(uint16_t *)((char *)(ey + c * es) + kmajor_off_host(k2, sp.KH + m2, sp.NB)) = si[c];
          }
        }
    }
  }
  sp.tyb_tile = tyt;
  sp.eyb_tile = eyt;
  sp.nchunks = (int)chunks.size();
  int rc = BFGT_OK;
  auto chk = [&](int x) {
    if (rc == BFGT_OK && x != BFGT_OK) rc = x;
  };
  chk(upload_vec(sp.chunks, chunks, msg));
  chk(upload_vec(sp.step_begin, step_begin, msg));
  chk(upload_vec(sp.steps, steps, msg));
  chk(upload_vec(sp.TyB, TyB, msg));
  chk(upload_vec(sp.EyB, EyB, msg));
  chk(upload_vec(sp.tyb_off, tyoff, msg));
  chk(upload_vec(sp.eyb_off, eyoff, msg));
  std::vector<int> zero(4, 0);
  chk(upload_vec(sp.err, zero, msg));
  if (rc != BFGT_OK) return rc;
  // the reduction and the rest of the pipeline use the tensor-core chunking
  if (dp.Mpart) cudaFree(dp.Mpart);
  dp.Mpart = nullptr;
  if (cudaMalloc(&dp.Mpart, sizeof(double2) * (size_t)dp.nd * dp.nexp * std::max<size_t>(chunks.size(), 1)) != cudaSuccess) {
    msg = "cudaMalloc failed (split partial expansions)";
    return BFGT_ERR_OOM;
  }
  {
    std::vector<int> cut_of_chunk(chunks.size());
    for (size_t c = 0; c < chunks.size(); c++) cut_of_chunk[c] = chunks[c].z;
    dp.nchunks = (int)chunks.size();
    // nd > 1: one CTA per density pass of a chunk (the passes write disjoint
    // densities; a wide chunk's passes would otherwise run one after another
    // in one CTA).  The pass count is the kernels' density_pass.
    std::vector<int> arrivals;
    if (dp.nd > 1) {
      std::vector<int2> items;
      arrivals.resize(chunks.size());
      for (size_t c = 0; c < chunks.size(); c++) {
        const int rpd = (chunks[c].y - chunks[c].x) * n;
        const int dpc = std::max(std::min(dp.nd, kRows / rpd), 1);
        const int npass = (dp.nd + dpc - 1) / dpc;
        arrivals[c] = npass;
        for (int p = 0; p < npass; p++) items.push_back(make_int2((int)c, p));
      }
      chk(upload_vec(sp.items, items, msg));
      sp.nitems = (int)items.size();
      sp.items_nd = dp.nd;
    }
    chk(build_reduce_groups(dp, cut_of_chunk, msg, arrivals));
  }
  dp.nchunks = (int)chunks.size();
  // shared memory
  {
    const int abytes = 3 * kRows * sp.KA * 2, bbytes = 3 * sp.NP * sp.KA * 2;
    // Y as float2 when, as double2, it would be the largest user of the area
    // (unpacked plans; the packed kernel keeps double2)
    const int ybytes_d = kRows * (hh | 1) * 16;
    sp.yfloat = hp.nd == 1 && ybytes_d > 2 * (abytes + bbytes);
    const int ybytes = sp.yfloat ? ybytes_d / 2 : ybytes_d;
    const int ubytes = ((std::max(2 * (abytes + bbytes), ybytes) + 127) / 128) * 128;
    sp.smem_form = 128 + ubytes + sizeof(double2) * (size_t)n * npw;
    // eval: operands, E, the chunk's phases and lslots densities' L.  Groups
    // of 8 steps, or of 4 if only that keeps two CTAs per SM with one L slot;
    // then as many L slots as keep two CTAs per SM (up to the densities a pass
    // can pack: cpc, and 3 nd for the gradient and Hessian views), at least one.
    const size_t lbytes = sizeof(double2) * (size_t)npw * hh;
    const int eab = 3 * kRows * sp.KE * 2;
    auto eval_base = [&](int eb) {
      const int ebb = 3 * (16 * eb) * sp.KE * 2;
      return 128 + ((eab + 127) / 128) * 128 + ((ebb + 127) / 128) * 128 +
             sizeof(double2) * ((size_t)npw * n + (size_t)sp.cpc * npw);
    };
    sp.ebatch = kEvalBatchMax;
    if (eval_base(kEvalBatchMax) + lbytes > (size_t)kEvalSmemTwoPerSm &&
        eval_base(kEvalBatchMax / 2) + lbytes <= (size_t)kEvalSmemTwoPerSm)
      sp.ebatch = kEvalBatchMax / 2;
    const size_t ebase = eval_base(sp.ebatch);
    const int lcap = std::min(sp.cpc, 3 * hp.nd);
    sp.lslots = 1;
    while (sp.lslots < lcap && ebase + (sp.lslots + 1) * lbytes <= (size_t)kEvalSmemTwoPerSm) sp.lslots++;
    sp.smem_eval = ebase + sp.lslots * lbytes;
  }
  // x-contraction tiles per form thread (npw <= 64: at most 256 tiles)
  sp.nt = ((((npw + 1) / 2) * ((hh + 3) / 4)) + kThreads - 1) / kThreads;
  if (sp.smem_form > (size_t)kMaxDynSmem || sp.smem_eval > (size_t)kMaxDynSmem) {
    msg = "split precision: shared memory need exceeds 227 KB";
    return BFGT_ERR_CAPACITY;
  }
  set_split_smem_attrs();
  sp.wait_iters = kWaitIters;
  // tensor-core FLOP issued per transform (every slice product counted)
  const double nsteps_total = (double)(steps.size() / (1 + sp.cpc));
  sp.tc_flops_form = nsteps_total * hp.nd * 6.0 * (sp.KA / 16) * 2.0 * kRows * sp.NP * 16;
  sp.tc_flops_eval = nsteps_total * hp.nd * 6.0 * (sp.KE / 16) * 2.0 * kRows * sp.NB * 16;
  return rc;
}

void split_plan_destroy(DevicePlan &dp) {
  SplitPlan &sp = dp.split;
  void *ptrs[] = {sp.chunks, sp.step_begin, sp.steps, sp.TyB, sp.EyB, sp.tyb_off, sp.eyb_off, sp.err, sp.items};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  sp = SplitPlan();
}

namespace {

// The plan's {chunk, pass} items if they were cut for its density count (a
// gradient or Hessian view of the eval stage has 2 nd or 3 nd densities and
// runs whole chunks), and the CTA count that goes with the choice.
const int2 *split_items(const DevicePlan &dp) {
  return dp.split.items && dp.nd == dp.split.items_nd ? dp.split.items : nullptr;
}
int split_ctas(const DevicePlan &dp) { return split_items(dp) ? dp.split.nitems : dp.split.nchunks; }

FormTcArgs form_args(const DevicePlan &dp, long long elem_off) {
  const SplitPlan &sp = dp.split;
  return FormTcArgs{sp.chunks, sp.step_begin, sp.steps, dp.columns, sp.TyB, sp.tyb_off, sp.tyb_tile, dp.T, dp.PH,
                    dp.ph_off, dp.Mpart, reduce_args(dp), sp.err, dp.nd, dp.n, dp.npw, dp.hh, dp.nexp, sp.cpc,
                    sp.NP, sp.KA, sp.wait_iters, elem_off, split_items(dp)};
}

EvalTcArgs eval_args(const DevicePlan &dp, long long elem_off) {
  const SplitPlan &sp = dp.split;
  return EvalTcArgs{sp.chunks, sp.step_begin, sp.steps, dp.columns, sp.EyB, sp.eyb_off, sp.eyb_tile, dp.E, dp.PH,
                    dp.ph_off, dp.L, sp.err, dp.nd, dp.n, dp.npw, dp.hh, dp.nexp, sp.cpc, sp.NB, sp.KE, sp.KH,
                    sp.lslots, sp.ebatch, sp.wait_iters, elem_off, split_items(dp)};
}

// variant: 0, 1 = unpacked with 1, 2 x-contraction tiles per thread (+2 with
// Y as float2); 4 = packed; +5 for n = 16
int form_variant(const DevicePlan &dp) {
  return (dp.nd > 1 ? 4 : dp.split.nt - 1 + (dp.split.yfloat ? 2 : 0)) + (dp.n == 16 ? 5 : 0);
}

void launch_form(int variant, int grid, size_t smem, cudaStream_t s, const FormTcLaunch &lp) {
  if (grid <= 0) return;
  const bool b = lp.descs != nullptr;
#define FORM_V(V, P, NT, YF, N)                                                 \
  case V:                                                                       \
    if (b) k_form_tc<true, P, NT, YF, N><<<grid, kThreads, smem, s>>>(lp);     \
    else k_form_tc<false, P, NT, YF, N><<<grid, kThreads, smem, s>>>(lp);      \
    break;
  switch (variant) {
    FORM_V(0, false, 1, false, 8) FORM_V(1, false, 2, false, 8) FORM_V(2, false, 1, true, 8)
    FORM_V(3, false, 2, true, 8) FORM_V(4, true, 1, false, 8)
    FORM_V(5, false, 1, false, 16) FORM_V(6, false, 2, false, 16) FORM_V(7, false, 1, true, 16)
    FORM_V(8, false, 2, true, 16) FORM_V(9, true, 1, false, 16)
  }
#undef FORM_V
}

void launch_eval(int nnt, bool pack, bool n16, int grid, size_t smem, cudaStream_t s, const EvalTcLaunch &lp) {
  if (grid <= 0) return;
  const bool b = lp.descs != nullptr;
  switch (nnt) {
#define EVAL_NNT(X)                                                         \
  case X:                                                                   \
    if (n16) {                                                               \
      if (pack) {                                                            \
        if (b) k_eval_tc<X, true, true, 16><<<grid, kEvalThreads, smem, s>>>(lp);  \
        else k_eval_tc<X, false, true, 16><<<grid, kEvalThreads, smem, s>>>(lp);  \
      } else {                                                               \
        if (b) k_eval_tc<X, true, false, 16><<<grid, kEvalThreads, smem, s>>>(lp); \
        else k_eval_tc<X, false, false, 16><<<grid, kEvalThreads, smem, s>>>(lp); \
      }                                                                      \
    } else {                                                                 \
      if (pack) {                                                            \
        if (b) k_eval_tc<X, true, true, 8><<<grid, kEvalThreads, smem, s>>>(lp);   \
        else k_eval_tc<X, false, true, 8><<<grid, kEvalThreads, smem, s>>>(lp);   \
      } else {                                                               \
        if (b) k_eval_tc<X, true, false, 8><<<grid, kEvalThreads, smem, s>>>(lp);  \
        else k_eval_tc<X, false, false, 8><<<grid, kEvalThreads, smem, s>>>(lp);  \
      }                                                                      \
    }                                                                        \
    break;
    EVAL_NNT(1) EVAL_NNT(2) EVAL_NNT(3) EVAL_NNT(4) EVAL_NNT(5) EVAL_NNT(6) EVAL_NNT(7) EVAL_NNT(8)
#undef EVAL_NNT
  }
}

}  // namespace

void split_form(DevicePlan &dp, const double *d_fvals, cudaStream_t s) {
  FormTcLaunch lp{form_args(dp, 0), nullptr, nullptr, d_fvals};
  launch_form(form_variant(dp), split_ctas(dp), dp.split.smem_form, s, lp);
}

void split_eval(DevicePlan &dp, double *d_pot, cudaStream_t s) {
  EvalTcLaunch lp{eval_args(dp, 0), nullptr, nullptr, d_pot};
  launch_eval((dp.hh + 3) / 4, dp.nd > 1, dp.n == 16, split_ctas(dp), dp.split.smem_eval, s, lp);
}

int split_batch_create(SplitBatch &b, const std::vector<DevicePlan *> &plans, const std::vector<long long> &offs,
                       std::string &msg) {
  split_batch_destroy(b);
  std::vector<FormTcArgs> fd;
  std::vector<EvalTcArgs> ed;
  // the plans' work items (chunks, or chunk passes), grouped by kernel variant: form_variant for
  // form; density packing (nd > 1), the column-tile count of H and the leaf
  // order for eval (variant = nnt + 16 pack + 32 (n = 16)); within a group the
  // plans keep their order
  std::vector<std::vector<int2>> fw(10), ew(64);
  std::vector<size_t> fsm(10, 0), esm(64, 0);
  for (size_t i = 0; i < plans.size(); i++) {
    DevicePlan &dp = *plans[i];
    fd.push_back(form_args(dp, offs[i]));
    ed.push_back(eval_args(dp, offs[i]));
    if (dp.precision != BFGT_PREC_SPLIT || dp.direct_only) continue;
    const int fv = form_variant(dp), ev = (dp.hh + 3) / 4 + 16 * (dp.nd > 1 ? 1 : 0) + 32 * (dp.n == 16 ? 1 : 0);
    for (int c = 0; c < split_ctas(dp); c++) {
      fw[fv].push_back(make_int2((int)i, c));
      ew[ev].push_back(make_int2((int)i, c));
    }
    fsm[fv] = std::max(fsm[fv], dp.split.smem_form);
    esm[ev] = std::max(esm[ev], dp.split.smem_eval);
  }
  std::vector<int2> fall, eall;
  for (int v = 0; v < 10; v++)
    if (!fw[v].empty()) {
      b.form_groups.push_back(SplitBatch::Group{v, (int)fall.size(), (int)fw[v].size(), fsm[v]});
      fall.insert(fall.end(), fw[v].begin(), fw[v].end());
    }
  for (int v = 0; v < 64; v++)
    if (!ew[v].empty()) {
      b.eval_groups.push_back(SplitBatch::Group{v, (int)eall.size(), (int)ew[v].size(), esm[v]});
      eall.insert(eall.end(), ew[v].begin(), ew[v].end());
    }
  int rc = BFGT_OK;
  auto chk = [&](int x) {
    if (rc == BFGT_OK && x != BFGT_OK) rc = x;
  };
  FormTcArgs *dfd = nullptr;
  EvalTcArgs *ded = nullptr;
  chk(upload_vec(dfd, fd, msg));
  chk(upload_vec(ded, ed, msg));
  chk(upload_vec(b.form_work, fall, msg));
  chk(upload_vec(b.eval_work, eall, msg));
  b.form_descs = dfd;
  b.eval_descs = ded;
  return rc;
}

void split_batch_form(const SplitBatch &b, const double *fbase, cudaStream_t s) {
  for (const SplitBatch::Group &g : b.form_groups) {
    FormTcLaunch lp{};
    lp.descs = static_cast<const FormTcArgs *>(b.form_descs);
    lp.work = b.form_work + g.begin;
    lp.fbase = fbase;
    launch_form(g.variant, g.count, g.smem, s, lp);
  }
}

void split_batch_eval(const SplitBatch &b, double *pbase, cudaStream_t s) {
  for (const SplitBatch::Group &g : b.eval_groups) {
    EvalTcLaunch lp{};
    lp.descs = static_cast<const EvalTcArgs *>(b.eval_descs);
    lp.work = b.eval_work + g.begin;
    lp.pbase = pbase;
    launch_eval(g.variant & 15, (g.variant & 16) != 0, g.variant >= 32, g.count, g.smem, s, lp);
  }
}

int split_batch_launches(const SplitBatch &b) { return (int)(b.form_groups.size() + b.eval_groups.size()); }

void split_batch_destroy(SplitBatch &b) {
  void *ptrs[] = {b.form_descs, b.eval_descs, b.form_work, b.eval_work};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  b = SplitBatch();
}

unsigned int split_default_wait_iters() { return kWaitIters; }

int split_check(DevicePlan &dp) {
  if (!dp.split.err) return BFGT_OK;
  int h[4] = {0, 0, 0, 0};
  if (cudaMemcpy(h, dp.split.err, sizeof(int) * 4, cudaMemcpyDeviceToHost) != cudaSuccess) return BFGT_ERR_CUDA;
  if (h[0]) {
    cudaMemset(dp.split.err, 0, sizeof(int) * 4);
    return BFGT_ERR_TIMEOUT;
  }
  return BFGT_OK;
}

}  // namespace bfgt
