// Near field on block work lists: on the tensor cores for split plans with
// floating slices (k_near_tc), in FP64 for the others (k_near_f64); see
// near_tc.cuh.
#include "near_tc.cuh"

#include <algorithm>
#include <cstring>
#include <vector>

#include "../../include/bfgt.h"
#include "tc_sm100.cuh"

namespace bfgt {

namespace {

constexpr int kNtThreads = 128;                       // one thread per MMA row
constexpr int kNtA = 128 * 16 * 2;                    // one BF16 slice of a 128 x 16 A operand
constexpr int kNtB = 16 * 16 * 2;                     // one slice of a 16 x 16 B operand
constexpr int kNtTab = 3 * kNtB / 2;                  // uint16 per table slot (3 slices)
constexpr int kTG = 1;                                // tiles (slots) per MMA round
constexpr size_t kNtFixed = kTG * 3 * (kNtA + kNtB);  // operand buffers
constexpr int kColB = 32 * kTG;                       // TMEM column of stage B's accumulators
constexpr int kTmemCols = kTG == 1 ? 64 : 128;        // 32 columns per stage-A tile of a round and stage B
constexpr size_t kNtMinSmem = kTG == 1 ? 29 * 1024 : 46 * 1024;  // CTAs per SM x kTmemCols <= 512
constexpr uint32_t kNtWaitIters = 1u << 26;

// host copy of tc::kmajor_off
inline uint32_t kmajor_off_host(int r, int k, int R) {
  return (uint32_t)((((k >> 3) * (R >> 3) + (r >> 3)) << 7) + ((r & 7) << 4) + ((k & 7) << 1));
}

// FP64 -> FP32 -> three BF16 slices by truncation (as tc::split3_bf16x1)
inline void split3_host(double v, uint16_t &s0, uint16_t &s1, uint16_t &s2) {
  auto hi = [](float x) {
    uint32_t u;
    std::memcpy(&u, &x, 4);
    u &= 0xFFFF0000u;
    float y;
    std::memcpy(&y, &u, 4);
    return y;
  };
  auto top = [](float x) {
    uint32_t u;
    std::memcpy(&u, &x, 4);
    return (uint16_t)(u >> 16);
  };
  const float a = (float)v;
  const float h = hi(a), r = a - h;
  const float m = hi(r), l = r - m;
  s0 = top(h);
  s1 = top(m);
  s2 = top(l);
}

template <typename T>
int upload_nt(T *&d, const std::vector<T> &v, std::string &msg) {
  d = nullptr;
  if (v.empty()) return BFGT_OK;
  if (cudaMalloc(&d, sizeof(T) * v.size()) != cudaSuccess) {
    cudaGetLastError();
    msg = "cudaMalloc failed (tensor-core near field)";
    return BFGT_ERR_OOM;
  }
  if (cudaMemcpy(d, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
    msg = "cudaMemcpy failed (tensor-core near field)";
    return BFGT_ERR_CUDA;
  }
  return BFGT_OK;
}

// Stores the 16 K values v[0..15] of MMA row r as three BF16 slices (K-major
// core layout, R = 128 rows).
__device__ __forceinline__ void store_row16(unsigned char *sA, int r, const float (&v)[16]) {
#pragma unroll
  for (int k0 = 0; k0 < 16; k0 += 8) {
    uint32_t p[3][4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const float a0 = v[k0 + 2 * q], a1 = v[k0 + 2 * q + 1];
      const float h0 = tc::bf16_hi(a0), h1 = tc::bf16_hi(a1);
      const float r0 = a0 - h0, r1 = a1 - h1;
      const float m0 = tc::bf16_hi(r0), m1 = tc::bf16_hi(r1);
      const float l0 = r0 - m0, l1 = r1 - m1;
      p[0][q] = __byte_perm(__float_as_uint(h0), __float_as_uint(h1), 0x7632);
      p[1][q] = __byte_perm(__float_as_uint(m0), __float_as_uint(m1), 0x7632);
      p[2][q] = __byte_perm(__float_as_uint(l0), __float_as_uint(l1), 0x7632);
    }
    const uint32_t o = tc::kmajor_off(r, k0, 128);
#pragma unroll
    for (int c = 0; c < 3; c++)
      *reinterpret_cast<uint4 *>(sA + c * kNtA + o) = make_uint4(p[c][0], p[c][1], p[c][2], p[c][3]);
  }
}

// The six slice products i + j <= 2 of one 128 x 16 x 16 MMA step: s0 s0 into
// D0, the corrections into D1.
__device__ __forceinline__ void near_mmas(uint32_t d0, uint32_t d1, uint32_t aA, uint32_t aB, uint32_t acc) {
  constexpr uint32_t idesc = tc::idesc_bf16_f32(128, 16);
  uint64_t ad[3], bd[3];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    ad[c] = tc::smem_desc(aA + c * kNtA, (128 / 8) * 128, 128);
    bd[c] = tc::smem_desc(aB + c * kNtB, (16 / 8) * 128, 128);
  }
  tc::mma_bf16(d0, ad[0], bd[0], idesc, acc);
  tc::mma_bf16(d1, ad[0], bd[1], idesc, acc);
  tc::mma_bf16(d1, ad[1], bd[0], idesc, 1u);
  tc::mma_bf16(d1, ad[0], bd[2], idesc, 1u);
  tc::mma_bf16(d1, ad[1], bd[1], idesc, 1u);
  tc::mma_bf16(d1, ad[2], bd[0], idesc, 1u);
}

// One CTA: up to 128/kN targets; per density, stage A over the CTA's block
// tiles into Q (shared memory), then stage B over the slots into pot.  Both
// stages take kTG tiles (slots) per round: their operands side by side in
// shared memory, their MMAs issued together under one commit, so that a
// round's loads are all in flight at once and the round trip (barrier, MMA,
// wait) is paid once per kTG tiles.  TMEM: tile g of a stage-A round in
// columns 32 g .. 32 g + 31 (D0, D1), stage B in the 32 after them.  One
// tile per round measured fastest on the regime-C benchmark tree (0.48 ms):
// rounds of 3 tiles cut the CTAs per SM from 5 to 3 (0.52 ms), and so did a
// cp.async staging of the next tile's rows during the MMAs (17 KB of shared
// memory more: 0.52 ms).  The kernel is bound by the latency of its rounds,
// and resident CTAs hide it best.  Q is
// [target][slot][k2][j1], rows of kN + 1 floats: the stage-A adds (fixed k2,
// consecutive j1 across threads) and the stage-B reads (fixed j1, consecutive
// k2) are both free of bank conflicts.
// (at least 5 CTAs per SM: without the hint ptxas settles at 64 registers
// with spills, 17% slower on the regime-C benchmark tree)
template <int kN>
__global__ void __launch_bounds__(kNtThreads, 5) k_near_tc(const __grid_constant__ NearTcLaunch lp) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t mbar[2];  // MMA rounds; the final drain
  __shared__ uint32_t tmem_slot;
  constexpr int kG = 128 / kN;  // blocks per stage-A tile, targets per CTA
  constexpr int kQr = kN + 1;   // Q row stride
  const NearTcArgs &a = lp.descs ? lp.descs[lp.work[blockIdx.x].x] : lp.one;
  const int cta = lp.descs ? lp.work[blockIdx.x].y : (int)blockIdx.x;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int4 c = a.ctas[cta];
  const int ntarget = c.w & 0xFF, nslot = c.w >> 8;
  const int nd = a.nd, npb = kN * kN;
  const double *fv = lp.fbase + a.elem_off;
  double *pot = lp.pbase + a.elem_off;
  unsigned char *sA = smem;                                // kTG x 3 slices
  unsigned char *sB = smem + kTG * 3 * kNtA;               // kTG x 3 slices
  float *sQ = reinterpret_cast<float *>(smem + kNtFixed);  // [tl][slot][k2][j1]
  const int qsz = kG * nslot * kN * kQr;

  if (warp == 0) tc::tmem_alloc(&tmem_slot, kTmemCols);
  if (tid == 0) {
    tc::mbar_init(&mbar[0], 1);
    tc::mbar_init(&mbar[1], 1);
    tc::fence_mbar_init();
  }
  // kN = 8: the K columns 8-15 of every A buffer are zero for the whole kernel
  if (kN == 8) {
    const float z[16] = {};
    for (int g = 0; g < kTG; g++) store_row16(sA + g * 3 * kNtA, tid, z);
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = tmem_slot;
  const uint32_t lane_base = (uint32_t)(32 * warp) << 16;
  const uint32_t aA = tc::smem_u32(sA), aB = tc::smem_u32(sB);
  bool ok = true;
  uint32_t phase = 0;
  // stage-A row: block i of a tile, grid index j1; stage-B row: target tl, k2
  const int ri = tid / kN, rj = tid % kN;
  const int *slot_q = a.slot_q + (size_t)cta * kNearTcSlots;
  auto round_trip = [&](int nmma_groups, auto &&issue) {
    tc::cp_async_wait_all();
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (tid == 0 && ok) {
      for (int g = 0; g < nmma_groups; g++) issue(g);
      tc::commit(&mbar[0]);
    }
    if (ok && !tc::mbar_wait(&mbar[0], phase & 1, a.wait_iters)) {
      ok = false;
      atomicExch(a.err, 1);
    }
    phase++;
    tc::fence_after_sync();
  };

  for (int ind = 0; ind < nd; ind++) {
    for (int e = tid; e < qsz; e += kNtThreads) sQ[e] = 0.0f;
    __syncthreads();
    for (int t0 = c.x; t0 < c.y; t0 += kTG) {
      const int ng = min(kTG, c.y - t0);
      int4 bk[kTG];
#pragma unroll
      for (int g = 0; g < kTG; g++) {
        bk[g] = make_int4(-1, 0, 0, 0);
        if (g < ng) {
          const int4 T = a.tiles[t0 + g];
          const uint16_t *tb = a.tabB + (size_t)(T.x + a.yoff) * kNtTab;
          for (int u = tid; u < 3 * kNtB / 16; u += kNtThreads) tc::cp_async16(sB + g * 3 * kNtB + 16 * u, tb + 8 * u);
          if (ri < T.z) bk[g] = a.blocks[T.y + ri];
        }
      }
      tc::cp_async_commit();
      // F(j1 = rj, j2) of each tile's block, all loads issued before any use
      float v[kTG][16];
#pragma unroll
      for (int g = 0; g < kTG; g++) {
        const double *src = fv + (size_t)(bk[g].x >= 0 ? bk[g].x : 0) * nd * npb + ind + (size_t)nd * rj;
#pragma unroll
        for (int j2 = 0; j2 < 16; j2++)
          v[g][j2] = (bk[g].x >= 0 && j2 < kN) ? __double2float_rn(src[(size_t)nd * kN * j2]) : 0.0f;
      }
#pragma unroll
      for (int g = 0; g < kTG; g++) {
        if (bk[g].x < 0) continue;
        if (kN == 16) {
          store_row16(sA + g * 3 * kNtA, tid, v[g]);
        } else {
          // only the first 8 K columns of the row (the rest stay zero)
          uint32_t p[3][4];
#pragma unroll
          for (int q = 0; q < 4; q++) {
            const float a0 = v[g][2 * q], a1 = v[g][2 * q + 1];
            const float h0 = tc::bf16_hi(a0), h1 = tc::bf16_hi(a1);
            const float r0 = a0 - h0, r1 = a1 - h1;
            const float m0 = tc::bf16_hi(r0), m1 = tc::bf16_hi(r1);
            const float l0 = r0 - m0, l1 = r1 - m1;
            p[0][q] = __byte_perm(__float_as_uint(h0), __float_as_uint(h1), 0x7632);
            p[1][q] = __byte_perm(__float_as_uint(m0), __float_as_uint(m1), 0x7632);
            p[2][q] = __byte_perm(__float_as_uint(l0), __float_as_uint(l1), 0x7632);
          }
          const uint32_t o = tc::kmajor_off(tid, 0, 128);
#pragma unroll
          for (int cc = 0; cc < 3; cc++)
            *reinterpret_cast<uint4 *>(sA + g * 3 * kNtA + cc * kNtA + o) = make_uint4(p[cc][0], p[cc][1], p[cc][2], p[cc][3]);
        }
      }
      round_trip(ng, [&](int g) {
        near_mmas(tmem + 32 * g, tmem + 32 * g + 16, aA + g * 3 * kNtA, aB + g * 3 * kNtB, 0u);
      });
      // G rows (block, j1 = rj) -> Q(t, slot, k2, j1) of each pair they serve,
      // tile after tile (two tiles of a round may serve the same Q rows), 8
      // columns at a time
      for (int g = 0; g < ng; g++) {
        if (g > 0) __syncthreads();
#pragma unroll
        for (int h = 0; h < kN; h += 8) {
          float d0[8], d1[8];
          tc::tmem_ld8(tmem + lane_base + 32 * g + h, d0);
          tc::tmem_ld8(tmem + lane_base + 32 * g + 16 + h, d1);
          tc::tmem_ld_wait();
          if (bk[g].x >= 0 && ok) {
#pragma unroll
            for (int k2 = 0; k2 < 8; k2++) d0[k2] += d1[k2];
            for (int u = 0; u < bk[g].w; u++) {
              const int cs = ((u < 2 ? bk[g].y : bk[g].z) >> (16 * (u & 1))) & 0xFFFF;
              const int tl = cs & 0xFF, slot = cs >> 8;
              float *q = sQ + (size_t)(tl * nslot + slot) * kN * kQr + rj;
#pragma unroll
              for (int k2 = 0; k2 < 8; k2++) q[(size_t)(h + k2) * kQr] += d0[k2];
            }
          }
        }
      }
      tc::fence_before_sync();
      __syncthreads();
    }
    // stage B: one K block per slot, kTG slots per round, accumulated in
    // TMEM columns kColB ..
    for (int s0 = 0; s0 < nslot; s0 += kTG) {
      const int ns = min(kTG, nslot - s0);
      for (int g = 0; g < ns; g++) {
        const uint16_t *tb = a.tabB + (size_t)(slot_q[s0 + g] + a.xoff) * kNtTab;
        for (int u = tid; u < 3 * kNtB / 16; u += kNtThreads) tc::cp_async16(sB + g * 3 * kNtB + 16 * u, tb + 8 * u);
      }
      tc::cp_async_commit();
      for (int g = 0; g < ns; g++) {
        // A row (tl = ri, k2 = rj): Q(tl, slot, k2, j1) over j1
        const float *q = sQ + ((size_t)(ri * nslot + s0 + g) * kN + rj) * kQr;
        float v[16];
#pragma unroll
        for (int j1 = 0; j1 < 16; j1++) v[j1] = j1 < kN ? q[j1] : 0.0f;
        store_row16(sA + g * 3 * kNtA, tid, v);
      }
      round_trip(ns, [&](int g) {
        near_mmas(tmem + kColB, tmem + kColB + 16, aA + g * 3 * kNtA, aB + g * 3 * kNtB, s0 + g > 0 ? 1u : 0u);
      });
      __syncthreads();  // every thread has read its Q rows and the MMAs are done: the buffers are free
    }
    if (nslot > 0) {
      // pot(k1, k2 = rj) of target ri, k1 = 0..kN-1, 8 at a time
      double *pb = ri < ntarget ? pot + (size_t)a.targets[c.z + ri] * a.out_nd * npb + a.out_off + ind +
                                      (size_t)a.out_nd * kN * rj
                                : nullptr;
#pragma unroll
      for (int h = 0; h < kN; h += 8) {
        float d0[8], d1[8];
        tc::tmem_ld8(tmem + lane_base + kColB + h, d0);
        tc::tmem_ld8(tmem + lane_base + kColB + 16 + h, d1);
        tc::tmem_ld_wait();
        if (ok && pb) {
#pragma unroll
          for (int k1 = 0; k1 < 8; k1++) pb[(size_t)a.out_nd * (h + k1)] += (double)d0[k1] + (double)d1[k1];
        }
      }
      tc::fence_before_sync();
      __syncthreads();
    }
  }
  // drain: no tensor-core operation of this CTA may be in flight when TMEM is freed
  if (tid == 0) tc::commit(&mbar[1]);
  if (!tc::mbar_wait(&mbar[1], 0, kNtWaitIters)) atomicExch(a.err, 2);
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, kTmemCols);
}

// The same CTA, tile and block lists on the FP64 pipes (FP64 plans and
// fixed-point split plans).  Stage A: G_b = F_b ty for the tile's blocks
// (shared memory, 4 x kN/4 output tiles per thread); stage B: each thread
// adds tx_slot^T G_b for the pairs of its own target into a 4 x kN/4 tile of
// that target's pot held in registers, so no Q is needed; pot is updated
// once per density at the end.  Rows of kN + 1 doubles in shared memory.
template <int kN>
__global__ void __launch_bounds__(kNtThreads) k_near_f64(const __grid_constant__ NearTcLaunch lp) {
  extern __shared__ __align__(16) double dsm[];
  __shared__ int4 s_blk[128 / kN];
  constexpr int kG = 128 / kN, kS = kN + 1, kTN = kN / 4;
  const NearTcArgs &a = lp.descs ? lp.descs[lp.work[blockIdx.x].x] : lp.one;
  const int cta = lp.descs ? lp.work[blockIdx.x].y : (int)blockIdx.x;
  const int tid = threadIdx.x;
  const int4 c = a.ctas[cta];
  const int ntarget = c.w & 0xFF, nslot = c.w >> 8;
  const int nd = a.nd, npb = kN * kN;
  const double *fv = lp.fbase + a.elem_off;
  double *pot = lp.pbase + a.elem_off;
  double *sF = dsm;                    // [block][j1][j2]
  double *sG = sF + kG * kN * kS;      // [block][j1][k2]
  double *sTY = sG + kG * kN * kS;     // [j2][k2]
  double *sTX = sTY + kN * kS;         // [slot][j1][k1]
  const int grp = tid / kN, sub = tid % kN;
  const int ra = (sub / 4) * 4, ca = (sub % 4) * kTN;  // rows ra..ra+3, columns ca..ca+kTN-1
  const int *slot_q = a.slot_q + (size_t)cta * kNearTcSlots;
  for (int e = tid; e < nslot * npb; e += kNtThreads) {
    const int sl = e / npb, r = e - sl * npb, j = r % kN, k = r / kN;
    sTX[((size_t)sl * kN + j) * kS + k] = a.tabD[(size_t)(slot_q[sl] + a.xoff) * npb + r];
  }
  for (int ind = 0; ind < nd; ind++) {
    double acc[4][kTN];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
      for (int u = 0; u < kTN; u++) acc[i][u] = 0.0;
    for (int t = c.x; t < c.y; t++) {
      const int4 T = a.tiles[t];
      __syncthreads();  // the previous tile's shared data has been read
      if (tid < T.z) s_blk[tid] = a.blocks[T.y + tid];
      for (int e = tid; e < npb; e += kNtThreads) {
        const int j = e % kN, k = e / kN;
        sTY[j * kS + k] = a.tabD[(size_t)(T.x + a.yoff) * npb + e];
      }
      __syncthreads();
      for (int e = tid; e < T.z * npb; e += kNtThreads) {
        const int b = e / npb, r = e - b * npb, j1 = r % kN, j2 = r / kN;
        sF[((size_t)b * kN + j1) * kS + j2] = fv[(size_t)s_blk[b].x * nd * npb + ind + (size_t)nd * r];
      }
      __syncthreads();
      if (grp < T.z) {
        double g[4][kTN];
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
          for (int u = 0; u < kTN; u++) g[i][u] = 0.0;
        const double *fr = sF + ((size_t)grp * kN + ra) * kS;
#pragma unroll 4
        for (int j2 = 0; j2 < kN; j2++) {
          double f[4], y[kTN];
#pragma unroll
          for (int i = 0; i < 4; i++) f[i] = fr[i * kS + j2];
#pragma unroll
          for (int u = 0; u < kTN; u++) y[u] = sTY[j2 * kS + ca + u];
#pragma unroll
          for (int i = 0; i < 4; i++)
#pragma unroll
            for (int u = 0; u < kTN; u++) g[i][u] = fma(f[i], y[u], g[i][u]);
        }
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
          for (int u = 0; u < kTN; u++) sG[((size_t)grp * kN + ra + i) * kS + ca + u] = g[i][u];
      }
      __syncthreads();
      // pairs of this thread's target: (block b, x slot) with target grp
      if (grp < ntarget) {
        for (int b = 0; b < T.z; b++) {
          const int4 bk = s_blk[b];
          for (int u = 0; u < bk.w; u++) {
            const int cs = ((u < 2 ? bk.y : bk.z) >> (16 * (u & 1))) & 0xFFFF;
            if ((cs & 0xFF) != grp) continue;
            const double *xr = sTX + (size_t)(cs >> 8) * kN * kS;
            const double *gr = sG + (size_t)b * kN * kS;
#pragma unroll 4
            for (int j1 = 0; j1 < kN; j1++) {
              double x[4], gv[kTN];
#pragma unroll
              for (int i = 0; i < 4; i++) x[i] = xr[j1 * kS + ra + i];
#pragma unroll
              for (int v = 0; v < kTN; v++) gv[v] = gr[j1 * kS + ca + v];
#pragma unroll
              for (int i = 0; i < 4; i++)
#pragma unroll
                for (int v = 0; v < kTN; v++) acc[i][v] = fma(x[i], gv[v], acc[i][v]);
            }
          }
        }
      }
    }
    if (grp < ntarget) {
      // pot(k1 = ra + i, k2 = ca + v) of target grp
      double *pb = pot + (size_t)a.targets[c.z + grp] * a.out_nd * npb + a.out_off + ind;
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int v = 0; v < kTN; v++) pb[(size_t)a.out_nd * ((ra + i) + kN * (ca + v))] += acc[i][v];
    }
  }
}

}  // namespace

int near_tc_create(DevicePlan &dp, const HostPlan &hp, std::string &msg, bool fp64) {
  near_tc_destroy(dp);
  const int n = hp.norder;
  if (hp.nf_target.empty() || (n != 8 && n != 16)) return BFGT_OK;
  const int nslots_tab = 13 * (hp.nlevels + 1);
  if ((int)hp.tab_loc.size() < n * n * nslots_tab || (int)hp.ind_loc.size() < 2 * (n + 1) * nslots_tab) return BFGT_OK;
  // the table operands: B(out k, in j) = tab_loc(j, k, slot) inside the band
  // pattern, 0 outside; slots whose band is empty are marked unused
  // three sets: values, and the first and second derivatives in the target
  // coordinate (tabx_loc, tabxx_loc) for the gradient and Hessian outputs,
  // all on the values' band pattern
  const bool derivs = hp.tabx_loc.size() >= (size_t)n * n * nslots_tab && hp.tabxx_loc.size() >= (size_t)n * n * nslots_tab;
  const std::vector<double> *sets[3] = {&hp.tab_loc, &hp.tabx_loc, &hp.tabxx_loc};
  std::vector<uint16_t> tab(fp64 ? 0 : (size_t)3 * nslots_tab * kNtTab, 0);
  std::vector<double> tabd(fp64 ? (size_t)3 * nslots_tab * n * n : 0, 0.0);
  std::vector<char> used(nslots_tab, 0);
  for (int q = 0; q < nslots_tab; q++) {
    const int *il = &hp.ind_loc[(size_t)2 * (n + 1) * q];
    const int k0 = il[2 * n], k1 = il[2 * n + 1];
    if (k1 - k0 + 1 <= 0) continue;
    used[q] = 1;
    for (int set = 0; set < (derivs ? 3 : 1); set++) {
      const double *t = &(*sets[set])[(size_t)n * n * q];
      for (int k = k0 - 1; k < k1; k++) {
        const int lo = il[2 * k], hi = il[2 * k + 1];
        for (int j = lo - 1; j < hi; j++) {
          if (fp64) {
            tabd[((size_t)set * nslots_tab + q) * n * n + j + (size_t)n * k] = t[j + (size_t)n * k];
            continue;
          }
          uint16_t s[3];
          split3_host(t[j + (size_t)n * k], s[0], s[1], s[2]);
          const uint32_t o = kmajor_off_host(k, j, 16) / 2;
          uint16_t *dst = &tab[((size_t)set * nslots_tab + q) * kNtTab];
          for (int cc = 0; cc < 3; cc++) dst[cc * (kNtB / 2) + o] = s[cc];
        }
      }
    }
  }
  // CTAs of up to kG targets whose entries use at most kNearTcSlots distinct
  // x tables; entries with an empty table contribute nothing and are dropped.
  // Within a CTA the pairs that share (source, y table) share one stage-A
  // block (up to 4 pairs each); blocks are cut into tiles of kG that share the
  // y table, and a block whose pairs meet one already in the tile (the same
  // target and x slot) starts a new tile, so that no two rows of a tile add
  // into the same Q rows.
  const int kG = 128 / n;
  struct Pair {
    int src, tl, slot, qy;
  };
  std::vector<int4> ctas, tiles, blocks;
  std::vector<int> targets, slot_q;
  std::vector<Pair> cur;
  std::vector<int> cur_q, cur_t;
  int maxslot = 0;
  auto close_cta = [&]() {
    if (cur_t.empty()) return;
    std::stable_sort(cur.begin(), cur.end(), [](const Pair &x, const Pair &y) {
      if (x.qy != y.qy) return x.qy < y.qy;
      if (x.src != y.src) return x.src < y.src;
      if (x.tl != y.tl) return x.tl < y.tl;
      return x.slot < y.slot;
    });
    // blocks: runs of equal (qy, src), at most 4 consumers each
    struct Blk {
      int qy, src, ncons, cons[4];
    };
    std::vector<Blk> bl;
    for (size_t i = 0; i < cur.size(); i++) {
      const int cs = cur[i].tl | (cur[i].slot << 8);
      if (!bl.empty() && bl.back().qy == cur[i].qy && bl.back().src == cur[i].src && bl.back().ncons < 4) {
        bl.back().cons[bl.back().ncons++] = cs;
      } else {
        bl.push_back(Blk{cur[i].qy, cur[i].src, 1, {cs, 0, 0, 0}});
      }
    }
    int4 c;
    c.x = (int)tiles.size();
    size_t i = 0;
    while (i < bl.size()) {
      const int begin = (int)blocks.size();
      std::vector<int> seen;
      size_t j = i;
      for (; j < bl.size() && bl[j].qy == bl[i].qy && (int)(j - i) < kG; j++) {
        bool clash = false;
        for (int u = 0; u < bl[j].ncons; u++) clash = clash || std::find(seen.begin(), seen.end(), bl[j].cons[u]) != seen.end();
        if (clash) break;
        for (int u = 0; u < bl[j].ncons; u++) seen.push_back(bl[j].cons[u]);
        const Blk &b = bl[j];
        blocks.push_back(make_int4(b.src, b.cons[0] | (b.cons[1] << 16), b.cons[2] | (b.cons[3] << 16), b.ncons));
      }
      tiles.push_back(make_int4(bl[i].qy, begin, (int)(j - i), 0));
      i = j;
    }
    c.y = (int)tiles.size();
    c.z = (int)targets.size();
    c.w = (int)cur_t.size() | ((int)cur_q.size() << 8);
    targets.insert(targets.end(), cur_t.begin(), cur_t.end());
    for (int q = 0; q < kNearTcSlots; q++) slot_q.push_back(q < (int)cur_q.size() ? cur_q[q] : 0);
    maxslot = std::max(maxslot, (int)cur_q.size());
    ctas.push_back(c);
    cur.clear();
    cur_q.clear();
    cur_t.clear();
  };
  for (size_t t = 0; t < hp.nf_target.size(); t++) {
    std::vector<int> ents, qxs;
    for (int e = hp.nf_begin[t]; e < hp.nf_begin[t + 1]; e++) {
      const int qx = hp.nf_elev[e] * 13 + hp.nf_ix[e] + 6, qy = hp.nf_elev[e] * 13 + hp.nf_iy[e] + 6;
      if (qx < 0 || qy < 0 || qx >= nslots_tab || qy >= nslots_tab || !used[qx] || !used[qy]) continue;
      ents.push_back(e);
      if (std::find(qxs.begin(), qxs.end(), qx) == qxs.end()) qxs.push_back(qx);
    }
    if (ents.empty()) continue;
    if ((int)qxs.size() > kNearTcSlots) return BFGT_OK;  // the FP64 kernel serves this plan
    int add = 0;
    for (int q : qxs)
      if (std::find(cur_q.begin(), cur_q.end(), q) == cur_q.end()) add++;
    if ((int)cur_t.size() == kG || (int)cur_q.size() + add > kNearTcSlots) close_cta();
    const int tl = (int)cur_t.size();
    cur_t.push_back(hp.nf_target[t]);
    for (int e : ents) {
      const int qx = hp.nf_elev[e] * 13 + hp.nf_ix[e] + 6, qy = hp.nf_elev[e] * 13 + hp.nf_iy[e] + 6;
      auto it = std::find(cur_q.begin(), cur_q.end(), qx);
      int slot = (int)(it - cur_q.begin());
      if (it == cur_q.end()) cur_q.push_back(qx);
      cur.push_back(Pair{hp.nf_src[e], tl, slot, qy});
    }
  }
  close_cta();
  if (ctas.empty()) return BFGT_OK;
  NearTcPlan &p = dp.ntc;
  int rc = BFGT_OK;
  auto chk = [&](int x) {
    if (rc == BFGT_OK && x != BFGT_OK) rc = x;
  };
  chk(upload_nt(p.ctas, ctas, msg));
  chk(upload_nt(p.tiles, tiles, msg));
  chk(upload_nt(p.blocks, blocks, msg));
  chk(upload_nt(p.targets, targets, msg));
  chk(upload_nt(p.slot_q, slot_q, msg));
  chk(upload_nt(p.tabB, tab, msg));
  chk(upload_nt(p.tabD, tabd, msg));
  if (rc != BFGT_OK) {
    near_tc_destroy(dp);
    return rc;
  }
  p.nctas = (int)ctas.size();
  p.maxslot = maxslot;
  p.fp64 = fp64;
  p.smem = fp64 ? sizeof(double) * ((size_t)2 * kG * n * (n + 1) + (size_t)n * (n + 1) + (size_t)maxslot * n * (n + 1))
                : std::max(kNtFixed + sizeof(float) * (size_t)kG * maxslot * n * (n + 1), kNtMinSmem);
  const int smax = 227 * 1024 - 1024;
  if (p.smem > (size_t)smax) {
    near_tc_destroy(dp);
    return BFGT_OK;
  }
  cudaFuncSetAttribute(k_near_tc<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax);
  cudaFuncSetAttribute(k_near_tc<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax);
  // all of the unified L1 as shared memory: as many CTAs per SM as their
  // shared memory allows
  cudaFuncSetAttribute(k_near_tc<8>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  cudaFuncSetAttribute(k_near_tc<16>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  cudaFuncSetAttribute(k_near_f64<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax);
  cudaFuncSetAttribute(k_near_f64<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax);
  cudaFuncSetAttribute(k_near_f64<8>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  cudaFuncSetAttribute(k_near_f64<16>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  if (cudaGetLastError() != cudaSuccess) {
    msg = "CUDA error while preparing the tensor-core near field";
    near_tc_destroy(dp);
    return BFGT_ERR_CUDA;
  }
  return BFGT_OK;
}

void near_tc_destroy(DevicePlan &dp) {
  NearTcPlan &p = dp.ntc;
  void *ptrs[] = {p.ctas, p.tiles, p.blocks, p.targets, p.slot_q, p.tabB, p.tabD};
  for (void *x : ptrs)
    if (x) cudaFree(x);
  p = NearTcPlan();
}

NearTcArgs near_tc_args(const DevicePlan &dp, long long elem_off) {
  const NearTcPlan &p = dp.ntc;
  return NearTcArgs{p.ctas, p.targets, p.tiles, p.blocks, p.slot_q, p.tabB, p.tabD, dp.split.err, dp.nd, dp.n, p.nctas,
                    dp.split.wait_iters ? dp.split.wait_iters : kNtWaitIters, elem_off, dp.nd, 0, 0, 0};
}

void near_f64_launch(int n, int grid, size_t smem, cudaStream_t s, const NearTcLaunch &lp) {
  if (grid <= 0) return;
  if (n == 16)
    k_near_f64<16><<<grid, kNtThreads, smem, s>>>(lp);
  else
    k_near_f64<8><<<grid, kNtThreads, smem, s>>>(lp);
}

void near_tc_launch(int n, int grid, size_t smem, cudaStream_t s, const NearTcLaunch &lp) {
  if (grid <= 0) return;
  if (n == 16)
    k_near_tc<16><<<grid, kNtThreads, smem, s>>>(lp);
  else
    k_near_tc<8><<<grid, kNtThreads, smem, s>>>(lp);
}

}  // namespace bfgt
