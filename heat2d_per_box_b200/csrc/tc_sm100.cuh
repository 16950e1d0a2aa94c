// Minimal sm_100a tensor-core (tcgen05) and mbarrier helpers, written as
// inline PTX.  Operands live in shared memory in the no-swizzle K-major
// "core matrix" layout: 8 rows x 16 bytes per core matrix, row groups 128 B
// apart (SBO), the two 8-element K halves of one MMA (K = 16 for 16-bit
// types) LBO bytes apart.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace bfgt {
namespace tc {

// byte offset of element (r, k) of a K-major operand with R rows (R % 8 == 0)
__device__ __forceinline__ uint32_t kmajor_off(int r, int k, int R) {
  return (uint32_t)((((k >> 3) * (R >> 3) + (r >> 3)) << 7) + ((r & 7) << 4) + ((k & 7) << 1));
}

// shared-memory matrix descriptor (sm_100 layout: version 1, no swizzle)
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for sm_100
  return d;                // base offset 0, layout type 0 (no swizzle)
}

// instruction descriptor: kind::f16 with BF16 A/B, FP32 accumulator, both K-major
__host__ __device__ constexpr uint32_t idesc_bf16_f32(int M, int N) {
  return (1u << 4)                       // D format F32
         | (1u << 7)                     // A format BF16
         | (1u << 10)                    // B format BF16
         | ((uint32_t)(N >> 3) << 17)    // N / 8
         | ((uint32_t)(M >> 4) << 24);   // M / 16
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void commit(uint64_t *mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
               : "memory");
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// warp-wide: allocate ncols TMEM columns, write the base address to *dst
__device__ __forceinline__ void tmem_alloc(uint32_t *dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 32 lanes x 16 consecutive 32-bit columns; thread t of the warp gets lane (base lane + t)
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}
// 32 lanes x 8 consecutive 32-bit columns
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float *v) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 8; i++) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t *mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// Bounded wait for the completion of the given phase parity.  Returns false
// (and leaves the barrier untouched) when the iteration limit is reached.
__device__ __forceinline__ bool mbar_wait(uint64_t *mbar, uint32_t parity, uint32_t max_iter) {
  const uint32_t a = smem_u32(mbar);
  for (uint32_t it = 0; it < max_iter; it++) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// FP64 tensor-core MMA, D(8x8) += A(8x4) B(4x8): lane (g = lane/4, t = lane%4)
// holds A[g][t], B[t][g] and D[g][2t], D[g][2t+1]
__device__ __forceinline__ void dmma_8x8x4(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

// FP32 -> its leading BF16 part by truncation: the top 16 bits of the FP32
// encoding (sign, exponent, 7 mantissa bits) are a BF16 number, and
// x - hi(x) is exact in FP32.  Integer operations only (no conversion
// instructions).
__device__ __forceinline__ float bf16_hi(float x) { return __uint_as_float(__float_as_uint(x) & 0xFFFF0000u); }

// FP64 value -> three BF16 slices through FP32 (see split3_bf16x2)
__device__ __forceinline__ void split3_bf16x1(double v, uint16_t &s0, uint16_t &s1, uint16_t &s2) {
  const float a = __double2float_rn(v);
  const float h = bf16_hi(a), r = a - h;
  const float m = bf16_hi(r), l = r - m;
  s0 = (uint16_t)(__float_as_uint(h) >> 16);
  s1 = (uint16_t)(__float_as_uint(m) >> 16);
  s2 = (uint16_t)(__float_as_uint(l) >> 16);
}

// 16-byte global -> shared copy that bypasses registers (completion: cp_async_wait_all)
__device__ __forceinline__ void cp_async16(void *smem_dst, const void *gsrc) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(smem_dst)), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

__device__ __forceinline__ uint32_t bf162_bits(__nv_bfloat162 h) { return *reinterpret_cast<uint32_t *>(&h); }

// Two FP64 values -> three packed BF16x2 slices.  The values are rounded to
// FP32 first (relative error 2^-24); the FP32 value is then cut exactly by
// truncation: s0 = the top 8 significant bits, the remainder (exact in FP32)
// has at most 16, s1 = its top 8, and what is left (exact) has at most 8
// significant bits, so it is a BF16 number s2 and s0 + s1 + s2 reproduces the
// FP32 value (FP32 values below the normal range aside, which lose their low
// bits: an absolute error below 2^-133).  One conversion per value; the cuts
// and the packing are integer operations.  Element v0 goes to the low half
// (the lower address of a packed pair).
__device__ __forceinline__ void split3_bf16x2(double v0, double v1, uint32_t &p0, uint32_t &p1, uint32_t &p2) {
  const float a0 = __double2float_rn(v0), a1 = __double2float_rn(v1);
  const float h0 = bf16_hi(a0), h1 = bf16_hi(a1);
  const float r0 = a0 - h0, r1 = a1 - h1;
  const float m0 = bf16_hi(r0), m1 = bf16_hi(r1);
  const float l0 = r0 - m0, l1 = r1 - m1;
  // bytes 2, 3 of the first word, then bytes 2, 3 (6, 7) of the second
  p0 = __byte_perm(__float_as_uint(h0), __float_as_uint(h1), 0x7632);
  p1 = __byte_perm(__float_as_uint(m0), __float_as_uint(m1), 0x7632);
  p2 = __byte_perm(__float_as_uint(l0), __float_as_uint(l1), 0x7632);
}

}  // namespace tc
}  // namespace bfgt
