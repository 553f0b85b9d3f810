// tcgen05 (5th-generation tensor core) helpers for sm_100a: TMEM allocation,
// shared-memory operand descriptors in the K-major no-swizzle canonical
// layout, single-thread MMA issue with commit to an mbarrier, bounded waits
// and TMEM -> register loads.
//
// Canonical K-major layout (SWIZZLE_NONE): the operand is tiled into "core
// matrices" of 8 rows x 16 bytes, each stored as 128 contiguous bytes (row r of
// the core matrix at +16 r).  We place core matrix (row group g, 16-byte K
// chunk c) at byte (g * KC + c) * 128, KC = K bytes / 16, so the descriptor's
// leading-dimension byte offset (between the two K chunks one MMA reads) is
// 128 and its stride-dimension byte offset (between row groups) is KC * 128.
#pragma once
#include "oqmc_common.cuh"

#define OQ_TC_SPIN_LIMIT (1u << 26)

__device__ __forceinline__ uint32_t oq_smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// 64-bit shared-memory matrix descriptor (sm_100): start, LBO, SBO in 16-byte
// units, version 1 at bits [46,48), swizzle mode 0 (none) at bits [61,64).
__device__ __forceinline__ uint64_t oq_desc_kmajor(uint32_t saddr, uint32_t lbo_bytes,
                                                   uint32_t sbo_bytes) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// Instruction descriptor, kind::tf32 (A, B TF32; D FP32), both K-major.
__host__ __device__ constexpr uint32_t oq_idesc_tf32(int M, int N) {
  return (1u << 4)                      // D format F32
         | (2u << 7) | (2u << 10)       // A, B format TF32
         | ((uint32_t)(N >> 3) << 17)   // N / 8
         | ((uint32_t)(M >> 4) << 24);  // M / 16
}

// Instruction descriptor, kind::f16 with BF16 A and B, FP32 D, both K-major.
__host__ __device__ constexpr uint32_t oq_idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

// One warp allocates ncols TMEM columns; the base address lands in *slot.
__device__ __forceinline__ void oq_tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
               ::"r"(oq_smem_addr(slot)), "r"(ncols));
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}

__device__ __forceinline__ void oq_tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}

__device__ __forceinline__ void oq_mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(oq_smem_addr(bar)), "r"(count));
  asm volatile("fence.mbarrier_init.release.cluster;");
}

// Bounded wait on an mbarrier phase; returns false on timeout.
__device__ __forceinline__ bool oq_mbar_wait(uint64_t* bar, uint32_t phase) {
  const uint32_t a = oq_smem_addr(bar);
  for (uint32_t it = 0; it < OQ_TC_SPIN_LIMIT; ++it) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(a), "r"(phase));
    if (done) return true;
  }
  return false;
}

// Generic-proxy shared-memory writes become visible to the tensor core.
__device__ __forceinline__ void oq_fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void oq_tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void oq_tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

// D[tmem] (+)= A[smem] * B[smem]^T, issued by one thread.
__device__ __forceinline__ void oq_mma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                            uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void oq_mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                            uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

// Arrive on *bar when every MMA this thread issued so far has completed.
__device__ __forceinline__ void oq_mma_commit(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          oq_smem_addr(bar)));
}

// 16 consecutive FP32 columns of this thread's TMEM lane (32x32b shape).
__device__ __forceinline__ void oq_tmem_ld16(uint32_t taddr, float v[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
      "%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Same load without the wait: several may be in flight before one
// oq_tmem_wait_ld(); the registers are valid only after the wait.
__device__ __forceinline__ void oq_tmem_ld16_nw(uint32_t taddr, uint32_t r[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
      "%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
__device__ __forceinline__ void oq_tmem_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Store 16 consecutive 32-bit columns of this thread's TMEM lane (32x32b
// shape); the data reach tensor memory only after oq_tmem_wait_st().
__device__ __forceinline__ void oq_tmem_st16(uint32_t taddr, const uint32_t r[16]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,"
      "%13,%14,%15,%16};" ::"r"(taddr),
      "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]),
      "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]),
      "r"(r[15])
      : "memory");
}
__device__ __forceinline__ void oq_tmem_wait_st() {
  asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

// D[tmem] (+)= A[tmem] * B[smem]^T (kind::f16, BF16): A as 128 lanes (rows)
// of K/2 32-bit columns, two consecutive K elements per column (the lower
// 16 bits hold the even element), issued by one thread.
__device__ __forceinline__ void oq_mma_bf16_ta(uint32_t tmem_d, uint32_t tmem_a, uint64_t bdesc,
                                               uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n}" ::"r"(tmem_d),
      "r"(tmem_a), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

// Round an FP32 value to TF32 (round to nearest, ties away) and return the
// rounded value; v - oq_tf32(v) is the low part of a 2-term split.
__device__ __forceinline__ float oq_tf32(float v) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(v));
  return __uint_as_float(r);
}

// Byte offset of element (row, k) of a 4-byte K-major canonical operand with
// KC 16-byte chunks per row.
__device__ __forceinline__ uint32_t oq_kmajor_off4(int row, int k, int KC) {
  return ((uint32_t)((row >> 3) * KC + (k >> 2)) << 7) + ((row & 7) << 4) + ((k & 3) << 2);
}
// Same for 2-byte elements (BF16): 8 elements per 16-byte chunk.
__device__ __forceinline__ uint32_t oq_kmajor_off2(int row, int k, int KC) {
  return ((uint32_t)((row >> 3) * KC + (k >> 3)) << 7) + ((row & 7) << 4) + ((k & 7) << 1);
}
