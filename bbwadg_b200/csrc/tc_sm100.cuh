// Minimal sm_100a tensor-core (tcgen05 / UMMA) primitives as inline PTX.
//
// Shared-memory operands use the canonical K-major layout without swizzle:
// 8-row x 16-byte "core matrices" (8 x 8 FP16), the two 16-byte K chunks of
// one MMA K step LBO bytes apart and consecutive 8-row groups SBO bytes
// apart.  The descriptor bit fields follow the PTX ISA matrix-descriptor
// format for tcgen05 (version 1); the instruction descriptor is the
// kind::f16 one (dense, FP32 accumulator).
//
// Accumulators live in tensor memory (TMEM): address = lane << 16 | column.
// For M = 128 row i of D is lane i; for M = 64 row m is lane
// (m % 16) + 32 (m / 16).  A warp reads only its 32-lane sub-partition
// (warp % 4).
#pragma once
#include <cstdint>

namespace bbw {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// canonical K-major, no swizzle: offset of element (row r, k) of an FP16
// operand whose K extent (padded) is kp
__host__ __device__ __forceinline__ int kmajor_offset_f16(int r, int k, int kp) {
  return ((r >> 3) * (kp >> 3) + (k >> 3)) * 64 + (r & 7) * 8 + (k & 7);
}

// shared-memory matrix descriptor (SWIZZLE_NONE)
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo_bytes,
                                              uint32_t sbo_bytes) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version (sm_100)
  return d;                // base offset 0, LBO mode 0, layout SWIZZLE_NONE
}

// instruction descriptor, kind::f16, FP32 accumulate, both operands K-major
// fmt: 0 = F16, 1 = BF16
__host__ __device__ constexpr uint32_t idesc_f16(int M, int N, int fmt) {
  return (1u << 4) | ((uint32_t)fmt << 7) | ((uint32_t)fmt << 10) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

// D (TMEM) (+)= A (smem) * B (smem)^T; issued by one thread
__device__ __forceinline__ void mma_f16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                        uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(
          tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

// arrive on mbar once all previously issued MMAs of this thread complete
__device__ __forceinline__ void mma_commit(void *mbar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
          smem_u32(mbar))
      : "memory");
}

__device__ __forceinline__ void mbar_init(void *mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(mbar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

// bounded wait for phase `parity` of mbar; false when the bound is hit
__device__ __forceinline__ bool mbar_wait(void *mbar, uint32_t parity, uint32_t max_iter) {
  const uint32_t a = smem_u32(mbar);
  for (uint32_t it = 0; it < max_iter; ++it) {
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

__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
}
// generic-proxy shared-memory writes -> visible to the tensor core (async proxy)
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}

// TMEM allocation: warp-collective; writes the base address to *slot
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                   smem_u32(slot)),
               "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(ncols)
               : "memory");
}

// 32 lanes x 32 bits, 16 consecutive columns -> 16 registers per thread;
// the wait is part of the same statement so the outputs are valid after it
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n\t"
      "tcgen05.wait::ld.sync.aligned;\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// 32 lanes x 32 bits, 8 consecutive columns -> 8 registers per thread
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8]) {
  uint32_t r[8];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n\t"
      "tcgen05.wait::ld.sync.aligned;\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

// four 32x32b.x8 loads at column offsets a0..a3 (8 columns each), then one
// wait: 32 registers valid after the statement
__device__ __forceinline__ void tmem_ld8x4(uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                           float (&v0)[8], float (&v1)[8], float (&v2)[8],
                                           float (&v3)[8]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%32];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%8,%9,%10,%11,%12,%13,%14,%15}, [%33];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%16,%17,%18,%19,%20,%21,%22,%23}, [%34];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%24,%25,%26,%27,%28,%29,%30,%31}, [%35];\n\t"
      "tcgen05.wait::ld.sync.aligned;\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
        "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3));
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    v0[i] = __uint_as_float(r[i]);
    v1[i] = __uint_as_float(r[8 + i]);
    v2[i] = __uint_as_float(r[16 + i]);
    v3[i] = __uint_as_float(r[24 + i]);
  }
}

// 16 lanes x 64 bits, 4 repetitions along the columns (8 consecutive
// columns): the warp's 16 TMEM lanes spread over all 32 threads, 4 registers
// per thread (the lane / column of each register: ep_row / ep_elem in
// kernels_tc.cu); the wait is part of the statement
__device__ __forceinline__ void tmem_ld16x64b_x4(uint32_t taddr, float (&v)[4]) {
  uint32_t r[4];
  asm volatile(
      "tcgen05.ld.sync.aligned.16x64b.x4.b32 {%0,%1,%2,%3}, [%4];\n\t"
      "tcgen05.wait::ld.sync.aligned;\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 4; ++i) v[i] = __uint_as_float(r[i]);
}

// four such loads at column addresses a0..a3, then one wait
__device__ __forceinline__ void tmem_ld16x64b_x4x4(uint32_t a0, uint32_t a1, uint32_t a2,
                                                   uint32_t a3, float (&v0)[4], float (&v1)[4],
                                                   float (&v2)[4], float (&v3)[4]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.16x64b.x4.b32 {%0,%1,%2,%3}, [%16];\n\t"
      "tcgen05.ld.sync.aligned.16x64b.x4.b32 {%4,%5,%6,%7}, [%17];\n\t"
      "tcgen05.ld.sync.aligned.16x64b.x4.b32 {%8,%9,%10,%11}, [%18];\n\t"
      "tcgen05.ld.sync.aligned.16x64b.x4.b32 {%12,%13,%14,%15}, [%19];\n\t"
      "tcgen05.wait::ld.sync.aligned;\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3));
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    v0[i] = __uint_as_float(r[i]);
    v1[i] = __uint_as_float(r[4 + i]);
    v2[i] = __uint_as_float(r[8 + i]);
    v3[i] = __uint_as_float(r[12 + i]);
  }
}

// ---- bulk (TMA, 1-D) copies global -> shared, completion on an mbarrier
__device__ __forceinline__ void mbar_expect_tx(void *mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(mbar)),
               "r"(bytes)
               : "memory");
}
// L2 prefetch of a global range (hint, no completion); src 16-byte aligned,
// bytes a multiple of 16
__device__ __forceinline__ void prefetch_l2(const void *src, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(src), "r"(bytes) : "memory");
}
// dst, src 16-byte aligned, bytes a multiple of 16
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, void *mbar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(mbar))
      : "memory");
}

}  // namespace tc
}  // namespace bbw
