// hml_tcgen05.cuh -- the tcgen05 (fifth-generation tensor core) and TMEM
// primitives shared by the split-BF16 SGEMM (sgemm_tc.cu) and the
// tensor-core k-means assignment (kmeans.cu): TMEM allocation, loads and
// stores, tcgen05.mma with A in TMEM, commits to mbarriers, and the shared-
// memory and instruction descriptors of the operand layouts they use.
#pragma once

#include <cstdint>

#include "hml_device.cuh"

namespace hml {

__device__ __forceinline__ void tmem_alloc(uint32_t *dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_u32(dst_smem)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// D (TMEM) (+)= A (TMEM, 128 lanes x 16 BF16 in 8 columns) * B (shared
// memory descriptor), kind::f16 with BF16 inputs and an FP32 accumulator.
__device__ __forceinline__ void mma_bf16_ts(uint32_t dtmem, uint32_t atmem, uint64_t bdesc,
                                            uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}" ::"r"(dtmem),
      "r"(atmem), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t *bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(bar))
      : "memory");
}

// 32 lanes x 8 / 16 consecutive 32-bit columns of TMEM into registers (the
// caller issues tmem_wait_ld before using them).
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&r)[8]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7])
      : "r"(taddr));
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}

__device__ __forceinline__ void tmem_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// 32 lanes x 16 consecutive 32-bit columns from registers into TMEM.
__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, "
      "%10, %11, %12, %13, %14, %15, %16};" ::"r"(taddr),
      "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]),
      "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]),
      "r"(r[15])
      : "memory");
}

__device__ __forceinline__ void tmem_wait_st() {
  asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

// Shared-memory matrix descriptor: K-major, 64-byte swizzle (rows of 64 B),
// 8-row atoms 512 B apart (stride byte offset), descriptor version 1.
__device__ __forceinline__ uint64_t sw64_desc(uint32_t saddr) {
  return static_cast<uint64_t>((saddr >> 4) & 0x3FFFu) | (static_cast<uint64_t>(1) << 16) |
         (static_cast<uint64_t>(512 >> 4) << 32) | (static_cast<uint64_t>(1) << 46) |
         (static_cast<uint64_t>(4) << 61);
}

// Instruction descriptor: BF16 x BF16 -> F32, both K-major, M = bm, N = bn.
__host__ __device__ constexpr uint32_t idesc_bf16(int bn, int bm = 128) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(bn >> 3) << 17) |
         (static_cast<uint32_t>(bm >> 4) << 24);
}

// The same for FP16 x FP16 -> F32 (kind::f16; A and B format code 0).
__host__ __device__ constexpr uint32_t idesc_f16(int bn, int bm = 128) {
  return (1u << 4) | (static_cast<uint32_t>(bn >> 3) << 17) |
         (static_cast<uint32_t>(bm >> 4) << 24);
}

// The same for TF32 x TF32 -> F32 (kind::tf32; A and B format code 2).
__host__ __device__ constexpr uint32_t idesc_tf32(int bn, int bm = 128) {
  return (1u << 4) | (2u << 7) | (2u << 10) | (static_cast<uint32_t>(bn >> 3) << 17) |
         (static_cast<uint32_t>(bm >> 4) << 24);
}

// Shared-memory matrix descriptor: K-major, 128-byte swizzle (rows of 128 B =
// 32 TF32), 8-row atoms 1024 B apart (stride byte offset), version 1.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  return static_cast<uint64_t>((saddr >> 4) & 0x3FFFu) | (static_cast<uint64_t>(1) << 16) |
         (static_cast<uint64_t>(1024 >> 4) << 32) | (static_cast<uint64_t>(1) << 46) |
         (static_cast<uint64_t>(2) << 61);
}

// D (TMEM) (+)= A (TMEM, 128 lanes x 8 TF32 in 8 columns) * B (shared
// memory descriptor, 8 TF32 deep), kind::tf32 with an FP32 accumulator.
__device__ __forceinline__ void mma_tf32_ts(uint32_t dtmem, uint32_t atmem, uint64_t bdesc,
                                            uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n\t}" ::"r"(dtmem),
      "r"(atmem), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// x rounded to TF32 (11 significant bits, nearest, ties away), in a 32-bit
// container whose low 13 bits are zero.
__device__ __forceinline__ uint32_t tf32_rna(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

// D (TMEM) (+)= A (shared memory descriptor, 128 rows x 8 TF32) * B (shared
// memory descriptor, 8 TF32 deep), kind::tf32 with an FP32 accumulator.
__device__ __forceinline__ void mma_tf32_ss(uint32_t dtmem, uint64_t adesc, uint64_t bdesc,
                                            uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(dtmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

}  // namespace hml
