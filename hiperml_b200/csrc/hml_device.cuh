// hml_device.cuh -- sm_100a device helpers shared by the kernels: mbarriers
// with bounded waits, TMA tile loads, thread-block-cluster barriers and
// distributed-shared-memory loads, and the device error word.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace hml {

// Error codes written to the device error word by a bounded wait that ran
// out.  The host reads and clears it with hml_device_error().
enum : int {
  kDevErrNone = 0,
  kDevErrFullBarrier = 1,   // a consumer waited too long for a TMA tile
  kDevErrEmptyBarrier = 2,  // the producer waited too long for a free stage
  kDevErrMmaBarrier = 3,    // the epilogue waited too long for tcgen05.commit
  kDevErrQueue = 4,         // a batched work-queue wait expired
};

// A bounded wait gives up after this many nanoseconds of %globaltimer.
constexpr uint64_t kWaitLimitNs = 2000000000ull;  // 2 s

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// `p` advanced to the next multiple of `align` (a power of two) bytes in the
// shared window.  Pointer arithmetic on a shared pointer, not a round trip
// through an integer, so that the compiler keeps the shared state space for
// everything derived from it (32-bit addresses and shared loads instead of
// generic 64-bit ones).
template <typename T>
__device__ __forceinline__ T *align_shared(T *p, uint32_t align) {
  const uint32_t pad = (align - (smem_u32(p) & (align - 1))) & (align - 1);
  return reinterpret_cast<T *>(reinterpret_cast<uint8_t *>(p) + pad);
}

__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void set_device_error(int *err, int code) {
  if (err) atomicCAS(err, 0, code);
}

// ------------------------------------------------------------- mbarrier
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// One try_wait with a suspend-time hint: the thread is parked until the
// phase completes or about `kSuspendNs` pass, instead of returning at once
// and re-polling (a polling warp takes issue slots from the warps doing the
// work).
constexpr uint32_t kSuspendNs = 1000000u;  // 1 ms

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity), "r"(kSuspendNs)
      : "memory");
  return ok != 0;
}

// Waits for the phase with the given parity to complete, for at most
// kWaitLimitNs (plus one suspend slice).  Returns false (and records `code`)
// when the limit expires.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, int *err, int code) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = globaltimer_ns();
  for (;;) {
    if (mbar_try_wait(bar, parity)) return true;
    if (globaltimer_ns() - t0 > kWaitLimitNs) {
      set_device_error(err, code);
      return false;
    }
  }
}

// ------------------------------------------------- dependent launches
// Lets the next kernel on the stream (launched as a programmatic dependent)
// begin as soon as every CTA of this grid has executed this.
__device__ __forceinline__ void allow_dependent_launch() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Waits until the grid this one was launched after has completed and its
// memory writes are visible (returns at once for a normal launch).
__device__ __forceinline__ void wait_prior_grid() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
}

// ------------------------------------------------------------------ TMA
// 2-D tiled bulk tensor load, global -> this CTA's own shared memory only,
// completing on `bar` with the tile's byte count.
__device__ __forceinline__ void tma_load_2d(void *smem_dst, const void *tmap, uint64_t *bar,
                                            int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4}], [%2];" ::"r"(smem_u32(smem_dst)),
      "l"(reinterpret_cast<uint64_t>(tmap)), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}

__device__ __forceinline__ void prefetch_tmap(const void *tmap) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(tmap)) : "memory");
}

// -------------------------------------------------------------- cluster
__device__ __forceinline__ uint32_t cluster_ctarank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}

__device__ __forceinline__ void cluster_sync() {
  asm volatile(
      "barrier.cluster.arrive.release.aligned;\n\t"
      "barrier.cluster.wait.acquire.aligned;" ::
          : "memory");
}

__device__ __forceinline__ uint32_t mapa_shared(uint32_t addr, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(addr), "r"(rank));
  return r;
}

__device__ __forceinline__ float ld_dsmem(uint32_t addr) {
  float v;
  asm volatile("ld.shared::cluster.f32 %0, [%1];" : "=f"(v) : "r"(addr) : "memory");
  return v;
}

__device__ __forceinline__ float4 ld_dsmem4(uint32_t addr) {
  float4 v;
  asm volatile("ld.shared::cluster.v4.f32 {%0, %1, %2, %3}, [%4];"
               : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
               : "r"(addr)
               : "memory");
  return v;
}

// ------------------------------------------------------------ streaming
// 16-byte global load that bypasses L1 allocation (A is read exactly once).
__device__ __forceinline__ float4 ldg_stream4(const float *p) {
  float4 v;
  asm volatile("ld.global.nc.L1::no_allocate.v4.f32 {%0, %1, %2, %3}, [%4];"
               : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
               : "l"(p));
  return v;
}

__device__ __forceinline__ float ldg_stream(const float *p) {
  float v;
  asm volatile("ld.global.nc.L1::no_allocate.f32 %0, [%1];" : "=f"(v) : "l"(p));
  return v;
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// BLAS epilogue: beta == 0 never reads the old value.
// alpha * acc + beta * c with one fixed rounding sequence, so that every
// kernel that finishes a C element the same way gives the same bits.
__device__ __forceinline__ float axpby(float alpha, float acc, float beta, const float *c) {
  return beta == 0.0f ? __fmul_rn(alpha, acc) : __fmaf_rn(alpha, acc, __fmul_rn(beta, *c));
}

}  // namespace hml
