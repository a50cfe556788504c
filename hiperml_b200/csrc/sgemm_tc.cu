// sgemm_tc.cu -- split-BF16 SGEMM on the B200 tensor cores (tcgen05 + TMEM).
//
// FP32 operands are split into BF16 terms, a = a0 + a1 (+ a2), each term the
// BF16 rounding of what the previous terms left (every residual is exact in
// FP32), and the products that carry FP32-level information are accumulated
// in FP32:
//   BF16X3: a0*b0 + a0*b1 + a1*b0                          (2 planes, 3 MMAs)
//   BF16X6: a0*b0 + a0*b1 + a1*b0 + a0*b2 + a1*b1 + a2*b0  (3 planes, 6 MMAs)
// The result is C = alpha * A * B + beta * C in FP32, the reference's
// hmlSgemm contract (src/hml_sgemm.cu:120-211) on a different machine.
//
// Data flow of one CTA (a 128-row tile of C, BN columns, a K range):
//   * B is small (K x N): a pre-pass splits it once into BF16 planes stored
//     K-contiguous in a workspace ([plane][N_pad][K_pad]); the kernel loads
//     plane tiles with TMA straight into the UMMA canonical K-major layout
//     (64-byte swizzle, 32 BF16 per row).
//   * A streams from HBM exactly once: a TMA thread loads 128 x 32 FP32 tiles
//     into a ring of `stages` slots, each released as soon as the converter
//     warps have read it (B tiles live in a separate ring released by the
//     MMAs, so HBM latency is hidden by the A ring alone).
//   * sixteen converter warps split each FP32 tile into BF16 planes written in
//     the same canonical layout (a transpose when A is M-contiguous) into one
//     of two converted buffers, then signal the MMA warp.
//   * one thread of the MMA warp issues tcgen05.mma (M=128, N=BN, K=16, both
//     operands from shared memory, FP32 accumulator in TMEM) and releases
//     ring slots and buffers with tcgen05.commit.
//   * the tensor core's FP32 accumulation truncates, so a long accumulation
//     chain in TMEM loses accuracy as K grows.  Each 64-deep chunk of K is
//     accumulated into one of two TMEM accumulators; the converter warps then
//     read it (tcgen05.ld) and add it into FP32 running sums held in
//     registers (round to nearest) while the tensor core fills the other.
//   * the converter warps apply alpha/beta from the running sums; with
//     split_k > 1 the CTAs of one thread-block cluster sum their tiles in
//     rank order through distributed shared memory.
// Every wait is bounded (2 s of %globaltimer); on expiry the device error
// word is set, the CTA skips ahead, frees its TMEM and returns.
#include <cuda_bf16.h>

#include <algorithm>
#include <cstring>
#include <mutex>

#include "hml_device.cuh"
#include "hml_internal.h"

namespace hml {
namespace {

constexpr int kBM = 128;        // rows of C per CTA = UMMA M
constexpr int kBK = 32;         // K per ring stage (one 64-byte BF16 swizzle row)
constexpr int kConvWarps = 16;  // converters + accumulator drain + epilogue
constexpr int kLoadAWarp = kConvWarps, kLoadBWarp = kConvWarps + 1, kMmaWarp = kConvWarps + 2;
constexpr int kThreads = (kConvWarps + 3) * 32;
constexpr int kChunkK = 64;     // K accumulated in TMEM before an FP32 drain

struct TcShape {
  int bn;
};
constexpr TcShape kTcShapes[] = {{16}, {32}, {64}, {128}};
constexpr int kNumTcShapes = sizeof(kTcShapes) / sizeof(kTcShapes[0]);

// ------------------------------------------------------------ tcgen05
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

__device__ __forceinline__ void mma_bf16(uint32_t dtmem, uint64_t adesc, uint64_t bdesc,
                                         uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(dtmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t *bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(bar))
      : "memory");
}

// 32 lanes x 4 / 8 / 16 consecutive 32-bit columns of TMEM into registers.
__device__ __forceinline__ void tmem_ld4(uint32_t taddr, float *v) {
  uint32_t r[4];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 4; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float *v) {
  uint32_t r[8];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Shared-memory matrix descriptor: K-major, 64-byte swizzle (rows of 64 B),
// 8-row atoms 512 B apart (stride byte offset), descriptor version 1.
__device__ __forceinline__ uint64_t sw64_desc(uint32_t saddr) {
  return static_cast<uint64_t>((saddr >> 4) & 0x3FFFu) | (static_cast<uint64_t>(1) << 16) |
         (static_cast<uint64_t>(512 >> 4) << 32) | (static_cast<uint64_t>(1) << 46) |
         (static_cast<uint64_t>(4) << 61);
}

// Byte offset of the 16-byte chunk `c` (0..3) of row `r` in a 64-byte-row
// tile with the 64-byte swizzle (chunk bits 4-5 XOR address bits 7-8).
__device__ __forceinline__ uint32_t sw64_off(int r, int c) {
  return static_cast<uint32_t>(r * 64 + ((c ^ ((r >> 1) & 3)) << 4));
}

// Instruction descriptor: BF16 x BF16 -> F32, both K-major, M = 128, N = bn.
__host__ __device__ constexpr uint32_t idesc_bf16(int bn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(bn >> 3) << 17) |
         (static_cast<uint32_t>(kBM >> 4) << 24);
}

// Split eight floats into NS BF16 planes, t0 = bf16(x), t1 = bf16(x - t0),
// ... (each residual is exact in FP32), packed two per 32-bit word with
// cvt.rn.bf16x2.f32.
__device__ __forceinline__ uint32_t bf16x2_rn(float lo, float hi) {
  uint32_t r;
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
  return r;
}

template <int NS>
__device__ __forceinline__ void pack8(const float (&x)[8], uint4 (&out)[NS]) {
  uint32_t w[NS][4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    float a = x[2 * j], b = x[2 * j + 1];
#pragma unroll
    for (int i = 0; i < NS; ++i) {
      const uint32_t t = bf16x2_rn(a, b);
      w[i][j] = t;
      if (i + 1 < NS) {
        a -= __uint_as_float(t << 16);
        b -= __uint_as_float(t & 0xFFFF0000u);
      }
    }
  }
#pragma unroll
  for (int i = 0; i < NS; ++i) out[i] = make_uint4(w[i][0], w[i][1], w[i][2], w[i][3]);
}

struct TcArgs {
  GemmProblem p;
  int split;       // CTAs per cluster along K
  int kc;          // K extent per split (multiple of kChunkK)
  int sa, so;      // A ring and operand ring depths
  int n_pad;       // rows of one B plane in the workspace
  int *err;
};

// ------------------------------------------------------------ B planes
// planes[p][n][k] (k contiguous, zero padded to n_pad x k_pad).
template <int NS>
__global__ void split_b_kernel(const float *B, int64_t sbk, int64_t sbn, int K, int N,
                               __nv_bfloat16 *planes, int k_pad, int n_pad) {
  const int64_t chunks = static_cast<int64_t>(n_pad) * (k_pad / 8);
  for (int64_t c = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; c < chunks;
       c += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int n = static_cast<int>(c / (k_pad / 8));
    const int k0 = static_cast<int>(c % (k_pad / 8)) * 8;
    float x[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int k = k0 + j;
      x[j] = (n < N && k < K)
                 ? B[static_cast<int64_t>(k) * sbk + static_cast<int64_t>(n) * sbn]
                 : 0.0f;
    }
    uint4 v[NS];
    pack8<NS>(x, v);
#pragma unroll
    for (int i = 0; i < NS; ++i)
      *reinterpret_cast<uint4 *>(planes + (static_cast<int64_t>(i) * n_pad + n) * k_pad + k0) =
          v[i];
  }
}

// ------------------------------------------------------------- kernel
// Shared-memory plan of one CTA (all tiles 1024-byte aligned):
//   A ring        sa slots of the FP32 A tile (16 KB), filled by TMA and
//                 released by the converter warps as soon as they have read
//                 it, so HBM latency is covered by this ring alone;
//   operand ring  so slots, each holding the NS B-plane tiles of one K block
//                 (filled by TMA) and the NS converted A planes of the same
//                 block (written by the converter warps).  One tcgen05.commit
//                 releases a whole slot: the MMA thread's issue rate (about
//                 30 ns a tcgen05.mma, 70 ns a tcgen05.commit) bounds the
//                 kernel for skinny N, so commits are kept to one per block.
struct TcPlan {
  int sa, so;
};

__host__ __device__ constexpr size_t tc_a_bytes() { return static_cast<size_t>(kBM) * kBK * 4; }
__host__ __device__ constexpr size_t tc_op_bytes(int bn, int ns) {
  return static_cast<size_t>(ns) * bn * kBK * 2 + static_cast<size_t>(ns) * kBM * kBK * 2;
}
size_t tc_plan_bytes(int bn, int ns, const TcPlan &pl) {
  return 1024 + pl.sa * tc_a_bytes() + pl.so * tc_op_bytes(bn, ns) + 8 * (2 * pl.sa + 2 * pl.so + 4) +
         16;
}

// The deepest operand ring (2..6 slots) that fits next to sa A slots.
bool tc_plan(int bn, int ns, int sa, TcPlan *out) {
  for (int so = 6; so >= 2; --so) {
    const TcPlan pl = {sa, so};
    if (tc_plan_bytes(bn, ns, pl) <= 227 * 1024) {
      *out = pl;
      return true;
    }
  }
  return false;
}

// Warps 0-15: convert A, drain the accumulator, epilogue.  Warp 16 loads A,
// warp 17 loads B (separate warps, so a load waiting on the MMA pipeline
// never holds back the HBM stream), warp 18 allocates TMEM and issues MMAs.
template <int BN, int NS, bool AK>
__global__ void __launch_bounds__(kThreads, 1)
    tc_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
              TcArgs args) {
  constexpr int A32_BYTES = static_cast<int>(tc_a_bytes());  // FP32 A slot (16 KB)
  constexpr int BPL_BYTES = BN * kBK * 2;                    // one B plane tile
  constexpr int APL_BYTES = kBM * kBK * 2;                   // one converted A plane (8 KB)
  constexpr int OP_BYTES = NS * (BPL_BYTES + APL_BYTES);     // one operand slot
  constexpr int QTR = BN / 4;                                // columns drained per thread
  constexpr uint32_t TMEM_COLS = 2 * BN < 32 ? 32 : 2 * BN;  // two accumulators
  constexpr uint32_t IDESC = idesc_bf16(BN);
  constexpr int P = kChunkK / kBK;                           // k-blocks per TMEM chunk

  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = reinterpret_cast<uint8_t *>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  const GemmProblem &p = args.p;
  const int SA = args.sa, SO = args.so;
  uint8_t *aring = smem;
  uint8_t *opring = aring + SA * A32_BYTES;  // slot: [A planes][B planes]
  uint64_t *afull32 = reinterpret_cast<uint64_t *>(opring + SO * OP_BYTES);  // [SA]
  uint64_t *aempty32 = afull32 + SA;                                         // [SA]
  uint64_t *opfull = aempty32 + SA;  // [SO] B planes landed and A planes written
  uint64_t *opempty = opfull + SO;   // [SO] the MMAs reading the slot are done
  uint64_t *tfull = opempty + SO;    // [2] TMEM accumulator holds a finished chunk
  uint64_t *tempty = tfull + 2;      // [2] TMEM accumulator drained
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(tempty + 2);
  int *bad_flag = reinterpret_cast<int *>(tmem_slot + 1);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int split = args.split;
  const int rank = split > 1 ? static_cast<int>(cluster_ctarank()) : 0;
  const int64_t m0 = static_cast<int64_t>(blockIdx.x / split) * kBM;
  const int n0 = blockIdx.y * BN;
  const int kbeg = rank * args.kc;
  const int kend = min(p.K, kbeg + args.kc);
  const int nkb = kend > kbeg ? (kend - kbeg + kBK - 1) / kBK : 0;
  const int nchunks = (nkb + P - 1) / P;

  if (tid == 0) {
    for (int s = 0; s < SA; ++s) {
      mbar_init(&afull32[s], 1);
      mbar_init(&aempty32[s], kConvWarps);
    }
    for (int o = 0; o < SO; ++o) {
      mbar_init(&opfull[o], kConvWarps + 1);  // converter warps + the B loader
      mbar_init(&opempty[o], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&tfull[b], 1);
      mbar_init(&tempty[b], kConvWarps);
    }
    *bad_flag = 0;
    fence_mbar_init();
  }
  if (warp == kMmaWarp) tmem_alloc(tmem_slot, TMEM_COLS);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  float sums[QTR];  // converter warps: FP32 running sums, a quarter row of C
#pragma unroll
  for (int i = 0; i < QTR; ++i) sums[i] = 0.0f;

  if (warp == kLoadAWarp) {
    // -------------------------------------------------------- TMA, A
    if (lane == 0) {
      prefetch_tmap(&tmA);
      for (int kb = 0; kb < nkb; ++kb) {
        const int s = kb % SA;
        if (!mbar_wait(&aempty32[s], ((kb / SA) & 1) ^ 1, args.err, kDevErrEmptyBarrier)) {
          *bad_flag = 1;
          break;
        }
        uint8_t *dst = aring + s * A32_BYTES;
        const int k0 = kbeg + kb * kBK;
        mbar_arrive_expect_tx(&afull32[s], A32_BYTES);
        if (AK)  // 128 rows of 32 floats (128-byte swizzle)
          tma_load_2d(dst, &tmA, &afull32[s], k0, static_cast<int>(m0));
        else     // 32 rows (k) of 128 floats (m)
          tma_load_2d(dst, &tmA, &afull32[s], static_cast<int>(m0), k0);
      }
    }
  } else if (warp == kLoadBWarp) {
    // -------------------------------------------------------- TMA, B
    if (lane == 0) {
      prefetch_tmap(&tmB);
      for (int kb = 0; kb < nkb; ++kb) {
        const int o = kb % SO;
        if (!mbar_wait(&opempty[o], ((kb / SO) & 1) ^ 1, args.err, kDevErrEmptyBarrier)) {
          *bad_flag = 1;
          break;
        }
        uint8_t *dst = opring + o * OP_BYTES + NS * APL_BYTES;
        const int k0 = kbeg + kb * kBK;
        mbar_arrive_expect_tx(&opfull[o], NS * BPL_BYTES);
#pragma unroll
        for (int i = 0; i < NS; ++i)
          tma_load_2d(dst + i * BPL_BYTES, &tmB, &opfull[o], k0, i * args.n_pad + n0);
      }
    }
  } else if (warp == kMmaWarp) {
    // ---------------------------------------------------------- MMA
    if (lane == 0) {
      for (int kb = 0; kb < nkb; ++kb) {
        const int o = kb % SO;
        const int q = kb / P, b = q & 1;
        const bool first = (kb % P) == 0;
        const bool last = (kb % P) == P - 1 || kb == nkb - 1;
        if ((first &&
             !mbar_wait(&tempty[b], ((q >> 1) & 1) ^ 1, args.err, kDevErrEmptyBarrier)) ||
            !mbar_wait(&opfull[o], (kb / SO) & 1, args.err, kDevErrFullBarrier)) {
          *bad_flag = 1;
          break;
        }
        tc_fence_after();
        const uint32_t dacc = tmem + static_cast<uint32_t>(b * BN);
        const uint64_t a_desc = sw64_desc(smem_u32(opring + o * OP_BYTES));
        const uint64_t b_desc = sw64_desc(smem_u32(opring + o * OP_BYTES + NS * APL_BYTES));
#pragma unroll
        for (int kk = 0; kk < kBK / 16; ++kk) {
#pragma unroll
          for (int i = 0; i < NS; ++i)
#pragma unroll
            for (int j = 0; j < NS - i; ++j) {
              // descriptor start addresses count 16-byte units
              const uint64_t ad = a_desc + static_cast<uint64_t>((i * APL_BYTES + kk * 32) >> 4);
              const uint64_t bd = b_desc + static_cast<uint64_t>((j * BPL_BYTES + kk * 32) >> 4);
              const uint32_t acc = (!first || kk > 0 || i > 0 || j > 0) ? 1u : 0u;
              mma_bf16(dacc, ad, bd, IDESC, acc);
            }
        }
        mma_commit(&opempty[o]);
        if (last) mma_commit(&tfull[b]);
      }
    }
  } else {
    // ------------------------------------ converters / drain (warps 0-15)
    const int m = tid & (kBM - 1);  // row of the tile == TMEM lane
    const int g = tid >> 7;         // 8-wide k chunk of each block, column quarter
    const int quarter = warp & 3;   // TMEM lanes 32*quarter .. +31 == rows of this warp
    bool ok = true;
    auto drain = [&](int q) -> bool {
      const int b = q & 1;
      bool w = mbar_wait(&tfull[b], (q >> 1) & 1, args.err, kDevErrMmaBarrier);
      w = __all_sync(0xffffffffu, w);  // tcgen05.ld is warp-collective
      if (!w) return false;
      tc_fence_after();
      const uint32_t taddr =
          tmem + (static_cast<uint32_t>(quarter * 32) << 16) + b * BN + g * QTR;
      if (QTR >= 16) {
#pragma unroll
        for (int nc = 0; nc < QTR; nc += 16) {
          float v[16];
          tmem_ld16(taddr + nc, v);
#pragma unroll
          for (int i = 0; i < 16; ++i) sums[nc + i] += v[i];
        }
      } else if (QTR == 8) {
        float v[8];
        tmem_ld8(taddr, v);
#pragma unroll
        for (int i = 0; i < 8; ++i) sums[i] += v[i];
      } else {
        float v[4];
        tmem_ld4(taddr, v);
#pragma unroll
        for (int i = 0; i < 4; ++i) sums[i] += v[i];
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&tempty[b]);
      return true;
    };
    int drained = 0;
    for (int kb = 0; kb < nkb && ok; ++kb) {
      const int s = kb % SA, o = kb % SO;
      // 1. the FP32 tile: read this thread's eight values and release the
      //    slot at once, so the HBM stream never waits for the MMA pipeline
      bool w = mbar_wait(&afull32[s], (kb / SA) & 1, args.err, kDevErrFullBarrier);
      if (!__all_sync(0xffffffffu, w)) {
        ok = false;
        break;
      }
      const float *a32 = reinterpret_cast<const float *>(aring + s * A32_BYTES);
      float x[8];
      if (AK) {
        // row m holds 32 floats in 128 bytes, 128-byte swizzle
#pragma unroll
        for (int hh = 0; hh < 2; ++hh) {
          const int qq = (2 * g + hh) ^ (m & 7);
          const float4 v = *reinterpret_cast<const float4 *>(a32 + m * 32 + qq * 4);
          x[4 * hh + 0] = v.x; x[4 * hh + 1] = v.y; x[4 * hh + 2] = v.z; x[4 * hh + 3] = v.w;
        }
      } else {
#pragma unroll
        for (int j = 0; j < 8; ++j) x[j] = a32[(g * 8 + j) * kBM + m];
      }
      // consume the values before the warp releases the slot: one lane
      // arrives for the warp, and __syncwarp alone does not wait for the
      // other lanes' shared-memory loads to return
      uint4 v[NS];
      pack8<NS>(x, v);
      __syncwarp();
      if (lane == 0) mbar_arrive(&aempty32[s]);
      // 2. the operand slot: wait until the MMAs that read it are done
      w = mbar_wait(&opempty[o], ((kb / SO) & 1) ^ 1, args.err, kDevErrEmptyBarrier);
      if (!__all_sync(0xffffffffu, w)) {
        ok = false;
        break;
      }
      uint8_t *dst = opring + o * OP_BYTES;
      const uint32_t off = sw64_off(m, g);
#pragma unroll
      for (int i = 0; i < NS; ++i) *reinterpret_cast<uint4 *>(dst + i * APL_BYTES + off) = v[i];
      fence_proxy_async_smem();  // generic-proxy writes -> tensor-core reads
      __syncwarp();
      if (lane == 0) mbar_arrive(&opfull[o]);
      // after the last block of chunk q, drain chunk q-1 (one chunk of slack
      // so the tensor core never waits for the drain)
      const bool chunk_end = (kb % P) == P - 1 || kb == nkb - 1;
      if (chunk_end && kb / P >= 1) {
        if (!drain(drained)) { ok = false; break; }
        ++drained;
      }
    }
    while (ok && drained < nchunks) {
      if (!drain(drained)) { ok = false; break; }
      ++drained;
    }
    if (!ok) *bad_flag = 1;
  }

  // ---------------------------------------------------------- epilogue
  __syncthreads();
  const bool failed = *bad_flag != 0;
  float *red = reinterpret_cast<float *>(smem);  // [BN][kBM], reuses the rings
  if (warp < kConvWarps) {
    const int m = tid & (kBM - 1);
    const int g = tid >> 7;
    const int64_t gm = m0 + m;
    if (failed) {
#pragma unroll
      for (int i = 0; i < QTR; ++i) sums[i] = 0.0f;
    }
    if (split > 1) {
#pragma unroll
      for (int i = 0; i < QTR; ++i) red[(g * QTR + i) * kBM + m] = sums[i];
    } else if (gm < p.M) {
#pragma unroll
      for (int i = 0; i < QTR; ++i) {
        const int gn = n0 + g * QTR + i;
        if (gn < p.N) {
          float *cp = p.C + gm * p.scm + static_cast<int64_t>(gn) * p.scn;
          *cp = axpby(p.alpha, sums[i], p.beta, cp);
        }
      }
    }
  }
  if (split > 1) {
    cluster_sync();
    constexpr int E = kBM * BN;
    const int per = E / split;
    const uint32_t base = smem_u32(red);
    for (int e4 = tid * 4; e4 < per; e4 += kThreads * 4) {
      const int e = rank * per + e4;
      float4 sum = make_float4(0.f, 0.f, 0.f, 0.f);
      for (int r = 0; r < split; ++r) {
        const float4 v = ld_dsmem4(mapa_shared(base + e * 4, r));
        sum.x += v.x; sum.y += v.y; sum.z += v.z; sum.w += v.w;
      }
      const float sv[4] = {sum.x, sum.y, sum.z, sum.w};
#pragma unroll
      for (int qq = 0; qq < 4; ++qq) {
        const int mm = (e + qq) % kBM, nn = (e + qq) / kBM;
        const int64_t gm = m0 + mm;
        const int gn = n0 + nn;
        if (gm < p.M && gn < p.N) {
          float *cp = p.C + gm * p.scm + static_cast<int64_t>(gn) * p.scn;
          *cp = axpby(p.alpha, sv[qq], p.beta, cp);
        }
      }
    }
    cluster_sync();
  }
  tc_fence_before();
  __syncthreads();
  if (warp == kMmaWarp) tmem_dealloc(tmem, TMEM_COLS);
}

}  // namespace

bool tc_config_fits(int bn, int ns, int stages) {
  TcPlan pl;
  return tc_plan(bn, ns, stages, &pl);
}

namespace {

template <int BN, int NS, bool AK>
hml_status run_tc(const GemmProblem &p, const hml_sgemm_config &c, cudaStream_t s) {
  const int k_pad = ((p.K + kChunkK - 1) / kChunkK) * kChunkK;
  const int n_pad = ((p.N + BN - 1) / BN) * BN;
  // B planes in the stream's workspace
  const size_t plane_bytes = static_cast<size_t>(n_pad) * k_pad * 2;
  void *ws = nullptr;
  hml_status st = workspace(NS * plane_bytes, s, &ws);
  if (st != HML_STATUS_SUCCESS) return st;
  auto *planes = static_cast<__nv_bfloat16 *>(ws);
  {
    const int64_t chunks = static_cast<int64_t>(n_pad) * (k_pad / 8);
    const int blocks = static_cast<int>(std::min<int64_t>((chunks + 255) / 256, 4 * sm_count()));
    count_launch();
    split_b_kernel<NS><<<blocks, 256, 0, s>>>(p.B, p.sbk, p.sbn, p.K, p.N, planes, k_pad, n_pad);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
      note_cuda_error(e, "split_b");
      return HML_STATUS_CUDA_ERROR;
    }
  }
  CUtensorMap ta, tb;
  memset(&ta, 0, sizeof ta);
  memset(&tb, 0, sizeof tb);
  bool ok;
  if (AK)
    ok = tensor_map_2d(&ta, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, p.A, p.K, p.M, p.sam * 4, kBK, kBM,
                       CU_TENSOR_MAP_SWIZZLE_128B);
  else
    ok = tensor_map_2d(&ta, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, p.A, p.M, p.K, p.sak * 4, kBM, kBK,
                       CU_TENSOR_MAP_SWIZZLE_NONE);
  if (ok)
    ok = tensor_map_2d(&tb, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, planes, k_pad,
                       static_cast<uint64_t>(NS) * n_pad, static_cast<uint64_t>(k_pad) * 2, kBK, BN,
                       CU_TENSOR_MAP_SWIZZLE_64B);
  if (!ok) return HML_STATUS_CUDA_ERROR;
  TcArgs args;
  args.p = p;
  args.split = c.split_k;
  const int kchunks = k_pad / kChunkK;
  args.kc = ((kchunks + c.split_k - 1) / c.split_k) * kChunkK;
  TcPlan plan;
  if (!tc_plan(BN, NS, c.stages, &plan)) return HML_STATUS_INVALID_VALUE;
  args.sa = plan.sa;
  args.so = plan.so;
  args.n_pad = n_pad;
  args.err = device_error_word();
  const size_t smem = tc_plan_bytes(BN, NS, plan);
  auto kern = tc_kernel<BN, NS, AK>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem));
  if (e == cudaSuccess && c.split_k > 8)
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  if (e != cudaSuccess) {
    note_cuda_error(e, "tc attributes");
    return HML_STATUS_CUDA_ERROR;
  }
  const int64_t tiles_m = (static_cast<int64_t>(p.M) + kBM - 1) / kBM;
  const int64_t tiles_n = n_pad / BN;
  if (tiles_m * c.split_k > 0x7fffffff || tiles_n > 65535) return HML_STATUS_NOT_SUPPORTED;
  dim3 grid(static_cast<unsigned>(tiles_m * c.split_k), static_cast<unsigned>(tiles_n));
  e = launch_k(kern, grid, dim3(kThreads), smem, s, c.split_k, ta, tb, args);
  note_cuda_error(e, "tc launch");
  return cuda_status(e);
}

template <int BN, int NS>
hml_status run_tc_layout(const GemmProblem &p, const hml_sgemm_config &c, cudaStream_t s) {
  return p.a_kcontig() ? run_tc<BN, NS, true>(p, c, s) : run_tc<BN, NS, false>(p, c, s);
}

template <int NS>
hml_status run_tc_ns(const GemmProblem &p, const hml_sgemm_config &c, cudaStream_t s) {
  switch (c.tile_n) {
    case 16: return run_tc_layout<16, NS>(p, c, s);
    case 32: return run_tc_layout<32, NS>(p, c, s);
    case 64: return run_tc_layout<64, NS>(p, c, s);
    case 128: return run_tc_layout<128, NS>(p, c, s);
    default: return HML_STATUS_INVALID_VALUE;
  }
}

bool aligned16(const void *ptr) { return (reinterpret_cast<uintptr_t>(ptr) & 15u) == 0; }

}  // namespace

int tc_num_shapes() { return kNumTcShapes; }
void tc_shape(int v, int *bm, int *bn) {
  *bm = kBM;
  *bn = kTcShapes[v].bn;
}

hml_status check_tc(const GemmProblem &p, const hml_sgemm_config &c) {
  if (c.algo != HML_ALGO_BF16X3 && c.algo != HML_ALGO_BF16X6) return HML_STATUS_INVALID_VALUE;
  if (c.variant < 0 || c.variant >= kNumTcShapes) return HML_STATUS_INVALID_VALUE;
  if (c.tile_m != kBM || c.tile_n != kTcShapes[c.variant].bn) return HML_STATUS_INVALID_VALUE;
  if (c.split_k < 1 || c.split_k > 16 || (c.split_k & (c.split_k - 1)) != 0)
    return HML_STATUS_INVALID_VALUE;
  if (c.stages < 2 || c.stages > 8) return HML_STATUS_INVALID_VALUE;
  const int ns = c.algo == HML_ALGO_BF16X3 ? 2 : 3;
  if (!tc_config_fits(c.tile_n, ns, c.stages)) return HML_STATUS_INVALID_VALUE;
  // the rings are reused for the split-K partial tile
  if (c.split_k > 1 &&
      static_cast<size_t>(kBM) * c.tile_n * 4 > static_cast<size_t>(c.stages) * tc_a_bytes())
    return HML_STATUS_INVALID_VALUE;
  // TMA on A: 16-byte aligned base and row stride
  const int64_t sa = p.a_kcontig() ? p.sam : p.sak;
  if (!aligned16(p.A) || (sa * 4) % 16 != 0) return HML_STATUS_NOT_SUPPORTED;
  if (p.a_kcontig() ? p.sak != 1 : p.sam != 1) return HML_STATUS_NOT_SUPPORTED;
  if (p.M < 1 || p.N < 1 || p.K < 1) return HML_STATUS_NOT_SUPPORTED;
  return HML_STATUS_SUCCESS;
}

hml_status launch_tc(const GemmProblem &p, const hml_sgemm_config &c, cudaStream_t s) {
  hml_status st = check_tc(p, c);
  if (st != HML_STATUS_SUCCESS) return st;
  return c.algo == HML_ALGO_BF16X3 ? run_tc_ns<2>(p, c, s) : run_tc_ns<3>(p, c, s);
}

}  // namespace hml

// ----------------------------------------------------- no-allocation variant
//
// hml_sgemm_ex_config_noalloc runs the split-BF16 kernel above without any
// device allocation.  Its only scratch, the BF16 planes of B, lives in a
// fixed-size array in this file's module instead of the per-stream workspace
// (which the library grows with cudaMalloc).  The array is part of the
// library's device image, so every GPU that loads the library holds it until
// the process exits.
namespace hml {
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(4) << 20;  // 4 MiB per device
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
void *g_noalloc_addr[kNoAllocMaxDevices];

// Device address of the scratch array on the current device.  In host code
// the array's name is only a host-side stand-in, so the address is looked up
// once per device (with that device current) and cached.
hml_status noalloc_scratch(void **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    note_cuda_error(e, "noalloc: cudaGetDevice");
    return HML_STATUS_CUDA_ERROR;
  }
  if (dev < 0 || dev >= kNoAllocMaxDevices) return HML_STATUS_NOT_SUPPORTED;
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void *addr = nullptr;
    e = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
    if (e != cudaSuccess || !addr) {
      note_cuda_error(e != cudaSuccess ? e : cudaErrorInvalidSymbol,
                      "noalloc: cudaGetSymbolAddress");
      return HML_STATUS_CUDA_ERROR;
    }
    g_noalloc_addr[dev] = addr;
  }
  *out = g_noalloc_addr[dev];
  return HML_STATUS_SUCCESS;
}

size_t noalloc_bytes_needed(const GemmProblem &p, const hml_sgemm_config &c) {
  const int ns = c.algo == HML_ALGO_BF16X3 ? 2 : 3;
  const size_t k_pad = ((static_cast<size_t>(p.K) + kChunkK - 1) / kChunkK) * kChunkK;
  const size_t n_pad = ((static_cast<size_t>(p.N) + c.tile_n - 1) / c.tile_n) * c.tile_n;
  return static_cast<size_t>(ns) * n_pad * k_pad * 2;
}

// The launch of run_tc with the B planes in `planes` (the static array) and
// no device error word (bounded waits still end; nothing is recorded).
template <int BN, int NS, bool AK>
hml_status run_tc_static(const GemmProblem &p, const hml_sgemm_config &c, void *scratch,
                         cudaStream_t s) {
  const int k_pad = ((p.K + kChunkK - 1) / kChunkK) * kChunkK;
  const int n_pad = ((p.N + BN - 1) / BN) * BN;
  auto *planes = static_cast<__nv_bfloat16 *>(scratch);
  {
    const int64_t chunks = static_cast<int64_t>(n_pad) * (k_pad / 8);
    const int blocks = static_cast<int>(std::min<int64_t>((chunks + 255) / 256, 4 * sm_count()));
    count_launch();
    split_b_kernel<NS><<<blocks, 256, 0, s>>>(p.B, p.sbk, p.sbn, p.K, p.N, planes, k_pad, n_pad);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
      note_cuda_error(e, "noalloc split_b");
      return HML_STATUS_CUDA_ERROR;
    }
  }
  CUtensorMap ta, tb;
  memset(&ta, 0, sizeof ta);
  memset(&tb, 0, sizeof tb);
  bool ok;
  if (AK)
    ok = tensor_map_2d(&ta, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, p.A, p.K, p.M, p.sam * 4, kBK, kBM,
                       CU_TENSOR_MAP_SWIZZLE_128B);
  else
    ok = tensor_map_2d(&ta, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, p.A, p.M, p.K, p.sak * 4, kBM, kBK,
                       CU_TENSOR_MAP_SWIZZLE_NONE);
  if (ok)
    ok = tensor_map_2d(&tb, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, planes, k_pad,
                       static_cast<uint64_t>(NS) * n_pad, static_cast<uint64_t>(k_pad) * 2, kBK, BN,
                       CU_TENSOR_MAP_SWIZZLE_64B);
  if (!ok) return HML_STATUS_CUDA_ERROR;
  TcArgs args;
  args.p = p;
  args.split = c.split_k;
  const int kchunks = k_pad / kChunkK;
  args.kc = ((kchunks + c.split_k - 1) / c.split_k) * kChunkK;
  TcPlan plan;
  if (!tc_plan(BN, NS, c.stages, &plan)) return HML_STATUS_INVALID_VALUE;
  args.sa = plan.sa;
  args.so = plan.so;
  args.n_pad = n_pad;
  args.err = nullptr;
  const size_t smem = tc_plan_bytes(BN, NS, plan);
  auto kern = tc_kernel<BN, NS, AK>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem));
  if (e == cudaSuccess && c.split_k > 8)
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  if (e != cudaSuccess) {
    note_cuda_error(e, "noalloc tc attributes");
    return HML_STATUS_CUDA_ERROR;
  }
  const int64_t tiles_m = (static_cast<int64_t>(p.M) + kBM - 1) / kBM;
  const int64_t tiles_n = n_pad / BN;
  if (tiles_m * c.split_k > 0x7fffffff || tiles_n > 65535) return HML_STATUS_NOT_SUPPORTED;
  dim3 grid(static_cast<unsigned>(tiles_m * c.split_k), static_cast<unsigned>(tiles_n));
  e = launch_k(kern, grid, dim3(kThreads), smem, s, c.split_k, ta, tb, args);
  note_cuda_error(e, "noalloc tc launch");
  return cuda_status(e);
}

template <int NS>
hml_status run_tc_static_ns(const GemmProblem &p, const hml_sgemm_config &c, void *scratch,
                            cudaStream_t s) {
  const bool ak = p.a_kcontig();
  switch (c.tile_n) {
    case 16: return ak ? run_tc_static<16, NS, true>(p, c, scratch, s)
                       : run_tc_static<16, NS, false>(p, c, scratch, s);
    case 32: return ak ? run_tc_static<32, NS, true>(p, c, scratch, s)
                       : run_tc_static<32, NS, false>(p, c, scratch, s);
    case 64: return ak ? run_tc_static<64, NS, true>(p, c, scratch, s)
                       : run_tc_static<64, NS, false>(p, c, scratch, s);
    case 128: return ak ? run_tc_static<128, NS, true>(p, c, scratch, s)
                        : run_tc_static<128, NS, false>(p, c, scratch, s);
    default: return HML_STATUS_INVALID_VALUE;
  }
}

}  // namespace
}  // namespace hml

extern "C" hml_status hml_sgemm_ex_config_noalloc(hml_order order, hml_op transA, hml_op transB,
                                                  int M, int N, int K, float alpha, const float *A,
                                                  int lda, const float *B, int ldb, float beta,
                                                  float *C, int ldc, const hml_sgemm_config *config,
                                                  void *stream) {
  using namespace hml;
  if (!config || (config->algo != HML_ALGO_BF16X3 && config->algo != HML_ALGO_BF16X6))
    return HML_STATUS_INVALID_VALUE;
  GemmProblem p;
  hml_status st = gemm_from_blas(order, transA, transB, M, N, K, alpha, A, lda, B, ldb, beta, C,
                                 ldc, &p);
  if (st != HML_STATUS_SUCCESS) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (p.M == 0 || p.N == 0) return HML_STATUS_SUCCESS;
  if (p.K == 0 || p.alpha == 0.0f) return launch_scale(p.C, p.M, p.N, p.scm, p.scn, p.beta, s);
  st = check_tc(p, *config);
  if (st != HML_STATUS_SUCCESS) return st;
  if (noalloc_bytes_needed(p, *config) > kNoAllocScratchBytes) {
    note_text_error("noalloc: the BF16 planes of B need more than the 4 MiB static scratch "
                    "(planes x ceil(N/tile_n)*tile_n x ceil(K/64)*64 x 2 bytes)");
    return HML_STATUS_INVALID_VALUE;
  }
  void *scratch = nullptr;
  st = noalloc_scratch(&scratch);
  if (st != HML_STATUS_SUCCESS) return st;
  return config->algo == HML_ALGO_BF16X3 ? run_tc_static_ns<2>(p, *config, scratch, s)
                                         : run_tc_static_ns<3>(p, *config, scratch, s);
}
