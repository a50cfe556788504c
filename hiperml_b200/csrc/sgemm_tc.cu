// sgemm_tc.cu -- split-BF16 SGEMM on the B200 tensor cores (tcgen05 + TMEM).
//
// FP32 operands are split into BF16 terms, a = a0 + a1 (+ a2), each term the
// BF16 rounding of what the previous terms left, and the products that carry
// FP32-level information are accumulated in FP32 in tensor memory:
//   BF16X3: a0*b0 + a0*b1 + a1*b0                       (2 planes, 3 MMAs)
//   BF16X6: a0*b0 + a0*b1 + a1*b0 + a0*b2 + a1*b1 + a2*b0 (3 planes, 6 MMAs)
// The result is C = alpha * A * B + beta * C in FP32, the reference's
// hmlSgemm contract (src/hml_sgemm.cu:120-211) with a different machine.
//
// Data flow per CTA (one 128-row tile of C, all BN columns, a K range):
//   * B is small (K x N): a pre-pass splits it once into BF16 planes stored
//     K-contiguous in a workspace ([plane][N_pad][K_pad]); the main kernel
//     loads plane tiles with TMA straight into the UMMA canonical K-major
//     128-byte-swizzled layout.
//   * A is streamed from HBM exactly once: a TMA warp loads 128 x 64 FP32
//     tiles into a ring; four converter warps split each tile into BF16
//     planes written in the canonical K-major swizzled layout (a transpose
//     when A is M-contiguous), then signal the MMA warp.
//   * one thread of the MMA warp issues tcgen05.mma (M=128, N=BN, K=16,
//     operands from shared memory, accumulator in TMEM) and releases ring
//     slots with tcgen05.commit.
//   * the converter warps then read the accumulator with tcgen05.ld and
//     apply alpha/beta; with split_k > 1 the CTAs of a cluster sum their
//     tiles in rank order through distributed shared memory.
// Every wait is bounded (2 s of %globaltimer); on expiry the device error
// word is set, the CTA skips ahead, frees its TMEM and returns.
#include <cuda_bf16.h>

#include <algorithm>
#include <cstring>

#include "hml_device.cuh"
#include "hml_internal.h"

namespace hml {
namespace {

constexpr int kBM = 128;  // rows of C per CTA = UMMA M
constexpr int kBK = 64;   // K per ring stage (one 128-byte BF16 swizzle row)
constexpr int kConvThreads = 128;
constexpr int kThreads = 192;  // warps 0-3 convert + epilogue, 4 TMA, 5 MMA

struct TcShape {
  int bn;
};
constexpr TcShape kTcShapes[] = {{16}, {32}, {64}, {128}, {256}};
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

// 32 lanes x 16 consecutive 32-bit columns of TMEM into 16 registers.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
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

// Shared-memory matrix descriptor: K-major, 128-byte swizzle, rows of 128 B,
// 8-row atoms 1024 B apart (SBO), descriptor version 1.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  return static_cast<uint64_t>((saddr >> 4) & 0x3FFFu) | (static_cast<uint64_t>(1) << 16) |
         (static_cast<uint64_t>(1024 >> 4) << 32) | (static_cast<uint64_t>(1) << 46) |
         (static_cast<uint64_t>(2) << 61);
}

// Instruction descriptor: BF16 x BF16 -> F32, both K-major, M = 128, N = bn.
__host__ __device__ constexpr uint32_t idesc_bf16(int bn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(bn >> 3) << 17) |
         (static_cast<uint32_t>(kBM >> 4) << 24);
}

// Split x into NS BF16 terms: t0 = bf16(x), t1 = bf16(x - t0), ...
// (each residual is exact in FP32).
template <int NS>
__device__ __forceinline__ void split_bf16(float x, unsigned short (&t)[NS]) {
  float r = x;
#pragma unroll
  for (int i = 0; i < NS; ++i) {
    const __nv_bfloat16 h = __float2bfloat16_rn(r);
    t[i] = __bfloat16_as_ushort(h);
    r = r - __bfloat162float(h);
  }
}

struct TcArgs {
  GemmProblem p;
  int split;     // CTAs per cluster along K
  int kc;        // K extent per split (multiple of kBK)
  int stages;    // FP32 A ring depth
  int cbufs;     // converted-A ring depth
  int n_pad;     // rows of one B plane in the workspace
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
    unsigned short t[NS][8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int k = k0 + j;
      const float x = (n < N && k < K) ? B[static_cast<int64_t>(k) * sbk + static_cast<int64_t>(n) * sbn] : 0.0f;
      unsigned short s[NS];
      split_bf16<NS>(x, s);
#pragma unroll
      for (int i = 0; i < NS; ++i) t[i][j] = s[i];
    }
#pragma unroll
    for (int i = 0; i < NS; ++i) {
      uint4 v;
      v.x = t[i][0] | (static_cast<uint32_t>(t[i][1]) << 16);
      v.y = t[i][2] | (static_cast<uint32_t>(t[i][3]) << 16);
      v.z = t[i][4] | (static_cast<uint32_t>(t[i][5]) << 16);
      v.w = t[i][6] | (static_cast<uint32_t>(t[i][7]) << 16);
      *reinterpret_cast<uint4 *>(planes + (static_cast<int64_t>(i) * n_pad + n) * k_pad + k0) = v;
    }
  }
}

// ------------------------------------------------------------- kernel
template <int BN, int NS, bool AK>
__global__ void __launch_bounds__(kThreads, 1)
    tc_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
              TcArgs args) {
  constexpr int A32_BYTES = kBM * kBK * 4;          // FP32 A stage (32 KB)
  constexpr int BPL_BYTES = BN * kBK * 2;           // one B plane tile
  constexpr int STAGE_BYTES = A32_BYTES + NS * BPL_BYTES;
  constexpr int APL_BYTES = kBM * kBK * 2;          // one converted A plane (16 KB)
  constexpr int CBUF_BYTES = NS * APL_BYTES;
  constexpr uint32_t TMEM_COLS = BN < 32 ? 32 : BN;
  constexpr uint32_t IDESC = idesc_bf16(BN);

  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = reinterpret_cast<uint8_t *>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  const GemmProblem &p = args.p;
  const int S = args.stages, CB = args.cbufs;
  uint8_t *ring = smem;                       // S x STAGE_BYTES
  uint8_t *cbuf = smem + S * STAGE_BYTES;     // CB x CBUF_BYTES (1024-aligned)
  uint64_t *full = reinterpret_cast<uint64_t *>(cbuf + CB * CBUF_BYTES);
  uint64_t *empty = full + S;
  uint64_t *cfull = empty + S;
  uint64_t *cempty = cfull + CB;
  uint64_t *accfull = cempty + CB;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(accfull + 1);
  int *bad_flag = reinterpret_cast<int *>(tmem_slot + 1);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int split = args.split;
  const int rank = split > 1 ? static_cast<int>(cluster_ctarank()) : 0;
  const int64_t m0 = static_cast<int64_t>(blockIdx.x / split) * kBM;
  const int n0 = blockIdx.y * BN;
  const int kbeg = rank * args.kc;
  const int kend = min(p.K, kbeg + args.kc);
  const int nkb = kend > kbeg ? (kend - kbeg + kBK - 1) / kBK : 0;

  if (tid == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int c = 0; c < CB; ++c) {
      mbar_init(&cfull[c], kConvThreads);
      mbar_init(&cempty[c], 1);
    }
    mbar_init(accfull, 1);
    *bad_flag = 0;
    fence_mbar_init();
  }
  if (warp == 5) tmem_alloc(tmem_slot, TMEM_COLS);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 4) {
    // ---------------------------------------------------------- TMA
    if (lane == 0) {
      prefetch_tmap(&tmA);
      prefetch_tmap(&tmB);
      for (int kb = 0; kb < nkb; ++kb) {
        const int s = kb % S;
        if (!mbar_wait(&empty[s], ((kb / S) & 1) ^ 1, args.err, kDevErrEmptyBarrier)) {
          *bad_flag = 1;
          break;
        }
        uint8_t *st = ring + s * STAGE_BYTES;
        const int k0 = kbeg + kb * kBK;
        mbar_arrive_expect_tx(&full[s], STAGE_BYTES);
        if (AK) {
          // two 32-float wide boxes (128-byte swizzle), rows = 128 m
          tma_load_2d(st, &tmA, &full[s], k0, static_cast<int>(m0));
          tma_load_2d(st + A32_BYTES / 2, &tmA, &full[s], k0 + 32, static_cast<int>(m0));
        } else {
          tma_load_2d(st, &tmA, &full[s], static_cast<int>(m0), k0);
        }
#pragma unroll
        for (int i = 0; i < NS; ++i)
          tma_load_2d(st + A32_BYTES + i * BPL_BYTES, &tmB, &full[s], k0, i * args.n_pad + n0);
      }
    }
  } else if (warp == 5) {
    // ---------------------------------------------------------- MMA
    if (lane == 0) {
      for (int kb = 0; kb < nkb; ++kb) {
        const int s = kb % S, c = kb % CB;
        if (!mbar_wait(&full[s], (kb / S) & 1, args.err, kDevErrFullBarrier) ||
            !mbar_wait(&cfull[c], (kb / CB) & 1, args.err, kDevErrFullBarrier)) {
          *bad_flag = 1;
          break;
        }
        tc_fence_after();
        const uint32_t a_base = smem_u32(cbuf + c * CBUF_BYTES);
        const uint32_t b_base = smem_u32(ring + s * STAGE_BYTES + A32_BYTES);
#pragma unroll
        for (int kk = 0; kk < kBK / 16; ++kk) {
          // products in increasing magnitude order is not needed: the FP32
          // accumulator holds every term's 16 leading bits
#pragma unroll
          for (int i = 0; i < NS; ++i)
#pragma unroll
            for (int j = 0; j < NS - i; ++j) {
              const uint64_t ad = sw128_desc(a_base + i * APL_BYTES + kk * 32);
              const uint64_t bd = sw128_desc(b_base + j * BPL_BYTES + kk * 32);
              const uint32_t acc = (kb > 0 || kk > 0 || i > 0 || j > 0) ? 1u : 0u;
              mma_bf16(tmem, ad, bd, IDESC, acc);
            }
        }
        mma_commit(&empty[s]);
        mma_commit(&cempty[c]);
      }
      mma_commit(accfull);
    }
  } else {
    // ---------------------------------------------------- converters
    const int m = tid;  // row of the tile, 0..127
    for (int kb = 0; kb < nkb; ++kb) {
      const int s = kb % S, c = kb % CB;
      if (!mbar_wait(&full[s], (kb / S) & 1, args.err, kDevErrFullBarrier) ||
          !mbar_wait(&cempty[c], ((kb / CB) & 1) ^ 1, args.err, kDevErrEmptyBarrier)) {
        *bad_flag = 1;
        break;
      }
      const float *a32 = reinterpret_cast<const float *>(ring + s * STAGE_BYTES);
      uint8_t *dst = cbuf + c * CBUF_BYTES;
#pragma unroll
      for (int ch = 0; ch < kBK / 8; ++ch) {  // 8 chunks of 8 k values
        float x[8];
        if (AK) {
          // box (ch / 4) holds k in [32*(ch/4), +32): 128-byte rows, swizzled
          const float *box = a32 + (ch >> 2) * (kBM * 32);
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int q = ((ch & 3) * 2 + h) ^ (m & 7);  // 16-byte chunk within the row
            const float4 v = *reinterpret_cast<const float4 *>(box + m * 32 + q * 4);
            x[4 * h + 0] = v.x; x[4 * h + 1] = v.y; x[4 * h + 2] = v.z; x[4 * h + 3] = v.w;
          }
        } else {
#pragma unroll
          for (int j = 0; j < 8; ++j) x[j] = a32[(ch * 8 + j) * kBM + m];
        }
        unsigned short t[NS][8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          unsigned short sp[NS];
          split_bf16<NS>(x[j], sp);
#pragma unroll
          for (int i = 0; i < NS; ++i) t[i][j] = sp[i];
        }
        const uint32_t off = static_cast<uint32_t>(m * 128 + ((ch ^ (m & 7)) << 4));
#pragma unroll
        for (int i = 0; i < NS; ++i) {
          uint4 v;
          v.x = t[i][0] | (static_cast<uint32_t>(t[i][1]) << 16);
          v.y = t[i][2] | (static_cast<uint32_t>(t[i][3]) << 16);
          v.z = t[i][4] | (static_cast<uint32_t>(t[i][5]) << 16);
          v.w = t[i][6] | (static_cast<uint32_t>(t[i][7]) << 16);
          *reinterpret_cast<uint4 *>(dst + i * APL_BYTES + off) = v;
        }
      }
      fence_proxy_async_smem();  // generic-proxy writes -> tensor-core reads
      mbar_arrive(&cfull[c]);
    }
  }

  // ---------------------------------------------------------- epilogue
  __syncthreads();
  const bool failed = *bad_flag != 0;
  float *red = reinterpret_cast<float *>(ring);  // [BN][kBM], reuses the ring
  if (warp < 4) {
    bool ok = !failed;
    if (ok && nkb > 0) ok = mbar_wait(accfull, 0, args.err, kDevErrMmaBarrier);
    ok = __all_sync(0xffffffffu, ok);  // tcgen05.ld is warp-collective
    tc_fence_after();
    const int m = warp * 32 + lane;
    const int64_t gm = m0 + m;
#pragma unroll 1
    for (int nc = 0; nc < BN; nc += 16) {
      float v[16];
      if (ok && nkb > 0) {
        tmem_ld16(tmem + (static_cast<uint32_t>(warp * 32) << 16) + nc, v);
      } else {
#pragma unroll
        for (int i = 0; i < 16; ++i) v[i] = 0.0f;
      }
      if (split > 1) {
#pragma unroll
        for (int i = 0; i < 16; ++i) red[(nc + i) * kBM + m] = v[i];
      } else if (gm < p.M) {
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          const int gn = n0 + nc + i;
          if (gn < p.N) {
            float *cp = p.C + gm * p.scm + static_cast<int64_t>(gn) * p.scn;
            *cp = axpby(p.alpha, v[i], p.beta, cp);
          }
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
      for (int q = 0; q < 4; ++q) {
        const int mm = (e + q) % kBM, nn = (e + q) / kBM;
        const int64_t gm = m0 + mm;
        const int gn = n0 + nn;
        if (gm < p.M && gn < p.N) {
          float *cp = p.C + gm * p.scm + static_cast<int64_t>(gn) * p.scn;
          *cp = axpby(p.alpha, sv[q], p.beta, cp);
        }
      }
    }
    cluster_sync();
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 5) tmem_dealloc(tmem, TMEM_COLS);
}

size_t tc_smem_bytes(int bn, int ns, int stages, int cbufs) {
  const size_t stage = static_cast<size_t>(kBM) * kBK * 4 + static_cast<size_t>(ns) * bn * kBK * 2;
  const size_t cb = static_cast<size_t>(ns) * kBM * kBK * 2;
  return 1024 + stages * stage + cbufs * cb + 8 * (2 * stages + 2 * cbufs + 1) + 16;
}

}  // namespace

bool tc_config_fits(int bn, int ns, int stages) {
  return tc_smem_bytes(bn, ns, stages, 1) <= 227 * 1024;
}

namespace {

int pick_cbufs(int bn, int ns, int stages) {
  return tc_smem_bytes(bn, ns, stages, 2) <= 227 * 1024 ? 2 : 1;
}

template <int BN, int NS, bool AK>
hml_status run_tc(const GemmProblem &p, const hml_sgemm_config &c, cudaStream_t s) {
  const int k_pad = ((p.K + kBK - 1) / kBK) * kBK;
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
    ok = tensor_map_2d(&ta, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, p.A, p.K, p.M, p.sam * 4, 32, kBM,
                       CU_TENSOR_MAP_SWIZZLE_128B);
  else
    ok = tensor_map_2d(&ta, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, p.A, p.M, p.K, p.sak * 4, kBM, kBK,
                       CU_TENSOR_MAP_SWIZZLE_NONE);
  if (ok)
    ok = tensor_map_2d(&tb, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, planes, k_pad,
                       static_cast<uint64_t>(NS) * n_pad, static_cast<uint64_t>(k_pad) * 2, kBK, BN,
                       CU_TENSOR_MAP_SWIZZLE_128B);
  if (!ok) return HML_STATUS_CUDA_ERROR;
  TcArgs args;
  args.p = p;
  args.split = c.split_k;
  const int kblocks = k_pad / kBK;
  args.kc = ((kblocks + c.split_k - 1) / c.split_k) * kBK;
  args.stages = c.stages;
  args.cbufs = pick_cbufs(BN, NS, c.stages);
  args.n_pad = n_pad;
  args.err = device_error_word();
  const size_t smem = tc_smem_bytes(BN, NS, c.stages, args.cbufs);
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
    case 256: return run_tc_layout<256, NS>(p, c, s);
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
  if (c.stages < 2 || c.stages > 4) return HML_STATUS_INVALID_VALUE;
  const int ns = c.algo == HML_ALGO_BF16X3 ? 2 : 3;
  if (tc_smem_bytes(c.tile_n, ns, c.stages, 1) > 227 * 1024) return HML_STATUS_INVALID_VALUE;
  // the ring is reused for the split-K partial tile
  if (c.split_k > 1 &&
      static_cast<size_t>(kBM) * c.tile_n * 4 >
          static_cast<size_t>(c.stages) * (kBM * kBK * 4 + ns * c.tile_n * kBK * 2))
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
