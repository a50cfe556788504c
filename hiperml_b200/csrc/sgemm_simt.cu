// sgemm_simt.cu -- plain FP32 SIMT skinny SGEMM for B200 (sm_100a).
//
// Replaces the reference's var-K / const-K kernels
// (include/hml_sgemm_kernel_template.h:19-191, 229-333): same result
// C = alpha * A * B + beta * C in FP32, different machine.
//
// Structure of one CTA (warp specialised):
//   * 32-deep K slabs of A (BM x 32) and B (32 x BN) are staged into a ring
//     of `stages` shared-memory buffers, stages-1 slabs ahead of the math.
//     When strides and base addresses allow it one thread issues 2-D TMA
//     tile loads (cp.async.bulk.tensor, no multicast) that complete on a
//     per-slot mbarrier; otherwise every thread issues 4-byte cp.async
//     copies with zero fill (cp.async groups).  A tile of K-contiguous A
//     uses the 128-byte swizzle so that it is read without bank conflicts.
//     There is no separate producer warp: a ninth warp would put three warps
//     on one SM sub-partition and cap registers at 168 per thread, too few
//     for the 8 x 16 micro-tiles.
//   * 8 warps, arranged WM x WN x WK.  Each lane owns TM rows x TN
//     columns of C in registers; all lanes of a warp share the same columns,
//     so B values are shared-memory broadcasts and A values are read once per
//     warp.  WK > 1 splits every K slab across warps (intra-CTA split-K) for
//     the skinny shapes, where a C tile is too small to occupy 8 warps.
//   * epilogue: the WK partial tiles are summed in shared memory; with
//     split_k > 1 the CTAs of one thread-block cluster each own a K range
//     and the cluster sums their tiles through distributed shared memory in
//     rank order.  No global workspace, deterministic results.  beta == 0
//     does not read C.
#include <algorithm>
#include <cstring>

#include "hml_device.cuh"
#include "hml_internal.h"

namespace hml {
namespace {

constexpr int kBK = 32;  // K depth of one pipeline stage (128 bytes of FP32)

struct SimtShape {
  int tm, tn, wm, wn, wk;
  int bm() const { return wm * 32 * tm; }
  int bn() const { return wn * tn; }
};

// The micro-tile table (index = hml_sgemm_config.variant for HML_ALGO_SIMT).
constexpr SimtShape kSimtShapes[] = {
    {4, 16, 1, 1, 8},  // 0: 128 x 16,  K split 8 ways across warps
    {4, 8, 1, 1, 8},   // 1: 128 x 8
    {4, 16, 1, 2, 4},  // 2: 128 x 32
    {8, 16, 1, 2, 4},  // 3: 256 x 32
    {8, 16, 1, 4, 2},  // 4: 256 x 64
    {8, 16, 1, 8, 1},  // 5: 256 x 128
    {4, 16, 2, 4, 1},  // 6: 256 x 64, two row groups
    {4, 16, 1, 4, 2},  // 7: 128 x 64
    {4, 16, 1, 8, 1},  // 8: 128 x 128
};
constexpr int kNumSimtShapes = sizeof(kSimtShapes) / sizeof(kSimtShapes[0]);

__device__ __forceinline__ float4 lds128(const float *p) {
  return *reinterpret_cast<const float4 *>(p);
}

__device__ __forceinline__ void cp_async4(uint32_t dst, const float *src, bool valid) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(dst), "l"(src),
               "r"(valid ? 4 : 0)
               : "memory");
}

struct SimtArgs {
  GemmProblem p;
  int split;      // CTAs per cluster along K
  int kc;         // K extent per split (multiple of kBK)
  int stages;
  int *err;
};

__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}

// cp.async.wait_group takes an immediate: dispatch the runtime ring depth.
__device__ __forceinline__ void cp_async_wait_ring(int stages) {
  switch (stages) {
    case 2: asm volatile("cp.async.wait_group 0;" ::: "memory"); break;
    case 3: asm volatile("cp.async.wait_group 1;" ::: "memory"); break;
    case 4: asm volatile("cp.async.wait_group 2;" ::: "memory"); break;
    case 5: asm volatile("cp.async.wait_group 3;" ::: "memory"); break;
    case 6: asm volatile("cp.async.wait_group 4;" ::: "memory"); break;
    case 7: asm volatile("cp.async.wait_group 5;" ::: "memory"); break;
    default: asm volatile("cp.async.wait_group 6;" ::: "memory"); break;
  }
}

template <int TM, int TN, int WM, int WN, int WK, bool AK, bool BK_, bool TMA>
__global__ void __launch_bounds__(256, 1)
    simt_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                SimtArgs args) {
  constexpr int BM = WM * 32 * TM;
  constexpr int BN = WN * TN;
  constexpr int NCW = WM * WN * WK;  // warps
  static_assert(NCW == 8, "8 warps");
  constexpr int NT = NCW * 32;
  constexpr int KW = kBK / WK;  // K values per warp per stage
  constexpr int A_BYTES = BM * kBK * 4;
  constexpr int B_BYTES = BN * kBK * 4;
  constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
  constexpr int RED_BYTES = WK * BM * BN * 4;  // epilogue reuse of the ring

  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = reinterpret_cast<uint8_t *>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  const GemmProblem &p = args.p;
  const int stages = args.stages;
  // barriers sit past both the ring and the epilogue's reduction buffer
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + max(stages * STAGE_BYTES, RED_BYTES));

  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const int split = args.split;
  const int rank = split > 1 ? static_cast<int>(cluster_ctarank()) : 0;
  const int64_t m0 = static_cast<int64_t>(blockIdx.x / split) * BM;
  const int n0 = blockIdx.y * BN;
  const int kbeg = rank * args.kc;
  const int kend = min(p.K, kbeg + args.kc);
  const int nk = kend > kbeg ? (kend - kbeg + kBK - 1) / kBK : 0;

  if (TMA && tid == 0) {
    for (int s = 0; s < stages; ++s) mbar_init(&full[s], 1);
    fence_mbar_init();
    prefetch_tmap(&tmA);
    prefetch_tmap(&tmB);
  }
  __syncthreads();

  // Stage `it` of this CTA's K range into ring slot it % stages.
  auto issue = [&](int it) {
    const int s = it % stages;
    const int k0 = kbeg + it * kBK;
    uint8_t *sa = smem + s * STAGE_BYTES;
    uint8_t *sb = sa + A_BYTES;
    if (TMA) {
      mbar_arrive_expect_tx(&full[s], STAGE_BYTES);
      if (AK)
        tma_load_2d(sa, &tmA, &full[s], k0, static_cast<int>(m0));
      else
        tma_load_2d(sa, &tmA, &full[s], static_cast<int>(m0), k0);
      if (BK_)
        tma_load_2d(sb, &tmB, &full[s], k0, n0);
      else
        tma_load_2d(sb, &tmB, &full[s], n0, k0);
    } else {
      const uint32_t ua = smem_u32(sa), ub = smem_u32(sb);
      for (int e = tid; e < BM * kBK; e += NT) {
        int m, k;
        uint32_t off;
        if (AK) {  // same 128-byte swizzle as the TMA path
          k = e % kBK;
          m = e / kBK;
          off = static_cast<uint32_t>(m * 128 + k * 4) ^ static_cast<uint32_t>((m & 7) << 4);
        } else {
          m = e % BM;
          k = e / BM;
          off = static_cast<uint32_t>((k * BM + m) * 4);
        }
        const int64_t gm = m0 + m;
        const int gk = k0 + k;
        const bool ok = gm < p.M && gk < kend;
        const float *src = ok ? p.A + gm * p.sam + static_cast<int64_t>(gk) * p.sak : p.A;
        cp_async4(ua + off, src, ok);
      }
      for (int e = tid; e < BN * kBK; e += NT) {
        int n, k;
        uint32_t off;
        if (BK_) {
          k = e % kBK;
          n = e / kBK;
          off = static_cast<uint32_t>((n * kBK + k) * 4);
        } else {
          n = e % BN;
          k = e / BN;
          off = static_cast<uint32_t>((k * BN + n) * 4);
        }
        const int gn = n0 + n;
        const int gk = k0 + k;
        const bool ok = gn < p.N && gk < kend;
        const float *src =
            ok ? p.B + static_cast<int64_t>(gk) * p.sbk + static_cast<int64_t>(gn) * p.sbn : p.B;
        cp_async4(ub + off, src, ok);
      }
    }
  };

  float acc[TM][TN];
#pragma unroll
  for (int i = 0; i < TM; ++i)
#pragma unroll
    for (int j = 0; j < TN; ++j) acc[i][j] = 0.0f;

  // prologue: stages-1 slabs in flight
  if (TMA) {
    if (tid == 0)
      for (int it = 0; it < stages - 1 && it < nk; ++it) issue(it);
  } else {
    for (int it = 0; it < stages - 1; ++it) {
      if (it < nk) issue(it);
      cp_async_commit();
    }
  }

  const int wk = warp % WK;
  const int wn = (warp / WK) % WN;
  const int wm = warp / (WK * WN);
  const int mrow = wm * 32 * TM;
  const int ncol = wn * TN;
  bool bad = false;
  for (int it = 0; it < nk; ++it) {
    const int s = it % stages;
    if (TMA) {
      // all threads finished slab it-1: its slot takes slab it+stages-1
      if (__syncthreads_or(bad)) break;
      if (tid == 0 && it + stages - 1 < nk) issue(it + stages - 1);
      bad = !mbar_wait(&full[s], (it / stages) & 1, args.err, kDevErrFullBarrier);
      if (bad) continue;
    } else {
      cp_async_wait_ring(stages);
      __syncthreads();
      if (it + stages - 1 < nk) issue(it + stages - 1);
      cp_async_commit();
    }
    const float *sa = reinterpret_cast<const float *>(smem + s * STAGE_BYTES);
    const float *sb = reinterpret_cast<const float *>(smem + s * STAGE_BYTES + A_BYTES);
#pragma unroll 2
    for (int k4 = 0; k4 < KW / 4; ++k4) {
      const int kb = wk * KW + k4 * 4;
      // A K-contiguous: one 16-byte read per row gives 4 k values
      float4 a4[AK ? TM : 1];
      if (AK) {
#pragma unroll
        for (int i = 0; i < TM; ++i) {
          const int m = mrow + lane + 32 * i;
          a4[i] = lds128(sa + m * kBK + (((kb >> 2) ^ (m & 7)) << 2));
        }
      }
#pragma unroll
      for (int kk = 0; kk < 4; ++kk) {
        float a[TM];
        if (AK) {
#pragma unroll
          for (int i = 0; i < TM; ++i)
            a[i] = kk == 0 ? a4[i].x : kk == 1 ? a4[i].y : kk == 2 ? a4[i].z : a4[i].w;
        } else {
#pragma unroll
          for (int j = 0; j < TM / 4; ++j) {
            const float4 v = lds128(sa + (kb + kk) * BM + mrow + 4 * lane + 128 * j);
            a[4 * j + 0] = v.x; a[4 * j + 1] = v.y; a[4 * j + 2] = v.z; a[4 * j + 3] = v.w;
          }
        }
        float b[TN];
        if (BK_) {
#pragma unroll
          for (int j = 0; j < TN; ++j) b[j] = sb[(ncol + j) * kBK + kb + kk];
        } else {
#pragma unroll
          for (int j = 0; j < TN / 4; ++j) {
            const float4 v = lds128(sb + (kb + kk) * BN + ncol + 4 * j);
            b[4 * j + 0] = v.x; b[4 * j + 1] = v.y; b[4 * j + 2] = v.z; b[4 * j + 3] = v.w;
          }
        }
#pragma unroll
        for (int i = 0; i < TM; ++i)
#pragma unroll
          for (int j = 0; j < TN; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
      }
    }
  }
  if (!TMA) asm volatile("cp.async.wait_all;" ::: "memory");

  // ---------------------------------------------------------- epilogue
  __syncthreads();  // every stage consumed: the ring can be reused
  float *red = reinterpret_cast<float *>(smem);  // [WK][BN][BM]
  {
    float *r = red + static_cast<size_t>(wk) * BM * BN;
#pragma unroll
    for (int j = 0; j < TN; ++j) {
      float *col = r + (wn * TN + j) * BM + wm * 32 * TM;
      if (AK) {
#pragma unroll
        for (int i = 0; i < TM; ++i) col[lane + 32 * i] = acc[i][j];
      } else {
#pragma unroll
        for (int q = 0; q < TM / 4; ++q)
          *reinterpret_cast<float4 *>(col + 4 * lane + 128 * q) =
              make_float4(acc[4 * q][j], acc[4 * q + 1][j], acc[4 * q + 2][j], acc[4 * q + 3][j]);
      }
    }
  }
  __syncthreads();
  constexpr int E = BM * BN;
  if (WK > 1) {
    for (int e = tid; e < E; e += NT) {
      float s = red[e];
#pragma unroll
      for (int w = 1; w < WK; ++w) s += red[w * E + e];
      red[e] = s;
    }
  }
  const bool c_ncontig = p.scn == 1 && p.scm != 1;
  if (split > 1) {
    cluster_sync();
    const int per = E / split;  // split divides E (E is a multiple of 1024)
    const uint32_t base = smem_u32(red);
    for (int e4 = tid * 4; e4 < per; e4 += NT * 4) {
      const int e = rank * per + e4;
      float4 s = make_float4(0.f, 0.f, 0.f, 0.f);
      for (int r = 0; r < split; ++r) {
        const float4 v = ld_dsmem4(mapa_shared(base + e * 4, r));
        s.x += v.x; s.y += v.y; s.z += v.z; s.w += v.w;
      }
      const float sv[4] = {s.x, s.y, s.z, s.w};
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int m = (e + q) % BM, n = (e + q) / BM;
        const int64_t gm = m0 + m;
        const int gn = n0 + n;
        if (gm < p.M && gn < p.N) {
          float *c = p.C + gm * p.scm + static_cast<int64_t>(gn) * p.scn;
          *c = axpby(p.alpha, sv[q], p.beta, c);
        }
      }
    }
    cluster_sync();
  } else {
    __syncthreads();
    if (c_ncontig) {
      // row-major C: walk n fastest so consecutive threads write adjacent
      // addresses (red is [n][m]; the strided smem read is the cheaper side)
      for (int e = tid; e < E; e += NT) {
        const int n = e % BN, m = e / BN;
        const int64_t gm = m0 + m;
        const int gn = n0 + n;
        if (gm < p.M && gn < p.N) {
          float *c = p.C + gm * p.scm + gn;
          *c = axpby(p.alpha, red[n * BM + m], p.beta, c);
        }
      }
    } else {
      for (int e = tid; e < E; e += NT) {
        const int m = e % BM, n = e / BM;
        const int64_t gm = m0 + m;
        const int gn = n0 + n;
        if (gm < p.M && gn < p.N) {
          float *c = p.C + gm * p.scm + static_cast<int64_t>(gn) * p.scn;
          *c = axpby(p.alpha, red[e], p.beta, c);
        }
      }
    }
  }
}

template <int TM, int TN, int WM, int WN, int WK, bool AK, bool BK_, bool TMA>
hml_status run_simt(const GemmProblem &p, const hml_sgemm_config &c, cudaStream_t s) {
  constexpr int BM = WM * 32 * TM, BN = WN * TN;
  constexpr int NT = 256;
  const int stages = c.stages;
  const size_t stage_bytes = static_cast<size_t>(BM + BN) * kBK * 4;
  const size_t red_bytes = static_cast<size_t>(WK) * BM * BN * 4;
  size_t smem = std::max(stage_bytes * stages, red_bytes);
  smem = ((smem + 15) & ~size_t(15)) + 2 * 8 * stages + 1024;  // barriers + alignment slack
  auto kern = simt_kernel<TM, TN, WM, WN, WK, AK, BK_, TMA>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem));
  if (e == cudaSuccess && c.split_k > 8)
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  if (e != cudaSuccess) {
    note_cuda_error(e, "simt attributes");
    return HML_STATUS_CUDA_ERROR;
  }
  CUtensorMap ta, tb;
  memset(&ta, 0, sizeof(ta));
  memset(&tb, 0, sizeof(tb));
  if (TMA) {
    bool ok;
    if (AK)
      ok = tensor_map_2d(&ta, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, p.A, p.K, p.M, p.sam * 4, kBK, BM,
                         CU_TENSOR_MAP_SWIZZLE_128B);
    else
      ok = tensor_map_2d(&ta, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, p.A, p.M, p.K, p.sak * 4, BM, kBK,
                         CU_TENSOR_MAP_SWIZZLE_NONE);
    if (ok) {
      if (BK_)
        ok = tensor_map_2d(&tb, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, p.B, p.K, p.N, p.sbn * 4, kBK, BN,
                           CU_TENSOR_MAP_SWIZZLE_NONE);
      else
        ok = tensor_map_2d(&tb, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, p.B, p.N, p.K, p.sbk * 4, BN, kBK,
                           CU_TENSOR_MAP_SWIZZLE_NONE);
    }
    if (!ok) return HML_STATUS_CUDA_ERROR;
  }
  SimtArgs args;
  args.p = p;
  args.split = c.split_k;
  const int ktiles = (p.K + kBK - 1) / kBK;
  args.kc = ((ktiles + c.split_k - 1) / c.split_k) * kBK;
  args.stages = stages;
  args.err = device_error_word();
  const int64_t tiles_m = (static_cast<int64_t>(p.M) + BM - 1) / BM;
  const int64_t tiles_n = (p.N + BN - 1) / BN;
  if (tiles_m * c.split_k > 0x7fffffff || tiles_n > 65535) return HML_STATUS_NOT_SUPPORTED;
  dim3 grid(static_cast<unsigned>(tiles_m * c.split_k), static_cast<unsigned>(tiles_n));
  e = launch_k(kern, grid, dim3(NT), smem, s, c.split_k, ta, tb, args);
  note_cuda_error(e, "simt launch");
  return cuda_status(e);
}

bool aligned16(const void *ptr) { return (reinterpret_cast<uintptr_t>(ptr) & 15u) == 0; }

bool tma_ok(const GemmProblem &p) {
  if (!aligned16(p.A) || !aligned16(p.B)) return false;
  const int64_t sa = p.a_kcontig() ? p.sam : p.sak;
  const int64_t sb = p.b_kcontig() ? p.sbn : p.sbk;
  if ((sa * 4) % 16 != 0 || (sb * 4) % 16 != 0) return false;
  if (sa * 4 >= (int64_t(1) << 40) || sb * 4 >= (int64_t(1) << 40)) return false;
  return true;
}

template <int V, bool AK, bool BK_, bool TMA>
hml_status run_v(const GemmProblem &p, const hml_sgemm_config &c, cudaStream_t s) {
  constexpr SimtShape sh = kSimtShapes[V];
  return run_simt<sh.tm, sh.tn, sh.wm, sh.wn, sh.wk, AK, BK_, TMA>(p, c, s);
}

template <int V>
hml_status run_layouts(const GemmProblem &p, const hml_sgemm_config &c, cudaStream_t s) {
  const bool ak = p.a_kcontig(), bk = p.b_kcontig(), tma = tma_ok(p);
  if (ak) {
    if (bk) return tma ? run_v<V, true, true, true>(p, c, s) : run_v<V, true, true, false>(p, c, s);
    return tma ? run_v<V, true, false, true>(p, c, s) : run_v<V, true, false, false>(p, c, s);
  }
  if (bk) return tma ? run_v<V, false, true, true>(p, c, s) : run_v<V, false, true, false>(p, c, s);
  return tma ? run_v<V, false, false, true>(p, c, s) : run_v<V, false, false, false>(p, c, s);
}

}  // namespace

hml_status check_simt(const GemmProblem &p, const hml_sgemm_config &c) {
  if (c.variant < 0 || c.variant >= kNumSimtShapes) return HML_STATUS_INVALID_VALUE;
  const SimtShape &sh = kSimtShapes[c.variant];
  if (c.tile_m != sh.bm() || c.tile_n != sh.bn()) return HML_STATUS_INVALID_VALUE;
  if (c.split_k < 1 || c.split_k > 16 || (c.split_k & (c.split_k - 1)) != 0)
    return HML_STATUS_INVALID_VALUE;
  if (c.stages < 2 || c.stages > 8) return HML_STATUS_INVALID_VALUE;
  const size_t stage_bytes = static_cast<size_t>(sh.bm() + sh.bn()) * kBK * 4;
  const size_t red_bytes = static_cast<size_t>(sh.wk) * sh.bm() * sh.bn() * 4;
  const size_t smem = std::max(stage_bytes * c.stages, red_bytes) + 2 * 8 * c.stages + 1024 + 16;
  if (smem > 227 * 1024) return HML_STATUS_INVALID_VALUE;
  if (p.a_kcontig() ? (p.sak != 1) : (p.sam != 1)) return HML_STATUS_NOT_SUPPORTED;
  if (p.b_kcontig() ? false : (p.sbn != 1)) return HML_STATUS_NOT_SUPPORTED;
  return HML_STATUS_SUCCESS;
}

hml_status launch_simt(const GemmProblem &p, const hml_sgemm_config &c, cudaStream_t s) {
  hml_status st = check_simt(p, c);
  if (st != HML_STATUS_SUCCESS) return st;
  switch (c.variant) {
    case 0: return run_layouts<0>(p, c, s);
    case 1: return run_layouts<1>(p, c, s);
    case 2: return run_layouts<2>(p, c, s);
    case 3: return run_layouts<3>(p, c, s);
    case 4: return run_layouts<4>(p, c, s);
    case 5: return run_layouts<5>(p, c, s);
    case 6: return run_layouts<6>(p, c, s);
    case 7: return run_layouts<7>(p, c, s);
    case 8: return run_layouts<8>(p, c, s);
    default: return HML_STATUS_INVALID_VALUE;
  }
}

// Shape table access for the configuration space.
int simt_num_shapes() { return kNumSimtShapes; }
void simt_shape(int v, int *bm, int *bn, int *wk) {
  *bm = kSimtShapes[v].bm();
  *bn = kSimtShapes[v].bn();
  *wk = kSimtShapes[v].wk;
}

}  // namespace hml
