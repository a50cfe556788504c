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
//     tile loads (cp.async.bulk.tensor into this CTA only) that complete on a
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
//     Micro-tiles of at most 64 accumulators are compiled for 128
//     registers a thread, so two CTAs share an SM and hide each other's
//     latencies; the 8 x 16 micro-tiles run one CTA an SM.
//   * epilogue: the WK partial tiles are summed in shared memory; with
//     split_k > 1 the CTAs of one thread-block cluster each own a K range
//     and the cluster sums their tiles through distributed shared memory in
//     rank order.  No global workspace, deterministic results.  beta == 0
//     does not read C.
#include <algorithm>
#include <cstring>

#include "hml_device.cuh"
#include "hml_internal.h"
#include "simt_tile.cuh"

namespace hml {
namespace {

struct SimtArgs {
  GemmProblem p;
  int split;      // CTAs per cluster along K
  int kc;         // K extent per split (multiple of kBK)
  int stages;
  int *err;
};

template <int TM, int TN, int WM, int WN, int WK, bool AK, bool BK_, bool TMA>
__global__ void __launch_bounds__(256, TMA && TM * TN <= 64 ? 2 : 1)  // see simt_ctas_per_sm
    simt_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                SimtArgs args) {
  using T = SimtTile<TM, TN, WM, WN, WK, AK, BK_>;
  constexpr int BM = T::BM, BN = T::BN, NT = T::NT;
  constexpr int A_BYTES = T::A_BYTES, STAGE_BYTES = T::STAGE_BYTES;

  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = align_shared(smem_raw, 1024);
  const GemmProblem &p = args.p;
  const int stages = args.stages;
  // barriers sit past both the ring and the epilogue's reduction buffer
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + max(stages * STAGE_BYTES, T::RED_BYTES));

  const int tid = threadIdx.x;
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
        const int m = AK ? e / kBK : e % BM;
        const int k = AK ? e % kBK : e / BM;
        const int64_t gm = m0 + m;
        const int gk = k0 + k;
        const bool ok = gm < p.M && gk < kend;
        const float *src = ok ? p.A + gm * p.sam + static_cast<int64_t>(gk) * p.sak : p.A;
        cp_async4(ua + T::a_off(m, k), src, ok);
      }
      for (int e = tid; e < BN * kBK; e += NT) {
        const int n = BK_ ? e / kBK : e % BN;
        const int k = BK_ ? e % kBK : e / BN;
        const int gn = n0 + n;
        const int gk = k0 + k;
        const bool ok = gn < p.N && gk < kend;
        const float *src =
            ok ? p.B + static_cast<int64_t>(gk) * p.sbk + static_cast<int64_t>(gn) * p.sbn : p.B;
        cp_async4(ub + T::b_off(n, k), src, ok);
      }
    }
  };

  float acc[TM][TN];
  T::zero(acc);

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

  const typename T::Coord co = T::coord(tid);
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
    T::slab(reinterpret_cast<const float *>(smem + s * STAGE_BYTES),
            reinterpret_cast<const float *>(smem + s * STAGE_BYTES + A_BYTES), acc, co);
  }
  if (!TMA) asm volatile("cp.async.wait_all;" ::: "memory");

  // ---------------------------------------------------------- epilogue
  __syncthreads();  // every stage consumed: the ring can be reused
  float *red = reinterpret_cast<float *>(smem);  // [WK][BN][BM]
  T::stash(red, acc, co);
  __syncthreads();
  T::reduce_wk(red, tid);
  constexpr int E = BM * BN;
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
    T::store_c(red, tid, m0, n0, p.M, p.N, p.C, p.scm, p.scn, p.alpha, p.beta);
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
  if (c.variant >= kNumSimtShapes && c.variant < kNumSimtShapes + stream_num_variants()) {
    if (c.tile_n != stream_tile_n(c.variant - kNumSimtShapes)) return HML_STATUS_INVALID_VALUE;
    return check_stream(p, c);
  }
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
  if (c.variant >= kNumSimtShapes) return launch_stream(p, c, s);
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
// CTAs of shape v one SM holds: two where the micro-tile has at most 64
// accumulators (the TMA instances are compiled for 128 registers a thread),
// given shared memory for both rings.
int simt_ctas_per_sm(int v) { return kSimtShapes[v].tm * kSimtShapes[v].tn <= 64 ? 2 : 1; }

}  // namespace hml
