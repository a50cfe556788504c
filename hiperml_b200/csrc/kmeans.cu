// kmeans.cu -- the k-means assignment step as a consumer of the skinny SGEMM.
//
// HiperML's assignment kernel (hmlKmeansAssignCtrdSmem,
// include/hml_kmeans_kernel_template.h:19-90) gives each point the index of
// its nearest centroid: dist_k = sum_d (x_d - c_kd)^2 accumulated in FP32 in
// dimension order (nvcc contracts `dist += delta * delta` into one fused
// multiply-add per dimension), the first k with the smallest dist winning
// (strict `<` from FLT_MAX).  Points are row-major [points][dims], centroids
// row-major [clusters][dims].
//
// Here the work goes through the tensor-core SGEMM: with ||x||^2 constant per
// point, argmin_k dist_k = argmin_k (||c_k||^2 - 2 x . c_k), and the dot
// products of every point with every centroid are one skinny GEMM
// S = X C^T (points x clusters), run by the library's FP32-accurate
// configuration (BF16X6 or SIMT; never the fast BF16X3 mode).  A second
// kernel reads S and picks the argmin.  Since S carries rounding errors that
// the reference's direct sums do not, the pick is made exact: with
// g_k = ||c_k||^2 - 2 S_k, every centroid whose g_k lies within a bound of
// the smallest (16 gamma_{dims+4} (||x||^2 + max_k ||c_k||^2), more than
// twice the sum of the worst-case errors of g and of the reference's dist)
// is a candidate, the reference's choice is always among them, and when
// there is more than one the kernel recomputes dist for the candidates with
// the reference's own arithmetic, in increasing k with strict `<`.  So every
// point gets the reference kernel's index, exact ties included.
#include <cfloat>

#include "hml_device.cuh"
#include "hml_internal.h"
#include "hml_select.h"
#include "hml_tune.h"

namespace hml {
namespace {

constexpr int kNormWarps = 8;

// ||c_k||^2 for every centroid, one warp per centroid (FP32; used only to
// screen candidates).
__global__ void centroid_norms_kernel(const float *cent, int k, int d, float *cnorm) {
  const int lane = threadIdx.x & 31;
  for (int c = blockIdx.x * kNormWarps + (threadIdx.x >> 5); c < k; c += gridDim.x * kNormWarps) {
    const float *row = cent + static_cast<int64_t>(c) * d;
    float s = 0.0f;
    for (int j = lane; j < d; j += 32) s = fmaf(row[j], row[j], s);
    cnorm[c] = warp_sum(s);
  }
}

// The reference's distance of point x to centroid c (the fused form nvcc
// gives `dist += delta * delta`).
__device__ __forceinline__ float ref_dist(const float *x, const float *c, int d) {
  float dist = 0.0f;
  for (int j = 0; j < d; ++j) {
    const float delta = __fsub_rn(x[j], c[j]);
    dist = __fmaf_rn(delta, delta, dist);
  }
  return dist;
}

// One thread per point: g_k = ||c_k||^2 - 2 S(p, k) (S column-major, ld lds),
// the candidates within `margin` of the smallest, and, when there is more
// than one, the reference's own pick among them.  `exact` counts the points
// that needed it.
__global__ void kmeans_pick_kernel(const float *points, int64_t np, int d, const float *cent,
                                   int k, const float *S, int64_t lds, const float *cnorm,
                                   uint32_t *out, unsigned *exact) {
  extern __shared__ float s_cnorm[];  // [k], then the block's max
  float cmax = 0.0f;
  for (int c = threadIdx.x; c < k; c += blockDim.x) {
    const float v = cnorm[c];
    s_cnorm[c] = v;
    cmax = fmaxf(cmax, v);
  }
  cmax = fmaxf(cmax, __shfl_xor_sync(0xffffffffu, cmax, 16));
  cmax = fmaxf(cmax, __shfl_xor_sync(0xffffffffu, cmax, 8));
  cmax = fmaxf(cmax, __shfl_xor_sync(0xffffffffu, cmax, 4));
  cmax = fmaxf(cmax, __shfl_xor_sync(0xffffffffu, cmax, 2));
  cmax = fmaxf(cmax, __shfl_xor_sync(0xffffffffu, cmax, 1));
  __shared__ float s_wmax[32];
  if ((threadIdx.x & 31) == 0) s_wmax[threadIdx.x >> 5] = cmax;
  __syncthreads();
  cmax = 0.0f;
  for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) cmax = fmaxf(cmax, s_wmax[w]);
  // 16 gamma_{d+4}, rounded up (gamma_n = n u / (1 - n u), u = 2^-24)
  const double nu = (d + 4) * 0x1p-24;
  const float bound = static_cast<float>(16.0 * nu / (1.0 - nu) * 1.001);
  unsigned my_exact = 0;
  for (int64_t p = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; p < np;
       p += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const float *x = points + p * d;
    float xn = 0.0f;
    for (int j = 0; j < d; ++j) xn = fmaf(x[j], x[j], xn);
    const float *sp = S + p;
    float gmin = INFINITY;
    int kmin = 0;
    for (int c = 0; c < k; ++c) {
      const float g = fmaf(-2.0f, sp[c * lds], s_cnorm[c]);
      if (g < gmin) {
        gmin = g;
        kmin = c;
      }
    }
    const float lim = gmin + bound * (xn + cmax) + 1e-37f;
    int cand = 0;
    for (int c = 0; c < k; ++c) cand += fmaf(-2.0f, sp[c * lds], s_cnorm[c]) <= lim;
    uint32_t pick = static_cast<uint32_t>(kmin);
    if (cand != 1) {
      // the reference's arithmetic over the candidates, in increasing k
      ++my_exact;
      float best = FLT_MAX;
      pick = 0;
      for (int c = 0; c < k; ++c) {
        if (!(fmaf(-2.0f, sp[c * lds], s_cnorm[c]) <= lim)) continue;
        const float dist = ref_dist(x, cent + static_cast<int64_t>(c) * d, d);
        if (dist < best) {
          best = dist;
          pick = static_cast<uint32_t>(c);
        }
      }
    }
    out[p] = pick;
  }
  if (exact && my_exact) atomicAdd(exact, my_exact);
}

// The fused form for dims <= 64: one thread per point, the point in
// registers (DP >= dims values, zero padded), the centroids streamed through
// shared memory KC at a time (all lanes read the same centroid: broadcasts),
// the dot products x . c_k as an FP32 fused multiply-add chain, and the
// argmin in registers: the smallest g_k = ||c_k||^2 - 2 x.c_k, its index and
// the second smallest.  A point whose second smallest lies within the bound
// of the smallest goes through a second pass over the centroids that
// compares the candidates with the reference's own distance.  The products
// never leave the SM.
constexpr int kFusedThreads = 256;
constexpr int kFusedKC = 64;  // centroids per shared-memory stage

template <int DP>
__global__ void __launch_bounds__(kFusedThreads) kmeans_fused_kernel(
    const float *points, int64_t np, int d, const float *cent, int k, const float *cnorm,
    uint32_t *out, unsigned *exact) {
  __shared__ float s_c[kFusedKC][DP];
  __shared__ float s_n[kFusedKC];
  __shared__ float s_wmax[kFusedThreads / 32];
  // max_k ||c_k||^2 over all centroids (for the bound)
  float cmax = 0.0f;
  for (int c = threadIdx.x; c < k; c += kFusedThreads) cmax = fmaxf(cmax, cnorm[c]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) cmax = fmaxf(cmax, __shfl_xor_sync(0xffffffffu, cmax, o));
  if ((threadIdx.x & 31) == 0) s_wmax[threadIdx.x >> 5] = cmax;
  __syncthreads();
  cmax = 0.0f;
#pragma unroll
  for (int w = 0; w < kFusedThreads / 32; ++w) cmax = fmaxf(cmax, s_wmax[w]);
  const double nu = (d + 4) * 0x1p-24;
  const float bound = static_cast<float>(16.0 * nu / (1.0 - nu) * 1.001);

  const int64_t p = blockIdx.x * static_cast<int64_t>(kFusedThreads) + threadIdx.x;
  const bool live = p < np;
  float x[DP];
#pragma unroll
  for (int j = 0; j < DP; ++j) x[j] = (live && j < d) ? points[p * d + j] : 0.0f;
  float xn = 0.0f;
#pragma unroll
  for (int j = 0; j < DP; ++j) xn = fmaf(x[j], x[j], xn);
  float g1 = INFINITY, g2 = INFINITY;
  int k1 = 0;
  for (int c0 = 0; c0 < k; c0 += kFusedKC) {
    const int kc = min(kFusedKC, k - c0);
    __syncthreads();
    for (int e = threadIdx.x; e < kc * DP; e += kFusedThreads) {
      const int c = e / DP, j = e % DP;
      s_c[c][j] = j < d ? cent[static_cast<int64_t>(c0 + c) * d + j] : 0.0f;
    }
    for (int c = threadIdx.x; c < kc; c += kFusedThreads) s_n[c] = cnorm[c0 + c];
    __syncthreads();
    for (int c = 0; c < kc; ++c) {
      float dot = 0.0f;
#pragma unroll
      for (int j = 0; j < DP; ++j) dot = fmaf(x[j], s_c[c][j], dot);
      const float g = fmaf(-2.0f, dot, s_n[c]);
      if (g < g1) {
        g2 = g1;
        g1 = g;
        k1 = c0 + c;
      } else if (g < g2) {
        g2 = g;
      }
    }
  }
  if (!live) return;
  const float lim = g1 + bound * (xn + cmax) + 1e-37f;
  uint32_t pick = static_cast<uint32_t>(k1);
  if (!(g2 > lim)) {
    // close call (or non-finite values): the candidates, in increasing k,
    // with the reference's own arithmetic; their g_k is recomputed exactly
    // as above
    if (exact) atomicAdd(exact, 1u);
    const float *xp = points + p * d;
    float best = FLT_MAX;
    pick = 0;
    for (int c = 0; c < k; ++c) {
      const float *cp = cent + static_cast<int64_t>(c) * d;
      float dot = 0.0f;
#pragma unroll
      for (int j = 0; j < DP; ++j) dot = fmaf(x[j], j < d ? cp[j] : 0.0f, dot);
      if (!(fmaf(-2.0f, dot, cnorm[c]) <= lim)) continue;
      const float dist = ref_dist(xp, cp, d);
      if (dist < best) {
        best = dist;
        pick = static_cast<uint32_t>(c);
      }
    }
  }
  out[p] = pick;
}

template <int DP>
hml_status launch_fused(const float *points, int np, int d, const float *cent, int k,
                        const float *cnorm, uint32_t *out, unsigned *exact, cudaStream_t s) {
  const int64_t blocks = (static_cast<int64_t>(np) + kFusedThreads - 1) / kFusedThreads;
  if (blocks > 0x7fffffff) return HML_STATUS_NOT_SUPPORTED;
  count_launch();
  kmeans_fused_kernel<DP><<<static_cast<unsigned>(blocks), kFusedThreads, 0, s>>>(
      points, np, d, cent, k, cnorm, out, exact);
  cudaError_t e = cudaGetLastError();
  note_cuda_error(e, "kmeans fused");
  return cuda_status(e);
}

}  // namespace

hml_status kmeans_assign(const float *points, int np, int d, const float *cent, int k,
                         uint32_t *out, unsigned *exact, cudaStream_t s) {
  if (np < 0 || d < 0 || k < 1) return HML_STATUS_INVALID_VALUE;
  if (np == 0) return HML_STATUS_SUCCESS;
  if (!out || (d > 0 && (!points || !cent))) return HML_STATUS_INVALID_VALUE;
  if (d <= 64) {
    // the fused SIMT form: ||c_k||^2 first (a small workspace), then one pass
    void *ws = nullptr;
    hml_status st = workspace_slot(1, static_cast<size_t>(k) * sizeof(float), s, &ws);
    if (st != HML_STATUS_SUCCESS) return st;
    float *cnorm = static_cast<float *>(ws);
    count_launch();
    const int nb = std::min((k + kNormWarps - 1) / kNormWarps, 4 * sm_count());
    centroid_norms_kernel<<<std::max(1, nb), 32 * kNormWarps, 0, s>>>(cent, k, d, cnorm);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
      note_cuda_error(e, "kmeans norms");
      return HML_STATUS_CUDA_ERROR;
    }
    if (d <= 8) return launch_fused<8>(points, np, d, cent, k, cnorm, out, exact, s);
    if (d <= 16) return launch_fused<16>(points, np, d, cent, k, cnorm, out, exact, s);
    if (d <= 32) return launch_fused<32>(points, np, d, cent, k, cnorm, out, exact, s);
    return launch_fused<64>(points, np, d, cent, k, cnorm, out, exact, s);
  }
  if (np < 0 || d < 0 || k < 1) return HML_STATUS_INVALID_VALUE;
  if (np == 0) return HML_STATUS_SUCCESS;
  if (!out || (d > 0 && (!points || !cent))) return HML_STATUS_INVALID_VALUE;
  const size_t s_bytes = static_cast<size_t>(np) * k * sizeof(float);
  const size_t n_off = (s_bytes + 255) & ~static_cast<size_t>(255);
  void *ws = nullptr;
  hml_status st = workspace_slot(1, n_off + static_cast<size_t>(k) * sizeof(float), s, &ws);
  if (st != HML_STATUS_SUCCESS) return st;
  float *S = static_cast<float *>(ws);
  float *cnorm = reinterpret_cast<float *>(static_cast<uint8_t *>(ws) + n_off);
  // S (points x clusters, column-major) = X C^T: X is the row-major points
  // (column-major d x np, transposed), C^T the row-major centroids
  // (column-major d x k)
  if (d > 0) {
    GemmProblem p;
    st = gemm_from_blas(HML_COL_MAJOR, HML_OP_T, HML_OP_N, np, k, d, 1.0f, points, d, cent, d,
                        0.0f, S, np, &p);
    if (st != HML_STATUS_SUCCESS) return st;
    GemvProblem g;
    if (as_gemv(p, &g)) {
      st = launch_gemv(g, kGemvTuned, s);
    } else {
      hml_sgemm_config c;
      st = select_config(p, &c, s);
      // the candidate bound assumes FP32-level dot products
      if (st == HML_STATUS_SUCCESS && c.algo == HML_ALGO_BF16X3) {
        c = heuristic_config(p, HML_ALGO_BF16X6);
        if (!check_config_ok(p, c)) c = heuristic_config(p, HML_ALGO_SIMT);
      }
      if (st == HML_STATUS_SUCCESS) st = run_config(p, c, s);
    }
    if (st != HML_STATUS_SUCCESS) return st;
  } else {
    cudaError_t e = cudaMemsetAsync(S, 0, s_bytes, s);
    if (e != cudaSuccess) {
      note_cuda_error(e, "kmeans: zero products");
      return HML_STATUS_CUDA_ERROR;
    }
  }
  count_launch(2);
  const int nblocks = std::min((k + kNormWarps - 1) / kNormWarps, 4 * sm_count());
  centroid_norms_kernel<<<std::max(1, nblocks), 32 * kNormWarps, 0, s>>>(cent, k, d, cnorm);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) {
    const size_t smem = static_cast<size_t>(k) * sizeof(float);
    if (smem > 48 * 1024) {
      e = cudaFuncSetAttribute(kmeans_pick_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(smem));
    }
    if (e == cudaSuccess) {
      const int64_t blocks = std::min<int64_t>((np + 255) / 256, 8LL * sm_count());
      kmeans_pick_kernel<<<static_cast<unsigned>(blocks), 256, smem, s>>>(
          points, np, d, cent, k, S, np, cnorm, out, exact);
      e = cudaGetLastError();
    }
  }
  note_cuda_error(e, "kmeans assign");
  return cuda_status(e);
}

}  // namespace hml

extern "C" hml_status hml_kmeans_assign(const float *points, int num_points, int dims,
                                        const float *centroids, int num_clusters,
                                        uint32_t *assignments, void *stream) {
  return hml::kmeans_assign(points, num_points, dims, centroids, num_clusters, assignments,
                            nullptr, static_cast<cudaStream_t>(stream));
}

extern "C" hml_status hml_kmeans_assign_stats(const float *points, int num_points, int dims,
                                              const float *centroids, int num_clusters,
                                              uint32_t *assignments, unsigned *exact_count,
                                              void *stream) {
  return hml::kmeans_assign(points, num_points, dims, centroids, num_clusters, assignments,
                            exact_count, static_cast<cudaStream_t>(stream));
}
