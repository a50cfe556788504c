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
// Here, with ||x||^2 constant per point, argmin_k dist_k = argmin_k
// (||c_k||^2 - 2 x . c_k), and the dot products of every point with every
// centroid are one skinny GEMM S = X C^T (points x clusters), in one of two
// forms: the tiled form (method 1, up to 256 dimensions by default) runs the
// GEMM as a register-tiled FP32 SIMT kernel with the argmin in its epilogue,
// the products never leaving the SM; the GEMM form (method 2, wider points)
// runs it through the library's SGEMM in an FP32-accurate configuration
// (BF16X6 or SIMT; never the fast BF16X3 mode), S in HBM, and a second
// kernel picks the argmin.  Since the products carry rounding errors that the
// reference's direct sums do not, the pick is made exact: with g_k =
// ||c_k||^2 - 2 S_k, every centroid whose g_k lies within a bound of the
// smallest (16 gamma_{dims+4} (||x||^2 + max_k ||c_k||^2), more than twice
// the sum of the worst-case errors of g and of the reference's dist) is a
// candidate, the reference's choice is always among them, and when there is
// more than one the kernel recomputes dist for the candidates with the
// reference's own arithmetic, in increasing k with strict `<`.  So every
// point gets the reference kernel's index, exact ties included.
#include <cfloat>

#include "hml_device.cuh"
#include "hml_internal.h"
#include "hml_select.h"
#include "hml_tune.h"

namespace hml {
namespace {

constexpr int kNormWarps = 8;
// Widest points the automatic choice gives the tiled form (method 1); wider
// ones go through the SGEMM (method 2).
constexpr int kKmeansTiledMaxDims = 256;

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

// The reference's pick for point x among the candidates -- the centroids
// whose g_k, recomputed, is at most lim -- by the G lanes of a group (lanes
// `gmask`, this one lane r of G): lane r takes centroids r, r + G, ...,
// keeping the first smallest dist below FLT_MAX (strict <, increasing k),
// and the group keeps the smallest dist, the lowest k among equal ones: the
// first minimum in k order, which is the reference's pick.  0 when no
// candidate's dist is below FLT_MAX (the reference leaves that case unset).
template <int G>
__device__ __noinline__ uint32_t exact_pick(const float *x, int d, const float *cent, int k,
                                            const float *cnorm, float lim, unsigned gmask,
                                            int r) {
  float bd = FLT_MAX;
  int bk = -1;
  for (int c = r; c < k; c += G) {
    const float *cp = cent + static_cast<int64_t>(c) * d;
    float dot = 0.0f;
    for (int j = 0; j < d; ++j) dot = fmaf(x[j], cp[j], dot);
    if (!(fmaf(-2.0f, dot, cnorm[c]) <= lim)) continue;
    const float dist = ref_dist(x, cp, d);
    if (dist < bd) {
      bd = dist;
      bk = c;
    }
  }
#pragma unroll
  for (int o = 1; o < G; o <<= 1) {
    const float od = __shfl_xor_sync(gmask, bd, o);
    const int ok = __shfl_xor_sync(gmask, bk, o);
    if (ok >= 0 && (bk < 0 || od < bd || (od == bd && ok < bk))) {
      bd = od;
      bk = ok;
    }
  }
  return bk < 0 ? 0u : static_cast<uint32_t>(bk);
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
  const int lane = threadIdx.x & 31;
  // the warp walks 32 consecutive points at a time (every lane takes every
  // step, so the warp can settle its close calls together)
  const int64_t wstride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t p0 = blockIdx.x * static_cast<int64_t>(blockDim.x) + (threadIdx.x & ~31); p0 < np;
       p0 += wstride) {
    const int64_t p = p0 + lane;
    const bool live = p < np;
    float lim = 0.0f;
    bool close = false;
    if (live) {
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
      lim = gmin + bound * (xn + cmax) + 1e-37f;
      int cand = 0;
      for (int c = 0; c < k; ++c) cand += fmaf(-2.0f, sp[c * lds], s_cnorm[c]) <= lim;
      close = cand != 1;
      if (!close) out[p] = static_cast<uint32_t>(kmin);
    }
    // close calls (or non-finite values): the warp settles each with the
    // reference's own arithmetic over the candidates
    unsigned todo = __ballot_sync(0xffffffffu, close);
    my_exact += __popc(todo) * (lane == 0);
    while (todo) {
      const int src = __ffs(todo) - 1;
      todo &= todo - 1;
      const int64_t q = p0 + src;
      const float ql = __shfl_sync(0xffffffffu, lim, src);
      const uint32_t pick = exact_pick<32>(points + q * d, d, cent, k, cnorm, ql, 0xffffffffu,
                                           lane);
      if (lane == 0) out[q] = pick;
    }
  }
  if (exact && my_exact) atomicAdd(exact, my_exact);
}

// The tiled form: the dot products of 128 points with 64 centroids at a
// time as a register-tiled FP32 SIMT GEMM with the argmin in its epilogue.
// A block of 256 threads takes 128 points; thread (tx, ty) of the 16 x 16
// grid owns points ty*4 .. ty*4+3 and 64+ty*4 .. 64+ty*4+3 and centroids
// tx*4 .. tx*4+3 of each 64-centroid pass.  Points and centroids are staged
// dimension-major in shared memory, 32 dimensions at a time (read from HBM
// with whole-row, coalesced loads), so each dimension step is three 16-byte
// shared-memory loads feeding 32 fused multiply-adds.  After a pass, g_k =
// ||c_k||^2 - 2 x.c_k updates the thread's smallest g, its index and the
// second smallest for each of its 8 points, in increasing k; at the end the
// 16 threads that share a point merge theirs (the smaller g, the lower index
// on equal g) with shuffles.  A point whose second smallest lies within the
// bound of the smallest is settled as in the GEMM form, by the reference's
// own distance over the candidates.  The products never leave the SM.
constexpr int kTP = 128;         // points per block
constexpr int kTC = 64;          // centroids per pass
constexpr int kTD = 32;          // dimensions per shared-memory stage
constexpr int kTThreads = 256;
constexpr int kXS = kTP + 4;     // row stride of the staged points (a 16-byte multiple)
constexpr int kCS = kTC + 4;     // row stride of the staged centroids

// Smallest g, its centroid and the second smallest g seen (values of g that
// compare false, i.e. NaN, are never taken).
struct Best {
  float g1;
  int k1;
  float g2;
};

__device__ __forceinline__ void best_add(Best &b, float g, int k) {
  if (g < b.g1) {
    b.g2 = b.g1;
    b.g1 = g;
    b.k1 = k;
  } else if (g < b.g2) {
    b.g2 = g;
  }
}

// Union of two disjoint centroid sets' states: (g1, k1) ordered by g, then
// k, so the merge is commutative and associative and keeps the first index.
__device__ __forceinline__ Best best_merge(const Best &a, const Best &b) {
  if (b.g1 < a.g1 || (b.g1 == a.g1 && b.k1 < a.k1)) return {b.g1, b.k1, fminf(b.g2, a.g1)};
  return {a.g1, a.k1, fminf(a.g2, b.g1)};
}

__global__ void __launch_bounds__(kTThreads, 2) kmeans_tile_kernel(
    const float *__restrict__ points, int np, int d, const float *__restrict__ cent, int k,
    const float *__restrict__ cnorm, uint32_t *__restrict__ out, unsigned *exact) {
  __shared__ __align__(16) float xs[kTD][kXS];
  __shared__ __align__(16) float cs[kTD][kCS];
  __shared__ float s_cn[kTC];
  __shared__ float s_xn[kTP];
  __shared__ float s_wmax[kTThreads / 32];
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int64_t p0 = static_cast<int64_t>(blockIdx.x) * kTP;
  const int nb = static_cast<int>(min(static_cast<int64_t>(kTP), np - p0));

  // max_k ||c_k||^2 (for the bound)
  float cmax = 0.0f;
  for (int c = tid; c < k; c += kTThreads) cmax = fmaxf(cmax, cnorm[c]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) cmax = fmaxf(cmax, __shfl_xor_sync(0xffffffffu, cmax, o));
  if ((tid & 31) == 0) s_wmax[tid >> 5] = cmax;

  Best best[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) best[i] = {INFINITY, 0, INFINITY};
  float xn = 0.0f;  // thread t < 128: ||x||^2 of point t, from the staged values
  const int dchunks = (d + kTD - 1) / kTD;
  const bool x_once = dchunks <= 1;

  // stage dimensions [d0, d0 + kTD) of the block's points, zero padded
  auto stage_points = [&](int d0, bool norms) {
    const int dn = min(kTD, d - d0);
    for (int e = tid; e < kTP * kTD; e += kTThreads) {
      const int pt = e / kTD, j = e % kTD;
      xs[j][pt] = (pt < nb && j < dn) ? points[(p0 + pt) * d + d0 + j] : 0.0f;
    }
    __syncthreads();
    if (norms && tid < kTP)
      for (int j = 0; j < dn; ++j) xn = fmaf(xs[j][tid], xs[j][tid], xn);
  };
  if (x_once && d > 0) stage_points(0, true);

  for (int c0 = 0; c0 < k; c0 += kTC) {
    __syncthreads();  // the previous pass is done with s_cn and the stages
    // ||c||^2 of the pass's centroids; NaN past the last (never taken)
    if (tid < kTC) s_cn[tid] = c0 + tid < k ? cnorm[c0 + tid] : __int_as_float(0x7fc00000);
    float acc[8][4];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[i][q] = 0.0f;
    for (int dc = 0; dc < dchunks; ++dc) {
      const int d0 = dc * kTD, dn = min(kTD, d - d0);
      if (dc > 0) __syncthreads();  // the previous stage's readers are done
      if (!x_once) stage_points(d0, c0 == 0);
      for (int e = tid; e < kTC * kTD; e += kTThreads) {
        const int c = e / kTD, j = e % kTD;
        cs[j][c] = (c0 + c < k && j < dn) ? cent[static_cast<int64_t>(c0 + c) * d + d0 + j] : 0.0f;
      }
      __syncthreads();
      const int jn = (dn + 3) & ~3;  // zero padded up to a multiple of 4
      for (int j0 = 0; j0 < jn; j0 += 4) {
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
          const int j = j0 + jj;
          const float4 xa = *reinterpret_cast<const float4 *>(&xs[j][ty * 4]);
          const float4 xb = *reinterpret_cast<const float4 *>(&xs[j][64 + ty * 4]);
          const float4 cv = *reinterpret_cast<const float4 *>(&cs[j][tx * 4]);
          const float xv[8] = {xa.x, xa.y, xa.z, xa.w, xb.x, xb.y, xb.z, xb.w};
          const float cw[4] = {cv.x, cv.y, cv.z, cv.w};
#pragma unroll
          for (int i = 0; i < 8; ++i)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[i][q] = fmaf(xv[i], cw[q], acc[i][q]);
        }
      }
    }
    if (dchunks == 0) __syncthreads();  // s_cn, written above, had no barrier after it
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int c = tx * 4 + q;
      const float cn = s_cn[c];
#pragma unroll
      for (int i = 0; i < 8; ++i) best_add(best[i], fmaf(-2.0f, acc[i][q], cn), c0 + c);
    }
  }
  if (tid < kTP) s_xn[tid] = xn;
  __syncthreads();
  cmax = 0.0f;
#pragma unroll
  for (int w = 0; w < kTThreads / 32; ++w) cmax = fmaxf(cmax, s_wmax[w]);
  const double nu = (d + 4) * 0x1p-24;
  const float bound = static_cast<float>(16.0 * nu / (1.0 - nu) * 1.001);

  // merge over the 16 threads of each point group (lanes of one half-warp)
#pragma unroll
  for (int i = 0; i < 8; ++i) {
#pragma unroll
    for (int o = 1; o < 16; o <<= 1) {
      const Best other = {__shfl_xor_sync(0xffffffffu, best[i].g1, o),
                          __shfl_xor_sync(0xffffffffu, best[i].k1, o),
                          __shfl_xor_sync(0xffffffffu, best[i].g2, o)};
      best[i] = best_merge(best[i], other);
    }
  }
  // the group's 8 points: a settled one is written by lane tx == i; a close
  // call (or non-finite values) is settled by the 16 lanes together with the
  // reference's own arithmetic over the candidates
  const unsigned hmask = 0xFFFFu << (threadIdx.x & 16);
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int pt = i < 4 ? ty * 4 + i : 64 + ty * 4 + (i - 4);
    if (pt >= nb) continue;  // the same for the whole half-warp
    const int64_t p = p0 + pt;
    const float lim = best[i].g1 + bound * (s_xn[pt] + cmax) + 1e-37f;
    if (best[i].g2 > lim) {
      if (tx == i) out[p] = static_cast<uint32_t>(best[i].k1);
      continue;
    }
    if (tx == 0 && exact) atomicAdd(exact, 1u);
    const uint32_t pick = exact_pick<16>(points + p * d, d, cent, k, cnorm, lim, hmask, tx);
    if (tx == 0) out[p] = pick;
  }
}

hml_status launch_norms(const float *cent, int k, int d, float *cnorm, cudaStream_t s) {
  count_launch();
  const int nb = std::min((k + kNormWarps - 1) / kNormWarps, 4 * sm_count());
  centroid_norms_kernel<<<std::max(1, nb), 32 * kNormWarps, 0, s>>>(cent, k, d, cnorm);
  cudaError_t e = cudaGetLastError();
  note_cuda_error(e, "kmeans norms");
  return cuda_status(e);
}

// The tiled SIMT form (method 1).
hml_status assign_tiled(const float *points, int np, int d, const float *cent, int k,
                        uint32_t *out, unsigned *exact, cudaStream_t s) {
  void *ws = nullptr;
  hml_status st = workspace_slot(1, static_cast<size_t>(k) * sizeof(float), s, &ws);
  if (st != HML_STATUS_SUCCESS) return st;
  float *cnorm = static_cast<float *>(ws);
  st = launch_norms(cent, k, d, cnorm, s);
  if (st != HML_STATUS_SUCCESS) return st;
  const int64_t blocks = (static_cast<int64_t>(np) + kTP - 1) / kTP;
  count_launch();
  kmeans_tile_kernel<<<static_cast<unsigned>(blocks), kTThreads, 0, s>>>(points, np, d, cent, k,
                                                                        cnorm, out, exact);
  cudaError_t e = cudaGetLastError();
  note_cuda_error(e, "kmeans tiled");
  return cuda_status(e);
}

// The GEMM form (method 2): S = X C^T through the library's SGEMM, then the
// pick kernel.
hml_status assign_gemm(const float *points, int np, int d, const float *cent, int k,
                       uint32_t *out, unsigned *exact, cudaStream_t s) {
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
  st = launch_norms(cent, k, d, cnorm, s);
  if (st != HML_STATUS_SUCCESS) return st;
  count_launch();
  cudaError_t e = cudaSuccess;
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
  note_cuda_error(e, "kmeans assign");
  return cuda_status(e);
}

}  // namespace

hml_status kmeans_assign(const float *points, int np, int d, const float *cent, int k,
                         uint32_t *out, int method, unsigned *exact, cudaStream_t s) {
  if (np < 0 || d < 0 || k < 1 || method < 0 || method > 2) return HML_STATUS_INVALID_VALUE;
  if (np == 0) return HML_STATUS_SUCCESS;
  if (!out || (d > 0 && (!points || !cent))) return HML_STATUS_INVALID_VALUE;
  // the pick kernel keeps ||c||^2 of every centroid in shared memory
  if (method == 2 && static_cast<size_t>(k) * sizeof(float) > 200 * 1024)
    return HML_STATUS_NOT_SUPPORTED;
  if (method == 0) method = d <= kKmeansTiledMaxDims ? 1 : 2;
  if (method == 2 && static_cast<size_t>(k) * sizeof(float) > 200 * 1024) method = 1;
  return method == 1 ? assign_tiled(points, np, d, cent, k, out, exact, s)
                     : assign_gemm(points, np, d, cent, k, out, exact, s);
}

}  // namespace hml

extern "C" hml_status hml_kmeans_assign(const float *points, int num_points, int dims,
                                        const float *centroids, int num_clusters,
                                        uint32_t *assignments, void *stream) {
  return hml::kmeans_assign(points, num_points, dims, centroids, num_clusters, assignments, 0,
                            nullptr, static_cast<cudaStream_t>(stream));
}

extern "C" hml_status hml_kmeans_assign_ex(const float *points, int num_points, int dims,
                                           const float *centroids, int num_clusters,
                                           uint32_t *assignments, int method,
                                           unsigned *exact_count, void *stream) {
  return hml::kmeans_assign(points, num_points, dims, centroids, num_clusters, assignments,
                            method, exact_count, static_cast<cudaStream_t>(stream));
}
