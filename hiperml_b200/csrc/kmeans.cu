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
// centroid are one skinny GEMM S = X C^T (points x clusters), in one of three
// forms:
//   * tensor-core (method 3, the default where it applies: dims a multiple of
//     4 up to 64, at most 256 centroids): TF32X3 products on tcgen05 into
//     TMEM, the argmin read back from the accumulator by the thread that owns
//     the point;
//   * tiled (method 1, the default otherwise up to 256 dimensions): a
//     register-tiled FP32 SIMT GEMM with the argmin in its epilogue;
//   * SGEMM (method 2, wider points): the library's SGEMM in an FP32-accurate
//     configuration (BF16X6 or SIMT; never the fast BF16X3 mode), S in HBM,
//     and a pick kernel.
// The products carry rounding errors that the reference's direct sums do
// not, so the pick is made exact: with g_k = ||c_k||^2 - 2 S_k, every
// centroid whose g_k lies within a bound of the smallest (16 gamma_{dims+4}
// (||x||^2 + max_k ||c_k||^2) for the FP32 forms, twice that for TF32X3: more
// than twice the sum of the worst-case errors of g and of the reference's
// dist) is a candidate, and the reference's choice is always among them.  A
// point with more than one candidate (or non-finite values) goes to a
// close-call list that a settle kernel resolves with the reference's own
// arithmetic over the candidates, the first smallest in increasing k.  So
// every point gets the reference kernel's index, exact ties included.
#include <cfloat>
#include <cstring>

#include "hml_device.cuh"
#include "hml_internal.h"
#include "hml_select.h"
#include "hml_tune.h"
#include "hml_tcgen05.cuh"
#include "simt_tile.cuh"

namespace hml {
namespace {

constexpr int kNormWarps = 8;
// Widest points the automatic choice gives the tiled form (method 1); wider
// ones go through the SGEMM (method 2).
constexpr int kKmeansTiledMaxDims = 256;

// ||c_k||^2 for every centroid, one warp per centroid (FP32; used only to
// screen candidates).  It runs first in every form, so it also empties the
// close-call list of the call.
__global__ void centroid_norms_kernel(const float *cent, int k, int d, float *cnorm,
                                      unsigned *ccount) {
  const int lane = threadIdx.x & 31;
  if (blockIdx.x == 0 && threadIdx.x == 0) *ccount = 0u;
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
// whose g_k, recomputed, is at most lim -- by one warp (every lane calls
// this with the same arguments).  For 16 centroids at a time, in increasing
// k, the lanes form x . c_k together (lane r takes dimensions r, r + 32,
// ...: coalesced loads of the rows; the partial sums added by xor shuffles,
// so every lane holds the same dot product: any FP32 evaluation of g stays
// within the bound the screen allowed for); for a candidate every lane forms
// the reference's own distance (sequential, subtract then FMA) and keeps the
// first smallest below FLT_MAX (strict <), which is the reference's pick.
// 0 when no candidate's distance is below FLT_MAX (the reference leaves that
// case unset).
__device__ __noinline__ uint32_t exact_pick(const float *x, int d, const float *cent, int k,
                                            const float *cnorm, float lim) {
  constexpr int U = 16;  // centroids in flight: their loads and shuffle trees interleave
  const int lane = threadIdx.x & 31;
  float bd = FLT_MAX;
  uint32_t bk = 0;
  for (int c0 = 0; c0 < k; c0 += U) {
    float part[U], cnv[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      part[u] = 0.0f;
      cnv[u] = c0 + u < k ? cnorm[c0 + u] : 0.0f;  // loaded ahead of the tests below
    }
    for (int j = lane; j < d; j += 32) {
      const float xj = x[j];
#pragma unroll
      for (int u = 0; u < U; ++u)
        if (c0 + u < k) part[u] = fmaf(xj, cent[static_cast<int64_t>(c0 + u) * d + j], part[u]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
      for (int u = 0; u < U; ++u) part[u] += __shfl_xor_sync(0xffffffffu, part[u], o);
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int c = c0 + u;
      if (c >= k || !(fmaf(-2.0f, part[u], cnv[u]) <= lim)) continue;
      const float dist = ref_dist(x, cent + static_cast<int64_t>(c) * d, d);
      if (dist < bd) {
        bd = dist;
        bk = static_cast<uint32_t>(c);
      }
    }
  }
  return bk;
}

// Close calls (a second smallest g within the bound of the smallest, or
// non-finite values) are not settled where they are found: the screening
// kernels append (point, bound) to a list, every lane of a warp calling this
// together (one atomic per warp), and kmeans_settle_kernel settles the list
// afterwards, a warp per point -- so a rare long settling never holds up the
// screening of the other points.
__device__ __forceinline__ void push_close(unsigned *ccount, uint2 *citems, int64_t p, float lim,
                                           bool close) {
  const unsigned m = __ballot_sync(0xffffffffu, close);
  if (!m) return;
  const int lane = threadIdx.x & 31, leader = __ffs(m) - 1;
  unsigned base = 0;
  if (lane == leader) base = atomicAdd(ccount, static_cast<unsigned>(__popc(m)));
  base = __shfl_sync(0xffffffffu, base, leader);
  if (close)
    citems[base + __popc(m & ((1u << lane) - 1u))] =
        make_uint2(static_cast<uint32_t>(p), __float_as_uint(lim));
}

// The same pick with the centroids staged in shared memory (rows padded to
// cs = d + 1 floats, so that lane r reading element j of centroid r + 32 i
// hits bank (r + j) % 32: no conflicts), their norms beside them and the
// point's row in `xs`: lane r takes whole centroids r, r + 32, ... (its dot
// products in dimension order, any FP32 order being within the bound), forms
// the reference's distance of its candidates and keeps the first smallest
// below FLT_MAX; the warp then keeps the smallest distance, the lowest index
// among equal ones -- the first minimum in k order, the reference's pick.
__device__ __forceinline__ uint32_t exact_pick_smem(const float *xs, int d, const float *cs,
                                                    int k, const float *cn, float lim) {
  const int lane = threadIdx.x & 31, st = d + 1;
  float bd = FLT_MAX;
  int bk = -1;
  for (int c = lane; c < k; c += 32) {
    const float *cp = cs + c * st;
    float dot = 0.0f;
    for (int j = 0; j < d; ++j) dot = fmaf(xs[j], cp[j], dot);
    if (!(fmaf(-2.0f, dot, cn[c]) <= lim)) continue;
    const float dist = ref_dist(xs, cp, d);
    if (dist < bd) {
      bd = dist;
      bk = c;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const float od = __shfl_xor_sync(0xffffffffu, bd, o);
    const int ok = __shfl_xor_sync(0xffffffffu, bk, o);
    if (ok >= 0 && (bk < 0 || od < bd || (od == bd && ok < bk))) {
      bd = od;
      bk = ok;
    }
  }
  return bk < 0 ? 0u : static_cast<uint32_t>(bk);
}

// Shared-memory floats the settle kernel stages (0: the centroids do not fit
// in 96 KB and are read from global memory): centroids with rows of d + 1,
// their norms, one point row per warp (8 warps).
__host__ __device__ constexpr int64_t settle_smem_floats(int k, int d) {
  return static_cast<int64_t>(k) * (d + 1) + k + 8 * static_cast<int64_t>(d);
}
constexpr int64_t kSettleSmemFloats = 96 * 1024 / 4;

__global__ void __launch_bounds__(256) kmeans_settle_kernel(
    const float *points, int d, const float *cent, int k, const float *cnorm,
    const unsigned *ccount, const uint2 *citems, uint32_t *out, unsigned *exact, int staged) {
  wait_prior_grid();  // launched as a programmatic dependent of the screening kernel
  extern __shared__ float s_set[];
  const unsigned n = *ccount;
  if (exact && n && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(exact, n);
  const unsigned wpb = blockDim.x >> 5, warps = gridDim.x * wpb;
  if (blockIdx.x * wpb >= n) return;  // no entry for this block's warps
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  float *cs = s_set, *cn = s_set + static_cast<int64_t>(k) * (d + 1);
  float *xs = cn + k + wib * d;
  if (staged) {
    for (int e = threadIdx.x; e < k * d; e += blockDim.x) {
      const int c = e / d, j = e - c * d;
      cs[c * (d + 1) + j] = cent[e];
    }
    for (int c = threadIdx.x; c < k; c += blockDim.x) cn[c] = cnorm[c];
    __syncthreads();
  }
  for (unsigned w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < n; w += warps) {
    const uint2 it = citems[w];
    const float *x = points + static_cast<int64_t>(it.x) * d;
    uint32_t pick;
    if (staged) {
      for (int j = lane; j < d; j += 32) xs[j] = x[j];
      __syncwarp();
      pick = exact_pick_smem(xs, d, cs, k, cn, __uint_as_float(it.y));
      __syncwarp();  // xs is rewritten for the warp's next entry
    } else {
      pick = exact_pick(x, d, cent, k, cnorm, __uint_as_float(it.y));
    }
    if (lane == 0) out[it.x] = pick;
  }
}

// One thread per point: g_k = ||c_k||^2 - 2 S(p, k) (S column-major, ld lds),
// the candidates within `margin` of the smallest; a point with more than
// one goes to the close-call list.
__global__ void kmeans_pick_kernel(const float *points, int64_t np, int d, int k, const float *S,
                                   int64_t lds, const float *cnorm, uint32_t *out,
                                   unsigned *ccount, uint2 *citems) {
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
  const int lane = threadIdx.x & 31;
  // the warp walks 32 consecutive points at a time (every lane takes every
  // step, so the warp can list its close calls together)
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
    push_close(ccount, citems, p, lim, close);
  }
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
// bound of the smallest goes to the close-call list.  The products never
// leave the SM.
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

__device__ __forceinline__ Best shfl_best(unsigned mask, const Best &b, int o) {
  return {__shfl_xor_sync(mask, b.g1, o), __shfl_xor_sync(mask, b.k1, o),
          __shfl_xor_sync(mask, b.g2, o)};
}

// End of a tile for the 16 lanes of a point group (one half-warp, lane tx):
// their states for the group's 8 points (thread-local point i = tile row
// ty*4+i for i < 4, 64+ty*4+i-4 otherwise) are merged by a reduce-scatter --
// at offsets 8, 4 and 2 a lane keeps half of the points it carries, merged
// with its partner's half, and at offset 1 the pair merges its one point --
// so lanes tx and tx^1 end with point 4*bit3 + 2*bit2 + bit1 of tx merged
// over all 16.  The even lane writes a settled point or lists a close call
// (all 32 lanes of the warp call this together).
__device__ __forceinline__ void settle_group(Best (&best)[8], int64_t p0, int nb, int ty, int tx,
                                             const float *s_xn, float cmax, float bound,
                                             uint32_t *out, unsigned *ccount, uint2 *citems) {
  const unsigned hmask = 0xFFFFu << (threadIdx.x & 16);
  Best b4[4];
  {
    const bool up = tx & 8;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const Best keep = up ? best[4 + i] : best[i];
      const Best send = up ? best[i] : best[4 + i];
      b4[i] = best_merge(keep, shfl_best(hmask, send, 8));
    }
  }
  Best b2[2];
  {
    const bool up = tx & 4;
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const Best keep = up ? b4[2 + i] : b4[i];
      const Best send = up ? b4[i] : b4[2 + i];
      b2[i] = best_merge(keep, shfl_best(hmask, send, 4));
    }
  }
  Best b;
  {
    const bool up = tx & 2;
    const Best keep = up ? b2[1] : b2[0];
    const Best send = up ? b2[0] : b2[1];
    b = best_merge(keep, shfl_best(hmask, send, 2));
  }
  b = best_merge(b, shfl_best(hmask, b, 1));
  const int i = ((tx >> 3) & 1) * 4 + ((tx >> 2) & 1) * 2 + ((tx >> 1) & 1);
  const int pt = i < 4 ? ty * 4 + i : 64 + ty * 4 + (i - 4);
  const bool mine = (tx & 1) == 0 && pt < nb;
  float lim = 0.0f;
  bool close = false;
  if (mine) {
    lim = b.g1 + bound * (s_xn[pt] + cmax) + 1e-37f;
    close = !(b.g2 > lim);
    if (!close) out[p0 + pt] = static_cast<uint32_t>(b.k1);
  }
  push_close(ccount, citems, p0 + pt, lim, close);
}

__global__ void __launch_bounds__(kTThreads, 2) kmeans_tile_kernel(
    const float *__restrict__ points, int np, int d, const float *__restrict__ cent, int k,
    const float *__restrict__ cnorm, uint32_t *__restrict__ out, unsigned *ccount,
    uint2 *citems) {
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

  settle_group(best, p0, nb, ty, tx, s_xn, cmax, bound, out, ccount, citems);
}

// The resident form of the tiled kernel, for centroids that fit in shared
// memory (k and dims padded to kp = 64-multiple and dp = 4-multiple, dp <= 64
// and kp * dp <= kResidentFloats, so two blocks fit on an SM): each block
// stages the transposed centroids and their norms once and then walks
// 128-point tiles (a persistent grid), the next tile's rows copied by
// cp.async into the other of two row-major buffers while the current tile
// is computed, so the loads' latency hides behind the arithmetic.  A
// thread's 8 points are read as 16-byte row pieces (4 dimensions each), the
// centroids as 16-byte pieces of a dimension row; the products, the running
// argmin, the merge and the close-call list are the tiled kernel's.
constexpr int kResidentFloats = 8192;

__global__ void __launch_bounds__(kTThreads, 2) kmeans_resident_kernel(
    const float *__restrict__ points, int np, int d, int dp, bool vec,
    const float *__restrict__ cent, int k, int kp, const float *__restrict__ cnorm,
    uint32_t *__restrict__ out, unsigned *ccount, uint2 *citems) {
  extern __shared__ __align__(16) float sm[];
  const int cst = kp + 4;                   // row stride of the transposed centroids
  float *ct = sm;                           // [dp][cst]
  float *cn = ct + dp * cst;                // [kp]
  float *xr = cn + kp;                      // [2][kTP][dp]
  float *s_xn = xr + 2 * kTP * dp;          // [kTP]
  __shared__ float s_wmax[kTThreads / 32];
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int64_t tiles = (static_cast<int64_t>(np) + kTP - 1) / kTP;

  // the next tile's rows into buffer `buf` (zero past d and past np when
  // copied element-wise)
  auto issue = [&](int64_t t, int buf) {
    const int64_t p0 = t * kTP;
    const int nbt = static_cast<int>(min(static_cast<int64_t>(kTP), np - p0));
    float *dst = xr + buf * kTP * dp;
    if (vec) {
      const int q = dp / 4;
      for (int e = tid; e < nbt * q; e += kTThreads) {
        const int pt = e / q, c4 = e - pt * q;
        cp_async16(smem_u32(dst + pt * dp + c4 * 4), points + (p0 + pt) * d + c4 * 4, 16);
      }
    } else {
      for (int e = tid; e < kTP * dp; e += kTThreads) {
        const int pt = e / dp, j = e - pt * dp;
        const bool v = pt < nbt && j < d;
        cp_async4(smem_u32(dst + e), v ? points + (p0 + pt) * d + j : points, v);
      }
    }
    cp_async_commit();
  };
  int64_t t = blockIdx.x;
  if (t < tiles) issue(t, 0);

  // centroids (transposed, zero padded) and norms (NaN past k: never taken)
  for (int e = tid; e < dp * kp; e += kTThreads) {
    const int j = e / kp, c = e - j * kp;
    ct[j * cst + c] = (c < k && j < d) ? cent[static_cast<int64_t>(c) * d + j] : 0.0f;
  }
  float cmax = 0.0f;
  for (int c = tid; c < kp; c += kTThreads) {
    const float v = c < k ? cnorm[c] : __int_as_float(0x7fc00000);
    cn[c] = v;
    if (c < k) cmax = fmaxf(cmax, v);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) cmax = fmaxf(cmax, __shfl_xor_sync(0xffffffffu, cmax, o));
  if ((tid & 31) == 0) s_wmax[tid >> 5] = cmax;
  __syncthreads();
  cmax = 0.0f;
#pragma unroll
  for (int w = 0; w < kTThreads / 32; ++w) cmax = fmaxf(cmax, s_wmax[w]);
  const double nu = (d + 4) * 0x1p-24;
  const float bound = static_cast<float>(16.0 * nu / (1.0 - nu) * 1.001);

  for (int buf = 0; t < tiles; t += gridDim.x, buf ^= 1) {
    const int64_t tn = t + gridDim.x;
    if (tn < tiles) {
      issue(tn, buf ^ 1);
      asm volatile("cp.async.wait_group 1;" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;" ::: "memory");
    }
    __syncthreads();  // this tile's rows are in place
    const float *x = xr + buf * kTP * dp;
    const int64_t p0 = t * kTP;
    const int nb = static_cast<int>(min(static_cast<int64_t>(kTP), np - p0));
    if (tid < kTP) {
      // ||x||^2 for the bound (the row's 16-byte pieces in a rotated order,
      // so that the lanes of a warp read different banks)
      const int q = dp / 4;
      float xn = 0.0f;
      for (int i = 0; i < q; ++i) {
        const float4 v = lds128(x + tid * dp + ((i + tid) % q) * 4);
        xn = fmaf(v.x, v.x, xn);
        xn = fmaf(v.y, v.y, xn);
        xn = fmaf(v.z, v.z, xn);
        xn = fmaf(v.w, v.w, xn);
      }
      s_xn[tid] = xn;
    }
    Best best[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) best[i] = {INFINITY, 0, INFINITY};
    const float *xa = x + (ty * 4) * dp, *xb = x + (64 + ty * 4) * dp;
    for (int c0 = 0; c0 < kp; c0 += kTC) {
      float acc[8][4];
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[i][q] = 0.0f;
      const float *cc = ct + c0 + tx * 4;
      for (int j0 = 0; j0 < dp; j0 += 4) {
        float4 xv[8];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          xv[i] = lds128(xa + i * dp + j0);
          xv[4 + i] = lds128(xb + i * dp + j0);
        }
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
          const float4 cv = lds128(cc + (j0 + jj) * cst);
          const float cw[4] = {cv.x, cv.y, cv.z, cv.w};
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            const float xi = jj == 0 ? xv[i].x : jj == 1 ? xv[i].y : jj == 2 ? xv[i].z : xv[i].w;
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[i][q] = fmaf(xi, cw[q], acc[i][q]);
          }
        }
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int c = tx * 4 + q;
        const float cnv = cn[c0 + c];
#pragma unroll
        for (int i = 0; i < 8; ++i) best_add(best[i], fmaf(-2.0f, acc[i][q], cnv), c0 + c);
      }
    }
    __syncthreads();  // s_xn is complete
    settle_group(best, p0, nb, ty, tx, s_xn, cmax, bound, out, ccount, citems);
    __syncthreads();  // the buffer and s_xn are free for the tile after next
  }
}

// ------------------------------------------------ the tensor-core form
// (method 3)  The dot products of a 128-point tile with all (up to 256)
// centroids as TF32X3 products on the tensor cores: x = xh + xl and
// c = ch + cl with xh = tf32(x), xl = tf32(x - xh) (22 significant bits
// together), and x.c ~ xh.ch + xh.cl + xl.ch accumulated in FP32 in TMEM.
// One CTA per SM walks the tiles of a persistent grid:
//   * warp 0, one lane: TMA of the centroids' TF32 planes (split once by
//     kmeans_tf32_planes_kernel, K-contiguous), resident in shared memory
//     in the UMMA K-major layout (128-byte swizzle), then of each point tile
//     (128 rows x 32 dimensions a box, 128-byte swizzle) into a ring;
//   * W warpgroups take the CTA's tiles round-robin.  Thread m of a group
//     owns point m of the tile, which is TMEM lane m: it reads the point's
//     row, forms ||x||^2 (for the bound) and the TF32 planes, writes them
//     into the group's TMEM A region with tcgen05.st; one elected thread
//     then issues the group's tcgen05.mma chain (A in TMEM, B from shared
//     memory, N = the padded number of centroids) into the group's TMEM
//     accumulator and commits it to the group's mbarrier; the group reads
//     its rows back with tcgen05.ld and takes the argmin of g_k =
//     ||c_k||^2 - 2 x.c_k in increasing k -- the whole row of a point in
//     one thread, so no merge.  W groups keep W tiles in flight, W issuing
//     threads in parallel (one thread issues a tcgen05.mma only every ~130
//     cycles).
// Close calls go to the close-call list, the margin being twice the SIMT
// forms' (32 gamma_{dims+4}), as the
// products' error is up to about four times a direct FP32 sum's (the split
// leaves 2^-22 per operand; the tensor core's accumulation truncates).
constexpr int kTcMaxD = 64;    // dimensions (padded to 32)
constexpr int kTcMaxK = 256;   // centroids (padded to 32): one MMA's N
constexpr int kTcBox = kTP * 32 * 4;  // bytes of one 128 x 32 FP32 box

struct KmTcArgs {
  int np, d, k, dp, kp, sa;
  int nc, passes;  // centroids per pass (a multiple of 32) and passes per tile
  const float *cnorm;
  uint32_t *out;
  unsigned *ccount;
  uint2 *citems;
  int *err;
};

// OR of `v` over the 128 threads of a warpgroup (named barrier `id`).
__device__ __forceinline__ bool group_any(bool v, int id) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "barrier.cta.red.or.pred q, %2, 128, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}"
      : "=r"(r)
      : "r"(static_cast<uint32_t>(v)), "r"(id)
      : "memory");
  return r != 0;
}

__device__ __forceinline__ void group_sync(int id) {
  asm volatile("barrier.cta.sync.aligned %0, 128;" ::"r"(id) : "memory");
}

__host__ __device__ constexpr int km_tc_threads(int w) { return (4 + 4 * w) * 32; }

template <int W>
__global__ void __launch_bounds__(km_tc_threads(W), 1)
    kmeans_tc_kernel(const __grid_constant__ CUtensorMap tmX,
                     const __grid_constant__ CUtensorMap tmB, const __grid_constant__ KmTcArgs a) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = align_shared(smem_raw, 1024);
  const int dp = a.dp, kp = a.kp, nkb = dp / 32, SA = a.sa;
  const int slot = nkb * kTcBox;   // bytes of one point tile
  const int btile = kp * 128;      // bytes of one (plane, 32-dim block) of the centroids
  uint8_t *xring = smem;                                  // [SA][nkb][128 x 128 B]
  uint8_t *bsm = xring + SA * slot;                       // [2][nkb][kp x 128 B]
  float *cn = reinterpret_cast<float *>(bsm + 2 * nkb * btile);  // [kp]
  uint64_t *afull = reinterpret_cast<uint64_t *>(cn + kp);
  uint64_t *aempty = afull + SA;
  uint64_t *accfull = aempty + SA;  // [W]
  uint64_t *bfull = accfull + W;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bfull + 1);
  float *s_cmax = reinterpret_cast<float *>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t tiles = (static_cast<int64_t>(a.np) + kTP - 1) / kTP;
  const int my_tiles = static_cast<int>((tiles - blockIdx.x + gridDim.x - 1) / gridDim.x);

  if (threadIdx.x == 0) {
    for (int i = 0; i < SA; ++i) {
      mbar_init(&afull[i], 1);
      mbar_init(&aempty[i], 4);  // the 4 warps of the group that read the tile
    }
    for (int g = 0; g < W; ++g) mbar_init(&accfull[g], 1);
    mbar_init(bfull, 1);
    fence_mbar_init();
    prefetch_tmap(&tmX);
    prefetch_tmap(&tmB);
  }
  // the planes and norms come from the prep kernel launched just before
  wait_prior_grid();
  if (warp == 1) {
    // ||c||^2 (+inf past k: never taken, and never the second smallest) and
    // its maximum over the centroids
    float cmax = 0.0f;
    for (int c = lane; c < kp; c += 32) {
      const float v = c < a.k ? a.cnorm[c] : INFINITY;
      cn[c] = v;
      if (c < a.k) cmax = fmaxf(cmax, v);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cmax = fmaxf(cmax, __shfl_xor_sync(0xffffffffu, cmax, o));
    if (lane == 0) *s_cmax = cmax;
  }
  if (warp == 2) tmem_alloc(tmem_slot, 512);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    // ------------------------------------------------------------ TMA
    if (lane == 0) {
      mbar_arrive_expect_tx(bfull, 2 * nkb * btile);
      for (int pl = 0; pl < 2; ++pl)
        for (int kb = 0; kb < nkb; ++kb)
          tma_load_2d(bsm + (pl * nkb + kb) * btile, &tmB, bfull, kb * 32, pl * kp);
      int j = 0;
      for (; j < my_tiles; ++j) {
        const int st = j % SA;
        if (j >= SA && !mbar_wait(&aempty[st], ((j / SA) - 1) & 1, a.err, kDevErrEmptyBarrier))
          break;
        const int64_t t = blockIdx.x + static_cast<int64_t>(j) * gridDim.x;
        mbar_arrive_expect_tx(&afull[st], slot);
        for (int kb = 0; kb < nkb; ++kb)
          tma_load_2d(xring + st * slot + kb * kTcBox, &tmX, &afull[st], kb * 32,
                      static_cast<int>(t * kTP));
      }
      // every load issued has landed before the CTA may exit
      for (int i = max(0, j - SA); i < j; ++i)
        mbar_wait(&afull[i % SA], (i / SA) & 1, a.err, kDevErrFullBarrier);
      mbar_wait(bfull, 0, a.err, kDevErrFullBarrier);
    }
  } else if (warp >= 4) {
    // ------------------------------------------------- point groups
    const int g = (warp - 4) >> 2, bar_id = 1 + g;
    const int m = (warp & 3) * 32 + lane;  // tile row == TMEM lane
    const uint32_t lanes = static_cast<uint32_t>((warp & 3) * 32) << 16;
    const int nc = a.nc, P = a.passes;
    const uint32_t tacc = tmem + static_cast<uint32_t>(g * (nc + 2 * dp));
    const uint32_t tA = tacc + static_cast<uint32_t>(nc);  // hi plane dp columns, then lo
    const bool issuer = warp == 4 + 4 * g && lane == 0;
    const float cmax = *s_cmax;
    const double nu = (a.d + 4) * 0x1p-24;
    const float bound = static_cast<float>(32.0 * nu / (1.0 - nu) * 1.001);
    const uint32_t idesc = idesc_tf32(nc);
    int it = 0, ph = 0;  // tiles done, phases of accfull[g] done
    for (int j = g; j < my_tiles; j += W, ++it) {
      const int st = j % SA;
      const bool w = mbar_wait(&afull[st], (j / SA) & 1, a.err, kDevErrFullBarrier);
      if (group_any(!w, bar_id)) break;
      __syncwarp();  // tcgen05.st is warp-collective
      // the point's row: ||x||^2 in dimension order, then its TF32 planes
      const float *xs = reinterpret_cast<const float *>(xring + st * slot);
      float xn = 0.0f;
      for (int kb = 0; kb < nkb; ++kb) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          float x[16];
#pragma unroll
          for (int c = 0; c < 4; ++c) {
            const float4 v = *reinterpret_cast<const float4 *>(
                xs + kb * (kTcBox / 4) + m * 32 + (((4 * h + c) ^ (m & 7)) * 4));
            x[4 * c] = v.x;
            x[4 * c + 1] = v.y;
            x[4 * c + 2] = v.z;
            x[4 * c + 3] = v.w;
          }
          uint32_t hi[16], lo[16];
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            xn = fmaf(x[i], x[i], xn);
            hi[i] = tf32_rna(x[i]);
            lo[i] = tf32_rna(__fsub_rn(x[i], __uint_as_float(hi[i])));
          }
          const uint32_t col = static_cast<uint32_t>(kb * 32 + h * 16);
          tmem_st16(tA + lanes + col, hi);
          tmem_st16(tA + lanes + static_cast<uint32_t>(dp) + col, lo);
        }
      }
      // the slot is consumed (every value above was used before this point)
      __syncwarp();
      if (lane == 0) mbar_arrive(&aempty[st]);
      __syncwarp();
      tmem_wait_st();
      tc_fence_before();
      group_sync(bar_id);
      // the centroids in P passes of nc (the accumulator holds one pass):
      // argmin of g_k over the point's row, without branches -- g1 the
      // smallest, k1 the first index reaching it, g2 the second smallest of
      // the multiset (equal to g1 on a tie; a NaN g makes it g1 too, which
      // only sends the point to the close-call list)
      float g1 = INFINITY, g2 = INFINITY;
      int k1 = 0;
      bool bad = false;
      for (int q = 0; q < P; ++q) {
        if (issuer) {
          tc_fence_after();
          bool bok = true;
          if (it == 0 && q == 0) bok = mbar_wait(bfull, 0, a.err, kDevErrFullBarrier);
          if (bok) {
            // products hh, hl, lh of every 8-deep step of every 32-dim block,
            // against centroids q*nc .. q*nc+nc-1 (rows of the B tiles)
            for (int kb = 0; kb < nkb; ++kb)
#pragma unroll
              for (int kk = 0; kk < 4; ++kk)
#pragma unroll
                for (int pr = 0; pr < 3; ++pr) {
                  const int ia = pr == 2 ? 1 : 0, jb = pr == 1 ? 1 : 0;
                  const uint32_t at = tA + static_cast<uint32_t>(ia * dp + kb * 32 + kk * 8);
                  const uint64_t bd =
                      sw128_desc(smem_u32(bsm + (jb * nkb + kb) * btile + q * nc * 128)) +
                      static_cast<uint64_t>((kk * 32) >> 4);
                  mma_tf32_ts(tacc, at, bd, idesc, (kb | kk | pr) != 0 ? 1u : 0u);
                }
          }
          mma_commit(&accfull[g]);  // arrives once the group's MMAs are done
        }
        const bool w2 = mbar_wait(&accfull[g], ph & 1, a.err, kDevErrMmaBarrier);
        ++ph;
        if (group_any(!w2, bar_id)) {
          bad = true;
          break;
        }
        __syncwarp();  // tcgen05.ld is warp-collective
        tc_fence_after();
        for (int c0 = 0; c0 < nc; c0 += 16) {
          uint32_t r[16];
          tmem_ld16(tacc + lanes + static_cast<uint32_t>(c0), r);
          float cv[16];
#pragma unroll
          for (int qq = 0; qq < 4; ++qq) {
            const float4 v = *reinterpret_cast<const float4 *>(cn + q * nc + c0 + 4 * qq);
            cv[4 * qq] = v.x;
            cv[4 * qq + 1] = v.y;
            cv[4 * qq + 2] = v.z;
            cv[4 * qq + 3] = v.w;
          }
          tmem_wait_ld();
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            const float gv = fmaf(-2.0f, __uint_as_float(r[i]), cv[i]);
            k1 = gv < g1 ? q * nc + c0 + i : k1;
            g2 = fminf(g2, fmaxf(g1, gv));
            g1 = fminf(g1, gv);
          }
        }
        tc_fence_before();  // the reads are done before the next MMAs
        if (q + 1 < P) group_sync(bar_id);
      }
      if (bad) break;
      const int64_t t = blockIdx.x + static_cast<int64_t>(j) * gridDim.x;
      const int64_t p = t * kTP + m;
      const bool live = p < a.np;
      const float lim = g1 + bound * (xn + cmax) + 1e-37f;
      const bool close = live && !(g2 > lim);
      if (live && !close) a.out[p] = static_cast<uint32_t>(k1);
      push_close(a.ccount, a.citems, p, lim, close);
    }
  }
  tc_fence_before();
  __syncthreads();
  // the settle kernel may now be scheduled (it waits for this grid itself);
  // earlier, its waiting CTAs would sit beside this kernel's on every SM
  allow_dependent_launch();
  if (warp == 2) {
    tc_fence_after();
    tmem_dealloc(tmem, 512);
  }
}

// Prep for the tensor-core form: the TF32 planes of the centroids and their
// norms (one warp per centroid row, the norm summed lane-wise -- it only
// enters the bound), and an empty close-call list.
__global__ void kmeans_tc_prep_kernel(const float *cent, int k, int d, int kp, int dp,
                                      uint32_t *planes, float *cnorm, unsigned *ccount) {
  allow_dependent_launch();
  if (blockIdx.x == 0 && threadIdx.x == 0) *ccount = 0u;
  const int lane = threadIdx.x & 31;
  const int c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (c >= kp) return;
  float sq = 0.0f;
  for (int j = lane; j < dp; j += 32) {
    const float v = (c < k && j < d) ? cent[static_cast<int64_t>(c) * d + j] : 0.0f;
    const uint32_t hi = tf32_rna(v);
    planes[c * dp + j] = hi;
    planes[kp * dp + c * dp + j] = tf32_rna(__fsub_rn(v, __uint_as_float(hi)));
    sq = fmaf(v, v, sq);
  }
  sq = warp_sum(sq);
  if (lane == 0 && c < k) cnorm[c] = sq;
}

// The call's workspace (the stream's second slot): `extra` bytes for the
// form (the products or the centroid planes), ||c||^2, and the close-call
// list (a count, then room for every point).
struct KmWs {
  uint8_t *extra;
  float *cnorm;
  unsigned *ccount;
  uint2 *citems;
};

hml_status km_workspace(size_t extra, int np, int k, cudaStream_t s, KmWs *w) {
  auto up = [](size_t b) { return (b + 255) & ~static_cast<size_t>(255); };
  const size_t o_norm = up(extra), o_cnt = o_norm + up(static_cast<size_t>(k) * sizeof(float));
  const size_t o_items = o_cnt + 256;
  void *ws = nullptr;
  hml_status st = workspace_slot(1, o_items + static_cast<size_t>(np) * sizeof(uint2), s, &ws);
  if (st != HML_STATUS_SUCCESS) return st;
  uint8_t *b = static_cast<uint8_t *>(ws);
  w->extra = b;
  w->cnorm = reinterpret_cast<float *>(b + o_norm);
  w->ccount = reinterpret_cast<unsigned *>(b + o_cnt);
  w->citems = reinterpret_cast<uint2 *>(b + o_items);
  return HML_STATUS_SUCCESS;
}

// ||c||^2 and an empty close-call list; first in every form.
hml_status launch_norms(const float *cent, int k, int d, const KmWs &w, cudaStream_t s) {
  count_launch();
  const int nb = std::min((k + kNormWarps - 1) / kNormWarps, 4 * sm_count());
  centroid_norms_kernel<<<std::max(1, nb), 32 * kNormWarps, 0, s>>>(cent, k, d, w.cnorm,
                                                                     w.ccount);
  cudaError_t e = cudaGetLastError();
  note_cuda_error(e, "kmeans norms");
  return cuda_status(e);
}

// The close calls the screening kernel listed; last in every form
// (`early`: as a programmatic dependent of a screening kernel that allows it).
hml_status launch_settle(const float *points, int d, const float *cent, int k, const KmWs &w,
                         uint32_t *out, unsigned *exact, cudaStream_t s, bool early = false) {
  // the centroids, norms and point rows in shared memory when they fit
  const int staged = settle_smem_floats(k, d) <= kSettleSmemFloats ? 1 : 0;
  const size_t smem = staged ? static_cast<size_t>(settle_smem_floats(k, d)) * 4 : 0;
  cudaError_t e = cudaSuccess;
  if (smem > 48 * 1024)
    e = cudaFuncSetAttribute(kmeans_settle_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(smem));
  if (e == cudaSuccess)
    e = launch_k_ex(kmeans_settle_kernel, dim3(2 * sm_count()), dim3(256), smem, s, 1, early,
                    points, d, cent, k, static_cast<const float *>(w.cnorm),
                    static_cast<const unsigned *>(w.ccount),
                    static_cast<const uint2 *>(w.citems), out, exact, staged);
  note_cuda_error(e, "kmeans settle");
  return cuda_status(e);
}

// The tiled SIMT form (method 1).
hml_status assign_tiled(const float *points, int np, int d, const float *cent, int k,
                        uint32_t *out, unsigned *exact, cudaStream_t s) {
  KmWs w;
  hml_status st = km_workspace(0, np, k, s, &w);
  if (st == HML_STATUS_SUCCESS) st = launch_norms(cent, k, d, w, s);
  if (st != HML_STATUS_SUCCESS) return st;
  const int64_t blocks = (static_cast<int64_t>(np) + kTP - 1) / kTP;
  const int dp = (d + 3) & ~3, kp = (k + kTC - 1) / kTC * kTC;
  cudaError_t e = cudaSuccess;
  count_launch();
  if (d > 0 && dp <= 64 && static_cast<int64_t>(dp) * kp <= kResidentFloats) {
    const size_t smem =
        (static_cast<size_t>(dp) * (kp + 4) + kp + 2 * kTP * dp + kTP) * sizeof(float);
    e = cudaFuncSetAttribute(kmeans_resident_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(smem));
    // 16-byte row copies when every row starts on a 16-byte boundary
    const bool vec = d % 4 == 0 && (reinterpret_cast<uintptr_t>(points) & 15u) == 0;
    const int64_t grid = std::min<int64_t>(blocks, 2LL * sm_count());
    if (e == cudaSuccess)
      kmeans_resident_kernel<<<static_cast<unsigned>(grid), kTThreads, smem, s>>>(
          points, np, d, dp, vec, cent, k, kp, w.cnorm, out, w.ccount, w.citems);
  } else {
    kmeans_tile_kernel<<<static_cast<unsigned>(blocks), kTThreads, 0, s>>>(
        points, np, d, cent, k, w.cnorm, out, w.ccount, w.citems);
  }
  if (e == cudaSuccess) e = cudaGetLastError();
  note_cuda_error(e, "kmeans tiled");
  if (e != cudaSuccess) return cuda_status(e);
  return launch_settle(points, d, cent, k, w, out, exact, s);
}

// The GEMM form (method 2): S = X C^T through the library's SGEMM, then the
// pick kernel.
hml_status assign_gemm(const float *points, int np, int d, const float *cent, int k,
                       uint32_t *out, unsigned *exact, cudaStream_t s) {
  const size_t s_bytes = static_cast<size_t>(np) * k * sizeof(float);
  KmWs w;
  hml_status st = km_workspace(s_bytes, np, k, s, &w);
  if (st != HML_STATUS_SUCCESS) return st;
  float *S = reinterpret_cast<float *>(w.extra);
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
  st = launch_norms(cent, k, d, w, s);
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
        points, np, d, k, S, np, w.cnorm, out, w.ccount, w.citems);
    e = cudaGetLastError();
  }
  note_cuda_error(e, "kmeans assign");
  if (e != cudaSuccess) return cuda_status(e);
  return launch_settle(points, d, cent, k, w, out, exact, s);
}

// The tensor-core form applies to points with 4 <= dims <= 64 (a multiple of
// 4, rows 16-byte aligned, for TMA) and at most 256 centroids.
bool tc_form_applies(const float *points, int d, int k) {
  return d >= 4 && d % 4 == 0 && (reinterpret_cast<uintptr_t>(points) & 15u) == 0 &&
         ((d + 31) & ~31) <= kTcMaxD && ((k + 31) & ~31) <= kTcMaxK;
}

template <int W>
hml_status launch_km_tc(const CUtensorMap &tx, const CUtensorMap &tb, const KmTcArgs &a,
                        int grid, size_t smem, cudaStream_t s) {
  auto kern = kmeans_tc_kernel<W>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem));
  if (e == cudaSuccess)
    e = launch_k_ex(kern, dim3(grid), dim3(km_tc_threads(W)), smem, s, 1, true, tx, tb, a);
  note_cuda_error(e, "kmeans tensor-core");
  return cuda_status(e);
}

// The tensor-core form (method 3): centroid planes and norms in one prep
// kernel, then the persistent screening kernel and the settle kernel, each a
// programmatic dependent of the kernel before it.
hml_status assign_tc(const float *points, int np, int d, const float *cent, int k,
                     uint32_t *out, unsigned *exact, cudaStream_t s) {
  const int dp = (d + 31) & ~31, kp = (k + 31) & ~31, nkb = dp / 32;
  // W groups, each with nc + 2 dp TMEM columns (a pass's accumulator, the A
  // planes): the fewest passes P (nc = kp / P, a multiple of 32) that give
  // the most groups, up to 4
  int W = 0, P = 1;
  for (int p = 1; p <= kp / 32; ++p) {
    if ((kp / 32) % p) continue;
    const int per = kp / p + 2 * dp;
    const int w = per <= 128 ? 4 : per <= 256 ? 2 : per <= 512 ? 1 : 0;
    if (w > W) {
      W = w;
      P = p;
    }
    if (W == 4) break;
  }
  if (W == 0) return HML_STATUS_NOT_SUPPORTED;
  const size_t pbytes = static_cast<size_t>(2) * kp * dp * sizeof(uint32_t);
  KmWs w;
  hml_status st = km_workspace(pbytes, np, k, s, &w);
  if (st != HML_STATUS_SUCCESS) return st;
  uint32_t *planes = reinterpret_cast<uint32_t *>(w.extra);
  count_launch();
  kmeans_tc_prep_kernel<<<(kp + 7) / 8, 256, 0, s>>>(cent, k, d, kp, dp, planes, w.cnorm,
                                                     w.ccount);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    note_cuda_error(e, "kmeans prep");
    return HML_STATUS_CUDA_ERROR;
  }
  CUtensorMap tx, tb;
  memset(&tx, 0, sizeof(tx));
  memset(&tb, 0, sizeof(tb));
  if (!tensor_map_2d(&tx, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, points, d, np,
                     static_cast<uint64_t>(d) * 4, 32, kTP, CU_TENSOR_MAP_SWIZZLE_128B) ||
      !tensor_map_2d(&tb, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, planes, dp, 2 * kp,
                     static_cast<uint64_t>(dp) * 4, 32, kp, CU_TENSOR_MAP_SWIZZLE_128B))
    return HML_STATUS_CUDA_ERROR;
  const size_t slot = static_cast<size_t>(nkb) * kTcBox;
  const size_t bbytes = static_cast<size_t>(2) * nkb * kp * 128;
  // a multiple of W (tiles go to group j % W and slot j % sa: each group
  // then waits for every phase of its slots in order)
  int sa = static_cast<int>(std::min<size_t>(6, (200 * 1024 - bbytes) / slot));
  sa -= sa % W;
  if (sa < 2) return HML_STATUS_NOT_SUPPORTED;
  size_t smem = 1024 + sa * slot + bbytes + static_cast<size_t>(kp) * 4 +
                static_cast<size_t>(2 * sa + W + 1) * 8 + 16;
  // one CTA per SM: each allocates all 512 TMEM columns
  smem = std::max<size_t>(smem, 120 * 1024);
  KmTcArgs a;
  a.np = np;
  a.d = d;
  a.k = k;
  a.dp = dp;
  a.kp = kp;
  a.sa = sa;
  a.nc = kp / P;
  a.passes = P;
  a.cnorm = w.cnorm;
  a.out = out;
  a.ccount = w.ccount;
  a.citems = w.citems;
  a.err = device_error_word();
  const int64_t tiles = (static_cast<int64_t>(np) + kTP - 1) / kTP;
  const int grid = static_cast<int>(std::min<int64_t>(tiles, sm_count()));
  switch (W) {
    case 4: st = launch_km_tc<4>(tx, tb, a, grid, smem, s); break;
    case 2: st = launch_km_tc<2>(tx, tb, a, grid, smem, s); break;
    default: st = launch_km_tc<1>(tx, tb, a, grid, smem, s); break;
  }
  if (st != HML_STATUS_SUCCESS) return st;
  return launch_settle(points, d, cent, k, w, out, exact, s, true);
}

}  // namespace

hml_status kmeans_assign(const float *points, int np, int d, const float *cent, int k,
                         uint32_t *out, int method, unsigned *exact, cudaStream_t s) {
  if (np < 0 || d < 0 || k < 1 || method < 0 || method > 3) return HML_STATUS_INVALID_VALUE;
  if (np == 0) return HML_STATUS_SUCCESS;
  if (!out || (d > 0 && (!points || !cent))) return HML_STATUS_INVALID_VALUE;
  // the pick kernel keeps ||c||^2 of every centroid in shared memory
  if (method == 2 && static_cast<size_t>(k) * sizeof(float) > 200 * 1024)
    return HML_STATUS_NOT_SUPPORTED;
  if (method == 3 && !tc_form_applies(points, d, k)) return HML_STATUS_NOT_SUPPORTED;
  if (method == 0) {
    method = tc_form_applies(points, d, k) ? 3 : d <= kKmeansTiledMaxDims ? 1 : 2;
    if (method == 2 && static_cast<size_t>(k) * sizeof(float) > 200 * 1024) method = 1;
  }
  switch (method) {
    case 1: return assign_tiled(points, np, d, cent, k, out, exact, s);
    case 2: return assign_gemm(points, np, d, cent, k, out, exact, s);
    default: return assign_tc(points, np, d, cent, k, out, exact, s);
  }
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
