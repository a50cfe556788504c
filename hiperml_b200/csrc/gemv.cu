// gemv.cu -- FP32 SIMT GEMV kernels for B200 (sm_100a).
//
// Two memory orders of A, each bound by HBM bandwidth (0.5 flop/byte):
//
//  gemv_rows  A(p,q) rows contiguous (sq == 1): the reference's row-major
//             hmlSgemv (src/hml_sgemv.cu:125-213) and the column-major
//             y = A^T x.  TPR threads share one row: coalesced 16-byte loads
//             along the row, warp-shuffle reduction, then a shared-memory
//             reduction across the row's warps.  Replaces the reference's
//             one-CTA-per-row hmlSgemvKernelBasicN
//             (include/hml_sgemv_kernel_template.h:19-106), whose volatile
//             warp-synchronous tail is unsafe under independent thread
//             scheduling.
//  gemv_cols  A(p,q) columns contiguous (sp == 1): column-major y = A x.
//             Each lane owns 4 consecutive rows (one 16-byte load per
//             column), the 8 warps of a CTA take interleaved columns, and
//             `split` CTAs of one thread-block cluster take disjoint column
//             ranges.  Partial sums are combined in a fixed order through
//             shared memory and then distributed shared memory, so results
//             are deterministic and no global workspace is used.
#include <algorithm>

#include "hml_device.cuh"
#include "hml_internal.h"

namespace hml {
namespace {

constexpr int kThreads = 256;

// ----------------------------------------------------------------- rows
template <int TPR, bool VEC>
__global__ void __launch_bounds__(kThreads) gemv_rows_kernel(GemvProblem p) {
  constexpr int RPC = kThreads / TPR;  // rows per CTA
  __shared__ float red[kThreads / 32];
  const int t = threadIdx.x % TPR;
  const int r = threadIdx.x / TPR;
  const int64_t row = static_cast<int64_t>(blockIdx.x) * RPC + r;
  float acc = 0.0f;
  if (row < p.P) {
    const float *a = p.A + row * p.sp;
    if (VEC) {
      const int Q4 = p.Q >> 2;
      const float4 *a4 = reinterpret_cast<const float4 *>(a);
      const float4 *x4 = reinterpret_cast<const float4 *>(p.x);
      float acc1 = 0.0f, acc2 = 0.0f, acc3 = 0.0f;
      int q = t;
      for (; q + 3 * TPR < Q4; q += 4 * TPR) {
        float4 v0 = ldg_stream4(reinterpret_cast<const float *>(a4 + q));
        float4 v1 = ldg_stream4(reinterpret_cast<const float *>(a4 + q + TPR));
        float4 v2 = ldg_stream4(reinterpret_cast<const float *>(a4 + q + 2 * TPR));
        float4 v3 = ldg_stream4(reinterpret_cast<const float *>(a4 + q + 3 * TPR));
        float4 w0 = __ldg(x4 + q), w1 = __ldg(x4 + q + TPR);
        float4 w2 = __ldg(x4 + q + 2 * TPR), w3 = __ldg(x4 + q + 3 * TPR);
        acc = fmaf(v0.x, w0.x, acc); acc = fmaf(v0.y, w0.y, acc);
        acc = fmaf(v0.z, w0.z, acc); acc = fmaf(v0.w, w0.w, acc);
        acc1 = fmaf(v1.x, w1.x, acc1); acc1 = fmaf(v1.y, w1.y, acc1);
        acc1 = fmaf(v1.z, w1.z, acc1); acc1 = fmaf(v1.w, w1.w, acc1);
        acc2 = fmaf(v2.x, w2.x, acc2); acc2 = fmaf(v2.y, w2.y, acc2);
        acc2 = fmaf(v2.z, w2.z, acc2); acc2 = fmaf(v2.w, w2.w, acc2);
        acc3 = fmaf(v3.x, w3.x, acc3); acc3 = fmaf(v3.y, w3.y, acc3);
        acc3 = fmaf(v3.z, w3.z, acc3); acc3 = fmaf(v3.w, w3.w, acc3);
      }
      for (; q < Q4; q += TPR) {
        float4 v = ldg_stream4(reinterpret_cast<const float *>(a4 + q));
        float4 w = __ldg(x4 + q);
        acc = fmaf(v.x, w.x, acc); acc = fmaf(v.y, w.y, acc);
        acc = fmaf(v.z, w.z, acc); acc = fmaf(v.w, w.w, acc);
      }
      acc += acc1 + (acc2 + acc3);
      const int qt = (Q4 << 2) + t;
      if (t < (p.Q & 3)) acc = fmaf(a[qt], __ldg(p.x + qt), acc);
    } else {
      float acc1 = 0.0f;
      int q = t;
      for (; q + TPR < p.Q; q += 2 * TPR) {
        acc = fmaf(ldg_stream(a + q), __ldg(p.x + q * p.incx), acc);
        acc1 = fmaf(ldg_stream(a + q + TPR), __ldg(p.x + (q + TPR) * p.incx), acc1);
      }
      if (q < p.Q) acc = fmaf(ldg_stream(a + q), __ldg(p.x + q * p.incx), acc);
      acc += acc1;
    }
  }
  // reduce the TPR partial sums of this row
  if (TPR >= 32) {
    acc = warp_sum(acc);
    if (TPR > 32) {
      if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
      __syncthreads();
      if (t == 0) {
        acc = 0.0f;
#pragma unroll
        for (int w = 0; w < TPR / 32; ++w) acc += red[r * (TPR / 32) + w];
      }
    }
  } else {
#pragma unroll
    for (int o = TPR / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  }
  if (t == 0 && row < p.P) {
    float *y = p.y + row * p.incy;
    *y = axpby(p.alpha, acc, p.beta, y);
  }
}

// ----------------------------------------------------------------- cols
// VEC: lane owns rows base + 4*lane .. +3 (16-byte loads); else rows
// base + lane + 32*j for j < 4.  Either way a warp covers 128 rows.
template <bool VEC>
__global__ void __launch_bounds__(kThreads) gemv_cols_kernel(GemvProblem p, int split) {
  constexpr int kRows = 128;
  __shared__ float4 part[kThreads / 32][kRows / 4];
  __shared__ float sum[kRows];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int rank = split > 1 ? static_cast<int>(cluster_ctarank()) : 0;
  const int64_t tile = blockIdx.x / split;
  const int64_t row0 = tile * kRows;
  const int qc = (p.Q + split - 1) / split;
  const int qbeg = rank * qc;
  const int qend = min(p.Q, qbeg + qc);

  float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
  const int64_t myrow = VEC ? row0 + 4 * lane : row0 + lane;
  const bool full = VEC ? (myrow + 3 < p.P) : (row0 + kRows <= p.P);
  if (full) {
    const float *a = p.A + myrow;
    float4 acc1 = make_float4(0.f, 0.f, 0.f, 0.f);
    int q = qbeg + warp;
    for (; q + 3 * 8 < qend; q += 4 * 8) {
      float4 v0, v1, v2, v3;
      if (VEC) {
        v0 = ldg_stream4(a + static_cast<int64_t>(q) * p.sq);
        v1 = ldg_stream4(a + static_cast<int64_t>(q + 8) * p.sq);
        v2 = ldg_stream4(a + static_cast<int64_t>(q + 16) * p.sq);
        v3 = ldg_stream4(a + static_cast<int64_t>(q + 24) * p.sq);
      } else {
        const float *c0 = a + static_cast<int64_t>(q) * p.sq;
        const float *c1 = a + static_cast<int64_t>(q + 8) * p.sq;
        const float *c2 = a + static_cast<int64_t>(q + 16) * p.sq;
        const float *c3 = a + static_cast<int64_t>(q + 24) * p.sq;
        v0 = make_float4(ldg_stream(c0), ldg_stream(c0 + 32), ldg_stream(c0 + 64), ldg_stream(c0 + 96));
        v1 = make_float4(ldg_stream(c1), ldg_stream(c1 + 32), ldg_stream(c1 + 64), ldg_stream(c1 + 96));
        v2 = make_float4(ldg_stream(c2), ldg_stream(c2 + 32), ldg_stream(c2 + 64), ldg_stream(c2 + 96));
        v3 = make_float4(ldg_stream(c3), ldg_stream(c3 + 32), ldg_stream(c3 + 64), ldg_stream(c3 + 96));
      }
      const float x0 = __ldg(p.x + static_cast<int64_t>(q) * p.incx);
      const float x1 = __ldg(p.x + static_cast<int64_t>(q + 8) * p.incx);
      const float x2 = __ldg(p.x + static_cast<int64_t>(q + 16) * p.incx);
      const float x3 = __ldg(p.x + static_cast<int64_t>(q + 24) * p.incx);
      acc.x = fmaf(v0.x, x0, acc.x); acc.y = fmaf(v0.y, x0, acc.y);
      acc.z = fmaf(v0.z, x0, acc.z); acc.w = fmaf(v0.w, x0, acc.w);
      acc1.x = fmaf(v1.x, x1, acc1.x); acc1.y = fmaf(v1.y, x1, acc1.y);
      acc1.z = fmaf(v1.z, x1, acc1.z); acc1.w = fmaf(v1.w, x1, acc1.w);
      acc.x = fmaf(v2.x, x2, acc.x); acc.y = fmaf(v2.y, x2, acc.y);
      acc.z = fmaf(v2.z, x2, acc.z); acc.w = fmaf(v2.w, x2, acc.w);
      acc1.x = fmaf(v3.x, x3, acc1.x); acc1.y = fmaf(v3.y, x3, acc1.y);
      acc1.z = fmaf(v3.z, x3, acc1.z); acc1.w = fmaf(v3.w, x3, acc1.w);
    }
    for (; q < qend; q += 8) {
      float4 v;
      if (VEC) {
        v = ldg_stream4(a + static_cast<int64_t>(q) * p.sq);
      } else {
        const float *c0 = a + static_cast<int64_t>(q) * p.sq;
        v = make_float4(ldg_stream(c0), ldg_stream(c0 + 32), ldg_stream(c0 + 64), ldg_stream(c0 + 96));
      }
      const float xv = __ldg(p.x + static_cast<int64_t>(q) * p.incx);
      acc.x = fmaf(v.x, xv, acc.x); acc.y = fmaf(v.y, xv, acc.y);
      acc.z = fmaf(v.z, xv, acc.z); acc.w = fmaf(v.w, xv, acc.w);
    }
    acc.x += acc1.x; acc.y += acc1.y; acc.z += acc1.z; acc.w += acc1.w;
  } else {
    // ragged last tile: element-wise with bounds checks
    float v[4] = {0.f, 0.f, 0.f, 0.f};
    for (int q = qbeg + warp; q < qend; q += 8) {
      const float xv = __ldg(p.x + static_cast<int64_t>(q) * p.incx);
      const float *col = p.A + static_cast<int64_t>(q) * p.sq;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int64_t rr = VEC ? myrow + j : myrow + 32 * j;
        if (rr < p.P) v[j] = fmaf(ldg_stream(col + rr), xv, v[j]);
      }
    }
    acc = make_float4(v[0], v[1], v[2], v[3]);
  }
  // combine the 8 warps: part[w][lane] holds this lane's 4 rows
  part[warp][lane] = acc;
  __syncthreads();
  if (threadIdx.x < kRows) {
    // thread i sums row slot i over warps in order 0..7
    const int slot_lane = VEC ? threadIdx.x >> 2 : threadIdx.x & 31;
    const int comp = VEC ? threadIdx.x & 3 : threadIdx.x >> 5;
    float s = 0.0f;
#pragma unroll
    for (int w = 0; w < kThreads / 32; ++w) {
      const float4 v = part[w][slot_lane];
      s += comp == 0 ? v.x : comp == 1 ? v.y : comp == 2 ? v.z : v.w;
    }
    // both lane-to-row maps give row offset == threadIdx.x for this slot
    sum[threadIdx.x] = s;
  }
  if (split > 1) {
    cluster_sync();
    // rank r finalises rows [r*len, (r+1)*len) of the tile, summing the
    // partials of ranks 0..split-1 in order
    const int len = (kRows + split - 1) / split;
    const int i = static_cast<int>(threadIdx.x);
    if (i < len) {
      const int roff = rank * len + i;
      if (roff < kRows) {
        const uint32_t base = smem_u32(&sum[roff]);
        float s = 0.0f;
        for (int r = 0; r < split; ++r) s += ld_dsmem(mapa_shared(base, r));
        const int64_t rr = row0 + roff;
        if (rr < p.P) {
          float *y = p.y + rr * p.incy;
          *y = axpby(p.alpha, s, p.beta, y);
        }
      }
    }
    cluster_sync();
  } else {
    __syncthreads();
    if (threadIdx.x < kRows) {
      const int64_t rr = row0 + threadIdx.x;
      if (rr < p.P) {
        float *y = p.y + rr * p.incy;
        *y = axpby(p.alpha, sum[threadIdx.x], p.beta, y);
      }
    }
  }
}

__global__ void scale_kernel(float *C, int M, int N, int64_t scm, int64_t scn, float beta) {
  const int64_t total = static_cast<int64_t>(M) * N;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t m = i % M, n = i / M;
    float *c = C + m * scm + n * scn;
    *c = beta == 0.0f ? 0.0f : beta * *c;
  }
}

template <int TPR>
hml_status run_rows(const GemvProblem &p, bool vec, cudaStream_t s) {
  constexpr int RPC = kThreads / TPR;
  const int64_t blocks = (static_cast<int64_t>(p.P) + RPC - 1) / RPC;
  if (blocks > 0x7fffffff) return HML_STATUS_NOT_SUPPORTED;
  count_launch();
  if (vec)
    gemv_rows_kernel<TPR, true><<<static_cast<unsigned>(blocks), kThreads, 0, s>>>(p);
  else
    gemv_rows_kernel<TPR, false><<<static_cast<unsigned>(blocks), kThreads, 0, s>>>(p);
  cudaError_t e = cudaGetLastError();
  note_cuda_error(e, "gemv_rows");
  return cuda_status(e);
}

bool aligned16(const void *ptr) { return (reinterpret_cast<uintptr_t>(ptr) & 15u) == 0; }

}  // namespace

// variant for the row kernel: threads per row (4..256), 0 = heuristic.
// variant for the column kernel: cluster split (1..8), 0 = heuristic.
hml_status launch_gemv(const GemvProblem &p, int variant, cudaStream_t s) {
  if (p.P == 0) return HML_STATUS_SUCCESS;
  if (p.sq != 1 && p.sp != 1) return HML_STATUS_NOT_SUPPORTED;
  if (p.sq == 1 && !(p.Q == 1 && p.sp == 1)) {
    const bool vec = aligned16(p.A) && (p.sp % 4 == 0 || p.P == 1) && p.incx == 1 &&
                     aligned16(p.x);
    int tpr = variant;
    if (tpr == 0) {
      // enough 16-byte loads per thread to keep 4 in flight, up to 128
      // (measured on B200, 32768 x 4096: 128 threads per row 6.37 TB/s,
      // 256 threads 6.23 TB/s)
      const int per_row4 = (p.Q + 3) / 4;
      tpr = 4;
      while (tpr < 128 && per_row4 / tpr > 16) tpr <<= 1;
    }
    switch (tpr) {
      case 4: return run_rows<4>(p, vec, s);
      case 8: return run_rows<8>(p, vec, s);
      case 16: return run_rows<16>(p, vec, s);
      case 32: return run_rows<32>(p, vec, s);
      case 64: return run_rows<64>(p, vec, s);
      case 128: return run_rows<128>(p, vec, s);
      case 256: return run_rows<256>(p, vec, s);
      default: return HML_STATUS_INVALID_VALUE;
    }
  }
  // columns contiguous
  const bool vec = aligned16(p.A) && (p.sq % 4 == 0 || p.Q == 1);
  const int64_t tiles = (static_cast<int64_t>(p.P) + 127) / 128;
  int split = variant;
  if (split == 0) {
    // aim for >= 4 CTAs per SM, each with >= 64 columns
    const int64_t want = 4 * static_cast<int64_t>(sm_count());
    split = static_cast<int>((want + tiles - 1) / tiles);
    split = max(1, min(split, 8));
    while (split > 1 && p.Q / split < 64) --split;
  }
  if (split < 1 || split > 8) return HML_STATUS_INVALID_VALUE;
  if (tiles * split > 0x7fffffff) return HML_STATUS_NOT_SUPPORTED;
  const dim3 grid(static_cast<unsigned>(tiles * split));
  cudaError_t e = vec ? launch_k(gemv_cols_kernel<true>, grid, dim3(kThreads), 0, s, split, p, split)
                      : launch_k(gemv_cols_kernel<false>, grid, dim3(kThreads), 0, s, split, p, split);
  note_cuda_error(e, "gemv_cols");
  return cuda_status(e);
}

hml_status launch_scale(float *C, int M, int N, int64_t scm, int64_t scn, float beta,
                        cudaStream_t s) {
  if (M == 0 || N == 0) return HML_STATUS_SUCCESS;
  const int64_t total = static_cast<int64_t>(M) * N;
  const int blocks = static_cast<int>(std::min<int64_t>((total + 255) / 256, 4 * 148 * 8));
  count_launch();
  scale_kernel<<<blocks, 256, 0, s>>>(C, M, N, scm, scn, beta);
  cudaError_t e = cudaGetLastError();
  note_cuda_error(e, "scale");
  return cuda_status(e);
}

}  // namespace hml
