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
//             scheduling.  Few long rows are split over several CTAs per
//             row (the reference's one CTA per row leaves most SMs idle).
//  gemv_cols  A(p,q) columns contiguous (sp == 1): column-major y = A x.
//             Each lane owns 4 consecutive rows (one 16-byte load per
//             column), the 8 warps of a CTA take 2 row groups x 4
//             interleaved column phases, and `split` CTAs take disjoint
//             column ranges of the same 256 rows.  Partial sums are combined
//             in a fixed order: the phases in shared memory, the split CTAs
//             through a per-stream workspace, summed in a fixed order
//             (fixed slices of the ranks, then the slices in order) by
//             whichever CTA of the tile finishes last (a per-tile arrival
//             counter, reset by that CTA), so results are deterministic.
//  gemv_short the same layout for P <= 128 with 16-byte loads: several
//             columns per warp so that every lane loads, one 128-row tile
//             split over up to 256 CTAs.
#include <algorithm>

#include "hml_device.cuh"
#include "hml_internal.h"
#include "hml_tune.h"

namespace hml {
namespace {

constexpr int kThreads = 256;

// ----------------------------------------------------------------- rows
// Sum of the TPR partial sums of each row of the CTA (threads r*TPR ..
// r*TPR+TPR-1); the result is valid in the row's thread t == 0.  The order
// is fixed: lanes by a shuffle tree, then the row's warps in index order.
template <int TPR, bool REUSE>
__device__ __forceinline__ float row_total(float acc, float *red, int r, int t) {
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
      if (REUSE) __syncthreads();  // red is read before anyone writes it again
    }
  } else {
#pragma unroll
    for (int o = TPR / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  }
  return acc;
}

// RPC = 256 / TPR rows per CTA, TPR threads per row.  With split > 1 (few
// long rows), `split` CTAs take disjoint ranges of the same rows' columns
// (whole float4 groups when VEC, the last rank also the Q % 4 tail) and
// publish per-rank row sums to `partial` ([split][P]); the last CTA of the
// row block to arrive (a per-block arrival counter, reset by that CTA) adds
// them up, rank j of a row summed by the row's thread j % TPR in rank order
// and the TPR results by the same tree as above, so results are
// deterministic.  SPLIT = false is the one-CTA-per-row-block form (split
// must be 1), compiled without the split bookkeeping (48 registers for the
// 16-byte form with 128 threads per row, 5 CTAs per SM, as before the split
// existed; 56 with it).
template <int TPR, bool VEC, bool SPLIT>
__global__ void __launch_bounds__(kThreads) gemv_rows_kernel(GemvProblem p, int split_arg,
                                                             float *partial, unsigned *arrivals) {
  constexpr int RPC = kThreads / TPR;  // rows per CTA
  __shared__ float red[kThreads / 32];
  __shared__ unsigned last;
  const int split = SPLIT ? split_arg : 1;
  const int t = threadIdx.x % TPR;
  const int r = threadIdx.x / TPR;
  const int rank = SPLIT ? static_cast<int>(blockIdx.x % split) : 0;
  const int64_t blk = SPLIT ? blockIdx.x / split : blockIdx.x;
  const int64_t row = blk * RPC + r;
  float acc = 0.0f;
  if (row < p.P) {
    const float *a = p.A + row * p.sp;
    if (VEC) {
      const int Q4 = p.Q >> 2;
      const int qc = (Q4 + split - 1) / split;
      const int qb = min(Q4, rank * qc), qe = min(Q4, qb + qc);
      const float4 *a4 = reinterpret_cast<const float4 *>(a);
      const float4 *x4 = reinterpret_cast<const float4 *>(p.x);
      float acc1 = 0.0f, acc2 = 0.0f, acc3 = 0.0f;
      int q = qb + t;
      for (; q + 3 * TPR < qe; q += 4 * TPR) {
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
      for (; q < qe; q += TPR) {
        float4 v = ldg_stream4(reinterpret_cast<const float *>(a4 + q));
        float4 w = __ldg(x4 + q);
        acc = fmaf(v.x, w.x, acc); acc = fmaf(v.y, w.y, acc);
        acc = fmaf(v.z, w.z, acc); acc = fmaf(v.w, w.w, acc);
      }
      acc += acc1 + (acc2 + acc3);
      const int qt = (Q4 << 2) + t;
      if (rank == split - 1 && t < (p.Q & 3)) acc = fmaf(a[qt], __ldg(p.x + qt), acc);
    } else {
      const int qc = (p.Q + split - 1) / split;
      const int64_t qb64 = static_cast<int64_t>(rank) * qc;
      const int qb = qb64 < p.Q ? static_cast<int>(qb64) : p.Q;
      const int qe = min(p.Q - qb, qc) + qb;
      float acc1 = 0.0f;
      int q = qb + t;
      for (; q + TPR < qe; q += 2 * TPR) {
        acc = fmaf(ldg_stream(a + q), __ldg(p.x + q * p.incx), acc);
        acc1 = fmaf(ldg_stream(a + q + TPR), __ldg(p.x + (q + TPR) * p.incx), acc1);
      }
      if (q < qe) acc = fmaf(ldg_stream(a + q), __ldg(p.x + q * p.incx), acc);
      acc += acc1;
    }
  }
  acc = row_total<TPR, SPLIT>(acc, red, r, t);
  if (!SPLIT) {
    if (t == 0 && row < p.P) {
      float *y = p.y + row * p.incy;
      *y = axpby(p.alpha, acc, p.beta, y);
    }
    return;
  }
  // publish this rank's row sums; the block's last CTA to arrive adds them
  if (t == 0 && row < p.P) __stcg(partial + static_cast<int64_t>(rank) * p.P + row, acc);
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(&arrivals[blk], 1u) == static_cast<unsigned>(split - 1);
  __syncthreads();
  if (!last) return;
  __threadfence();
  float s = 0.0f;
  if (row < p.P)
    for (int j = t; j < split; j += TPR) s += __ldcg(partial + static_cast<int64_t>(j) * p.P + row);
  s = row_total<TPR, false>(s, red, r, t);
  if (t == 0 && row < p.P) {
    float *y = p.y + row * p.incy;
    *y = axpby(p.alpha, s, p.beta, y);
  }
  if (threadIdx.x == 0) arrivals[blk] = 0u;  // ready for the next call
}

// ----------------------------------------------------------------- cols
// A CTA covers a tile of kColRows = 256 rows: warp w takes row group w & 1
// (128 rows) and column phase w >> 1 (columns qbeg + phase, + 4, + 8, ...).
// NARROW (P <= 128, a single 128-row tile): all 8 warps take the one row
// group, in 8 column phases.  VEC: lane owns rows group_base + 4*lane .. +3
// (16-byte loads); else rows group_base + lane + 32*j for j < 4; a lane
// whose rows all lie past P does no loads.  Eight columns are loaded before
// any is used, and registers are capped at 32 so that 8 CTAs fit on an SM
// (measured on B200, 32768 x 4096, split 8: 6.6 TB/s; with 48 registers and
// 5 CTAs per SM 6.1 TB/s; the earlier 128-row CTAs with 4 loads in flight
// reduced through cluster shared memory 5.3 TB/s).
constexpr int kColRows = 256;
constexpr int kColUnroll = 8;
constexpr int kMaxColSplit = kGemvMaxColSplit;
static_assert(kColRows == kThreads, "thread i finalises row i of the tile");

// End of a column-kernel CTA: sum[i] holds this CTA's sum for row i of its
// tile.  split == 1: write y.  Otherwise publish the partial ([tile][rank]
// [kTileRows] in the workspace); the tile's last CTA to arrive sums the
// split partials with 16-byte loads: thread i adds 4 rows (quad i % QUADS)
// over the ranks k = slice, slice + SLICES, ... in order, and the SLICES
// sums of a row are then added in slice order through shared memory
// (`flat`, 256 float4), so results are deterministic.
template <int kTileRows>
__device__ __forceinline__ void finish_tile(const GemvProblem &p, int64_t tile, int rank, int split,
                                            float *partial, unsigned *arrivals, const float *sum,
                                            float4 *flat, unsigned *last) {
  const int64_t rr = tile * kTileRows + threadIdx.x;
  if (split == 1) {
    __syncthreads();
    if (threadIdx.x < kTileRows && rr < p.P) {
      float *y = p.y + rr * p.incy;
      *y = axpby(p.alpha, sum[threadIdx.x], p.beta, y);
    }
    return;
  }
  float *tp = partial + tile * split * kTileRows;
  if (threadIdx.x < kTileRows) __stcg(tp + rank * kTileRows + threadIdx.x, sum[threadIdx.x]);
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) *last = atomicAdd(&arrivals[tile], 1u) == static_cast<unsigned>(split - 1);
  __syncthreads();
  if (!*last) return;
  __threadfence();
  constexpr int QUADS = kTileRows / 4, SLICES = kThreads / QUADS;
  const int quad = static_cast<int>(threadIdx.x) % QUADS;
  const int slice = static_cast<int>(threadIdx.x) / QUADS;
  float4 t4 = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll 8
  for (int k = slice; k < split; k += SLICES) {
    const float4 v = __ldcg(reinterpret_cast<const float4 *>(tp + k * kTileRows) + quad);
    t4.x += v.x; t4.y += v.y; t4.z += v.z; t4.w += v.w;
  }
  flat[slice * QUADS + quad] = t4;
  __syncthreads();
  if (threadIdx.x < kTileRows && rr < p.P) {
    const int q = static_cast<int>(threadIdx.x) >> 2, c = threadIdx.x & 3;
    float total = 0.0f;
#pragma unroll
    for (int sl = 0; sl < SLICES; ++sl) {
      const float4 v = flat[sl * QUADS + q];
      total += c == 0 ? v.x : c == 1 ? v.y : c == 2 ? v.z : v.w;
    }
    float *y = p.y + rr * p.incy;
    *y = axpby(p.alpha, total, p.beta, y);
  }
  if (threadIdx.x == 0) arrivals[tile] = 0u;  // ready for the next call
}

template <bool VEC, bool NARROW>
__global__ void __launch_bounds__(kThreads, 8) gemv_cols_kernel(GemvProblem p, int split,
                                                             float *partial, unsigned *arrivals) {
  constexpr int kTileRows = NARROW ? 128 : kColRows;
  constexpr int S = NARROW ? kThreads / 32 : kThreads / 32 / 2;  // column phases
  __shared__ float4 part[kThreads / 32][32];
  __shared__ float sum[kColRows];
  __shared__ unsigned last;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int group = NARROW ? 0 : warp & 1, phase = NARROW ? warp : warp >> 1;
  const int rank = static_cast<int>(blockIdx.x % split);
  const int64_t tile = blockIdx.x / split;
  const int64_t row0 = tile * kTileRows;
  const int64_t gbase = row0 + group * 128;
  const int qc = (p.Q + split - 1) / split;
  const int64_t qbeg64 = static_cast<int64_t>(rank) * qc;
  const int qbeg = qbeg64 < p.Q ? static_cast<int>(qbeg64) : p.Q;
  const int qend = min(p.Q - qbeg, qc) + qbeg;

  float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
  const int64_t myrow = VEC ? gbase + 4 * lane : gbase + lane;
  const bool full = VEC ? (myrow + 3 < p.P) : (gbase + 128 <= p.P);
  if (full) {
    const float *a = p.A + myrow;
    float4 acc1 = make_float4(0.f, 0.f, 0.f, 0.f);
    int q = qbeg + phase;
    const int64_t astep = static_cast<int64_t>(S) * p.sq, xstep = static_cast<int64_t>(S) * p.incx;
    const float *ac = a + static_cast<int64_t>(q) * p.sq;
    const float *xc = p.x + static_cast<int64_t>(q) * p.incx;
    for (; q + (kColUnroll - 1) * S < qend;
         q += kColUnroll * S, ac += kColUnroll * astep, xc += kColUnroll * xstep) {
      float4 v[kColUnroll];
#pragma unroll
      for (int u = 0; u < kColUnroll; ++u) {
        const float *c = ac + u * astep;
        v[u] = VEC ? ldg_stream4(c)
                   : make_float4(ldg_stream(c), ldg_stream(c + 32), ldg_stream(c + 64),
                                 ldg_stream(c + 96));
      }
#pragma unroll
      for (int u = 0; u < kColUnroll; u += 2) {
        const float x0 = __ldg(xc + u * xstep);
        const float x1 = __ldg(xc + (u + 1) * xstep);
        acc.x = fmaf(v[u].x, x0, acc.x); acc.y = fmaf(v[u].y, x0, acc.y);
        acc.z = fmaf(v[u].z, x0, acc.z); acc.w = fmaf(v[u].w, x0, acc.w);
        acc1.x = fmaf(v[u + 1].x, x1, acc1.x); acc1.y = fmaf(v[u + 1].y, x1, acc1.y);
        acc1.z = fmaf(v[u + 1].z, x1, acc1.z); acc1.w = fmaf(v[u + 1].w, x1, acc1.w);
      }
    }
    for (; q < qend; q += S) {
      const float *c = a + static_cast<int64_t>(q) * p.sq;
      const float4 v = VEC ? ldg_stream4(c)
                           : make_float4(ldg_stream(c), ldg_stream(c + 32), ldg_stream(c + 64),
                                         ldg_stream(c + 96));
      const float xv = __ldg(p.x + static_cast<int64_t>(q) * p.incx);
      acc.x = fmaf(v.x, xv, acc.x); acc.y = fmaf(v.y, xv, acc.y);
      acc.z = fmaf(v.z, xv, acc.z); acc.w = fmaf(v.w, xv, acc.w);
    }
    acc.x += acc1.x; acc.y += acc1.y; acc.z += acc1.z; acc.w += acc1.w;
  } else if (myrow < p.P) {
    // ragged last tile: element-wise with bounds checks
    float v[4] = {0.f, 0.f, 0.f, 0.f};
    for (int q = qbeg + phase; q < qend; q += S) {
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
  // combine the column phases: part[w][lane] holds this lane's 4 rows
  part[warp][lane] = acc;
  __syncthreads();
  if (threadIdx.x < kTileRows) {
    // thread i owns row offset i of the tile: group i / 128, and within the
    // group the lane slot / component that holds it; phases summed in order
    const int i = static_cast<int>(threadIdx.x);
    const int g = i >> 7, r = i & 127;
    const int slot_lane = VEC ? r >> 2 : r & 31;
    const int comp = VEC ? r & 3 : r >> 5;
    float s = 0.0f;
#pragma unroll
    for (int ph = 0; ph < S; ++ph) {
      const float4 v = part[NARROW ? ph : 2 * ph + g][slot_lane];
      s += comp == 0 ? v.x : comp == 1 ? v.y : comp == 2 ? v.z : v.w;
    }
    sum[i] = s;
  }
  finish_tile<kTileRows>(p, tile, rank, split, partial, arrivals, sum, &part[0][0], &last);
}

// Short results (P <= 128) with 16-byte loads: LPC lanes share a column
// (LPC = the power of two >= ceil(P / 4); lane l takes the 4 rows of quad
// l % LPC in column slot l / LPC), so a warp covers 32 / LPC columns per
// step and every lane loads; the 8 warps take interleaved column slots, 8
// steps loaded before any is used.  The column slots of a warp are added by
// a fixed shuffle tree, the warps in index order through shared memory;
// `split` CTAs take column ranges and finish as the column kernel does.
// A single tile runs at most 256 CTAs (under 2 per SM), so registers are
// not capped for occupancy: 16 columns per lane are loaded before any is
// used, twice the column kernel's, to halve the memory round trips of a
// CTA's short column range.
constexpr int kShortUnroll = 16;
template <int LPC>
__global__ void __launch_bounds__(kThreads, 2) gemv_short_kernel(GemvProblem p, int split,
                                                              float *partial, unsigned *arrivals) {
  constexpr int kTileRows = 128;
  constexpr int CPW = 32 / LPC;                // column slots per warp
  constexpr int CS = CPW * (kThreads / 32);    // columns per CTA step
  __shared__ float4 part[kThreads / 32][32];
  __shared__ float sum[kColRows];
  __shared__ unsigned last;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int quad = lane % LPC, slot = lane / LPC;
  const int rank = static_cast<int>(blockIdx.x);  // a single row tile
  const int qc = (p.Q + split - 1) / split;
  const int64_t qbeg64 = static_cast<int64_t>(rank) * qc;
  const int qbeg = qbeg64 < p.Q ? static_cast<int>(qbeg64) : p.Q;
  const int qend = min(p.Q - qbeg, qc) + qbeg;
  const int row = 4 * quad;
  const int first = qbeg + warp * CPW + slot;  // this lane's first column

  float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
  if (row + 3 < p.P) {
    float4 acc1 = make_float4(0.f, 0.f, 0.f, 0.f);
    const int64_t astep = static_cast<int64_t>(CS) * p.sq, xstep = static_cast<int64_t>(CS) * p.incx;
    int q = first;
    const float *ac = p.A + row + static_cast<int64_t>(q) * p.sq;
    const float *xc = p.x + static_cast<int64_t>(q) * p.incx;
    for (; q + (kShortUnroll - 1) * CS < qend;
         q += kShortUnroll * CS, ac += kShortUnroll * astep, xc += kShortUnroll * xstep) {
      float4 v[kShortUnroll];
#pragma unroll
      for (int u = 0; u < kShortUnroll; ++u) v[u] = ldg_stream4(ac + u * astep);
#pragma unroll
      for (int u = 0; u < kShortUnroll; u += 2) {
        const float x0 = __ldg(xc + u * xstep);
        const float x1 = __ldg(xc + (u + 1) * xstep);
        acc.x = fmaf(v[u].x, x0, acc.x); acc.y = fmaf(v[u].y, x0, acc.y);
        acc.z = fmaf(v[u].z, x0, acc.z); acc.w = fmaf(v[u].w, x0, acc.w);
        acc1.x = fmaf(v[u + 1].x, x1, acc1.x); acc1.y = fmaf(v[u + 1].y, x1, acc1.y);
        acc1.z = fmaf(v[u + 1].z, x1, acc1.z); acc1.w = fmaf(v[u + 1].w, x1, acc1.w);
      }
    }
    for (; q < qend; q += CS) {
      const float4 v = ldg_stream4(p.A + row + static_cast<int64_t>(q) * p.sq);
      const float xv = __ldg(p.x + static_cast<int64_t>(q) * p.incx);
      acc.x = fmaf(v.x, xv, acc.x); acc.y = fmaf(v.y, xv, acc.y);
      acc.z = fmaf(v.z, xv, acc.z); acc.w = fmaf(v.w, xv, acc.w);
    }
    acc.x += acc1.x; acc.y += acc1.y; acc.z += acc1.z; acc.w += acc1.w;
  } else if (row < p.P) {
    // the last, partial quad: element-wise (a 16-byte load could pass the
    // end of the last column)
    float v[4] = {0.f, 0.f, 0.f, 0.f};
    for (int q = first; q < qend; q += CS) {
      const float xv = __ldg(p.x + static_cast<int64_t>(q) * p.incx);
      const float *col = p.A + static_cast<int64_t>(q) * p.sq;
#pragma unroll
      for (int j = 0; j < 4; ++j)
        if (row + j < p.P) v[j] = fmaf(ldg_stream(col + row + j), xv, v[j]);
    }
    acc = make_float4(v[0], v[1], v[2], v[3]);
  }
  // column slots of the warp: lanes quad, quad + LPC, ... (xor over the
  // slot bits, fixed order)
#pragma unroll
  for (int o = 16; o >= LPC; o >>= 1) {
    acc.x += __shfl_xor_sync(0xffffffffu, acc.x, o);
    acc.y += __shfl_xor_sync(0xffffffffu, acc.y, o);
    acc.z += __shfl_xor_sync(0xffffffffu, acc.z, o);
    acc.w += __shfl_xor_sync(0xffffffffu, acc.w, o);
  }
  if (lane < LPC) part[warp][lane] = acc;
  __syncthreads();
  if (threadIdx.x < kTileRows) {
    const int i = static_cast<int>(threadIdx.x), qd = i >> 2, c = i & 3;
    float sv = 0.0f;
    if (qd < LPC) {
#pragma unroll
      for (int w = 0; w < kThreads / 32; ++w) {
        const float4 v = part[w][qd];
        sv += c == 0 ? v.x : c == 1 ? v.y : c == 2 ? v.z : v.w;
      }
    }
    sum[i] = sv;
  }
  finish_tile<kTileRows>(p, 0, rank, split, partial, arrivals, sum, &part[0][0], &last);
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

// Few long rows: the columns of each row are split over several CTAs so
// that about 7/8 of the CTAs that fit on the GPU at once (8 per SM) run,
// each thread keeping at least 8 float4 of its row (measured on B200,
// 64 x 200000: one CTA per row 65.7 us).
constexpr int kMaxRowSplit = 64;

template <int TPR>
hml_status run_rows(const GemvProblem &p, bool vec, cudaStream_t s) {
  constexpr int RPC = kThreads / TPR;
  const int64_t blocks = (static_cast<int64_t>(p.P) + RPC - 1) / RPC;
  if (blocks > 0x7fffffff) return HML_STATUS_NOT_SUPPORTED;
  int split = 1;
  const int64_t want = static_cast<int64_t>(sm_count()) * 8 * 7 / 8;
  if (blocks < want) {
    split = static_cast<int>(std::min<int64_t>(kMaxRowSplit, want / blocks));
    while (split > 1 && p.Q / (static_cast<int64_t>(split) * TPR * 4) < 8) --split;
  }
  float *partial = nullptr;
  unsigned *arrivals = nullptr;
  if (split > 1) {
    void *ws = nullptr;
    hml_status st = workspace(static_cast<size_t>(split) * p.P * sizeof(float), s, &ws);
    if (st != HML_STATUS_SUCCESS) return st;
    st = tile_counters(static_cast<size_t>(blocks), s, &arrivals);
    if (st != HML_STATUS_SUCCESS) return st;
    partial = static_cast<float *>(ws);
  }
  const dim3 grid(static_cast<unsigned>(blocks * split));
  auto kernel = vec ? (split > 1 ? gemv_rows_kernel<TPR, true, true>
                                  : gemv_rows_kernel<TPR, true, false>)
                    : (split > 1 ? gemv_rows_kernel<TPR, false, true>
                                 : gemv_rows_kernel<TPR, false, false>);
  cudaError_t e = launch_k(kernel, grid, dim3(kThreads), 0, s, 1, p, split, partial, arrivals);
  note_cuda_error(e, "gemv_rows");
  return cuda_status(e);
}

bool aligned16(const void *ptr) { return (reinterpret_cast<uintptr_t>(ptr) & 15u) == 0; }

}  // namespace

// variant for the row kernel: threads per row (4..256), 0 = heuristic (the
// split of long rows over CTAs is always the heuristic's).  variant for the
// column kernel: CTAs per row tile along the columns (1..256), 0 =
// heuristic.  kGemvTuned: the measured table's variant for this shape when
// it holds one, else the heuristic.
hml_status launch_gemv(const GemvProblem &p, int variant, cudaStream_t s) {
  if (p.P == 0) return HML_STATUS_SUCCESS;
  if (p.sq != 1 && p.sp != 1) return HML_STATUS_NOT_SUPPORTED;
  if (variant == kGemvTuned) {
    int v = 0;
    variant = gemv_tuned_lookup(p, &v) && gemv_variant_valid(gemv_rows_layout(p), v) ? v : 0;
  }
  if (gemv_rows_layout(p)) {
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
  const bool narrow = p.P <= 128;
  const int tile_rows = narrow ? 128 : kColRows;
  const int64_t tiles = (static_cast<int64_t>(p.P) + tile_rows - 1) / tile_rows;
  int split = variant;
  if (split == 0) {
    // about 7/8 of the CTAs that fit on the GPU at once, in one wave
    // (measured on B200, 32768 x 4096, 8 CTAs per SM resident: split 8 =
    // 1024 CTAs 6.6 TB/s, split 9 = 1152 CTAs 5.9 TB/s, split 10 (a second
    // wave) 5.3 TB/s), each with >= 64 columns; few row tiles take up to
    // kMaxColSplit CTAs each
    static const int per_sm = [] {
      int n = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, gemv_cols_kernel<true, false>,
                                                        kThreads, 0) != cudaSuccess ||
          n < 1)
        n = 1;
      return n;
    }();
    // (one 128-row tile of a short result may take up to 256 CTAs, a wider
    // tile 128: the tile's last CTA reads split x rows partials)
    const int64_t resident = static_cast<int64_t>(per_sm) * sm_count() * 7 / 8;
    const int cap = narrow ? kMaxColSplit : kMaxColSplit / 2;
    split = static_cast<int>(std::min<int64_t>(cap, resident / tiles));
    split = max(1, split);
    while (split > 1 && p.Q / split < 64) --split;
  }
  if (split < 1 || split > kMaxColSplit) return HML_STATUS_INVALID_VALUE;
  if (tiles * split > 0x7fffffff) return HML_STATUS_NOT_SUPPORTED;
  float *partial = nullptr;
  unsigned *arrivals = nullptr;
  if (split > 1) {
    void *ws = nullptr;
    hml_status st = workspace(static_cast<size_t>(tiles) * split * tile_rows * sizeof(float), s,
                              &ws);
    if (st != HML_STATUS_SUCCESS) return st;
    st = tile_counters(static_cast<size_t>(tiles), s, &arrivals);
    if (st != HML_STATUS_SUCCESS) return st;
    partial = static_cast<float *>(ws);
  }
  const dim3 grid(static_cast<unsigned>(tiles * split));
  auto kernel = vec ? (narrow ? gemv_cols_kernel<true, true> : gemv_cols_kernel<true, false>)
                    : (narrow ? gemv_cols_kernel<false, true> : gemv_cols_kernel<false, false>);
  if (vec && narrow) {
    // every lane on columns: LPC lanes per column, LPC >= ceil(P / 4)
    const int p4 = (p.P + 3) / 4;
    kernel = p4 <= 1   ? gemv_short_kernel<1>
             : p4 <= 2 ? gemv_short_kernel<2>
             : p4 <= 4 ? gemv_short_kernel<4>
             : p4 <= 8 ? gemv_short_kernel<8>
             : p4 <= 16 ? gemv_short_kernel<16>
                        : gemv_short_kernel<32>;
  }
  cudaError_t e = launch_k(kernel, grid, dim3(kThreads), 0, s, 1, p, split, partial, arrivals);
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
