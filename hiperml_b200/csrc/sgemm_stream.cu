// sgemm_stream.cu -- FP32 SIMT SGEMM for the bandwidth-bound skinny shapes
// with contiguous columns of A (column-major C = A * B, or C^T = B^T A^T
// row-major) and few columns of C (N <= 8).
//
// The work is A's 128-row strips x 32-column blocks ("units", one 16 KB TMA
// box each), and every CTA takes one contiguous, equally long range of the
// units in strip-major order (stream-K): all SMs stream A from HBM for the
// whole kernel, with no tail of idle SMs whatever M and K are.
//
// Structure of one CTA (2 per SM):
//   * warp 8, one lane: TMA of each unit's A box (128 x 32 FP32, column
//     after column) and of the matching 32 rows of B (N-contiguous: a
//     K-contiguous B is first copied so by gather_b_kernel, launched just
//     before, this kernel being its programmatic dependent) into a ring of
//     `stages` shared-memory slots;
//     a slot is refilled once the 8 consumer warps have released it.  (With
//     the loads issued by a consumer lane instead, that warp waits for the
//     slowest one before each refill, and the last warp to release a slot
//     issuing its refill was no better: both measured 1.3x slower on B200.)
//   * warps 0..7 ("column phases"): warp w takes the box's columns 4w ..
//     4w + 3; a lane owns 4 consecutive rows (one 16-byte shared-memory load
//     per column) and all NB columns of C for them, the values of B read as
//     16-byte shared-memory broadcasts.
//   * at the end of each strip in the range: the 8 phases are summed in
//     order in shared memory.  A strip owned by one CTA is written to C
//     (alpha, beta applied; beta == 0 does not read C).  A strip shared by
//     several CTAs (at most at the two ends of a range) is written to that
//     CTA's slot of a per-stream workspace; the CTA of the strip that
//     arrives last (a per-strip counter, which it resets) sums the slots in
//     CTA order and writes C.  Results are deterministic.  This epilogue
//     is inlined.  Built as a separate __noinline__ function (the same code,
//     with the named barrier in its non-aligned form) it gives wrong and
//     run-to-run different results on B200 in 3 of the 18 stream-kernel
//     tests, while the inlined build passes all of them bitwise-repeatably;
//     the cause was not found by reading (barrier participation, the reuse
//     of `red` and `s_last` across strips and the workspace hand-off check
//     out), so the function stays inlined.
//
// Measured on B200 (M = 65536, K = 4096, column-major A, 4 stages): N = 8
// 180 us with N-contiguous B (6.0 TB/s of A), and 194 us streaming a
// K-contiguous B as stored (before the copy), against 220 us for the tiled
// SIMT kernel; N = 4 165 us (6.5 TB/s).  The packed FMAs took N = 8 from 214 to 194 us: the kernel
// is bound by instruction issue as much as by HBM.  Reading B through the L1
// cache (LDG broadcasts) instead of staging it in shared memory capped the
// same structure at 5.0 TB/s with either B.  For 8 < N <= 16 the 64
// accumulators a thread cost the second CTA on each SM, and the split-BF16
// tensor-core kernel is faster there (an NB = 16 instantiation at one CTA
// per SM, measured: 4096 x 16 x 4096 with L2 flushed 58 us against 29.7 us,
// 65536 x 16 x 4096 320 us against 336 us, i.e. A at 3.4 TB/s).
#include <algorithm>
#include <cstring>

#include "hml_device.cuh"
#include "hml_internal.h"

namespace hml {
namespace {

constexpr int kSRows = 128;                  // rows of A per strip
constexpr int kSCols = 32;                   // columns of A per unit
constexpr int kSPhases = 8;                  // consumer warps, one column phase each
constexpr int kSThreads = 32 * (kSPhases + 1);  // + the TMA producer warp
constexpr int kMaxStreamStages = 8;
// CTAs per SM.  Registers are allocated per SM sub-partition (4 x 16K): the
// 18 warps of 2 CTAs put 5 warps on one and cap registers at 96 a thread,
// enough for the 4 x NB accumulators of a lane up to NB = 8.
constexpr int kSCtasPerSm = 2;
constexpr int kStreamNb[] = {4, 8};
constexpr int kNumStreamNb = 2;

struct StreamArgs {
  GemmProblem p;
  int kblocks;          // units per strip
  long long units;      // strips * kblocks
  int stages;
  float *partial;       // [gridDim.x][2][kSRows * NB]
  unsigned *arrivals;   // [strips], zero between calls
  int *err;
};

// First unit of CTA c's range: ranges are [begin(c), begin(c + 1)).
__device__ __forceinline__ long long range_begin(long long c, long long units, int ctas) {
  return c * units / ctas;
}

// The CTA whose range holds unit u (the last c with range_begin(c) <= u).
__device__ __forceinline__ int unit_owner(long long u, long long units, int ctas) {
  return static_cast<int>(((u + 1) * ctas - 1) / units);
}

// A lane's accumulators: rows j = 0..3 of its 4, columns of C in pairs
// (acc[j][h] = columns 2h, 2h + 1), updated with sm_100's packed FP32 FMA
// (fma.rn.f32x2): each half is rounded exactly as the scalar fma.rn, so the
// sums are bitwise those of scalar FMAs in the same order, with half the
// FMA instructions issued.
template <int NB>
__device__ __forceinline__ void zero_acc(float2 (&acc)[4][NB / 2]) {
#pragma unroll
  for (int j = 0; j < 4; ++j)
#pragma unroll
    for (int h = 0; h < NB / 2; ++h) acc[j][h] = make_float2(0.0f, 0.0f);
}

// acc[j][*] += a.j * (b pairs), j = 0..3 for the four components of a
template <int NB>
__device__ __forceinline__ void fma_rows(float2 (&acc)[4][NB / 2], float4 a, int h, float2 b) {
  acc[0][h] = __ffma2_rn(make_float2(a.x, a.x), b, acc[0][h]);
  acc[1][h] = __ffma2_rn(make_float2(a.y, a.y), b, acc[1][h]);
  acc[2][h] = __ffma2_rn(make_float2(a.z, a.z), b, acc[2][h]);
  acc[3][h] = __ffma2_rn(make_float2(a.w, a.w), b, acc[3][h]);
}

// Returns only once every accumulator holds its value, i.e. once every
// shared-memory load feeding it has returned: a slot may be released only
// after that, as __syncwarp does not wait for other lanes' loads and the
// compiler may otherwise sink the FMAs (and so the loads' completion) past
// the release.
template <int NB>
__device__ __forceinline__ void loads_consumed(const float2 (&acc)[4][NB / 2]) {
#pragma unroll
  for (int j = 0; j < 4; ++j)
#pragma unroll
    for (int h = 0; h < NB / 2; ++h) asm volatile("" ::"f"(acc[j][h].x), "f"(acc[j][h].y));
}

// Named barrier 1 over the 8 consumer warps.  The non-aligned form:
// barrier.sync.aligned (what bar.sync means) requires every thread of a warp
// to execute the same barrier instruction together, which the epilogue's
// one-thread branches (tid == 0) do not promise by themselves; the
// non-aligned form is defined for threads that arrive separately.
__device__ __forceinline__ void consumers_sync() {
  asm volatile("barrier.sync 1, %0;" ::"n"(kSPhases * 32) : "memory");
}

// End of this CTA's segment of `strip`, after every warp has stashed its
// accumulators in `red` ([phase][row][n]): the 8 column phases are summed
// in order; a strip owned by this CTA alone goes to C, a shared one through
// the CTA's workspace slot to whichever CTA of the strip arrives last, which
// sums the slots of CTAs owner0..owner1 in that order.
template <int NB>
__device__ __forceinline__ void finish_strip(const StreamArgs &args, int strip, int cta, int ctas,
                                          int first_strip, int tid, const float *red,
                                          unsigned *s_last) {
  const GemmProblem &p = args.p;
  const long long units = args.units;
  const int kblocks = args.kblocks;
  const long long first_unit = static_cast<long long>(strip) * kblocks;
  const int owner0 = unit_owner(first_unit, units, ctas);
  const int owner1 = unit_owner(first_unit + kblocks - 1, units, ctas);
  const bool shared = owner0 != owner1;
  const int64_t row0 = static_cast<int64_t>(strip) * kSRows;
  // this CTA's slot: 0 for the first strip of its range, 1 for the last
  float *mine = args.partial +
                (static_cast<int64_t>(cta) * 2 + (strip == first_strip ? 0 : 1)) * (kSRows * NB);
  for (int e = tid; e < kSRows * NB; e += kSPhases * 32) {
    float sum = 0.0f;
#pragma unroll
    for (int ph = 0; ph < kSPhases; ++ph) sum += red[ph * kSRows * NB + e];
    if (shared) {
      __stcg(mine + e, sum);
    } else {
      const int r = e / NB, n = e % NB;
      if (row0 + r < p.M && n < p.N) {
        float *cp = p.C + (row0 + r) * p.scm + static_cast<int64_t>(n) * p.scn;
        *cp = axpby(p.alpha, sum, p.beta, cp);
      }
    }
  }
  if (shared) {
    __threadfence();
    consumers_sync();
    if (tid == 0)
      *s_last = atomicAdd(&args.arrivals[strip], 1u) == static_cast<unsigned>(owner1 - owner0);
    consumers_sync();
    if (*s_last) {
      __threadfence();
      for (int e = tid; e < kSRows * NB; e += kSPhases * 32) {
        float sum = 0.0f;
        for (int c = owner0; c <= owner1; ++c) {
          const int cs =
              (strip == static_cast<int>(range_begin(c, units, ctas) / kblocks)) ? 0 : 1;
          sum += __ldcg(args.partial + (static_cast<int64_t>(c) * 2 + cs) * (kSRows * NB) + e);
        }
        const int r = e / NB, n = e % NB;
        if (row0 + r < p.M && n < p.N) {
          float *cp = p.C + (row0 + r) * p.scm + static_cast<int64_t>(n) * p.scn;
          *cp = axpby(p.alpha, sum, p.beta, cp);
        }
      }
      if (tid == 0) args.arrivals[strip] = 0u;  // ready for the next call
    }
  }
  consumers_sync();  // red and s_last are rewritten at the next strip end
}

template <int NB>
__global__ void __launch_bounds__(kSThreads, kSCtasPerSm)
    stream_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                  const __grid_constant__ StreamArgs args) {
  constexpr int A_BYTES = kSRows * kSCols * 4;
  constexpr int B_BYTES = kSCols * NB * 4;
  constexpr int STAGE = A_BYTES + B_BYTES;  // a multiple of 128 bytes
  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = align_shared(smem_raw, 1024);
  const int stages = args.stages;
  float *red = reinterpret_cast<float *>(smem + stages * STAGE);  // [phase][row][NB]
  uint64_t *full = reinterpret_cast<uint64_t *>(red + kSPhases * kSRows * NB);
  uint64_t *empty = full + stages;
  __shared__ unsigned s_last;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ctas = static_cast<int>(gridDim.x);
  const int cta = static_cast<int>(blockIdx.x);
  const long long units = args.units;
  const int kblocks = args.kblocks;
  const long long u0 = range_begin(cta, units, ctas);
  const int nunits = static_cast<int>(range_begin(cta + 1, units, ctas) - u0);
  // (strip, block) of the range's first unit; later units follow by a
  // cursor, without 64-bit divisions
  const int strip0 = static_cast<int>(u0 / kblocks);
  const int kb0 = static_cast<int>(u0 - static_cast<long long>(strip0) * kblocks);

  if (threadIdx.x == 0) {
    for (int s = 0; s < stages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kSPhases);
    }
    fence_mbar_init();
    prefetch_tmap(&tmA);
    prefetch_tmap(&tmB);
  }
  __syncthreads();

  // TMA of unit j of the range (at strip, block kb) into slot j % stages
  auto issue = [&](int j, int strip, int kb) {
    const int s = j % stages;
    const int k0 = kb * kSCols;
    uint8_t *dst = smem + s * STAGE;
    mbar_arrive_expect_tx(&full[s], STAGE);
    tma_load_2d(dst, &tmA, &full[s], strip * kSRows, k0);
    tma_load_2d(dst + A_BYTES, &tmB, &full[s], 0, k0);
  };
  if (warp == kSPhases) {
    // ------------------------------------------------------------ producer
    if (lane == 0) {
      // B may be a copy written by the kernel launched just before this one
      // (a programmatic dependent launch); A and C do not depend on it
      wait_prior_grid();
      int strip = strip0, kb = kb0, j = 0;
      for (; j < nunits; ++j) {
        const int s = j % stages;
        if (j >= stages &&
            !mbar_wait(&empty[s], ((j / stages) - 1) & 1, args.err, kDevErrEmptyBarrier))
          break;
        issue(j, strip, kb);
        if (++kb == kblocks) {
          kb = 0;
          ++strip;
        }
      }
      // every box issued has landed before the CTA may exit
      for (int i = max(0, j - stages); i < j; ++i)
        mbar_wait(&full[i % stages], (i / stages) & 1, args.err, kDevErrFullBarrier);
    }
    return;
  }

  // -------------------------------------------------------------- consumers
  const int phase = warp;
  const int tid = static_cast<int>(threadIdx.x);  // 0..255
  float2 acc[4][NB / 2];
  zero_acc<NB>(acc);
  bool bad = false;  // after an expired wait: no more waits, same barriers
  int strip = strip0, kb = kb0;
  for (int it = 0; it < nunits; ++it) {
    const int s = it % stages;
    if (!bad && !mbar_wait(&full[s], (it / stages) & 1, args.err, kDevErrFullBarrier)) bad = true;
    const float *ta = reinterpret_cast<const float *>(smem + s * STAGE);
    const float *tb = reinterpret_cast<const float *>(smem + s * STAGE + A_BYTES);
    {
      // B box stored [k][n]: this warp's 4 consecutive columns, NB / 4
      // vector broadcasts each
      constexpr int CW = kSCols / kSPhases;
      const int c0 = phase * CW;
#pragma unroll
      for (int q = 0; q < CW; ++q) {
        const float4 v = *reinterpret_cast<const float4 *>(ta + (c0 + q) * kSRows + lane * 4);
#pragma unroll
        for (int n4 = 0; n4 < NB; n4 += 4) {
          const float4 b4 = *reinterpret_cast<const float4 *>(tb + (c0 + q) * NB + n4);
          fma_rows<NB>(acc, v, n4 / 2, make_float2(b4.x, b4.y));
          fma_rows<NB>(acc, v, n4 / 2 + 1, make_float2(b4.z, b4.w));
        }
      }
    }
    // release the slot once every load from it has returned
    loads_consumed<NB>(acc);
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s]);

    const int cur = strip;
    const bool strip_end = ++kb == kblocks;
    if (strip_end) {
      kb = 0;
      ++strip;
    }
    if (!strip_end && it + 1 != nunits) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int n4 = 0; n4 < NB; n4 += 4)
        *reinterpret_cast<float4 *>(red + (phase * kSRows + lane * 4 + j) * NB + n4) =
            make_float4(acc[j][n4 / 2].x, acc[j][n4 / 2].y, acc[j][n4 / 2 + 1].x,
                        acc[j][n4 / 2 + 1].y);
    consumers_sync();
    finish_strip<NB>(args, cur, cta, ctas, strip0, tid, red, &s_last);
    zero_acc<NB>(acc);
  }
}

int nb_index(int tile_n) {
  for (int i = 0; i < kNumStreamNb; ++i)
    if (kStreamNb[i] == tile_n) return i;
  return -1;
}

size_t stream_smem(int nb, int stages) {
  const size_t stage = static_cast<size_t>(kSRows) * kSCols * 4 + static_cast<size_t>(kSCols) * nb * 4;
  return stage * stages + static_cast<size_t>(kSPhases) * kSRows * nb * 4 + 16 * stages + 1024;
}

bool aligned16(const void *ptr) { return (reinterpret_cast<uintptr_t>(ptr) & 15u) == 0; }

// Byte stride between the rows of a 2-D operand as the tensor map takes it.
// With a single row the stride is never used and may be anything the
// caller passed (e.g. ldb = 1 for one column of B): a padded row length
// stands in for it.
int64_t row_stride_bytes(int64_t stride, int64_t inner, int64_t outer) {
  return outer == 1 ? ((inner * 4 + 15) / 16) * 16 : stride * 4;
}

// K-contiguous B (K x N) -> an N-contiguous copy [K][nb] with columns N..nb-1
// zero: the kernel streams that layout faster (B box one contiguous 32 x nb
// block; measured N = 8, M = 65536, K = 4096: 180 against 194 us).
__global__ void gather_b_kernel(const float *__restrict__ B, int64_t sbk, int64_t sbn, int K,
                                int N, float *__restrict__ out, int nb) {
  allow_dependent_launch();  // the stream kernel waits for the copy itself
  for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < K;
       k += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    float v[8];
#pragma unroll
    for (int n = 0; n < 8; ++n) v[n] = (n < N) ? B[k * sbk + n * sbn] : 0.0f;
    float4 *o = reinterpret_cast<float4 *>(out + k * nb);
    o[0] = make_float4(v[0], v[1], v[2], v[3]);
    if (nb == 8) o[1] = make_float4(v[4], v[5], v[6], v[7]);
  }
}

// One launch of stream_kernel<NB> on p (B N-contiguous); `partial` is the
// workspace slot area, `early` makes it a programmatic dependent of the
// previous kernel on the stream (which then wrote B).
template <int NB>
hml_status launch_stream_kernel(const GemmProblem &p, const hml_sgemm_config &c, float *partial,
                                int ctas, bool early, cudaStream_t s) {
  const size_t smem = stream_smem(NB, c.stages);
  auto kern = stream_kernel<NB>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem));
  if (e != cudaSuccess) {
    note_cuda_error(e, "stream attributes");
    return HML_STATUS_CUDA_ERROR;
  }
  CUtensorMap ta, tb;
  memset(&ta, 0, sizeof(ta));
  memset(&tb, 0, sizeof(tb));
  bool ok = tensor_map_2d(&ta, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, p.A, p.M, p.K,
                          row_stride_bytes(p.sak, p.M, p.K), kSRows, kSCols,
                          CU_TENSOR_MAP_SWIZZLE_NONE);
  if (ok)
    ok = tensor_map_2d(&tb, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, p.B, p.N, p.K,
                       row_stride_bytes(p.sbk, p.N, p.K), NB, kSCols, CU_TENSOR_MAP_SWIZZLE_NONE);
  if (!ok) return HML_STATUS_CUDA_ERROR;

  const int strips = (p.M + kSRows - 1) / kSRows;
  StreamArgs args;
  args.p = p;
  args.kblocks = (p.K + kSCols - 1) / kSCols;
  args.units = static_cast<long long>(strips) * args.kblocks;
  args.stages = c.stages;
  args.err = device_error_word();
  args.partial = partial;
  hml_status st = tile_counters(static_cast<size_t>(strips), s, &args.arrivals);
  if (st != HML_STATUS_SUCCESS) return st;
  e = launch_k_ex(kern, dim3(ctas), dim3(kSThreads), smem, s, 1, early, ta, tb, args);
  note_cuda_error(e, "stream launch");
  return cuda_status(e);
}

// K-contiguous B is first copied N-contiguous ([K][NB], in the workspace
// after the partial-sum slots) and the N-contiguous kernel runs on the copy.
template <int NB>
hml_status run_stream(const GemmProblem &p, const hml_sgemm_config &c, cudaStream_t s) {
  const int strips = (p.M + kSRows - 1) / kSRows;
  const long long units = static_cast<long long>(strips) * ((p.K + kSCols - 1) / kSCols);
  const int ctas = static_cast<int>(std::min<long long>(units, kSCtasPerSm * sm_count()));
  const size_t part_bytes = static_cast<size_t>(ctas) * 2 * kSRows * NB * sizeof(float);
  const bool copy_b = p.b_kcontig();
  const size_t copy_bytes = copy_b ? static_cast<size_t>(p.K) * NB * sizeof(float) : 0;
  void *ws = nullptr;
  hml_status st = workspace(part_bytes + copy_bytes, s, &ws);
  if (st != HML_STATUS_SUCCESS) return st;
  float *partial = static_cast<float *>(ws);
  if (!copy_b) return launch_stream_kernel<NB>(p, c, partial, ctas, false, s);
  float *bcopy = partial + part_bytes / sizeof(float);
  const int blocks = static_cast<int>(std::min<int64_t>((p.K + 255) / 256, 4 * sm_count()));
  count_launch();
  gather_b_kernel<<<blocks, 256, 0, s>>>(p.B, p.sbk, p.sbn, p.K, p.N, bcopy, NB);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    note_cuda_error(e, "stream B copy");
    return HML_STATUS_CUDA_ERROR;
  }
  GemmProblem q = p;
  q.B = bcopy;
  q.sbk = NB;
  q.sbn = 1;
  return launch_stream_kernel<NB>(q, c, partial, ctas, true, s);
}

}  // namespace

int stream_num_variants() { return kNumStreamNb; }
int stream_tile_n(int i) { return kStreamNb[i]; }
int stream_max_stages(int nb) {
  int st = 2;
  while (st < kMaxStreamStages && (stream_smem(nb, st + 1) + 1024) * kSCtasPerSm <= 228 * 1024)
    ++st;
  return st;
}

// tile_m 128, tile_n = NB in {4, 8} (N <= NB), split_k 1 (the balance across
// SMs is built in), stages 2.. ring slots within the shared memory of 2 CTAs
// per SM.  A needs contiguous columns (sam == 1), 16-byte aligned with lda a
// multiple of 4.  B: K-contiguous with any leading dimension (it is copied
// first), or N-contiguous, 16-byte aligned with ldb a multiple of 4.
hml_status check_stream(const GemmProblem &p, const hml_sgemm_config &c) {
  const int i = nb_index(c.tile_n);
  if (i < 0 || c.tile_m != kSRows || c.split_k != 1) return HML_STATUS_INVALID_VALUE;
  if (c.stages < 2 || c.stages > kMaxStreamStages) return HML_STATUS_INVALID_VALUE;
  if ((stream_smem(c.tile_n, c.stages) + 1024) * kSCtasPerSm > 228 * 1024)
    return HML_STATUS_INVALID_VALUE;
  if (p.N > c.tile_n) return HML_STATUS_NOT_SUPPORTED;
  if (p.sam != 1 || p.a_kcontig()) return HML_STATUS_NOT_SUPPORTED;
  if (!(p.b_kcontig() || p.sbn == 1)) return HML_STATUS_NOT_SUPPORTED;
  const int64_t sa = row_stride_bytes(p.sak, p.M, p.K);
  if (!aligned16(p.A) || sa % 16 != 0 || sa >= (int64_t(1) << 40)) return HML_STATUS_NOT_SUPPORTED;
  if (!p.b_kcontig()) {
    const int64_t sb = row_stride_bytes(p.sbk, p.N, p.K);
    if (!aligned16(p.B) || sb % 16 != 0 || sb >= (int64_t(1) << 40))
      return HML_STATUS_NOT_SUPPORTED;
  }
  return HML_STATUS_SUCCESS;
}

hml_status launch_stream(const GemmProblem &p, const hml_sgemm_config &c, cudaStream_t s) {
  hml_status st = check_stream(p, c);
  if (st != HML_STATUS_SUCCESS) return st;
  switch (c.tile_n) {
    case 4: return run_stream<4>(p, c, s);
    case 8: return run_stream<8>(p, c, s);
    default: return HML_STATUS_INVALID_VALUE;
  }
}

}  // namespace hml
