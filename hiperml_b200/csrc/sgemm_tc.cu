// sgemm_tc.cu -- split-BF16 SGEMM on the B200 tensor cores (tcgen05 + TMEM).
//
// FP32 operands are split into BF16 terms, a = a0 + a1 (+ a2), each term the
// BF16 rounding of what the previous terms left (every residual is exact in
// FP32), and the products that carry FP32-level information are accumulated
// in FP32:
//   BF16X3: a0*b0 + a0*b1 + a1*b0                          (2 planes, 3 MMAs)
//   BF16X6: a0*b0 + a0*b1 + a1*b0 + a0*b2 + a1*b1 + a2*b0  (3 planes, 6 MMAs)
// and two explicit forms with 11-bit planes: TF32X3 (kind::tf32) and FP16X3
// (FP16 hi/lo planes of operands scaled by powers of two: per row of each
// 32-deep block of A, per column of B; each block is accumulated in TMEM on
// its own and rescaled by the drain).
// The result is C = alpha * A * B + beta * C in FP32, the reference's
// hmlSgemm contract (src/hml_sgemm.cu:120-211) on a different machine.
//
// Data flow of one CTA (a 128-row tile of C, BN columns, a K range), in
// 32-deep K blocks:
//   * B is small (K x N): a pre-pass splits it once into BF16 planes stored
//     K-contiguous in a workspace ([plane][N_pad][K_pad]); a TMA warp loads
//     plane tiles straight into the UMMA canonical K-major layout (64-byte
//     swizzle, 32 BF16 per row).
//   * A streams from HBM exactly once: a TMA warp loads 128 x 32 FP32 tiles
//     into a ring of shared-memory slots.
//   * G converter warpgroups take the blocks round-robin (group g converts
//     blocks g, g+G, ...), so G blocks are in conversion at once.  Thread m of
//     a group owns row m of the tile, which is also TMEM lane m: it reads the
//     row's 32 FP32 values, splits them, and writes the BF16 planes into a
//     TMEM stage with tcgen05.st (two BF16 per 32-bit column).  The MMAs read
//     A from TMEM (the tcgen05.mma form with A in tensor memory), so the
//     converted planes never touch shared memory.
//   * NI threads (2 to 4, one per accumulator) issue tcgen05.mma (M=128,
//     N=BN, K=16; A from TMEM, B from shared memory; FP32 accumulator in
//     TMEM), each for every NI-th 64-deep chunk, and release each operand
//     stage (B slot + A stage) with one tcgen05.commit.
//   * the tensor core's FP32 accumulation truncates, so a long accumulation
//     chain in TMEM loses accuracy as K grows.  Each 64-deep chunk of K is
//     accumulated into one of NI TMEM accumulators; drain warpgroups read it
//     (tcgen05.ld) and add it into FP32 running sums held in registers
//     (round to nearest) while the tensor core fills the others.
//   * the drain warps apply alpha/beta; with split_k > 1 the CTAs of one
//     thread-block cluster sum their tiles in rank order through distributed
//     shared memory.
// Every wait is bounded (2 s of %globaltimer); on expiry the device error
// word is set, the CTA skips ahead, waits for its issued MMAs, frees its TMEM
// and returns.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <new>
#include <utility>
#include <vector>

#include "hml_device.cuh"
#include "hml_internal.h"
#include "hml_tcgen05.cuh"

namespace hml {
namespace {

constexpr int kBM = 128;      // rows of C per CTA = UMMA M = TMEM lanes
constexpr int kBK = 32;       // K per block (one 64-byte BF16 swizzle row)
constexpr int kChunkK = 64;   // K accumulated in TMEM before an FP32 drain
constexpr int kTmemCols = 512;

// Tile shapes: 128-row tiles, one per CTA.  (256-row tiles on a CTA pair,
// tcgen05.mma.cta_group::2, were bitwise equal but slower on every measured
// shape -- the cross-CTA handshakes cost about 1 us per 32-deep block -- and
// are not built.)
struct TcShape {
  int bm, bn;
};
constexpr TcShape kTcShapes[] = {{128, 16}, {128, 32}, {128, 64}, {128, 128}};
constexpr int kNumTcShapes = sizeof(kTcShapes) / sizeof(kTcShapes[0]);

// Warp roles of one CTA:
//   warp 0       TMA loads of A (FP32 tiles)
//   warp 1       TMA loads of B (BF16 plane tiles)
//   warps 2..    NI MMA issuers (warp 2 also allocates TMEM); issuer i takes
//                the 64-deep chunks q = i, i+NI, ... into accumulator i
//   then, from the next warp index divisible by 4: G converter warpgroups,
//   then D drain warpgroups.
// A warp can reach only TMEM lanes 32 * (warp % 4) .. +31, so every
// warpgroup that touches TMEM starts at a warp index divisible by 4 and its
// warp q covers rows 32q .. 32q+31.
//
// Each thread's tcgen05.mma issue is serial (tens of ns an instruction), so
// at small N one thread cannot keep up with the HBM stream; NI threads issue
// into NI accumulators.  TMEM holds the NI accumulators (BN columns each)
// and so A stages (NS x 16 columns each, two BF16 per 32-bit column).
__host__ __device__ constexpr int tc_groups() { return 2; }
__host__ __device__ constexpr int tc_drain_groups(int bn) { return bn > 64 ? 2 : 1; }
// BF16-plane equivalents of a form's operand planes: NS = 2 and 3 (BF16X3,
// BF16X6), 4 (TF32X3: two 32-bit planes), 5 (FP16X3: two FP16 planes).
__host__ __device__ constexpr int tc_geom(int ns) { return ns == 5 ? 2 : ns; }
// TMEM columns of one converted A block: NS planes x 32 BF16 (2 per column).
__host__ __device__ constexpr int tc_stage_cols(int ns) { return tc_geom(ns) * kBK / 2; }
// Operand stages (B slot + A TMEM stage) with ni issuers: a multiple of
// 2 * ni (blocks per chunk x issuers), so that every stage is only ever used
// by one issuer and, as 2 * ni is even, by one converter group; at most 8.
__host__ __device__ constexpr int tc_stage_mult(int ni) { return 2 * ni; }
__host__ __device__ constexpr int tc_stages_for(int bn, int ns, int ni) {
  return (((kTmemCols - ni * bn) / tc_stage_cols(ns) < 8 ? (kTmemCols - ni * bn) /
                                                               tc_stage_cols(ns)
                                                         : 8) /
          tc_stage_mult(ni)) *
         tc_stage_mult(ni);
}
// The most issuers (4 at most, 2 at least) whose accumulators leave room
// for at least one stage multiple.
__host__ __device__ constexpr int tc_issuers(int bn, int ns) {
  return tc_stages_for(bn, ns, 4) >= tc_stage_mult(4)   ? 4
         : tc_stages_for(bn, ns, 3) >= tc_stage_mult(3) ? 3
                                                        : 2;
}
__host__ __device__ constexpr int tc_max_stages(int bn, int ns) {
  return tc_stages_for(bn, ns, tc_issuers(bn, ns));
}
__host__ __device__ constexpr int tc_conv_warp0(int bn, int ns) {
  return ((2 + tc_issuers(bn, ns) + 3) / 4) * 4;
}
__host__ __device__ constexpr int tc_warps(int bn, int ns) {
  return tc_conv_warp0(bn, ns) + 4 * tc_groups() + 4 * tc_drain_groups(bn);
}


// Split eight floats into NS BF16 planes, t0 = bf16(x), t1 = bf16(x - t0),
// ... (each residual is exact in FP32), packed two per 32-bit word with
// cvt.rn.bf16x2.f32 (the lower k in the low half, as in memory order).
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

// One plane of the same split for 32 consecutive values of one row: word j
// holds elements 2j and 2j+1 rounded to BF16; unless this is the last plane,
// x is left holding the residuals for the next one.
template <bool LAST>
__device__ __forceinline__ void split_plane32(float (&x)[32], uint32_t (&w)[16]) {
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const uint32_t t = bf16x2_rn(x[2 * j], x[2 * j + 1]);
    w[j] = t;
    if (!LAST) {
      // both residuals with one packed FMA: fma(hi, -1, x) rounds the exact
      // x - hi, so the bits are those of the two subtractions
      const float2 h = make_float2(__uint_as_float(t << 16), __uint_as_float(t & 0xFFFF0000u));
      const float2 r =
          __ffma2_rn(h, make_float2(-1.0f, -1.0f), make_float2(x[2 * j], x[2 * j + 1]));
      x[2 * j] = r.x;
      x[2 * j + 1] = r.y;
    }
  }
}

// ------------------------------------------------------- FP16X3 split
// FP16 keeps 11 significant bits but only 5 exponent bits, so each FP32 row
// block of A (and each column of B) is first scaled by a power of two 2^S
// that brings its largest magnitude into [2^14, 2^15): then x*2^S = hi + lo
// with hi = fp16(x*2^S) and lo = fp16(x*2^S - hi) keeps 22 significant bits
// of every element within 2^-17 of the largest (the scaling is exact), and
// hi*hi + hi*lo + lo*hi (3 products) carries FP32-level information.  The
// biased exponent of the scale is clamped to [1, 253] so that both 2^S and
// 2^-S are normal floats; an all-zero or denormal block gets 2^126.
__device__ __forceinline__ int fh_scale_biased(float maxabs) {
  const int e = __float_as_int(maxabs) >> 23;  // biased exponent (maxabs >= 0)
  return min(max(268 - e, 1), 253);            // 127 + (14 - (e - 127))
}

// Two FP32 values rounded to FP16 (nearest even), packed: lo in the low half.
__device__ __forceinline__ uint32_t f16x2_rn(float lo, float hi) {
  uint32_t r;
  asm("cvt.rn.f16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
  return r;
}

__device__ __forceinline__ float2 f16x2_to_f32(uint32_t h) {
  return __half22float2(*reinterpret_cast<const __half2 *>(&h));
}

// The hi and lo FP16 planes of 32 scaled values of one row: word j holds
// elements 2j and 2j+1; hi = fp16(v), lo = fp16(v - hi) with v = x * s, the
// residual exact in FP32 (hi is converted back to FP32 to form it).
__device__ __forceinline__ void split_fh32(const float (&x)[32], float s, uint32_t (&wh)[16],
                                           uint32_t (&wl)[16]) {
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const float a = __fmul_rn(x[2 * j], s), b = __fmul_rn(x[2 * j + 1], s);
    const uint32_t h = f16x2_rn(a, b);
    const float2 hf = f16x2_to_f32(h);
    wh[j] = h;
    wl[j] = f16x2_rn(__fsub_rn(a, hf.x), __fsub_rn(b, hf.y));
  }
}

// Largest magnitude of 32 values (a tree of maxima of absolute values).
__device__ __forceinline__ float maxabs32(const float (&x)[32]) {
  float m[16];
#pragma unroll
  for (int j = 0; j < 16; ++j) m[j] = fmaxf(fabsf(x[2 * j]), fabsf(x[2 * j + 1]));
#pragma unroll
  for (int w = 8; w >= 1; w >>= 1)
#pragma unroll
    for (int j = 0; j < w; ++j) m[j] = fmaxf(m[j], m[j + w]);
  return m[0];
}

// 2^e as a float for e in [-149, 127] (denormal below -126), 0 below.
__device__ __forceinline__ float exp2_int(int e) {
  if (e >= -126) return __int_as_float((min(e, 127) + 127) << 23);
  if (e >= -149) return __int_as_float(1 << (e + 149));
  return 0.0f;
}

// x * 2^e for an integer e, exact unless the result leaves the float range.
__device__ __forceinline__ float scale_pow2(float x, int e) {
  while (e > 126) { x *= 0x1p126f; e -= 126; }
  while (e < -126) { x *= 0x1p-126f; e += 126; }
  return x * __int_as_float((e + 127) << 23);
}

struct TcArgs {
  GemmProblem p;
  int split;       // CTAs per cluster along K
  int kc;          // K extent per split (multiple of kChunkK)
  int sa, so;      // A ring and operand-stage depths
  int n_pad;       // rows of one B plane in the workspace
  int *err;
  const int *bexp;  // FP16X3: per column of B, the scale exponent S_n of its planes
};

// ------------------------------------------------------------ B planes
// planes[p][n][k] (k contiguous, zero padded to n_pad x k_pad): NS BF16
// planes, or for NS = 4 two 32-bit TF32 planes, hi = TF32(x) and
// lo = TF32(x - hi).
template <int NS>
__global__ void split_b_kernel(const float *B, int64_t sbk, int64_t sbn, int K, int N,
                               void *planes_out, int k_pad, int n_pad) {
  // the tensor-core kernel that reads the planes is launched as a
  // programmatic dependent: its set-up and A loads overlap this kernel
  allow_dependent_launch();
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
    if constexpr (NS == 4) {
      uint32_t *planes = static_cast<uint32_t *>(planes_out);
      uint32_t h[8], l[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        h[j] = tf32_rna(x[j]);
        l[j] = tf32_rna(x[j] - __uint_as_float(h[j]));
      }
      uint32_t *ph = planes + static_cast<int64_t>(n) * k_pad + k0;
      uint32_t *pl = planes + (static_cast<int64_t>(n_pad) + n) * k_pad + k0;
      reinterpret_cast<uint4 *>(ph)[0] = make_uint4(h[0], h[1], h[2], h[3]);
      reinterpret_cast<uint4 *>(ph)[1] = make_uint4(h[4], h[5], h[6], h[7]);
      reinterpret_cast<uint4 *>(pl)[0] = make_uint4(l[0], l[1], l[2], l[3]);
      reinterpret_cast<uint4 *>(pl)[1] = make_uint4(l[4], l[5], l[6], l[7]);
    } else {
      __nv_bfloat16 *planes = static_cast<__nv_bfloat16 *>(planes_out);
      uint4 v[NS];
      pack8<NS>(x, v);
#pragma unroll
      for (int i = 0; i < NS; ++i)
        *reinterpret_cast<uint4 *>(planes + (static_cast<int64_t>(i) * n_pad + n) * k_pad + k0) =
            v[i];
    }
  }
}

// FP16X3 planes of B: column n is scaled by 2^S_n, which brings its largest
// magnitude over K into [2^14, 2^15), and split into planes[0][n][k] =
// fp16(b * 2^S_n) and planes[1][n][k] = fp16(b * 2^S_n - hi); S_n goes to
// bexp[n].  Padding columns (n >= N) get zero planes and kNoColumn.  One
// warp per column: the column's maximum, then its conversion, 8 values a
// lane at a time (16-byte stores).
constexpr int kNoColumn = -100000;

__global__ void split_b_fh_kernel(const float *B, int64_t sbk, int64_t sbn, int K, int N,
                                  uint32_t *planes, int *bexp, int k_pad, int n_pad) {
  allow_dependent_launch();
  const int wpb = blockDim.x >> 5, lane = threadIdx.x & 31;
  for (int n = blockIdx.x * wpb + (threadIdx.x >> 5); n < n_pad; n += gridDim.x * wpb) {
    const float *col = B + static_cast<int64_t>(n) * sbn;
    float mx = 0.0f;
    if (n < N)
      for (int k = lane; k < K; k += 32) mx = fmaxf(mx, fabsf(col[static_cast<int64_t>(k) * sbk]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    const int sb = fh_scale_biased(mx);
    const float sc = __int_as_float(sb << 23);
    if (lane == 0) bexp[n] = n < N ? sb - 127 : kNoColumn;
    // planes as 32-bit words: two FP16 per word, k_pad / 2 words per row
    uint32_t *ph = planes + static_cast<int64_t>(n) * (k_pad / 2);
    uint32_t *pl = planes + (static_cast<int64_t>(n_pad) + n) * (k_pad / 2);
    for (int k0 = lane * 8; k0 < k_pad; k0 += 256) {
      float x[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int k = k0 + j;
        x[j] = (n < N && k < K) ? col[static_cast<int64_t>(k) * sbk] : 0.0f;
      }
      uint32_t h[4], l[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const float a = x[2 * j] * sc, b = x[2 * j + 1] * sc;
        h[j] = f16x2_rn(a, b);
        const float2 hf = f16x2_to_f32(h[j]);  // hi exactly as stored
        l[j] = f16x2_rn(a - hf.x, b - hf.y);
      }
      *reinterpret_cast<uint4 *>(ph + k0 / 2) = make_uint4(h[0], h[1], h[2], h[3]);
      *reinterpret_cast<uint4 *>(pl + k0 / 2) = make_uint4(l[0], l[1], l[2], l[3]);
    }
  }
}

// ------------------------------------------------------------- kernel
// Shared-memory plan of one CTA (tiles 1024-byte aligned):
//   A ring    sa slots of the FP32 A tile (16 KB), filled by TMA, released
//             by the converter group that read it;
//   B ring    so slots, each the NS B-plane tiles of one K block (TMA).
// TMEM: NI accumulators of BN columns, then so A stages of NS x 16 columns.
// Operand stage o = B slot o + A stage o, released together by one commit.
// sa is a multiple of G and so a multiple of 2 * NI, so each slot is only
// ever used by one converter group and each stage by one MMA issuer: a
// waiter has always seen the previous phase of its barrier complete.
struct TcPlan {
  int sa, so;
};

__host__ __device__ constexpr size_t tc_a_bytes() { return static_cast<size_t>(kBM) * kBK * 4; }
__host__ __device__ constexpr size_t tc_b_bytes(int bn, int ns) {
  return static_cast<size_t>(tc_geom(ns)) * bn * kBK * 2;
}
// FP16X3: the ring of per-row scale exponents the converters hand to the
// drain warps, one entry per K block in flight (2 x the operand stages).
__host__ __device__ constexpr int tc_fh_ring(int so) { return 2 * so; }
size_t tc_plan_bytes(int bn, int ns, const TcPlan &pl) {
  const size_t ring = ns == 5 ? static_cast<size_t>(tc_fh_ring(pl.so)) * (8 + kBM * 4) : 0;
  return 1024 + pl.sa * tc_a_bytes() + pl.so * tc_b_bytes(bn, ns) +
         8 * (2 * pl.sa + 2 * pl.so + 2 * 4 + 1) + 16 + ring + 16;
}

// The deepest operand-stage ring that fits TMEM and shared memory next to
// sa A slots; sa must be a multiple of G.
bool tc_plan(int bn, int ns, int sa, TcPlan *out) {
  const int g = tc_groups();
  if (sa < g || sa % g != 0) return false;
  const int mult = tc_stage_mult(tc_issuers(bn, ns));
  for (int so = tc_max_stages(bn, ns); so >= mult; so -= mult) {
    const TcPlan pl = {sa, so};
    if (tc_plan_bytes(bn, ns, pl) <= 227 * 1024) {
      *out = pl;
      return true;
    }
  }
  return false;
}

__host__ __device__ constexpr uint32_t tc_pow2_cols(int cols) {
  return cols <= 32 ? 32 : cols <= 64 ? 64 : cols <= 128 ? 128 : cols <= 256 ? 256 : 512;
}
__host__ __device__ constexpr uint32_t tc_tmem_alloc_cols(int bn, int ns, int so) {
  return tc_pow2_cols(tc_issuers(bn, ns) * bn + so * tc_stage_cols(ns));
}

template <int BN, int NS, bool AK>
__global__ void __launch_bounds__(tc_warps(BN, NS) * 32, 1)
    tc_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
              TcArgs args) {
  // NS = 4 is the TF32 form: 2 planes of 32-bit TF32 (hi, lo), the TMEM and
  // shared-memory footprint of 4 BF16 planes
  constexpr bool TF = NS == 4;
  // NS = 5 is the FP16X3 form: 2 FP16 planes of scaled values (the footprint
  // of 2 BF16 planes), a power-of-two scale per row and 32-deep block of A
  // and per column of B, each block accumulated and drained on its own
  constexpr bool FH = NS == 5;
  constexpr int PL = TF ? 2 : tc_geom(NS);                   // planes
  constexpr int PLC = TF ? kBK : kBK / 2;                    // TMEM columns of a plane
  constexpr int KMMA = TF ? 8 : 16;                          // K of one MMA
  constexpr int G = tc_groups();
  constexpr int D = tc_drain_groups(BN);
  constexpr int DC = BN / D;                                 // columns per drain thread
  constexpr int NI = tc_issuers(BN, NS);                     // MMA issuers = accumulators
  constexpr int kThreads = tc_warps(BN, NS) * 32;
  constexpr int kConvWarp0 = tc_conv_warp0(BN, NS), kDrainWarp0 = kConvWarp0 + 4 * G;
  constexpr int A32_BYTES = static_cast<int>(tc_a_bytes());  // FP32 A slot (16 KB)
  constexpr int BPL_BYTES = BN * kBK * (TF ? 4 : 2);         // one B plane tile
  constexpr int BSLOT = PL * BPL_BYTES;                      // one B slot
  constexpr int SC = tc_stage_cols(NS);                      // TMEM columns of an A stage
  static_assert(SC == PL * PLC, "stage columns");
  constexpr uint32_t IDESC =
      TF ? idesc_tf32(BN) : FH ? idesc_f16(BN) : idesc_bf16(BN);
  // blocks per TMEM chunk (FP16X3: one, the row scales change every block)
  constexpr int P = FH ? 1 : kChunkK / kBK;

  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = align_shared(smem_raw, 1024);
  const GemmProblem &p = args.p;
  const int SA = args.sa, SO = args.so;
  uint8_t *aring = smem;
  uint8_t *bring = aring + SA * A32_BYTES;
  uint64_t *afull = reinterpret_cast<uint64_t *>(bring + SO * BSLOT);  // [SA] tile landed
  uint64_t *aempty = afull + SA;     // [SA] the converter group has read the tile
  uint64_t *opfull = aempty + SA;    // [SO] B tiles landed and the A stage written
  uint64_t *opempty = opfull + SO;   // [SO] the MMAs reading the stage are done
  uint64_t *accfull = opempty + SO;   // [NI] accumulator holds a finished chunk
  uint64_t *accempty = accfull + NI;  // [NI] accumulator drained
  uint64_t *mmadone = accempty + NI;  // every issued MMA has completed
  // FP16X3: ring of R entries, one per K block in flight, each the 128 row
  // scale exponents of a block (sexp) and the barrier the converters arrive
  // on once they are written (sfull)
  const int R = FH ? tc_fh_ring(SO) : 0;
  uint64_t *sfull = mmadone + 1;      // [R]
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(sfull + R);
  int *bad_flag = reinterpret_cast<int *>(tmem_slot + 1);
  int *tmax_sh = bad_flag + 1;        // FP16X3: the largest column scale exponent of the tile
  int *sexp = align_shared(tmax_sh + 1, 16);  // [R][kBM]

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int split = args.split;
  const int rank = split > 1 ? static_cast<int>(cluster_ctarank()) : 0;
  const int64_t m0 = static_cast<int64_t>(blockIdx.x / split) * kBM;
  const int n0 = blockIdx.y * BN;
  const int kbeg = rank * args.kc;
  const int kend = min(p.K, kbeg + args.kc);
  const int nkb = kend > kbeg ? (kend - kbeg + kBK - 1) / kBK : 0;
  const int nchunks = (nkb + P - 1) / P;
  const uint32_t tmem_cols = tc_tmem_alloc_cols(BN, NS, SO);

  if (tid == 0) {
    for (int s = 0; s < SA; ++s) {
      mbar_init(&afull[s], 1);
      mbar_init(&aempty[s], 4);
    }
    for (int o = 0; o < SO; ++o) {
      mbar_init(&opfull[o], 4 + 1);  // the converter group's warps + the B loader
      mbar_init(&opempty[o], 1);
    }
    for (int b = 0; b < NI; ++b) {
      mbar_init(&accfull[b], 1);
      mbar_init(&accempty[b], 4 * D);
    }
    mbar_init(mmadone, NI);  // one commit per MMA issuer
    for (int r = 0; r < R; ++r) mbar_init(&sfull[r], 4);  // the converter group's warps
    *bad_flag = 0;
    fence_mbar_init();
  }
  if (warp == 2) tmem_alloc(tmem_slot, tmem_cols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const uint32_t tacc = tmem;           // accumulator b: columns b*BN .. +BN-1
  const uint32_t tA = tmem + NI * BN;   // A stage o: columns NI*BN + o*SC .. +SC-1

  if (warp == 0) {
    // -------------------------------------------------------- TMA, A
    if (lane == 0) {
      prefetch_tmap(&tmA);
      for (int kb = 0; kb < nkb; ++kb) {
        const int s = kb % SA;
        if (!mbar_wait(&aempty[s], ((kb / SA) & 1) ^ 1, args.err, kDevErrEmptyBarrier)) {
          *bad_flag = 1;
          break;
        }
        uint8_t *dst = aring + s * A32_BYTES;
        const int k0 = kbeg + kb * kBK;
        mbar_arrive_expect_tx(&afull[s], A32_BYTES);
        if (AK)  // 128 rows of 32 floats (128-byte swizzle)
          tma_load_2d(dst, &tmA, &afull[s], k0, static_cast<int>(m0));
        else     // 32 rows (k) of 128 floats (m)
          tma_load_2d(dst, &tmA, &afull[s], static_cast<int>(m0), k0);
      }
    }
  } else if (warp == 1) {
    // -------------------------------------------------------- TMA, B
    if (lane == 0) {
      prefetch_tmap(&tmB);
      // the B planes come from the kernel launched just before this one,
      // which may still be running (programmatic dependent launch); nothing
      // else this kernel reads depends on it
      wait_prior_grid();
      for (int kb = 0; kb < nkb; ++kb) {
        const int o = kb % SO;
        if (!mbar_wait(&opempty[o], ((kb / SO) & 1) ^ 1, args.err, kDevErrEmptyBarrier)) {
          *bad_flag = 1;
          break;
        }
        uint8_t *dst = bring + o * BSLOT;
        const int k0 = kbeg + kb * kBK;
        mbar_arrive_expect_tx(&opfull[o], BSLOT);
#pragma unroll
        for (int i = 0; i < PL; ++i)
          tma_load_2d(dst + i * BPL_BYTES, &tmB, &opfull[o], k0, i * args.n_pad + n0);
      }
    }
  } else if (warp >= 2 && warp < 2 + NI) {
    // ---------------------------------------------------------- MMA
    // NI issuing threads, one per accumulator: issuer b takes the chunks
    // q = b, b+NI, ...  A commit tracks only the MMAs of the thread that
    // issues it.
    if (lane == 0) {
      const int b = warp - 2;
      const uint32_t dacc = tacc + static_cast<uint32_t>(b * BN);
      bool ok = true;
      for (int q = b; q < nchunks && ok; q += NI) {
        const bool w =
            mbar_wait(&accempty[b], ((q / NI) & 1) ^ 1, args.err, kDevErrEmptyBarrier);
        if (!w) {
          ok = false;
          break;
        }
        const int kb1 = min(nkb, (q + 1) * P);
        for (int kb = q * P; kb < kb1; ++kb) {
          const int o = kb % SO;
          const bool first = kb == q * P;
          const bool w = mbar_wait(&opfull[o], (kb / SO) & 1, args.err, kDevErrFullBarrier);
          if (!w) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t astage = tA + static_cast<uint32_t>(o * SC);
          const uint64_t b_desc = TF ? sw128_desc(smem_u32(bring + o * BSLOT))
                                     : sw64_desc(smem_u32(bring + o * BSLOT));
#pragma unroll
          for (int kk = 0; kk < kBK / KMMA; ++kk) {
#pragma unroll
            for (int i = 0; i < PL; ++i)
#pragma unroll
              for (int j = 0; j < PL - i; ++j) {
                // A plane i: PLC columns per plane, 8 per MMA step (16 BF16
                // or 8 TF32 deep); B: 32 bytes per step; descriptor start
                // addresses count 16-byte units
                const uint32_t at = astage + static_cast<uint32_t>(i * PLC + kk * 8);
                const uint64_t bd =
                    b_desc + static_cast<uint64_t>((j * BPL_BYTES + kk * 32) >> 4);
                const uint32_t acc = (!first || kk > 0 || i > 0 || j > 0) ? 1u : 0u;
                if constexpr (TF)
                  mma_tf32_ts(dacc, at, bd, IDESC, acc);
                else
                  mma_bf16_ts(dacc, at, bd, IDESC, acc);
              }
          }
          mma_commit(&opempty[o]);
        }
        if (ok) mma_commit(&accfull[b]);
      }
      if (!ok) *bad_flag = 1;
      // tracks every MMA this thread issued
      mma_commit(mmadone);
    }
  } else if (warp >= kConvWarp0 && warp < kDrainWarp0) {
    // ------------------------------------------ converters (G groups)
    const int g = (warp - kConvWarp0) >> 2;
    const int m = tid & (kBM - 1);  // row of the tile == TMEM lane
    const uint32_t lanes = static_cast<uint32_t>((warp & 3) * 32) << 16;
    for (int kb = g; kb < nkb; kb += G) {
      const int s = kb % SA, o = kb % SO;
      bool w = mbar_wait(&afull[s], (kb / SA) & 1, args.err, kDevErrFullBarrier);
      if (!__all_sync(0xffffffffu, w)) {
        *bad_flag = 1;
        break;
      }
      const float *a32 = reinterpret_cast<const float *>(aring + s * A32_BYTES);
      float x[32];
      if (AK) {
        // row m holds 32 floats in 128 bytes, 128-byte swizzle
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          const float4 v = *reinterpret_cast<const float4 *>(a32 + m * 32 + ((c ^ (m & 7)) * 4));
          x[4 * c + 0] = v.x; x[4 * c + 1] = v.y; x[4 * c + 2] = v.z; x[4 * c + 3] = v.w;
        }
      } else {
#pragma unroll
        for (int k = 0; k < 32; ++k) x[k] = a32[k * kBM + m];
      }
      // consume the values (the first plane's split reads every one) before
      // the warp releases the slot: one lane arrives for the warp, and
      // __syncwarp alone does not wait for the other lanes' shared-memory
      // loads to return
      uint32_t wv[16];
      [[maybe_unused]] uint32_t wl[16];
      [[maybe_unused]] int sexp_m = 0;
      if constexpr (TF) {
        // hi of the first 16 values; the other 16 only need to have arrived
#pragma unroll
        for (int k = 0; k < 16; ++k) wv[k] = tf32_rna(x[k]);
#pragma unroll
        for (int k = 16; k < 32; ++k) asm volatile("" ::"f"(x[k]));
      } else if constexpr (FH) {
        // the row's scale for this block from its largest magnitude, then
        // both planes
        const int sb = fh_scale_biased(maxabs32(x));
        sexp_m = sb - 127;
        split_fh32(x, __int_as_float(sb << 23), wv, wl);
      } else {
        split_plane32<NS == 1>(x, wv);
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&aempty[s]);
      // the A stage: wait until the MMAs that read it are done
      w = mbar_wait(&opempty[o], ((kb / SO) & 1) ^ 1, args.err, kDevErrEmptyBarrier);
      if (!__all_sync(0xffffffffu, w)) {
        *bad_flag = 1;
        break;
      }
      tc_fence_after();
      if constexpr (FH) {
        // the drain of this block reads the row's scale exponent (the entry
        // is free: the drain of block kb - R finished before the MMAs of
        // block kb - SO, which released this operand stage)
        sexp[(kb % R) * kBM + m] = sexp_m;
        __syncwarp();
        if (lane == 0) mbar_arrive(&sfull[kb % R]);
      }
      const uint32_t dst = tA + lanes + static_cast<uint32_t>(o * SC);
      if constexpr (TF) {
        // one TF32 per column: plane hi in columns 0..31 (k), lo in 32..63;
        // lo = TF32(x - hi), the residual being exact in FP32
        tmem_st16(dst, wv);
#pragma unroll
        for (int k = 0; k < 16; ++k) x[k] -= __uint_as_float(wv[k]);
#pragma unroll
        for (int k = 0; k < 16; ++k) wv[k] = tf32_rna(x[16 + k]);
        tmem_st16(dst + 16u, wv);
#pragma unroll
        for (int k = 0; k < 16; ++k) x[16 + k] -= __uint_as_float(wv[k]);
#pragma unroll
        for (int k = 0; k < 16; ++k) wv[k] = tf32_rna(x[k]);
        tmem_st16(dst + 32u, wv);
#pragma unroll
        for (int k = 0; k < 16; ++k) wv[k] = tf32_rna(x[16 + k]);
        tmem_st16(dst + 48u, wv);
      } else if constexpr (FH) {
        tmem_st16(dst, wv);
        tmem_st16(dst + 16u, wl);
      } else {
        tmem_st16(dst, wv);
        split_plane32<NS == 2>(x, wv);
        tmem_st16(dst + 16u, wv);
        if constexpr (NS == 3) {
          split_plane32<true>(x, wv);
          tmem_st16(dst + 32u, wv);
        }
      }
      tmem_wait_st();
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&opfull[o]);
    }
  } else if (warp >= kDrainWarp0) {
    // ------------------------------------------ drain (D groups)
    const int d = (warp - kDrainWarp0) >> 2;
    const uint32_t lanes = static_cast<uint32_t>((warp & 3) * 32) << 16;
    const int mrow = tid & (kBM - 1);
    float sums[DC];  // FP32 running sums of row m, DC columns
#pragma unroll
    for (int i = 0; i < DC; ++i) sums[i] = 0.0f;
    [[maybe_unused]] int tmax = kNoColumn;
    if constexpr (FH) {
      // the tile's largest column scale exponent: the running sums hold
      // C(m, n) * 2^(S_n - tmax), never above |C(m, n)| (the column scales
      // come from the B-splitting kernel launched just before this one)
      wait_prior_grid();
      for (int c = lane; c < BN; c += 32)
        if (n0 + c < p.N) tmax = max(tmax, args.bexp[n0 + c]);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) tmax = max(tmax, __shfl_xor_sync(0xffffffffu, tmax, o));
      if (tid == kDrainWarp0 * 32) *tmax_sh = tmax;
    }
    for (int q = 0; q < nchunks; ++q) {
      const int b = q % NI;
      bool w = mbar_wait(&accfull[b], (q / NI) & 1, args.err, kDevErrMmaBarrier);
      [[maybe_unused]] float mult = 1.0f, mult2 = 1.0f;
      [[maybe_unused]] bool twostep = false;
      if constexpr (FH) {
        // block q's partial of row m is scaled by 2^(S_m,q + S_n): undo the
        // row's scale and the tile's largest column scale, 2^e.  Outside
        // the normal range the factor is applied in two exact steps
        // (2^(e -+ 126), then 2^(+-126)), so no contribution is lost or
        // clamped that FP32 itself would represent.
        if (w) w = mbar_wait(&sfull[q % R], (q / R) & 1, args.err, kDevErrFullBarrier);
        if (w) {
          const int e = -sexp[(q % R) * kBM + mrow] - tmax;
          twostep = e < -126 || e > 127;
          mult = exp2_int(e < -126 ? e + 126 : e > 127 ? e - 126 : e);
          mult2 = e < -126 ? 0x1p-126f : 0x1p126f;
        }
      }
      if (!__all_sync(0xffffffffu, w)) {  // tcgen05.ld is warp-collective
        *bad_flag = 1;
        break;
      }
      tc_fence_after();
      const uint32_t src = tacc + lanes + static_cast<uint32_t>(b * BN + d * DC);
      if constexpr (FH && DC >= 16) {
        // up to 32 columns loaded before one wait (16 when the running sums
        // take 64 registers); packed FP32x2 FMAs
        constexpr int W = DC >= 64 ? 16 : DC >= 32 ? 32 : DC;
        const float2 m2 = make_float2(mult, mult), m22 = make_float2(mult2, mult2);
#pragma unroll
        for (int c = 0; c < DC; c += W) {
          uint32_t r0[W];
#pragma unroll
          for (int h = 0; h < W; h += 16)
            tmem_ld16(src + c + h, *reinterpret_cast<uint32_t(*)[16]>(r0 + h));
          tmem_wait_ld();
          if (!twostep) {
#pragma unroll
            for (int i = 0; i < W; i += 2) {
              const float2 r = make_float2(__uint_as_float(r0[i]), __uint_as_float(r0[i + 1]));
              const float2 t = __ffma2_rn(r, m2, make_float2(sums[c + i], sums[c + i + 1]));
              sums[c + i] = t.x;
              sums[c + i + 1] = t.y;
            }
          } else {
#pragma unroll
            for (int i = 0; i < W; i += 2) {
              const float2 r = make_float2(__uint_as_float(r0[i]), __uint_as_float(r0[i + 1]));
              const float2 t = __ffma2_rn(__fmul2_rn(r, m2), m22,
                                          make_float2(sums[c + i], sums[c + i + 1]));
              sums[c + i] = t.x;
              sums[c + i + 1] = t.y;
            }
          }
        }
      } else if constexpr (DC >= 16) {
#pragma unroll
        for (int c = 0; c < DC; c += 16) {
          uint32_t r0[16];
          tmem_ld16(src + c, r0);
          tmem_wait_ld();
#pragma unroll
          for (int i = 0; i < 16; ++i) sums[c + i] += __uint_as_float(r0[i]);
        }
      } else {
        static_assert(DC % 8 == 0, "drain width");
        uint32_t r0[8];
        tmem_ld8(src, r0);
        tmem_wait_ld();
        if constexpr (FH) {
          if (!twostep) {
#pragma unroll
            for (int i = 0; i < 8; ++i) sums[i] = __fmaf_rn(__uint_as_float(r0[i]), mult, sums[i]);
          } else {
#pragma unroll
            for (int i = 0; i < 8; ++i)
              sums[i] = __fmaf_rn(__fmul_rn(__uint_as_float(r0[i]), mult), mult2, sums[i]);
          }
        } else {
#pragma unroll
          for (int i = 0; i < 8; ++i) sums[i] += __uint_as_float(r0[i]);
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&accempty[b]);
    }
    // ---------------------------------------------------- epilogue
    // (the running sums stay in this branch's registers; the barrier is the
    // one every other thread reaches below)
    __syncthreads();
    const bool failed = *bad_flag != 0;
    float *red = reinterpret_cast<float *>(smem);  // [BN][kBM], reuses the A ring
    const int m = tid & (kBM - 1);
    const int64_t gm = m0 + m;
    if (failed) {
#pragma unroll
      for (int i = 0; i < DC; ++i) sums[i] = 0.0f;
    }
    if (split > 1) {
#pragma unroll
      for (int i = 0; i < DC; ++i) red[(d * DC + i) * kBM + m] = sums[i];
    } else if (gm < p.M) {
#pragma unroll
      for (int i = 0; i < DC; ++i) {
        const int gn = n0 + d * DC + i;
        if (gn < p.N) {
          float *cp = p.C + gm * p.scm + static_cast<int64_t>(gn) * p.scn;
          float v = sums[i];
          if constexpr (FH) v = scale_pow2(v, tmax - args.bexp[gn]);
          *cp = axpby(p.alpha, v, p.beta, cp);
        }
      }
    }
  }
  if (warp < kDrainWarp0) __syncthreads();
  if (split > 1) {
    [[maybe_unused]] int tmax_all = 0;
    if constexpr (FH) {
      wait_prior_grid();  // the column scale exponents below
      tmax_all = *tmax_sh;
    }
    cluster_sync();
    const float *red = reinterpret_cast<const float *>(smem);
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
          float v = sv[qq];
          if constexpr (FH) v = scale_pow2(v, tmax_all - args.bexp[gn]);
          *cp = axpby(p.alpha, v, p.beta, cp);
        }
      }
    }
    cluster_sync();
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 2) {
    // the TMEM is freed only once every issued MMA has completed
    bool w = true;
    if (lane == 0) w = mbar_wait(mmadone, 0, args.err, kDevErrMmaBarrier);
    __syncwarp();
    (void)w;
    tc_fence_after();
  }
  if (warp == 2) tmem_dealloc(tmem, tmem_cols);
}

}  // namespace

bool tc_config_fits(int bn, int ns, int stages) {
  TcPlan pl;
  return tc_plan(bn, ns, stages, &pl);
}

namespace {

// Launch of the kernel with the B planes already split into `planes`.
template <int BN, int NS, bool AK>
hml_status launch_tc_planes(const GemmProblem &p, const hml_sgemm_config &c,
                            const __nv_bfloat16 *planes, int k_pad, int n_pad, int *err,
                            cudaStream_t s, const int *bexp = nullptr) {
  if (NS == 5 && !bexp) return HML_STATUS_INVALID_VALUE;
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
  if (ok) {
    if (NS == 4)  // two TF32 planes: rows of 32 x 4 bytes, 128-byte swizzle
      ok = tensor_map_2d(&tb, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, planes, k_pad,
                         static_cast<uint64_t>(2) * n_pad, static_cast<uint64_t>(k_pad) * 4, kBK,
                         BN, CU_TENSOR_MAP_SWIZZLE_128B);
    else  // 16-bit planes (BF16, or FP16 for NS = 5: TMA only moves the bytes)
      ok = tensor_map_2d(&tb, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, planes, k_pad,
                         static_cast<uint64_t>(tc_geom(NS)) * n_pad,
                         static_cast<uint64_t>(k_pad) * 2, kBK, BN,
                         CU_TENSOR_MAP_SWIZZLE_64B);
  }
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
  args.err = err;
  args.bexp = bexp;
  const size_t smem = tc_plan_bytes(BN, NS, plan);
  void (*kern)(CUtensorMap, CUtensorMap, TcArgs) = tc_kernel<BN, NS, AK>;
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
  // launched right after split_b_kernel wrote the planes: a programmatic
  // dependent whose B loader waits for it (wait_prior_grid)
  e = launch_k_ex(kern, grid, dim3(tc_warps(BN, NS) * 32), smem, s, c.split_k, true,
                  ta, tb, args);
  note_cuda_error(e, "tc launch");
  return cuda_status(e);
}

// launch_tc_planes for a split_k = 1 configuration whose grid ends in a
// partial wave: the whole waves of row tiles run as configured and the rows
// of the last wave, when it would leave at least half of the SMs idle, run
// as a second grid with K split across the idle SMs (disjoint rows of C, so
// the results are those of split_k = 2..8 on those rows).  One CTA per SM:
// M = 65536, N = 32 is 3 full waves of 148 tiles and 68 more.
template <int BN, int NS, bool AK>
hml_status launch_tc_waves(const GemmProblem &p, const hml_sgemm_config &c,
                           const __nv_bfloat16 *planes, int k_pad, int n_pad, int *err,
                           cudaStream_t s) {
  const int64_t tiles = (static_cast<int64_t>(p.M) + kBM - 1) / kBM;
  const int64_t slots = sm_count();
  const int64_t full = (tiles / slots) * slots;
  const int64_t rest = tiles - full;
  if (c.split_k != 1 || n_pad != BN || full == 0 || rest == 0 || 2 * rest > slots)
    return launch_tc_planes<BN, NS, AK>(p, c, planes, k_pad, n_pad, err, s);
  int split = 1;
  while (split < 8 && 2 * split * rest <= slots && k_pad / (2 * split) >= 4 * kChunkK) split *= 2;
  if (split == 1) return launch_tc_planes<BN, NS, AK>(p, c, planes, k_pad, n_pad, err, s);
  const int64_t m1 = full * kBM;
  GemmProblem head = p, tail = p;
  head.M = static_cast<int>(m1);
  tail.M = p.M - static_cast<int>(m1);
  tail.A = p.A + m1 * p.sam;
  tail.C = p.C + m1 * p.scm;
  hml_sgemm_config ct = c;
  ct.split_k = split;
  hml_status st = launch_tc_planes<BN, NS, AK>(head, c, planes, k_pad, n_pad, err, s);
  if (st != HML_STATUS_SUCCESS) return st;
  return launch_tc_planes<BN, NS, AK>(tail, ct, planes, k_pad, n_pad, err, s);
}

// B -> BF16 planes in `planes` ([NS][n_pad][k_pad]).
template <int NS>
hml_status split_b(const GemmProblem &p, __nv_bfloat16 *planes, int k_pad, int n_pad,
                   cudaStream_t s) {
  const int64_t chunks = static_cast<int64_t>(n_pad) * (k_pad / 8);
  const int blocks = static_cast<int>(std::min<int64_t>((chunks + 255) / 256, 4 * sm_count()));
  count_launch();
  split_b_kernel<NS><<<blocks, 256, 0, s>>>(p.B, p.sbk, p.sbn, p.K, p.N, planes, k_pad, n_pad);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    note_cuda_error(e, "split_b");
    return HML_STATUS_CUDA_ERROR;
  }
  return HML_STATUS_SUCCESS;
}

// B -> the two FP16 planes of the FP16X3 form and the column scale
// exponents (bexp, n_pad ints).
hml_status split_b_fh(const GemmProblem &p, void *planes, int *bexp, int k_pad, int n_pad,
                      cudaStream_t s) {
  const int blocks = std::min(std::max(1, (n_pad + 7) / 8), 4 * sm_count());
  count_launch();
  split_b_fh_kernel<<<blocks, 256, 0, s>>>(p.B, p.sbk, p.sbn, p.K, p.N,
                                           static_cast<uint32_t *>(planes), bexp, k_pad, n_pad);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    note_cuda_error(e, "split_b_fh");
    return HML_STATUS_CUDA_ERROR;
  }
  return HML_STATUS_SUCCESS;
}

template <int BN, int NS, bool AK>
hml_status run_tc(const GemmProblem &p, const hml_sgemm_config &c, cudaStream_t s, bool waves) {
  const int k_pad = ((p.K + kChunkK - 1) / kChunkK) * kChunkK;
  const int n_pad = ((p.N + BN - 1) / BN) * BN;
  // B planes in the stream's workspace (FP16X3: then the column exponents)
  const size_t plane_bytes = static_cast<size_t>(n_pad) * k_pad * 2;
  const size_t planes_total = tc_geom(NS) * plane_bytes;
  const size_t extra = NS == 5 ? static_cast<size_t>(n_pad) * sizeof(int) : 0;
  void *ws = nullptr;
  hml_status st = workspace(planes_total + extra, s, &ws);
  if (st != HML_STATUS_SUCCESS) return st;
  auto *planes = static_cast<__nv_bfloat16 *>(ws);
  if constexpr (NS == 5) {
    // planes_total is a multiple of 128 bytes (k_pad a multiple of 64)
    int *bexp = reinterpret_cast<int *>(static_cast<uint8_t *>(ws) + planes_total);
    st = split_b_fh(p, ws, bexp, k_pad, n_pad, s);
    if (st != HML_STATUS_SUCCESS) return st;
    return launch_tc_planes<BN, NS, AK>(p, c, planes, k_pad, n_pad, device_error_word(), s,
                                        bexp);
  } else {
    st = split_b<NS>(p, planes, k_pad, n_pad, s);
    if (st != HML_STATUS_SUCCESS) return st;
    if (waves)
      return launch_tc_waves<BN, NS, AK>(p, c, planes, k_pad, n_pad, device_error_word(), s);
    return launch_tc_planes<BN, NS, AK>(p, c, planes, k_pad, n_pad, device_error_word(), s);
  }
}

template <int BN, int NS>
hml_status run_tc_layout(const GemmProblem &p, const hml_sgemm_config &c, cudaStream_t s,
                         bool waves) {
  return p.a_kcontig() ? run_tc<BN, NS, true>(p, c, s, waves)
                       : run_tc<BN, NS, false>(p, c, s, waves);
}

template <int NS>
hml_status run_tc_ns(const GemmProblem &p, const hml_sgemm_config &c, cudaStream_t s,
                     bool waves) {
  switch (c.tile_n) {
    case 16: return run_tc_layout<16, NS>(p, c, s, waves);
    case 32: return run_tc_layout<32, NS>(p, c, s, waves);
    case 64: return run_tc_layout<64, NS>(p, c, s, waves);
    case 128: return run_tc_layout<128, NS>(p, c, s, waves);
    default: return HML_STATUS_INVALID_VALUE;
  }
}

bool aligned16(const void *ptr) { return (reinterpret_cast<uintptr_t>(ptr) & 15u) == 0; }

}  // namespace

int tc_num_shapes() { return kNumTcShapes; }
void tc_shape(int v, int *bm, int *bn) {
  *bm = kTcShapes[v].bm;
  *bn = kTcShapes[v].bn;
}

// Planes of a split-precision family, in units of BF16 planes: TF32X3's two
// 32-bit planes take the room of four (its kernels are instantiated NS = 4).
// (FP16X3 is instantiated NS = 5: two 16-bit planes, the room of two BF16 ones)
int tc_ns(int algo) {
  return algo == HML_ALGO_BF16X3   ? 2
         : algo == HML_ALGO_BF16X6 ? 3
         : algo == HML_ALGO_FP16X3 ? 5
                                   : 4;
}

hml_status check_tc(const GemmProblem &p, const hml_sgemm_config &c) {
  if (c.algo != HML_ALGO_BF16X3 && c.algo != HML_ALGO_BF16X6 && c.algo != HML_ALGO_TF32X3 &&
      c.algo != HML_ALGO_FP16X3)
    return HML_STATUS_INVALID_VALUE;
  if (c.variant < 0 || c.variant >= kNumTcShapes) return HML_STATUS_INVALID_VALUE;
  if (c.tile_m != kTcShapes[c.variant].bm || c.tile_n != kTcShapes[c.variant].bn)
    return HML_STATUS_INVALID_VALUE;
  if (c.split_k < 1 || c.split_k > 16 || (c.split_k & (c.split_k - 1)) != 0)
    return HML_STATUS_INVALID_VALUE;
  if (c.stages < 2 || c.stages > 8) return HML_STATUS_INVALID_VALUE;
  if (!tc_config_fits(c.tile_n, tc_ns(c.algo), c.stages)) return HML_STATUS_INVALID_VALUE;
  // the A ring is reused for the split-K partial tile
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

hml_status launch_tc(const GemmProblem &p, const hml_sgemm_config &c, cudaStream_t s,
                     bool waves) {
  hml_status st = check_tc(p, c);
  if (st != HML_STATUS_SUCCESS) return st;
  switch (c.algo) {
    case HML_ALGO_BF16X3: return run_tc_ns<2>(p, c, s, waves);
    case HML_ALGO_BF16X6: return run_tc_ns<3>(p, c, s, waves);
    case HML_ALGO_FP16X3: return run_tc_ns<5>(p, c, s, waves);
    default: return run_tc_ns<4>(p, c, s, waves);
  }
}

}  // namespace hml

// ------------------------------------------- batched split-BF16 (persistent)
//
// The batched plan (batched.cu) hands the problems it routes to the tensor
// cores to tc_batch_create.  Each tile width class (BN = 32, 64, 128) gets one
// persistent launch of tc_batch_kernel with one CTA per SM.  The class's
// (problem, 128-row tile, BN-column tile) items sit in device memory longest
// first, and a device-side work queue hands them out: the CTA's TMA-A thread
// takes the next item with an atomic on the class's queue head and publishes
// it to the CTA's other roles through a ring of item slots in shared memory
// (one mbarrier each way per slot), so every SM keeps pulling work until the
// queue is empty.  The pipeline inside a CTA is the single-problem kernel's
// (TMA warps, converter groups, MMA issuers with one TMEM accumulator each,
// drain warps) walking the 64-deep chunks of its items in the order taken;
// the TMA descriptors of every problem sit in device memory.  The last CTA
// to finish resets the queue, so a graph replays the launch as it is.  A
// tile's arithmetic is the single-problem kernel's with split_k = 1, so each
// result equals hml_sgemm_ex_config's for the same tile width, bit for bit,
// whichever CTA took it.
namespace hml {
namespace {

struct TcBatchProblem {
  float *C;
  int64_t scm, scn;
  int M, N;
  float alpha, beta;
  int akc;    // 1: A is K-contiguous (128 x 32 boxes, 128-byte swizzle)
  int cpt;    // 64-deep chunks of K (K padded to 64)
  int n_pad;  // rows of one B plane
  int pad_;
};

struct TcBatchItem {
  int prob, tm, tn, pad_;
};

struct TcBatchArgs {
  const CUtensorMap *tmA;       // [problems], 64-byte aligned
  const CUtensorMap *tmB;       // [problems]
  const TcBatchProblem *probs;  // [problems]
  const TcBatchItem *items;     // this class's items, longest first
  int nitems;
  unsigned *queue;              // [2]: queue head, CTAs finished (zero between launches)
  int sa, so;
  int *err;
};

// Item slots between the CTA's TMA-A thread (which takes items from the
// queue) and its other roles.  More than the items a CTA can have in flight:
// an item is at least one chunk, and the pipeline holds at most
// sa + so blocks (<= 16) plus NI chunks (<= 4).
constexpr int kItemRing = 32;
constexpr int kNoItem = -1;  // the sentinel published once the queue is empty
constexpr int kQueueAhead = 4;  // queue indices a CTA's producer takes ahead

// A role's walk through the items its CTA takes, in the order taken: item j
// of the sequence is read from ring slot j % kItemRing once published, and
// the slot is released right after the read (every role reads every item:
// the roles count chunks across item boundaries).
struct QueueCursor {
  TcBatchItem it;
  const TcBatchProblem *pr;
  int j = 0, c = 0;
  bool end = false;
  // Reads item j; false when the wait for it expired.  `warp_role`: every
  // lane of the warp calls this, lane 0 releases the slot for the warp.
  __device__ __forceinline__ bool fetch(const TcBatchArgs &a, uint64_t *ifull, uint64_t *iempty,
                                        const TcBatchItem *ring, bool warp_role, int lane) {
    const int r = j % kItemRing;
    bool w = mbar_wait(&ifull[r], (j / kItemRing) & 1, a.err, kDevErrFullBarrier);
    if (warp_role) w = __all_sync(0xffffffffu, w);
    if (!w) return false;
    it = ring[r];
    if (warp_role) {
      __syncwarp();
      if (lane == 0) mbar_arrive(&iempty[r]);
    } else {
      mbar_arrive(&iempty[r]);
    }
    end = it.prob == kNoItem;
    if (!end) pr = a.probs + it.prob;
    c = 0;
    return true;
  }
  // Advances past the current chunk, reading the next item at an item
  // boundary; false when a wait expired.
  __device__ __forceinline__ bool next(const TcBatchArgs &a, uint64_t *ifull, uint64_t *iempty,
                                       const TcBatchItem *ring, bool warp_role, int lane) {
    if (++c < pr->cpt) return true;
    ++j;
    return fetch(a, ifull, iempty, ring, warp_role, lane);
  }
};

// Drain warpgroups of the batched kernel: 32 columns each (its drain also
// finishes C tiles, so it keeps fewer running sums per thread).
__host__ __device__ constexpr int tcb_drain_groups(int bn) { return bn >= 32 ? bn / 32 : 1; }
__host__ __device__ constexpr int tcb_warps(int bn, int ns) {
  return tc_conv_warp0(bn, ns) + 4 * tc_groups() + 4 * tcb_drain_groups(bn);
}

template <int BN, int NS>
__global__ void __launch_bounds__(tcb_warps(BN, NS) * 32, 1) tc_batch_kernel(TcBatchArgs args) {
  allow_dependent_launch();  // the next tile kernel may take SMs this one leaves
  constexpr int G = tc_groups();
  constexpr int D = tcb_drain_groups(BN);
  constexpr int DC = BN / D;
  constexpr int NI = tc_issuers(BN, NS);
  constexpr int kConvWarp0 = tc_conv_warp0(BN, NS), kDrainWarp0 = kConvWarp0 + 4 * G;
  constexpr int A32_BYTES = static_cast<int>(tc_a_bytes());
  constexpr int BPL_BYTES = BN * kBK * 2;
  constexpr int BSLOT = NS * BPL_BYTES;
  constexpr int SC = tc_stage_cols(NS);
  constexpr uint32_t IDESC = idesc_bf16(BN);
  constexpr int P = kChunkK / kBK;
  static_assert(G == P, "converter group g converts block g of every chunk");

  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = align_shared(smem_raw, 1024);
  const int SA = args.sa, SO = args.so;
  uint8_t *aring = smem;
  uint8_t *bring = aring + SA * A32_BYTES;
  uint64_t *afull = reinterpret_cast<uint64_t *>(bring + SO * BSLOT);
  uint64_t *aempty = afull + SA;
  uint64_t *opfull = aempty + SA;
  uint64_t *opempty = opfull + SO;
  uint64_t *accfull = opempty + SO;
  uint64_t *accempty = accfull + NI;
  uint64_t *mmadone = accempty + NI;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(mmadone + 1);
  // item ring: slot published (producer) / slot read by every role
  uint64_t *ifull = reinterpret_cast<uint64_t *>(tmem_slot + 2);
  uint64_t *iempty = ifull + kItemRing;
  TcBatchItem *iring = reinterpret_cast<TcBatchItem *>(iempty + kItemRing);
  // readers of every item: the B loader, NI issuers, the converter and drain warps
  constexpr int kItemReaders = 1 + NI + 4 * G + 4 * D;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t tmem_cols = tc_tmem_alloc_cols(BN, NS, SO);

  if (tid == 0) {
    for (int s = 0; s < SA; ++s) {
      mbar_init(&afull[s], 1);
      mbar_init(&aempty[s], 4);
    }
    for (int o = 0; o < SO; ++o) {
      mbar_init(&opfull[o], 4 + 1);
      mbar_init(&opempty[o], 1);
    }
    for (int b = 0; b < NI; ++b) {
      mbar_init(&accfull[b], 1);
      mbar_init(&accempty[b], 4 * D);
    }
    mbar_init(mmadone, NI);
    for (int r = 0; r < kItemRing; ++r) {
      mbar_init(&ifull[r], 1);
      mbar_init(&iempty[r], kItemReaders);
    }
    fence_mbar_init();
  }
  if (warp == 2) tmem_alloc(tmem_slot, tmem_cols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const uint32_t tacc = tmem;
  const uint32_t tA = tmem + NI * BN;

  if (warp == 0) {
    // ------------------------------------------- queue + TMA, A
    // takes items from the class's queue, publishes each to the ring, then
    // loads its A blocks; a sentinel ends every role's walk
    if (lane == 0) {
      int blk = 0;
      // the indices of the next kQueueAhead items are taken ahead and the
      // record of the next one is loaded ahead, so the atomics' and the
      // load's round trips overlap the current item's loads (a CTA holds at
      // most kQueueAhead - 1 items it has not started: at the end of the
      // longest-first queue, short ones)
      unsigned q[kQueueAhead];
#pragma unroll
      for (int i = 0; i < kQueueAhead; ++i) q[i] = atomicAdd(&args.queue[0], 1u);
      const unsigned nitems = static_cast<unsigned>(args.nitems);
      TcBatchItem nxt = {kNoItem, 0, 0, 0};
      if (q[0] < nitems) nxt = args.items[q[0]];
      for (int j = 0;; ++j) {
        const int r = j % kItemRing;
        if (!mbar_wait(&iempty[r], ((j / kItemRing) & 1) ^ 1, args.err, kDevErrEmptyBarrier))
          break;
        const TcBatchItem it = nxt;
        iring[r] = it;
        mbar_arrive(&ifull[r]);  // release: the slot's item is visible to the waiters
        if (it.prob == kNoItem) break;
        // slide the window: one more index taken, the next record loaded
#pragma unroll
        for (int i = 0; i + 1 < kQueueAhead; ++i) q[i] = q[i + 1];
        q[kQueueAhead - 1] = atomicAdd(&args.queue[0], 1u);  // past the end: harmless
        nxt = {kNoItem, 0, 0, 0};
        if (q[0] < nitems) nxt = args.items[q[0]];
        const TcBatchProblem &pr = args.probs[it.prob];
        const CUtensorMap *tm = args.tmA + it.prob;
        const int m0 = it.tm * kBM;
        bool ok = true;
        for (int kq = 0; kq < pr.cpt * P && ok; ++kq, ++blk) {
          const int k0 = kq * kBK;
          const int s = blk % SA;
          if (!mbar_wait(&aempty[s], ((blk / SA) & 1) ^ 1, args.err, kDevErrEmptyBarrier)) {
            ok = false;
            break;
          }
          mbar_arrive_expect_tx(&afull[s], A32_BYTES);
          // k beyond K (the last chunk of a problem) reads TMA's zero fill
          if (pr.akc)
            tma_load_2d(aring + s * A32_BYTES, tm, &afull[s], k0, m0);
          else
            tma_load_2d(aring + s * A32_BYTES, tm, &afull[s], m0, k0);
        }
        if (!ok) break;
      }
      // every atomic taken ahead has returned (its register is read) before
      // this thread's arrival on the finish counter, so the last CTA's reset
      // of the head comes after all of them
#pragma unroll
      for (int i = 0; i < kQueueAhead; ++i) asm volatile("" ::"r"(q[i]));
    }
  } else if (warp == 1) {
    // -------------------------------------------------------- TMA, B
    if (lane == 0) {
      // launched as a programmatic dependent of the previous kernel of the
      // plan: the B planes are complete once that kernel is (the kernel
      // before a tile kernel is the splitting kernel or another tile
      // kernel, itself complete only after the splitting kernel)
      wait_prior_grid();
      QueueCursor cur;
      bool ok = cur.fetch(args, ifull, iempty, iring, false, lane);
      for (int blk = 0; ok && !cur.end;) {
        const CUtensorMap *tm = args.tmB + cur.it.prob;
        const int n0 = cur.it.tn * BN;
        const int np = cur.pr->n_pad;
        for (int kb = 0; kb < P; ++kb, ++blk) {
          const int k0 = (cur.c * P + kb) * kBK;
          const int o = blk % SO;
          if (!mbar_wait(&opempty[o], ((blk / SO) & 1) ^ 1, args.err, kDevErrEmptyBarrier)) {
            ok = false;
            break;
          }
          uint8_t *dst = bring + o * BSLOT;
          mbar_arrive_expect_tx(&opfull[o], BSLOT);
#pragma unroll
          for (int i = 0; i < NS; ++i)
            tma_load_2d(dst + i * BPL_BYTES, tm, &opfull[o], k0, i * np + n0);
        }
        if (ok) ok = cur.next(args, ifull, iempty, iring, false, lane);
      }
    }
  } else if (warp >= 2 && warp < 2 + NI) {
    // ---------------------------------------------------------- MMA
    // issuer b takes the chunks q = b, b + NI, ... of the CTA's sequence
    if (lane == 0) {
      const int b = warp - 2;
      const uint32_t dacc = tacc + static_cast<uint32_t>(b * BN);
      QueueCursor cur;
      bool ok = cur.fetch(args, ifull, iempty, iring, false, lane);
      for (int q = 0; ok && !cur.end; ++q) {
        if (q % NI == b) {
          const int jq = q / NI;
          if (!mbar_wait(&accempty[b], (jq & 1) ^ 1, args.err, kDevErrEmptyBarrier)) break;
          for (int kb = 0; kb < P; ++kb) {
            const int blk = q * P + kb;
            const int o = blk % SO;
            if (!mbar_wait(&opfull[o], (blk / SO) & 1, args.err, kDevErrFullBarrier)) {
              ok = false;
              break;
            }
            tc_fence_after();
            const uint32_t astage = tA + static_cast<uint32_t>(o * SC);
            const uint64_t b_desc = sw64_desc(smem_u32(bring + o * BSLOT));
#pragma unroll
            for (int kk = 0; kk < kBK / 16; ++kk) {
#pragma unroll
              for (int i = 0; i < NS; ++i)
#pragma unroll
                for (int jj = 0; jj < NS - i; ++jj) {
                  const uint32_t at = astage + static_cast<uint32_t>(i * 16 + kk * 8);
                  const uint64_t bd =
                      b_desc + static_cast<uint64_t>((jj * BPL_BYTES + kk * 32) >> 4);
                  const uint32_t acc = (kb > 0 || kk > 0 || i > 0 || jj > 0) ? 1u : 0u;
                  mma_bf16_ts(dacc, at, bd, IDESC, acc);
                }
            }
            mma_commit(&opempty[o]);
          }
          if (!ok) break;
          mma_commit(&accfull[b]);
        }
        ok = cur.next(args, ifull, iempty, iring, false, lane);
      }
      mma_commit(mmadone);
    }
  } else if (warp >= kConvWarp0 && warp < kDrainWarp0) {
    // ------------------------------------------ converters (G groups)
    // group g converts block g of every chunk (G == P)
    const int g = (warp - kConvWarp0) >> 2;
    const int m = tid & (kBM - 1);
    const uint32_t lanes = static_cast<uint32_t>((warp & 3) * 32) << 16;
    QueueCursor cur;
    bool ok = cur.fetch(args, ifull, iempty, iring, true, lane);
    for (int q = 0; ok && !cur.end; ++q) {
      const int blk = q * P + g;
      const int s = blk % SA, o = blk % SO;
      bool w = mbar_wait(&afull[s], (blk / SA) & 1, args.err, kDevErrFullBarrier);
      if (!__all_sync(0xffffffffu, w)) break;
      const float *a32 = reinterpret_cast<const float *>(aring + s * A32_BYTES);
      float x[32];
      if (cur.pr->akc) {
        // row m holds 32 floats in 128 bytes, 128-byte swizzle
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          const float4 v = *reinterpret_cast<const float4 *>(a32 + m * 32 + ((c ^ (m & 7)) * 4));
          x[4 * c + 0] = v.x; x[4 * c + 1] = v.y; x[4 * c + 2] = v.z; x[4 * c + 3] = v.w;
        }
      } else {
#pragma unroll
        for (int k = 0; k < 32; ++k) x[k] = a32[k * kBM + m];
      }
      uint32_t wv[16];
      split_plane32<NS == 1>(x, wv);
      __syncwarp();
      if (lane == 0) mbar_arrive(&aempty[s]);
      w = mbar_wait(&opempty[o], ((blk / SO) & 1) ^ 1, args.err, kDevErrEmptyBarrier);
      if (!__all_sync(0xffffffffu, w)) break;
      tc_fence_after();
      const uint32_t dst = tA + lanes + static_cast<uint32_t>(o * SC);
      tmem_st16(dst, wv);
      split_plane32<NS == 2>(x, wv);
      tmem_st16(dst + 16u, wv);
      if constexpr (NS == 3) {
        split_plane32<true>(x, wv);
        tmem_st16(dst + 32u, wv);
      }
      tmem_wait_st();
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&opfull[o]);
      ok = cur.next(args, ifull, iempty, iring, true, lane);
    }
  } else if (warp >= kDrainWarp0) {
    // ------------------------------------------ drain (D groups)
    const int d = (warp - kDrainWarp0) >> 2;
    const int m = tid & (kBM - 1);
    const uint32_t lanes = static_cast<uint32_t>((warp & 3) * 32) << 16;
    float sums[DC];
#pragma unroll
    for (int i = 0; i < DC; ++i) sums[i] = 0.0f;
    QueueCursor cur;
    bool ok = cur.fetch(args, ifull, iempty, iring, true, lane);
    for (int q = 0; ok && !cur.end; ++q) {
      const int b = q % NI;
      const bool w = mbar_wait(&accfull[b], (q / NI) & 1, args.err, kDevErrMmaBarrier);
      if (!__all_sync(0xffffffffu, w)) break;
      tc_fence_after();
      const uint32_t src = tacc + lanes + static_cast<uint32_t>(b * BN + d * DC);
      if constexpr (DC >= 16) {
#pragma unroll
        for (int c = 0; c < DC; c += 16) {
          uint32_t r0[16];
          tmem_ld16(src + c, r0);
          tmem_wait_ld();
#pragma unroll
          for (int i = 0; i < 16; ++i) sums[c + i] += __uint_as_float(r0[i]);
        }
      } else {
        static_assert(DC % 8 == 0, "drain width");
        uint32_t r0[8];
        tmem_ld8(src, r0);
        tmem_wait_ld();
#pragma unroll
        for (int i = 0; i < 8; ++i) sums[i] += __uint_as_float(r0[i]);
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&accempty[b]);
      if (cur.c == cur.pr->cpt - 1) {
        // the item's last chunk: C tile (row m, columns d*DC ..) and reset
        const TcBatchProblem &pr = *cur.pr;
        const int64_t gm = static_cast<int64_t>(cur.it.tm) * kBM + m;
        const int nb = cur.it.tn * BN + d * DC;
        if (gm < pr.M) {
#pragma unroll
          for (int i = 0; i < DC; ++i) {
            if (nb + i < pr.N) {
              float *cp = pr.C + gm * pr.scm + static_cast<int64_t>(nb + i) * pr.scn;
              *cp = axpby(pr.alpha, sums[i], pr.beta, cp);
            }
          }
        }
#pragma unroll
        for (int i = 0; i < DC; ++i) sums[i] = 0.0f;
      }
      ok = cur.next(args, ifull, iempty, iring, true, lane);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 2) {
    bool w = true;
    if (lane == 0) w = mbar_wait(mmadone, 0, args.err, kDevErrMmaBarrier);
    __syncwarp();
    (void)w;
    tc_fence_after();
    tmem_dealloc(tmem, tmem_cols);
  }
  if (tid == 0) {
    // the last CTA out resets the queue for the next launch (every CTA's
    // last atomic on the head came before its own increment here)
    __threadfence();
    if (atomicAdd(&args.queue[1], 1u) == gridDim.x - 1) {
      args.queue[0] = 0u;
      args.queue[1] = 0u;
      __threadfence();
    }
  }
}

// B of every routed problem -> its BF16 planes, one launch: blockIdx.y is the
// problem, the x blocks stride over its (n, 8-deep k) chunks.
struct TcSplitDesc {
  const float *B;
  int64_t sbk, sbn;
  int K, N, k_pad, n_pad;
  __nv_bfloat16 *planes;
};

template <int NS>
__global__ void split_b_batch_kernel(const TcSplitDesc *descs) {
  allow_dependent_launch();  // the tensor-core kernels wait for the planes
  const TcSplitDesc d = descs[blockIdx.y];
  const int64_t chunks = static_cast<int64_t>(d.n_pad) * (d.k_pad / 8);
  for (int64_t c = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; c < chunks;
       c += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int n = static_cast<int>(c / (d.k_pad / 8));
    const int k0 = static_cast<int>(c % (d.k_pad / 8)) * 8;
    float x[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int k = k0 + j;
      x[j] = (n < d.N && k < d.K)
                 ? d.B[static_cast<int64_t>(k) * d.sbk + static_cast<int64_t>(n) * d.sbn]
                 : 0.0f;
    }
    uint4 v[NS];
    pack8<NS>(x, v);
#pragma unroll
    for (int i = 0; i < NS; ++i)
      *reinterpret_cast<uint4 *>(d.planes + (static_cast<int64_t>(i) * d.n_pad + n) * d.k_pad +
                                 k0) = v[i];
  }
}

constexpr int kBatchTcNS = 3;                     // BF16X6: FP32-level accuracy
constexpr int kBatchTcBN[] = {32, 64, 128};       // tile width classes

int batch_tc_class(int N) { return N <= 32 ? 0 : N <= 64 ? 1 : 2; }

}  // namespace

// Host side of the batched split-BF16 part of a plan.
struct TcBatch {
  int nprob = 0;
  int items = 0;
  int ctas = 0;                   // the widest class launch
  void *dev = nullptr;            // one device allocation holding everything below
  cudaStream_t owner = nullptr;   // stream of a stream-ordered allocation, if any
  const TcSplitDesc *splits = nullptr;
  int split_blocks = 1;
  struct Class {
    int grid = 0;
    size_t smem = 0;
    TcBatchArgs args = {};
  } cls[3];
};

// Problems the batched plan can run on the tensor cores: A addressable by TMA
// (16-byte aligned base, leading dimension a multiple of 16 bytes), a real
// product (K > 0, alpha != 0) and N > 8 (at N <= 8 the FP32 SIMT tile is
// faster).
bool tc_batch_eligible(const GemmProblem &p) {
  if (p.N <= 8 || p.M < 1 || p.K < 1 || p.alpha == 0.0f) return false;
  const int64_t sa = p.a_kcontig() ? p.sam : p.sak;
  if ((reinterpret_cast<uintptr_t>(p.A) & 15u) != 0 || (sa * 4) % 16 != 0) return false;
  if (p.a_kcontig() ? p.sak != 1 : p.sam != 1) return false;
  return true;
}

namespace {

size_t up256(size_t b) { return (b + 255) & ~static_cast<size_t>(255); }

// Shared memory of the item ring: slots plus their two barriers.
constexpr size_t kItemRingBytes = kItemRing * (sizeof(TcBatchItem) + 2 * sizeof(uint64_t)) + 16;

template <int BN>
hml_status tc_batch_class_setup(TcBatch::Class &c) {
  TcPlan plan;
  int sa = 8;
  while (sa >= 2 && !(tc_plan(BN, kBatchTcNS, sa, &plan) &&
                      tc_plan_bytes(BN, kBatchTcNS, plan) + kItemRingBytes <= 227 * 1024))
    sa -= 2;
  if (sa < 2) return HML_STATUS_NOT_SUPPORTED;
  c.args.sa = plan.sa;
  c.args.so = plan.so;
  c.smem = tc_plan_bytes(BN, kBatchTcNS, plan) + kItemRingBytes;
  const cudaError_t e = cudaFuncSetAttribute(tc_batch_kernel<BN, kBatchTcNS>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             static_cast<int>(c.smem));
  if (e != cudaSuccess) {
    note_cuda_error(e, "tc batch attributes");
    return HML_STATUS_CUDA_ERROR;
  }
  return HML_STATUS_SUCCESS;
}

}  // namespace

hml_status tc_batch_create(const GemmProblem *probs, int count, cudaStream_t stream_ordered,
                           TcBatch **out) {
  *out = nullptr;
  if (count <= 0) return HML_STATUS_SUCCESS;
  if (count > 65535) return HML_STATUS_NOT_SUPPORTED;  // grid.y of the split launch
  const int sms = sm_count();
  // per problem: class, padded sizes, planes
  std::vector<int> cls(count), k_pad(count), n_pad(count);
  std::vector<size_t> plane_off(count);
  size_t planes_bytes = 0;
  std::vector<std::vector<std::pair<int, TcBatchItem>>> items(3);  // (cost, item)
  int64_t max_chunks = 1;
  for (int i = 0; i < count; ++i) {
    const GemmProblem &p = probs[i];
    cls[i] = batch_tc_class(p.N);
    const int bn = kBatchTcBN[cls[i]];
    k_pad[i] = ((p.K + kChunkK - 1) / kChunkK) * kChunkK;
    n_pad[i] = ((p.N + bn - 1) / bn) * bn;
    plane_off[i] = planes_bytes;
    planes_bytes += up256(static_cast<size_t>(kBatchTcNS) * n_pad[i] * k_pad[i] * 2);
    max_chunks = std::max<int64_t>(max_chunks, static_cast<int64_t>(n_pad[i]) * (k_pad[i] / 8));
    const int64_t tm = (static_cast<int64_t>(p.M) + kBM - 1) / kBM, tn = n_pad[i] / bn;
    if (tm > 0x7fffffff) return HML_STATUS_NOT_SUPPORTED;
    for (int64_t x = 0; x < tm; ++x)
      for (int64_t y = 0; y < tn; ++y)
        items[cls[i]].push_back({k_pad[i] / kChunkK, TcBatchItem{i, static_cast<int>(x),
                                                                 static_cast<int>(y), 0}});
  }
  // per class: the items longest first, the order the queue hands them out
  // (each CTA takes the next when it can: longest-processing-time first)
  std::vector<TcBatchItem> cls_items[3];
  size_t total_items = 0;
  for (int c = 0; c < 3; ++c) {
    auto &v = items[c];
    if (v.empty()) continue;
    if (v.size() > 0x7fffffffu) return HML_STATUS_NOT_SUPPORTED;
    std::stable_sort(v.begin(), v.end(),
                     [](const std::pair<int, TcBatchItem> &a, const std::pair<int, TcBatchItem> &b) {
                       return a.first > b.first;
                     });
    for (const auto &e : v) cls_items[c].push_back(e.second);
    total_items += v.size();
  }
  // device layout: tensor maps | problems | split descriptors | queues |
  // per class items | planes
  const size_t o_tmA = 0, o_tmB = up256(count * sizeof(CUtensorMap));
  const size_t o_prob = o_tmB + up256(count * sizeof(CUtensorMap));
  const size_t o_split = o_prob + up256(count * sizeof(TcBatchProblem));
  const size_t o_queue = o_split + up256(count * sizeof(TcSplitDesc));
  size_t o = o_queue + up256(3 * 2 * sizeof(unsigned));
  size_t o_items[3];
  for (int c = 0; c < 3; ++c) {
    o_items[c] = o;
    o += up256(cls_items[c].size() * sizeof(TcBatchItem));
  }
  const size_t o_planes = o;
  const size_t total = o_planes + planes_bytes;

  TcBatch *b = new (std::nothrow) TcBatch;
  if (!b) return HML_STATUS_ALLOC_FAILED;
  cudaError_t e = stream_ordered ? cudaMallocAsync(&b->dev, total, stream_ordered)
                                 : cudaMalloc(&b->dev, total);
  if (e != cudaSuccess) {
    note_cuda_error(e, "tc batch allocation");
    delete b;
    return HML_STATUS_ALLOC_FAILED;
  }
  b->owner = stream_ordered;
  uint8_t *base = static_cast<uint8_t *>(b->dev);
  // host images
  std::vector<CUtensorMap> tmA(count), tmB(count);
  std::vector<TcBatchProblem> hp(count);
  std::vector<TcSplitDesc> hs(count);
  bool ok = true;
  for (int i = 0; i < count && ok; ++i) {
    const GemmProblem &p = probs[i];
    const int bn = kBatchTcBN[cls[i]];
    auto *planes = reinterpret_cast<__nv_bfloat16 *>(base + o_planes + plane_off[i]);
    memset(&tmA[i], 0, sizeof(CUtensorMap));
    memset(&tmB[i], 0, sizeof(CUtensorMap));
    if (p.a_kcontig())
      ok = tensor_map_2d(&tmA[i], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, p.A, p.K, p.M, p.sam * 4, kBK,
                         kBM, CU_TENSOR_MAP_SWIZZLE_128B);
    else
      ok = tensor_map_2d(&tmA[i], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, p.A, p.M, p.K, p.sak * 4, kBM,
                         kBK, CU_TENSOR_MAP_SWIZZLE_NONE);
    if (ok)
      ok = tensor_map_2d(&tmB[i], CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, planes, k_pad[i],
                         static_cast<uint64_t>(kBatchTcNS) * n_pad[i],
                         static_cast<uint64_t>(k_pad[i]) * 2, kBK, bn, CU_TENSOR_MAP_SWIZZLE_64B);
    TcBatchProblem &q = hp[i];
    memset(&q, 0, sizeof q);
    q.C = p.C;
    q.scm = p.scm;
    q.scn = p.scn;
    q.M = p.M;
    q.N = p.N;
    q.alpha = p.alpha;
    q.beta = p.beta;
    q.akc = p.a_kcontig() ? 1 : 0;
    q.cpt = k_pad[i] / kChunkK;
    q.n_pad = n_pad[i];
    hs[i] = TcSplitDesc{p.B, p.sbk, p.sbn, p.K, p.N, k_pad[i], n_pad[i], planes};
  }
  auto upload = [&](size_t off, const void *src, size_t bytes) {
    if (e != cudaSuccess || bytes == 0) return;
    e = stream_ordered ? cudaMemcpyAsync(base + off, src, bytes, cudaMemcpyHostToDevice,
                                         stream_ordered)
                       : cudaMemcpy(base + off, src, bytes, cudaMemcpyHostToDevice);
  };
  if (ok) {
    upload(o_tmA, tmA.data(), count * sizeof(CUtensorMap));
    upload(o_tmB, tmB.data(), count * sizeof(CUtensorMap));
    upload(o_prob, hp.data(), count * sizeof(TcBatchProblem));
    upload(o_split, hs.data(), count * sizeof(TcSplitDesc));
    for (int c = 0; c < 3; ++c)
      upload(o_items[c], cls_items[c].data(), cls_items[c].size() * sizeof(TcBatchItem));
    const unsigned zeros[6] = {0u, 0u, 0u, 0u, 0u, 0u};  // queue heads and finished counts
    upload(o_queue, zeros, sizeof zeros);
    // pageable sources: a synchronous copy has consumed them on return; the
    // stream-ordered ones have been staged by the driver before returning
  }
  hml_status st = ok ? cuda_status(e) : HML_STATUS_CUDA_ERROR;
  for (int c = 0; c < 3 && st == HML_STATUS_SUCCESS; ++c) {
    TcBatch::Class &k = b->cls[c];
    k.grid = static_cast<int>(std::min<size_t>(cls_items[c].size(), static_cast<size_t>(sms)));
    if (k.grid == 0) continue;
    st = c == 0   ? tc_batch_class_setup<32>(k)
         : c == 1 ? tc_batch_class_setup<64>(k)
                  : tc_batch_class_setup<128>(k);
    k.args.tmA = reinterpret_cast<const CUtensorMap *>(base + o_tmA);
    k.args.tmB = reinterpret_cast<const CUtensorMap *>(base + o_tmB);
    k.args.probs = reinterpret_cast<const TcBatchProblem *>(base + o_prob);
    k.args.items = reinterpret_cast<const TcBatchItem *>(base + o_items[c]);
    k.args.nitems = static_cast<int>(cls_items[c].size());
    k.args.queue = reinterpret_cast<unsigned *>(base + o_queue) + 2 * c;
    k.args.err = device_error_word();
    b->ctas = std::max(b->ctas, k.grid);
  }
  if (st != HML_STATUS_SUCCESS) {
    if (e != cudaSuccess) note_cuda_error(e, "tc batch upload");
    tc_batch_destroy(b);
    return st;
  }
  b->nprob = count;
  b->items = static_cast<int>(total_items);
  b->splits = reinterpret_cast<const TcSplitDesc *>(base + o_split);
  b->split_blocks = static_cast<int>(std::min<int64_t>((max_chunks + 255) / 256, 64));
  *out = b;
  return HML_STATUS_SUCCESS;
}

hml_status tc_batch_launch(const TcBatch *b, cudaStream_t s) {
  if (!b || b->nprob == 0) return HML_STATUS_SUCCESS;
  count_launch();
  split_b_batch_kernel<kBatchTcNS>
      <<<dim3(static_cast<unsigned>(b->split_blocks), static_cast<unsigned>(b->nprob)), 256, 0,
         s>>>(b->splits);
  cudaError_t e = cudaGetLastError();
  // each tile kernel is a programmatic dependent of the kernel before it:
  // its CTAs start on the SMs that kernel has finished with, and only its B
  // loader waits for that kernel to complete
  for (int c = 0; c < 3 && e == cudaSuccess; ++c) {
    const TcBatch::Class &k = b->cls[c];
    if (k.grid == 0) continue;
    if (c == 0)
      e = launch_k_ex(tc_batch_kernel<32, kBatchTcNS>, dim3(k.grid),
                      dim3(tcb_warps(32, kBatchTcNS) * 32), k.smem, s, 1, true, k.args);
    else if (c == 1)
      e = launch_k_ex(tc_batch_kernel<64, kBatchTcNS>, dim3(k.grid),
                      dim3(tcb_warps(64, kBatchTcNS) * 32), k.smem, s, 1, true, k.args);
    else
      e = launch_k_ex(tc_batch_kernel<128, kBatchTcNS>, dim3(k.grid),
                      dim3(tcb_warps(128, kBatchTcNS) * 32), k.smem, s, 1, true, k.args);
  }
  note_cuda_error(e, "tc batch launch");
  return cuda_status(e);
}

void tc_batch_destroy(TcBatch *b) {
  if (!b) return;
  if (b->dev) {
    if (b->owner)
      cudaFreeAsync(b->dev, b->owner);
    else
      cudaFree(b->dev);
  }
  delete b;
}

// The configuration under which a batched plan runs an eligible problem:
// its tile width class and the A-ring depth the class launch uses; the
// single-problem kernel with this configuration computes the same bits.
hml_sgemm_config tc_batch_config(const GemmProblem &p) {
  const int bn = kBatchTcBN[batch_tc_class(p.N)];
  int sa = 8;
  TcPlan plan;
  while (sa > 2 && !tc_plan(bn, kBatchTcNS, sa, &plan)) sa -= 2;
  int var = 0;
  while (var + 1 < kNumTcShapes && kTcShapes[var].bn != bn) ++var;
  return hml_sgemm_config{HML_ALGO_BF16X6, kBM, bn, 1, sa, var};
}

int tc_batch_items(const TcBatch *b) { return b ? b->items : 0; }
int tc_batch_ctas(const TcBatch *b) { return b ? b->ctas : 0; }

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
// The error word of the bounded waits of calls made through this entry point:
// file scope too, so that no call allocates it.  hml_device_error reads and
// clears it together with the library's other error word.
static __device__ int g_noalloc_error;

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
struct NoAllocAddrs {
  void *scratch = nullptr;
  int *err = nullptr;
};
NoAllocAddrs g_noalloc_addr[kNoAllocMaxDevices];

// Device addresses of the scratch array and the error word on the current
// device.  In host code the arrays' names are only host-side stand-ins, so
// the addresses are looked up once per device (with that device current) and
// cached.
hml_status noalloc_setup(NoAllocAddrs *out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    note_cuda_error(e, "noalloc: cudaGetDevice");
    return HML_STATUS_CUDA_ERROR;
  }
  if (dev < 0 || dev >= kNoAllocMaxDevices) return HML_STATUS_NOT_SUPPORTED;
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  NoAllocAddrs &a = g_noalloc_addr[dev];
  if (!a.scratch) {
    void *scratch = nullptr, *err = nullptr;
    e = cudaGetSymbolAddress(&scratch, g_noalloc_scratch);
    if (e == cudaSuccess) e = cudaGetSymbolAddress(&err, g_noalloc_error);
    if (e != cudaSuccess || !scratch || !err) {
      note_cuda_error(e != cudaSuccess ? e : cudaErrorInvalidSymbol,
                      "noalloc: cudaGetSymbolAddress");
      return HML_STATUS_CUDA_ERROR;
    }
    a.err = static_cast<int *>(err);
    a.scratch = scratch;
  }
  *out = a;
  return HML_STATUS_SUCCESS;
}

size_t noalloc_bytes_needed(const GemmProblem &p, const hml_sgemm_config &c) {
  const int ns = c.algo == HML_ALGO_BF16X3 ? 2 : 3;
  const size_t k_pad = ((static_cast<size_t>(p.K) + kChunkK - 1) / kChunkK) * kChunkK;
  const size_t n_pad = ((static_cast<size_t>(p.N) + c.tile_n - 1) / c.tile_n) * c.tile_n;
  return static_cast<size_t>(ns) * n_pad * k_pad * 2;
}

// The launch of run_tc with the B planes in the static array and the static
// error word.
template <int BN, int NS, bool AK>
hml_status run_tc_static(const GemmProblem &p, const hml_sgemm_config &c, const NoAllocAddrs &a,
                         cudaStream_t s) {
  const int k_pad = ((p.K + kChunkK - 1) / kChunkK) * kChunkK;
  const int n_pad = ((p.N + BN - 1) / BN) * BN;
  auto *planes = static_cast<__nv_bfloat16 *>(a.scratch);
  hml_status st = split_b<NS>(p, planes, k_pad, n_pad, s);
  if (st != HML_STATUS_SUCCESS) return st;
  return launch_tc_planes<BN, NS, AK>(p, c, planes, k_pad, n_pad, a.err, s);
}

template <int NS>
hml_status run_tc_static_ns(const GemmProblem &p, const hml_sgemm_config &c,
                            const NoAllocAddrs &a, cudaStream_t s) {
  const bool ak = p.a_kcontig();
  switch (c.tile_n) {
    case 16: return ak ? run_tc_static<16, NS, true>(p, c, a, s)
                       : run_tc_static<16, NS, false>(p, c, a, s);
    case 32: return ak ? run_tc_static<32, NS, true>(p, c, a, s)
                       : run_tc_static<32, NS, false>(p, c, a, s);
    case 64: return ak ? run_tc_static<64, NS, true>(p, c, a, s)
                       : run_tc_static<64, NS, false>(p, c, a, s);
    case 128: return ak ? run_tc_static<128, NS, true>(p, c, a, s)
                        : run_tc_static<128, NS, false>(p, c, a, s);
    default: return HML_STATUS_INVALID_VALUE;
  }
}

}  // namespace

// Reads and clears the error word of the allocation-free entry point on the
// current device; 0 when that entry point was never set up there.  Copies to
// and from the symbol allocate nothing.
hml_status noalloc_take_error(int *code) {
  *code = 0;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    note_cuda_error(e, "noalloc: cudaGetDevice");
    return HML_STATUS_CUDA_ERROR;
  }
  if (dev < 0 || dev >= kNoAllocMaxDevices) return HML_STATUS_SUCCESS;
  {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_addr[dev].err) return HML_STATUS_SUCCESS;
  }
  int h = 0;
  e = cudaMemcpyFromSymbol(&h, g_noalloc_error, sizeof(int));
  if (e == cudaSuccess && h != 0) {
    const int zero = 0;
    e = cudaMemcpyToSymbol(g_noalloc_error, &zero, sizeof(int));
  }
  note_cuda_error(e, "noalloc: error word");
  *code = h;
  return cuda_status(e);
}
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
                    "(planes x ceil(min(M,N)/tile_n)*tile_n x ceil(K/64)*64 x 2 bytes)");
    return HML_STATUS_INVALID_VALUE;
  }
  NoAllocAddrs addrs;
  st = noalloc_setup(&addrs);
  if (st != HML_STATUS_SUCCESS) return st;
  return config->algo == HML_ALGO_BF16X3 ? run_tc_static_ns<2>(p, *config, addrs, s)
                                         : run_tc_static_ns<3>(p, *config, addrs, s);
}
