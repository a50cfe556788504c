// simt_tile.cuh -- the FP32 SIMT tile arithmetic shared by the single-problem
// kernel (sgemm_simt.cu) and the persistent batched kernel (batched.cu).
//
// Both kernels stage 32-deep K slabs of A (BM x 32) and B (32 x BN) in shared
// memory and run the same per-slab FMA schedule and the same epilogue sum
// over the intra-CTA K split, so a tile computed by either kernel with the
// same shape gives the same bits.
#pragma once

#include "hml_device.cuh"

namespace hml {

constexpr int kBK = 32;  // K depth of one pipeline stage (128 bytes of FP32)

struct SimtShape {
  int tm, tn, wm, wn, wk;
  constexpr int bm() const { return wm * 32 * tm; }
  constexpr int bn() const { return wn * tn; }
};

// The micro-tile table (index = hml_sgemm_config.variant for HML_ALGO_SIMT).
// 8 warps per CTA arranged wm x wn x wk; each lane owns tm rows x tn columns.
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

// 16-byte shared-memory load at a 32-bit shared address.
__device__ __forceinline__ float4 lds128(uint32_t addr) {
  float4 v;
  asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];"
               : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
               : "r"(addr));
  return v;
}

// 4-byte asynchronous copy, zero-filled when !valid.
__device__ __forceinline__ void cp_async4(uint32_t dst, const float *src, bool valid) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(dst), "l"(src),
               "r"(valid ? 4 : 0)
               : "memory");
}

// 16-byte asynchronous copy of `bytes` (0..16) valid bytes, the rest zero.
__device__ __forceinline__ void cp_async16(uint32_t dst, const float *src, int bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}

// cp.async.wait_group takes an immediate: dispatch the runtime ring depth
// (wait until at most stages-2 groups are pending).
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

// Tile geometry and arithmetic of one micro-tile shape and operand layout.
//   AK : A is K-contiguous; its slab is stored [m][32 k] with the 128-byte
//        swizzle (16-byte granule g of row m at g ^ (m & 7)), else [k][BM].
//   BK_: B is K-contiguous; its slab is stored [n][32 k], else [k][BN].
template <int TM, int TN, int WM, int WN, int WK, bool AK, bool BK_>
struct SimtTile {
  static constexpr int BM = WM * 32 * TM;
  static constexpr int BN = WN * TN;
  static constexpr int NT = WM * WN * WK * 32;
  static_assert(NT == 256, "8 warps");
  static constexpr int KW = kBK / WK;  // K values per warp per slab
  static constexpr int A_BYTES = BM * kBK * 4;
  static constexpr int B_BYTES = BN * kBK * 4;
  static constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
  static constexpr int RED_BYTES = WK * BM * BN * 4;  // epilogue reuse of the ring

  // shared-memory byte offset of A(m, k) inside a slab
  __device__ static __forceinline__ uint32_t a_off(int m, int k) {
    return AK ? (static_cast<uint32_t>(m * 128 + k * 4) ^ static_cast<uint32_t>((m & 7) << 4))
              : static_cast<uint32_t>((k * BM + m) * 4);
  }
  __device__ static __forceinline__ uint32_t b_off(int n, int k) {
    return BK_ ? static_cast<uint32_t>((n * kBK + k) * 4) : static_cast<uint32_t>((k * BN + n) * 4);
  }

  // Warp coordinates of this thread's accumulators.
  struct Coord {
    int wk, wn, wm, mrow, ncol, lane;
  };
  __device__ static __forceinline__ Coord coord(int tid) {
    Coord c;
    const int warp = tid >> 5;
    c.lane = tid & 31;
    c.wk = warp % WK;
    c.wn = (warp / WK) % WN;
    c.wm = warp / (WK * WN);
    c.mrow = c.wm * 32 * TM;
    c.ncol = c.wn * TN;
    return c;
  }

  __device__ static __forceinline__ void zero(float (&acc)[TM][TN]) {
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
      for (int j = 0; j < TN; ++j) acc[i][j] = 0.0f;
  }

  // The TM rows of A this lane owns at k values kb..kb+3: a[kk][i].
  __device__ static __forceinline__ void a_frag(uint32_t ua, int kb, const Coord &c,
                                                float (&a)[4][TM]) {
    if (AK) {
      // A K-contiguous: one 16-byte read per row gives 4 k values
#pragma unroll
      for (int i = 0; i < TM; ++i) {
        const int m = c.mrow + c.lane + 32 * i;
        const float4 v = lds128(ua + m * 128 + ((((kb >> 2) ^ (m & 7))) << 4));
        a[0][i] = v.x; a[1][i] = v.y; a[2][i] = v.z; a[3][i] = v.w;
      }
    } else {
#pragma unroll
      for (int kk = 0; kk < 4; ++kk)
#pragma unroll
        for (int j = 0; j < TM / 4; ++j) {
          const float4 v = lds128(ua + ((kb + kk) * BM + c.mrow + 4 * c.lane + 128 * j) * 4);
          a[kk][4 * j + 0] = v.x; a[kk][4 * j + 1] = v.y;
          a[kk][4 * j + 2] = v.z; a[kk][4 * j + 3] = v.w;
        }
    }
  }

  // acc += this warp's K share of one staged slab.  Every accumulator takes
  // its products in k order, whatever the operand layouts.
  __device__ static __forceinline__ void slab(const float *sa, const float *sb,
                                              float (&acc)[TM][TN], const Coord &c) {
    // 32-bit shared addresses and a fully unrolled slab: every fragment
    // load is a base register plus an immediate offset (generic 64-bit
    // pointers measured 1.65 ms against 1.31 at 65536 x 128 x 4096)
    const uint32_t ua = smem_u32(sa), ub = smem_u32(sb);
#pragma unroll
    for (int k4 = 0; k4 < KW / 4; ++k4) {
      const int kb = c.wk * KW + k4 * 4;
      if (BK_) {
        float a[4][TM];
        a_frag(ua, kb, c, a);
        // B K-contiguous: one 16-byte broadcast per column gives its 4 k
        // values (all lanes read the same column); each column is used as
        // soon as it arrives, so only 4 B values are live at a time
#pragma unroll
        for (int j = 0; j < TN; ++j) {
          const float4 v = lds128(ub + ((c.ncol + j) * kBK + kb) * 4);
          if (!AK && WK > 1) {
            // rows 2q and 2q+1 are adjacent in the A fragment: one packed
            // FP32x2 FMA (two independent round-to-nearest FMAs, the same
            // bits) per row pair and k.  Only where warps split the slab
            // (8 k values a warp, so fewer FMAs between the per-slab waits):
            // 65536 x 32 x 4096 on 128 x 32 tiles 0.408 ms against 0.437;
            // the whole-slab tiles measured 0.5 % slower with it
            const float2 b0 = make_float2(v.x, v.x), b1 = make_float2(v.y, v.y);
            const float2 b2 = make_float2(v.z, v.z), b3 = make_float2(v.w, v.w);
#pragma unroll
            for (int q = 0; q < TM / 2; ++q) {
              float2 s = make_float2(acc[2 * q][j], acc[2 * q + 1][j]);
              s = __ffma2_rn(make_float2(a[0][2 * q], a[0][2 * q + 1]), b0, s);
              s = __ffma2_rn(make_float2(a[1][2 * q], a[1][2 * q + 1]), b1, s);
              s = __ffma2_rn(make_float2(a[2][2 * q], a[2][2 * q + 1]), b2, s);
              s = __ffma2_rn(make_float2(a[3][2 * q], a[3][2 * q + 1]), b3, s);
              acc[2 * q][j] = s.x;
              acc[2 * q + 1][j] = s.y;
            }
          } else {
#pragma unroll
            for (int i = 0; i < TM; ++i) {
              float s = acc[i][j];
              s = fmaf(a[0][i], v.x, s);
              s = fmaf(a[1][i], v.y, s);
              s = fmaf(a[2][i], v.z, s);
              acc[i][j] = fmaf(a[3][i], v.w, s);
            }
          }
        }
      } else {
        // A K-contiguous: one 16-byte read per row gives 4 k values
        float4 a4[AK ? TM : 1];
        if (AK) {
#pragma unroll
          for (int i = 0; i < TM; ++i) {
            const int m = c.mrow + c.lane + 32 * i;
            a4[i] = lds128(ua + m * 128 + (((kb >> 2) ^ (m & 7)) << 4));
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
              const float4 v = lds128(ua + ((kb + kk) * BM + c.mrow + 4 * c.lane + 128 * j) * 4);
              a[4 * j + 0] = v.x; a[4 * j + 1] = v.y; a[4 * j + 2] = v.z; a[4 * j + 3] = v.w;
            }
          }
          float b[TN];
#pragma unroll
          for (int j = 0; j < TN / 4; ++j) {
            const float4 v = lds128(ub + ((kb + kk) * BN + c.ncol + 4 * j) * 4);
            b[4 * j + 0] = v.x; b[4 * j + 1] = v.y; b[4 * j + 2] = v.z; b[4 * j + 3] = v.w;
          }
#pragma unroll
          for (int i = 0; i < TM; ++i)
#pragma unroll
            for (int j = 0; j < TN; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
      }
    }
  }

  // Writes this thread's partial tile into red = [WK][BN][BM] (the ring,
  // once every slab is consumed).
  __device__ static __forceinline__ void stash(float *red, const float (&acc)[TM][TN],
                                               const Coord &c) {
    float *r = red + static_cast<size_t>(c.wk) * BM * BN;
#pragma unroll
    for (int j = 0; j < TN; ++j) {
      float *col = r + (c.wn * TN + j) * BM + c.wm * 32 * TM;
      if (AK) {
#pragma unroll
        for (int i = 0; i < TM; ++i) col[c.lane + 32 * i] = acc[i][j];
      } else {
#pragma unroll
        for (int q = 0; q < TM / 4; ++q)
          *reinterpret_cast<float4 *>(col + 4 * c.lane + 128 * q) =
              make_float4(acc[4 * q][j], acc[4 * q + 1][j], acc[4 * q + 2][j], acc[4 * q + 3][j]);
      }
    }
  }

  // red[0] = sum over the WK partial tiles, in warp order.
  __device__ static __forceinline__ void reduce_wk(float *red, int tid) {
    constexpr int E = BM * BN;
    if (WK > 1) {
      for (int e = tid; e < E; e += NT) {
        float s = red[e];
#pragma unroll
        for (int w = 1; w < WK; ++w) s += red[w * E + e];
        red[e] = s;
      }
    }
  }

  // C tile = alpha * red[0] + beta * C for rows m0.. and columns n0.. of a
  // canonical problem (M, N, C strides scm, scn).
  __device__ static __forceinline__ void store_c(const float *red, int tid, int64_t m0, int n0,
                                                 int M, int N, float *C, int64_t scm,
                                                 int64_t scn, float alpha, float beta) {
    constexpr int E = BM * BN;
    if (scn == 1 && scm != 1) {
      // row-major C: walk n fastest so consecutive threads write adjacent
      // addresses (red is [n][m]; the strided smem read is the cheaper side)
      for (int e = tid; e < E; e += NT) {
        const int n = e % BN, m = e / BN;
        const int64_t gm = m0 + m;
        const int gn = n0 + n;
        if (gm < M && gn < N) {
          float *cp = C + gm * scm + gn;
          *cp = axpby(alpha, red[n * BM + m], beta, cp);
        }
      }
    } else {
      for (int e = tid; e < E; e += NT) {
        const int m = e % BM, n = e / BM;
        const int64_t gm = m0 + m;
        const int gn = n0 + n;
        if (gm < M && gn < N) {
          float *cp = C + gm * scm + static_cast<int64_t>(gn) * scn;
          *cp = axpby(alpha, red[e], beta, cp);
        }
      }
    }
  }
};

}  // namespace hml
