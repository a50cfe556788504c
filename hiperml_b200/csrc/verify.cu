// verify.cu -- accuracy reporting and synthetic data on the GPU.
//
//  * hml_fill_random: the counter-based SplitMix64 generator of
//    hiperml_b200/datagen.py (same integer stream, same FP32 uniforms).
//  * hml_sgemm_error_fp64: an FP64 GEMM over the same operands and the
//    error reductions (max |dC| / max |C64|, RMS, componentwise).  FP64 is
//    used only here, never on the SGEMM/SGEMV hot path.
#include <cmath>

#include "hml_device.cuh"
#include "hml_internal.h"

namespace hml {
namespace {

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

uint64_t mix64_host(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__global__ void fill_kernel(float *out, size_t n, uint64_t key, int dist) {
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const uint64_t z = mix64(key + (i + 1) * 0x9E3779B97F4A7C15ull);
    const double hi24 = static_cast<double>(z >> 40);
    float v;
    if (dist == 0) {
      v = static_cast<float>(2.0 * (hi24 * 0x1p-24) - 1.0);
    } else if (dist == 1) {
      const double u1 = (hi24 + 1.0) * 0x1p-24;
      const double u2 = static_cast<double>((z >> 16) & 0xFFFFFFull) * 0x1p-24;
      v = static_cast<float>(sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2));
    } else {
      const double mag = pow(10.0, 6.0 * (hi24 * 0x1p-24) - 3.0);
      v = static_cast<float>(((z >> 39) & 1ull) ? -mag : mag);
    }
    out[i] = v;
  }
}

// FP64 reference GEMM, 64 x 64 tiles, 256 threads, 4 x 4 outputs a thread.
// D(m,n) = alpha*sum A B + beta*C0 and Dabs = |alpha| sum|A||B| + |beta||C0|,
// both dense column-major (ld = M).
constexpr int kT = 64, kKB = 16;
__global__ void __launch_bounds__(256) dgemm_ref_kernel(GemmProblem p, const float *C0,
                                                        double *D, double *Dabs) {
  __shared__ double As[kKB][kT + 1];
  __shared__ double Bs[kKB][kT + 1];
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  const int64_t m0 = static_cast<int64_t>(blockIdx.x) * kT;
  const int64_t n0 = static_cast<int64_t>(blockIdx.y) * kT;
  double acc[4][4] = {}, aacc[4][4] = {};
  for (int k0 = 0; k0 < p.K; k0 += kKB) {
    for (int e = threadIdx.x; e < kKB * kT; e += 256) {
      const int mm = e % kT, kk = e / kT;
      const int64_t gm = m0 + mm, gn = n0 + mm;
      const int gk = k0 + kk;
      As[kk][mm] = (gm < p.M && gk < p.K) ? static_cast<double>(p.A[gm * p.sam + gk * p.sak]) : 0.0;
      Bs[kk][mm] = (gn < p.N && gk < p.K) ? static_cast<double>(p.B[gk * p.sbk + gn * p.sbn]) : 0.0;
    }
    __syncthreads();
#pragma unroll 4
    for (int kk = 0; kk < kKB; ++kk) {
      double a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[kk][tx + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[kk][ty + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          acc[i][j] = fma(a[i], b[j], acc[i][j]);
          aacc[i][j] = fma(fabs(a[i]), fabs(b[j]), aacc[i][j]);
        }
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int64_t gm = m0 + tx + 16 * i, gn = n0 + ty + 16 * j;
      if (gm < p.M && gn < p.N) {
        double c = 0.0;
        if (p.beta != 0.0f && C0) c = static_cast<double>(C0[gm * p.scm + gn * p.scn]);
        const double al = static_cast<double>(p.alpha), be = static_cast<double>(p.beta);
        // two rounded products and a rounded sum, no contraction: the same
        // operations as the CPU oracle, so both give the same FP64 value
        // (the k sums above agree too: FP32 x FP32 products are exact in
        // FP64, and both add them in increasing k from zero)
        D[gm + gn * p.M] = __dadd_rn(__dmul_rn(al, acc[i][j]), __dmul_rn(be, c));
        Dabs[gm + gn * p.M] =
            __dadd_rn(__dmul_rn(fabs(al), aacc[i][j]), __dmul_rn(fabs(be), fabs(c)));
      }
    }
}

__device__ __forceinline__ void atomic_max_nonneg(double *addr, double v) {
  atomicMax(reinterpret_cast<unsigned long long *>(addr),
            static_cast<unsigned long long>(__double_as_longlong(v)));
}

// out[0] = max|dC|, out[1] = sum dC^2, out[2] = sum C64^2, out[3] = max|C64|,
// out[4] = max |dC| / Dabs
__global__ void err_kernel(GemmProblem p, const double *D, const double *Dabs, double *out) {
  double mx = 0.0, s2 = 0.0, r2 = 0.0, mref = 0.0, cw = 0.0;
  const int64_t total = static_cast<int64_t>(p.M) * p.N;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t m = i % p.M, n = i / p.M;
    const double ref = D[i];
    const double got = static_cast<double>(p.C[m * p.scm + n * p.scn]);
    const double d = fabs(got - ref);
    mx = fmax(mx, d);
    s2 += d * d;
    r2 += ref * ref;
    mref = fmax(mref, fabs(ref));
    if (Dabs[i] > 0.0) cw = fmax(cw, d / Dabs[i]);
    else if (d > 0.0) cw = INFINITY;
    if (d != d) mx = INFINITY;  // NaN in the result
  }
  __shared__ double sh[5][8];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) {
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    r2 += __shfl_xor_sync(0xffffffffu, r2, o);
    mref = fmax(mref, __shfl_xor_sync(0xffffffffu, mref, o));
    cw = fmax(cw, __shfl_xor_sync(0xffffffffu, cw, o));
  }
  if (lane == 0) {
    sh[0][w] = mx; sh[1][w] = s2; sh[2][w] = r2; sh[3][w] = mref; sh[4][w] = cw;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < (int)(blockDim.x / 32); ++k) {
      mx = fmax(mx, sh[0][k]); s2 += sh[1][k]; r2 += sh[2][k];
      mref = fmax(mref, sh[3][k]); cw = fmax(cw, sh[4][k]);
    }
    atomic_max_nonneg(&out[0], mx);
    atomicAdd(&out[1], s2);
    atomicAdd(&out[2], r2);
    atomic_max_nonneg(&out[3], mref);
    atomic_max_nonneg(&out[4], cw);
  }
}

// A wait that nothing ends: thread 0 waits on an mbarrier no thread arrives
// on, with the bounded wait of every kernel of the library; it gives up
// after the limit, records the full-barrier code in the device error word
// and returns, leaving the context usable.
__global__ void expired_wait_kernel(int *err) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) mbar_wait(&bar, 0, err, kDevErrFullBarrier);
}

}  // namespace

hml_status check_wait_limit(cudaStream_t s) {
  int *err = device_error_word();
  if (!err) return HML_STATUS_ALLOC_FAILED;
  count_launch();
  expired_wait_kernel<<<1, 32, 0, s>>>(err);
  cudaError_t e = cudaGetLastError();
  note_cuda_error(e, "expired wait");
  return cuda_status(e);
}

hml_status fill_random(float *out, size_t n, uint64_t seed, uint64_t stream_id, int dist,
                       cudaStream_t s) {
  if (n == 0) return HML_STATUS_SUCCESS;
  if (!out || dist < 0 || dist > 2) return HML_STATUS_INVALID_VALUE;
  const uint64_t key = mix64_host(mix64_host(seed) ^ (stream_id * 0xD6E8FEB86659FD93ull));
  const size_t blocks = std::min<size_t>((n + 255) / 256, static_cast<size_t>(sm_count()) * 16);
  count_launch();
  fill_kernel<<<static_cast<unsigned>(blocks), 256, 0, s>>>(out, n, key, dist);
  cudaError_t e = cudaGetLastError();
  note_cuda_error(e, "fill_random");
  return cuda_status(e);
}

hml_status sgemm_error_fp64(const GemmProblem &p, const float *C0, double err[4], cudaStream_t s) {
  for (int i = 0; i < 4; ++i) err[i] = 0.0;
  if (p.M == 0 || p.N == 0) return HML_STATUS_SUCCESS;
  const size_t mn = static_cast<size_t>(p.M) * p.N;
  double *D = nullptr;
  cudaError_t e = cudaMalloc(&D, (2 * mn + 8) * sizeof(double));
  if (e != cudaSuccess) {
    note_cuda_error(e, "error_fp64 alloc");
    return HML_STATUS_ALLOC_FAILED;
  }
  double *Dabs = D + mn, *out = D + 2 * mn;
  hml_status st = HML_STATUS_SUCCESS;
  e = cudaMemsetAsync(out, 0, 8 * sizeof(double), s);
  if (e == cudaSuccess) {
    dim3 grid(static_cast<unsigned>((p.M + kT - 1) / kT), static_cast<unsigned>((p.N + kT - 1) / kT));
    count_launch(2);
    dgemm_ref_kernel<<<grid, 256, 0, s>>>(p, C0, D, Dabs);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    err_kernel<<<sm_count() * 4, 256, 0, s>>>(p, D, Dabs, out);
    e = cudaGetLastError();
  }
  double h[8] = {};
  if (e == cudaSuccess) e = cudaMemcpyAsync(h, out, 8 * sizeof(double), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    note_cuda_error(e, "error_fp64");
    st = HML_STATUS_CUDA_ERROR;
  } else {
    err[0] = h[3] > 0 ? h[0] / h[3] : h[0];
    err[1] = h[2] > 0 ? std::sqrt(h[1] / h[2]) : std::sqrt(h[1]);
    err[2] = h[4];
    err[3] = h[3];
  }
  cudaFree(D);
  return st;
}

}  // namespace hml
