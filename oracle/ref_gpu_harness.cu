// ref_gpu_harness.cu -- TEST INFRASTRUCTURE ONLY.  Entry points (extern "C")
// into the reference's own SGEMM / SGEMV kernel repositories and selectors,
// compiled from the reference sources with ref_gpu_compat.h (oracle/Makefile):
// the GPU baseline that the benchmark times and the parity tests compare
// with.  Each call follows the reference's host-pointer entry point --
// hmlSgemm (src/hml_sgemm.cu:153-195) and hmlSgemv (src/hml_sgemv.cu:
// 157-199): bind A and B (or x) to the textures, pick the kernel with the
// loaded rules (hmlSgemmKernelSelect / hmlSgemvKernelSelect), launch it with
// the same grid and block -- but on operands already on the device, `reps`
// times between CUDA events, so that the kernel alone is timed.  Row-major
// layout, the reference's only one.
#include <cuda_runtime.h>

#if defined(HML_REF_SGEMM)
#include "hml_sgemm_kernel.h"
extern bool sgemmKernelRepoInitialized;
extern bool sgemmKernelConfigDone;
#elif defined(HML_REF_SGEMV)
#include "hml_sgemv_kernel.h"
extern bool hmlSgemvKernelInitialized;
extern bool hmlSgemvKernelConfigDone;
#endif

namespace {
int timed(cudaEvent_t a, cudaEvent_t b, int reps, float *ms) {
  cudaError_t e = cudaEventSynchronize(b);
  float t = 0.0f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&t, a, b);
  if (ms) *ms = reps > 0 ? t / reps : 0.0f;
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return static_cast<int>(e);
}
}  // namespace

#if defined(HML_REF_SGEMM)
extern "C" int ref_gpu_sgemm_config(const char *path) {
  if (!sgemmKernelRepoInitialized) hmlSgemmKernelRepoInit();
  hmlSgemmKernelConfigReadFile(path);
  return sgemmKernelConfigDone ? 0 : 1;
}

// The kernel the rules pick: *is_const, grid and block of the launch.
extern "C" int ref_gpu_sgemm_select(int M, int N, int K, int *is_const, int *grid, int *block) {
  if (!sgemmKernelRepoInitialized || !sgemmKernelConfigDone) return 1;
  HmlSgemmKernelConstK constK = 0;
  HmlSgemmKernelVarK varK = 0;
  HmlKernelArg karg;
  hmlSgemmKernelSelect(&varK, &constK, &karg, M, N, K);
  *is_const = constK != 0;
  grid[0] = karg.grid.x; grid[1] = karg.grid.y; grid[2] = karg.grid.z;
  block[0] = karg.block.x; block[1] = karg.block.y; block[2] = karg.block.z;
  return 0;
}

// C = alpha A B + beta C (row-major, device pointers), `reps` launches.
extern "C" int ref_gpu_sgemm(float *C, const float *A, const float *B, int M, int N, int K,
                             float alpha, float beta, int reps, float *ms) {
  if (!sgemmKernelRepoInitialized || !sgemmKernelConfigDone) return 1;
  size_t off = 0;
  cudaError_t e = cudaBindTexture(&off, texFloatA, A, static_cast<size_t>(M) * K * sizeof(float));
  if (e == cudaSuccess)
    e = cudaBindTexture(&off, texFloatB, B, static_cast<size_t>(N) * K * sizeof(float));
  if (e != cudaSuccess) return static_cast<int>(e);
  HmlSgemmKernelConstK constK = 0;
  HmlSgemmKernelVarK varK = 0;
  HmlKernelArg karg;
  hmlSgemmKernelSelect(&varK, &constK, &karg, M, N, K);
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  cudaEventRecord(a);
  for (int r = 0; r < reps; ++r) {
    if (constK)
      constK<<<karg.grid, karg.block>>>(C, A, B, M, N, alpha, beta);
    else
      varK<<<karg.grid, karg.block>>>(C, A, B, M, N, K, alpha, beta);
  }
  cudaEventRecord(b);
  e = cudaGetLastError();
  const int st = timed(a, b, reps, ms);
  cudaUnbindTexture(texFloatA);
  cudaUnbindTexture(texFloatB);
  return e != cudaSuccess ? static_cast<int>(e) : st;
}
#endif

#if defined(HML_REF_SGEMV)
extern "C" int ref_gpu_sgemv_config(const char *path) {
  if (!hmlSgemvKernelInitialized) hmlSgemvKernelInit();
  hmlSgemvKernelConfigReadFile(path);
  return hmlSgemvKernelConfigDone ? 0 : 1;
}

extern "C" int ref_gpu_sgemv_select(int M, int N, int *is_const, int *grid, int *block) {
  if (!hmlSgemvKernelInitialized || !hmlSgemvKernelConfigDone) return 1;
  HmlSgemvKernelConstN constN = 0;
  HmlSgemvKernelVarN varN = 0;
  HmlKernelArg karg;
  hmlSgemvKernelSelect(&varN, &constN, &karg, M, N);
  *is_const = constN != 0;
  grid[0] = karg.grid.x; grid[1] = karg.grid.y; grid[2] = karg.grid.z;
  block[0] = karg.block.x; block[1] = karg.block.y; block[2] = karg.block.z;
  return 0;
}

// y = alpha A x + beta y (A row-major M x N, device pointers), `reps` launches.
extern "C" int ref_gpu_sgemv(float *y, const float *A, const float *x, int M, int N,
                             float alpha, float beta, int reps, float *ms) {
  if (!hmlSgemvKernelInitialized || !hmlSgemvKernelConfigDone) return 1;
  size_t off = 0;
  cudaError_t e = cudaBindTexture(&off, texFloatA, A, static_cast<size_t>(M) * N * sizeof(float));
  if (e == cudaSuccess) e = cudaBindTexture(&off, texFloatx, x, static_cast<size_t>(N) * sizeof(float));
  if (e != cudaSuccess) return static_cast<int>(e);
  HmlSgemvKernelConstN constN = 0;
  HmlSgemvKernelVarN varN = 0;
  HmlKernelArg karg;
  hmlSgemvKernelSelect(&varN, &constN, &karg, M, N);
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  cudaEventRecord(a);
  for (int r = 0; r < reps; ++r) {
    if (constN)
      constN<<<karg.grid, karg.block>>>(y, A, x, M, alpha, beta);
    else
      varN<<<karg.grid, karg.block>>>(y, A, x, M, N, alpha, beta);
  }
  cudaEventRecord(b);
  e = cudaGetLastError();
  const int st = timed(a, b, reps, ms);
  cudaUnbindTexture(texFloatA);
  cudaUnbindTexture(texFloatx);
  return e != cudaSuccess ? static_cast<int>(e) : st;
}
#endif
