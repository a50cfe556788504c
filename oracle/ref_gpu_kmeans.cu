// ref_gpu_kmeans.cu -- TEST INFRASTRUCTURE ONLY.  The reference's k-means
// assignment kernel, hmlKmeansAssignCtrdSmem (include/hml_kmeans_kernel_
// template.h:19-90), compiled from its header with ref_gpu_compat.h and
// launched as the reference launches it (setKmeansAssignSmemArg,
// src/hml_kmeans_kernel.cu:214-224: 256 threads, 1024 blocks, the centroids
// in dynamic shared memory), without textures (the repository's
// shared-memory entries use useTextureMem = false,
// src/hml_kmeans_kernel_init.cu:100-).  The parity target of the library's
// hml_kmeans_assign.
#include <cuda_runtime.h>
#include <stdint.h>

#include "hml_common.h"
#include "hml_kmeans_kernel_template.h"

// the texture object the header names (unused by the texture-free kernels)
texture<float, 1> texData1;

namespace {
template <uint32_t D>
cudaError_t launch(uint32_t *asg, const float *rows, uint32_t n, const float *ctrds, uint32_t k) {
  const size_t smem = sizeof(float) * D * k;
  cudaError_t e = cudaSuccess;
  if (smem > 48 * 1024)
    e = cudaFuncSetAttribute(hmlKmeansAssignCtrdSmem<D, false>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  hmlKmeansAssignCtrdSmem<D, false><<<1024, 256, smem>>>(asg, rows, n, ctrds, k);
  return cudaGetLastError();
}
}  // namespace

// Dimensions with an instantiation here: 4, 8, 16, 32, 64.
extern "C" int ref_gpu_kmeans_assign(uint32_t *asg, const float *rows, uint32_t num_rows,
                                     const float *ctrds, uint32_t num_clusts, uint32_t num_dims,
                                     int reps, float *ms) {
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  cudaEventRecord(a);
  cudaError_t e = cudaSuccess;
  for (int r = 0; r < reps && e == cudaSuccess; ++r) {
    switch (num_dims) {
      case 4: e = launch<4>(asg, rows, num_rows, ctrds, num_clusts); break;
      case 8: e = launch<8>(asg, rows, num_rows, ctrds, num_clusts); break;
      case 16: e = launch<16>(asg, rows, num_rows, ctrds, num_clusts); break;
      case 32: e = launch<32>(asg, rows, num_rows, ctrds, num_clusts); break;
      case 64: e = launch<64>(asg, rows, num_rows, ctrds, num_clusts); break;
      default: e = cudaErrorInvalidValue;
    }
  }
  cudaEventRecord(b);
  cudaError_t e2 = cudaEventSynchronize(b);
  float t = 0.0f;
  if (e2 == cudaSuccess) e2 = cudaEventElapsedTime(&t, a, b);
  if (ms) *ms = reps > 0 ? t / reps : 0.0f;
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return static_cast<int>(e != cudaSuccess ? e : e2);
}
