/*
 * ref_compat.h -- forced-include header for compiling the reference's own
 * CPU verification sources with CUDA 12, where legacy texture references
 * (texture<>, cudaBindTexture, cudaUnbindTexture, tex1Dfetch) no longer
 * exist.  TEST INFRASTRUCTURE ONLY: used by oracle/Makefile to build
 * oracle/_ref from the reference's unmodified sources.
 *
 * The stand-ins are inert: binding reports cudaErrorNotSupported and a fetch
 * yields 0.  None of them is reached by the functions the oracle calls
 * (hmlSgemmCpu, hmlSgemvCpu, hmlComputeCsum, hmlComputeYsum), which are
 * plain host loops.
 */
#ifndef HML_ORACLE_REF_COMPAT_H_
#define HML_ORACLE_REF_COMPAT_H_
#include <cuda_runtime.h>

template <class T, int dim = 1,
          enum cudaTextureReadMode mode = cudaReadModeElementType>
struct texture {
  int unused_;
};

template <class T, int dim, enum cudaTextureReadMode mode>
static inline cudaError_t cudaBindTexture(size_t *, const texture<T, dim, mode> &,
                                          const void *, size_t = ~(size_t)0) {
  return cudaErrorNotSupported;
}

template <class T, int dim, enum cudaTextureReadMode mode>
static inline cudaError_t cudaUnbindTexture(const texture<T, dim, mode> &) {
  return cudaSuccess;
}

#define tex1Dfetch(tex, idx) (0)
#endif
