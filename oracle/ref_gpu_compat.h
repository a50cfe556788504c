/*
 * ref_gpu_compat.h -- forced-include header for compiling the reference's own
 * SGEMM / SGEMV GPU kernels (and their selectors) with CUDA 12, which
 * removed legacy texture references.  TEST INFRASTRUCTURE ONLY: used by
 * oracle/Makefile to build oracle/_ref/libhml_ref_gpu_{sgemm,sgemv}.so from
 * the reference's unmodified sources, as the GPU baseline and a parity
 * target; nothing in hiperml_b200/ uses it.
 *
 * The reference reads A, B and x through 1-D texture references bound to
 * linear device memory (src/hml_utils.cu:175-230) and relies on a fetch past
 * the bound range returning 0 (its last row blocks and K tails read past the
 * arrays).  The stand-in keeps that behaviour without textures:
 *   - `texture<T, 1>` objects stay host objects (their identity is all the
 *     binding needs), registered by address under the name they have in the
 *     reference (texFloatA, texFloatB, texFloatx);
 *   - cudaBindTexture / cudaUnbindTexture record the bound (pointer, length)
 *     in a small __device__ table of every translation unit of the library;
 *   - tex1Dfetch(t, i) reads element i of the range bound to t, 0 outside it.
 * One library is built per reference API (HML_REF_SGEMM, HML_REF_SGEMV or
 * HML_REF_KMEANS), because the SGEMM and SGEMV sources both define a texture
 * named texFloatA.
 */
#ifndef HML_ORACLE_REF_GPU_COMPAT_H_
#define HML_ORACLE_REF_GPU_COMPAT_H_
#include <cuda_runtime.h>
#include <stddef.h>

struct HmlRefTexRange {
  const void *ptr;
  size_t n;  /* elements */
};

template <class T, int dim = 1, enum cudaTextureReadMode mode = cudaReadModeElementType>
struct texture {
  int unused_;
};

/* registry shared by the library's translation units (ref_gpu_registry.cu) */
void hml_ref_register_texture(const void *host_obj, int id);
void hml_ref_register_table(cudaError_t (*update)(int id, const void *ptr, size_t n));
cudaError_t hml_ref_bind(const void *host_obj, const void *ptr, size_t n);

enum {
  hml_ref_tex_texFloatA = 0,
  hml_ref_tex_texFloatB = 1,
  hml_ref_tex_texFloatx = 2,
  hml_ref_tex_texData1 = 3
};

/* this translation unit's table, and its update hook */
static __device__ HmlRefTexRange hml_ref_tex_table[4];
static cudaError_t hml_ref_update_table(int id, const void *ptr, size_t n) {
  HmlRefTexRange r;
  r.ptr = ptr;
  r.n = n;
  return cudaMemcpyToSymbol(hml_ref_tex_table, &r, sizeof r, id * sizeof r);
}
static int hml_ref_table_registered = (hml_ref_register_table(&hml_ref_update_table), 0);

#if defined(HML_REF_SGEMM)
extern texture<float, 1> texFloatA;
extern texture<float, 1> texFloatB;
static int hml_ref_textures_registered =
    (hml_ref_register_texture(&texFloatA, hml_ref_tex_texFloatA),
     hml_ref_register_texture(&texFloatB, hml_ref_tex_texFloatB), 0);
#elif defined(HML_REF_SGEMV)
extern texture<float, 1> texFloatA;
extern texture<float, 1> texFloatx;
static int hml_ref_textures_registered =
    (hml_ref_register_texture(&texFloatA, hml_ref_tex_texFloatA),
     hml_ref_register_texture(&texFloatx, hml_ref_tex_texFloatx), 0);
#endif

template <class T, int dim, enum cudaTextureReadMode mode>
static inline cudaError_t cudaBindTexture(size_t *offset, const texture<T, dim, mode> &tex,
                                          const void *ptr, size_t size = ~(size_t)0) {
  if (offset) *offset = 0;
  return hml_ref_bind(&tex, ptr, size / sizeof(T));
}

template <class T, int dim, enum cudaTextureReadMode mode>
static inline cudaError_t cudaUnbindTexture(const texture<T, dim, mode> &tex) {
  return hml_ref_bind(&tex, NULL, 0);
}

static __device__ __forceinline__ float hml_ref_fetch(int id, int i) {
  const HmlRefTexRange r = hml_ref_tex_table[id];
  return (i >= 0 && (size_t)i < r.n) ? static_cast<const float *>(r.ptr)[i] : 0.0f;
}
#define tex1Dfetch(t, i) hml_ref_fetch(hml_ref_tex_##t, (i))

#endif
