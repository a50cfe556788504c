// hml_internal.h -- host-side internals shared by the library's translation
// units: the canonical problem forms, launch helpers, tensor-map encoding
// and per-device resources.
#pragma once

#include <cuda.h>  // CUtensorMap and its enums (header only; the driver
                   // entry point is looked up at run time)
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/hml_b200.h"

namespace hml {

// Canonical SGEMM: C(m,n) = alpha * sum_k A(m,k) B(k,n) + beta * C(m,n),
// with A(m,k) = A[m*sam + k*sak], B(k,n) = B[k*sbk + n*sbn],
// C(m,n) = C[m*scm + n*scn].  After normalisation M >= N (M is the long
// dimension) and each operand has one unit stride.
struct GemmProblem {
  int M, N, K;
  float alpha, beta;
  const float *A;
  int64_t sam, sak;
  const float *B;
  int64_t sbk, sbn;
  float *C;
  int64_t scm, scn;
  bool a_kcontig() const { return sak == 1 && !(sam == 1 && K == 1); }
  bool b_kcontig() const { return sbk == 1; }
};

// Canonical SGEMV: y[p*incy] = alpha * sum_q A(p,q) x[q*incx] + beta * y,
// A(p,q) = A[p*sp + q*sq].
struct GemvProblem {
  int P, Q;
  float alpha, beta;
  const float *A;
  int64_t sp, sq;
  const float *x;
  int64_t incx;
  float *y;
  int64_t incy;
};

hml_status gemm_from_blas(hml_order order, hml_op ta, hml_op tb, int M, int N, int K,
                          float alpha, const float *A, int lda, const float *B, int ldb,
                          float beta, float *C, int ldc, GemmProblem *out);

hml_status gemv_from_blas(hml_order order, hml_op trans, int M, int N, float alpha,
                          const float *A, int lda, const float *x, float beta, float *y,
                          GemvProblem *out);

// Kernels (one launcher per family).  All are stream ordered.
// launch_gemv's variant: threads per row (4..256, powers of two) when the
// rows of A are contiguous, CTAs per row tile (1..kGemvMaxColSplit; a tile
// is 256 rows, or 128 when P <= 128) when the columns are; 0 = the
// heuristic; kGemvTuned = the autotuner's measured table, else the
// heuristic.
constexpr int kGemvTuned = -1;
constexpr int kGemvMaxColSplit = 256;
hml_status launch_gemv(const GemvProblem &p, int variant, cudaStream_t s);
// A GEMM with N == 1 as the GEMV it is (false when N != 1; api.cu).
bool as_gemv(const GemmProblem &p, GemvProblem *g);
// Which GEMV kernel serves p: the row kernel (rows of A contiguous) or the
// column kernel.
inline bool gemv_rows_layout(const GemvProblem &p) {
  return p.sq == 1 && !(p.Q == 1 && p.sp == 1);
}
inline bool gemv_variant_valid(bool rows, int v) {
  return rows ? (v >= 4 && v <= 256 && (v & (v - 1)) == 0) : (v >= 1 && v <= kGemvMaxColSplit);
}
hml_status launch_scale(float *C, int M, int N, int64_t scm, int64_t scn, float beta,
                        cudaStream_t s);
hml_status launch_simt(const GemmProblem &p, const hml_sgemm_config &c, cudaStream_t s);
// waves: a split_k = 1 configuration whose grid would end in a partial wave
// runs that wave's rows as a second grid split in K (automatic selection
// only; an explicitly given configuration runs exactly as given).
hml_status launch_tc(const GemmProblem &p, const hml_sgemm_config &c, cudaStream_t s,
                     bool waves = false);
hml_status check_simt(const GemmProblem &p, const hml_sgemm_config &c);
// The stream-K SIMT kernel for N <= 8 with contiguous columns of A
// (sgemm_stream.cu); reached through the SIMT family's variants
// simt_num_shapes() .. simt_num_shapes() + stream_num_variants() - 1.
int stream_num_variants();
int stream_tile_n(int i);
int stream_max_stages(int nb);  // deepest ring that fits
hml_status check_stream(const GemmProblem &p, const hml_sgemm_config &c);
hml_status launch_stream(const GemmProblem &p, const hml_sgemm_config &c, cudaStream_t s);
hml_status check_tc(const GemmProblem &p, const hml_sgemm_config &c);

// The split-BF16 part of a batched plan (sgemm_tc.cu): problems that
// tc_batch_eligible accepts run as persistent tensor-core launches, one per
// tile-width class, after one launch that splits every B into BF16 planes.
// With `stream_ordered` the device memory is allocated and freed on that
// stream.
struct TcBatch;
bool tc_batch_eligible(const GemmProblem &p);
hml_status tc_batch_create(const GemmProblem *probs, int count, cudaStream_t stream_ordered,
                           TcBatch **out);
hml_status tc_batch_launch(const TcBatch *b, cudaStream_t s);
void tc_batch_destroy(TcBatch *b);
hml_sgemm_config tc_batch_config(const GemmProblem &p);
int tc_batch_items(const TcBatch *b);
int tc_batch_ctas(const TcBatch *b);

// Launches a kernel whose bounded wait expires (verify.cu).
hml_status check_wait_limit(cudaStream_t s);

// Per-device resources.
int *device_error_word();  // nullptr on failure
int *device_error_word_if_any();  // nullptr when not allocated yet (allocates nothing)
// Reads and clears the allocation-free entry point's error word (sgemm_tc.cu).
hml_status noalloc_take_error(int *code);
hml_status workspace(size_t bytes, cudaStream_t s, void **ptr);
// The same for a second, independent buffer per (device, stream): slot 1 holds
// data that outlives a library call made in between (which uses slot 0).
hml_status workspace_slot(int slot, size_t bytes, cudaStream_t s, void **ptr);
// n zero-initialised counters private to (device, stream).  Kernels that use
// them leave every counter at zero again when they finish.
hml_status tile_counters(size_t n, cudaStream_t s, unsigned **ptr);

// Tensor maps.
bool tensor_map_2d(CUtensorMap *map, CUtensorMapDataType dtype, const void *base,
                   uint64_t dim0, uint64_t dim1, uint64_t stride1_bytes, uint32_t box0,
                   uint32_t box1, CUtensorMapSwizzle swizzle);

inline hml_status cuda_status(cudaError_t e) {
  return e == cudaSuccess ? HML_STATUS_SUCCESS : HML_STATUS_CUDA_ERROR;
}

// Remember the last CUDA error text for diagnostics.
void note_cuda_error(cudaError_t e, const char *where);
void note_text_error(const char *text);
const char *last_error_text();

int sm_count();

// Number of kernels this library has launched (all devices, all threads).
void count_launch(int n = 1);
uint64_t launch_count();

// Launch with an optional thread-block cluster along x.
// `early`: programmatic dependent launch -- the kernel may start while the
// previous kernel on the stream is still running (once all of that kernel's
// CTAs have executed griddepcontrol.launch_dependents); the kernel must
// execute griddepcontrol.wait before it reads anything that kernel writes.
template <typename... KArgs, typename... Args>
cudaError_t launch_k_ex(void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem,
                        cudaStream_t s, int cluster_x, bool early, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[2];
  int n = 0;
  if (cluster_x > 1) {
    attr[n].id = cudaLaunchAttributeClusterDimension;
    attr[n].val.clusterDim.x = cluster_x;
    attr[n].val.clusterDim.y = 1;
    attr[n].val.clusterDim.z = 1;
    ++n;
  }
  if (early) {
    attr[n].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[n].val.programmaticStreamSerializationAllowed = 1;
    ++n;
  }
  cfg.attrs = n ? attr : nullptr;
  cfg.numAttrs = n;
  count_launch();
  return cudaLaunchKernelEx(&cfg, k, static_cast<KArgs>(args)...);
}

template <typename... KArgs, typename... Args>
cudaError_t launch_k(void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                     int cluster_x, Args... args) {
  return launch_k_ex(k, grid, block, smem, s, cluster_x, false, args...);
}

}  // namespace hml
