// api.cu -- the extern "C" entry points of include/hml_b200.h: argument
// validation, normalisation of BLAS problems to the canonical long-M form,
// configuration space and selection, and dispatch to the kernel families.
#include <algorithm>
#include <cstring>
#include <vector>

#include "hml_internal.h"
#include "hml_select.h"
#include "hml_tune.h"

namespace hml {

hml_status fill_random(float *out, size_t n, uint64_t seed, uint64_t stream_id, int dist,
                       cudaStream_t s);
hml_status sgemm_error_fp64(const GemmProblem &p, const float *C0, double err[4], cudaStream_t s);
hml_status release_all();
int simt_num_shapes();
void simt_shape(int v, int *bm, int *bn, int *wk);
int tc_num_shapes();
void tc_shape(int v, int *bm, int *bn);
bool tc_config_fits(int bn, int ns, int stages);

// ---------------------------------------------------------- normalisation
hml_status gemm_from_blas(hml_order order, hml_op ta, hml_op tb, int M, int N, int K,
                          float alpha, const float *A, int lda, const float *B, int ldb,
                          float beta, float *C, int ldc, GemmProblem *out) {
  if (order != HML_COL_MAJOR && order != HML_ROW_MAJOR) return HML_STATUS_INVALID_VALUE;
  if ((ta != HML_OP_N && ta != HML_OP_T) || (tb != HML_OP_N && tb != HML_OP_T))
    return HML_STATUS_INVALID_VALUE;
  if (M < 0 || N < 0 || K < 0) return HML_STATUS_INVALID_VALUE;
  // storage extents (rows x cols) of each operand in its own order
  const bool cm = order == HML_COL_MAJOR;
  // op(A) is M x K.  Stored as (M x K) when N-op, (K x M) when T-op.
  const int a_rows = (ta == HML_OP_N) ? M : K, a_cols = (ta == HML_OP_N) ? K : M;
  const int b_rows = (tb == HML_OP_N) ? K : N, b_cols = (tb == HML_OP_N) ? N : K;
  const int a_ld_min = std::max(1, cm ? a_rows : a_cols);
  const int b_ld_min = std::max(1, cm ? b_rows : b_cols);
  const int c_ld_min = std::max(1, cm ? M : N);
  if (lda < a_ld_min || ldb < b_ld_min || ldc < c_ld_min) return HML_STATUS_INVALID_VALUE;
  if (M > 0 && N > 0 && !C) return HML_STATUS_INVALID_VALUE;
  if (M > 0 && N > 0 && K > 0 && alpha != 0.0f && (!A || !B)) return HML_STATUS_INVALID_VALUE;
  GemmProblem p;
  p.M = M; p.N = N; p.K = K;
  p.alpha = alpha; p.beta = beta;
  p.A = A; p.B = B; p.C = C;
  // element strides of the logical operands
  int64_t s_row, s_col;  // stride between consecutive rows / cols of storage
  s_row = cm ? 1 : lda; s_col = cm ? lda : 1;
  if (ta == HML_OP_N) { p.sam = s_row; p.sak = s_col; } else { p.sam = s_col; p.sak = s_row; }
  s_row = cm ? 1 : ldb; s_col = cm ? ldb : 1;
  if (tb == HML_OP_N) { p.sbk = s_row; p.sbn = s_col; } else { p.sbk = s_col; p.sbn = s_row; }
  p.scm = cm ? 1 : ldc;
  p.scn = cm ? ldc : 1;
  // the long dimension becomes M:  C^T = B^T A^T
  if (p.N > p.M) {
    GemmProblem q = p;
    q.M = p.N; q.N = p.M;
    q.A = p.B; q.sam = p.sbn; q.sak = p.sbk;
    q.B = p.A; q.sbk = p.sak; q.sbn = p.sam;
    q.scm = p.scn; q.scn = p.scm;
    p = q;
  }
  // a unit dimension can carry any stride: make the unit-stride side explicit
  if (p.K == 1) { p.sak = 1; p.sbk = 1; }
  if (p.M == 1) p.sam = 1;
  if (p.N == 1) p.sbn = 1;
  if (p.sam != 1 && p.sak != 1) return HML_STATUS_INVALID_VALUE;
  *out = p;
  return HML_STATUS_SUCCESS;
}

hml_status gemv_from_blas(hml_order order, hml_op trans, int M, int N, float alpha,
                          const float *A, int lda, const float *x, float beta, float *y,
                          GemvProblem *out) {
  if (order != HML_COL_MAJOR && order != HML_ROW_MAJOR) return HML_STATUS_INVALID_VALUE;
  if (trans != HML_OP_N && trans != HML_OP_T) return HML_STATUS_INVALID_VALUE;
  if (M < 0 || N < 0) return HML_STATUS_INVALID_VALUE;
  const bool cm = order == HML_COL_MAJOR;
  if (lda < std::max(1, cm ? M : N)) return HML_STATUS_INVALID_VALUE;
  const int P = trans == HML_OP_N ? M : N, Q = trans == HML_OP_N ? N : M;
  if (P > 0 && !y) return HML_STATUS_INVALID_VALUE;
  if (P > 0 && Q > 0 && alpha != 0.0f && (!A || !x)) return HML_STATUS_INVALID_VALUE;
  GemvProblem g;
  g.P = P; g.Q = Q; g.alpha = alpha; g.beta = beta;
  g.A = A; g.x = x; g.y = y; g.incx = 1; g.incy = 1;
  const int64_t s_row = cm ? 1 : lda, s_col = cm ? lda : 1;
  if (trans == HML_OP_N) { g.sp = s_row; g.sq = s_col; } else { g.sp = s_col; g.sq = s_row; }
  // a unit dimension can carry any stride
  if (g.Q == 1) g.sq = 1;
  else if (g.P == 1) g.sp = 1;
  *out = g;
  return HML_STATUS_SUCCESS;
}

// ------------------------------------------------------ configuration space
namespace {

std::vector<hml_sgemm_config> build_space() {
  std::vector<hml_sgemm_config> v;
  for (int var = 0; var < simt_num_shapes(); ++var) {
    int bm, bn, wk;
    simt_shape(var, &bm, &bn, &wk);
    for (int split : {1, 2, 4, 8, 16})
      for (int stages : {2, 3, 4, 6}) {
        hml_sgemm_config c = {HML_ALGO_SIMT, bm, bn, split, stages, var};
        const size_t smem = std::max<size_t>(static_cast<size_t>(bm + bn) * 128 * stages,
                                             static_cast<size_t>(wk) * bm * bn * 4);
        if (smem + 1024 + 128 > 227 * 1024) continue;
        v.push_back(c);
      }
  }
  // the stream-K kernel for N <= 8 (variants after the tiled shapes)
  for (int i = 0; i < stream_num_variants(); ++i) {
    const int nb = stream_tile_n(i), top = stream_max_stages(nb);
    for (int stages : {top - 2, top - 1, top}) {
      hml_sgemm_config c = {HML_ALGO_SIMT, 128, nb, 1, stages, simt_num_shapes() + i};
      v.push_back(c);
    }
  }
  // (TF32X3 is an explicit configuration only: as accurate as BF16X6 and
  // measured no faster -- slower up to N = 64, 2 % faster at N = 128)
  for (int algo : {HML_ALGO_BF16X3, HML_ALGO_BF16X6})
    for (int var = 0; var < tc_num_shapes(); ++var) {
      int bm, bn;
      tc_shape(var, &bm, &bn);
      // CTA-pair tiles are explicit configurations only: correct (bitwise
      // equal to the 128-row tile) but measured slower on B200, the
      // per-block handshakes between the two CTAs costing about 1 us
      if (bm != 128) continue;
      for (int split : {1, 2, 4, 8, 16})
        for (int stages : {2, 4, 6, 8}) {  // A-ring depths: multiples of the converter groups
          if (!tc_config_fits(bn, algo == HML_ALGO_BF16X3 ? 2 : 3, stages)) continue;
          hml_sgemm_config c = {algo, bm, bn, split, stages, var};
          v.push_back(c);
        }
    }
  return v;
}

const std::vector<hml_sgemm_config> &space() {
  static const std::vector<hml_sgemm_config> s = build_space();
  return s;
}

bool same_config(const hml_sgemm_config &a, const hml_sgemm_config &b) {
  return a.algo == b.algo && a.tile_m == b.tile_m && a.tile_n == b.tile_n &&
         a.split_k == b.split_k && a.stages == b.stages && a.variant == b.variant;
}

hml_status run(const GemmProblem &p, const hml_sgemm_config &c, cudaStream_t s, bool auto_choice) {
  if (p.M == 0 || p.N == 0) return HML_STATUS_SUCCESS;
  if (p.K == 0 || p.alpha == 0.0f) return launch_scale(p.C, p.M, p.N, p.scm, p.scn, p.beta, s);
  switch (c.algo) {
    case HML_ALGO_SIMT: return launch_simt(p, c, s);
    case HML_ALGO_BF16X3:
    case HML_ALGO_BF16X6:
    case HML_ALGO_TF32X3:
    case HML_ALGO_FP16X3: return launch_tc(p, c, s, auto_choice);
    default: return HML_STATUS_INVALID_VALUE;
  }
}

}  // namespace

// N == 1 is a GEMV: route it to the GEMV kernels.
bool as_gemv(const GemmProblem &p, GemvProblem *g) {
  if (p.N != 1) return false;
  g->P = p.M; g->Q = p.K; g->alpha = p.alpha; g->beta = p.beta;
  g->A = p.A; g->sp = p.sam; g->sq = p.sak;
  g->x = p.B; g->incx = p.sbk;
  g->y = p.C; g->incy = p.scm;
  return true;
}

const std::vector<hml_sgemm_config> &config_space() { return space(); }

hml_status check_config(const GemmProblem &p, const hml_sgemm_config &c) {
  switch (c.algo) {
    case HML_ALGO_SIMT: return check_simt(p, c);
    case HML_ALGO_BF16X3:
    case HML_ALGO_BF16X6:
    case HML_ALGO_TF32X3:
    case HML_ALGO_FP16X3: return check_tc(p, c);
    default: return HML_STATUS_INVALID_VALUE;
  }
}

bool check_config_ok(const GemmProblem &p, const hml_sgemm_config &c) {
  return check_config(p, c) == HML_STATUS_SUCCESS;
}

hml_status run_config(const GemmProblem &p, const hml_sgemm_config &c, cudaStream_t s,
                      bool auto_choice) {
  hml_status st = check_config(p, c);
  if (st != HML_STATUS_SUCCESS) return st;
  return run(p, c, s, auto_choice);
}

}  // namespace hml

using namespace hml;

extern "C" {

const char *hml_status_string(hml_status s) {
  switch (s) {
    case HML_STATUS_SUCCESS: return "success";
    case HML_STATUS_INVALID_VALUE: return "invalid value";
    case HML_STATUS_NOT_SUPPORTED: return "not supported";
    case HML_STATUS_CUDA_ERROR: return "CUDA error";
    case HML_STATUS_ALLOC_FAILED: return "allocation failed";
    case HML_STATUS_CONFIG_ERROR: return "configuration error";
    case HML_STATUS_TIMEOUT: return "device wait timed out";
    case HML_STATUS_IO_ERROR: return "I/O error";
  }
  return "unknown status";
}

const char *hml_version(void) { return "hml-b200 0.1 (sm_100a)"; }

const char *hml_last_error(void) { return last_error_text(); }

hml_status hml_sgemm_ex(hml_order order, hml_op transA, hml_op transB, int M, int N, int K,
                        float alpha, const float *A, int lda, const float *B, int ldb,
                        float beta, float *C, int ldc, void *stream) {
  GemmProblem p;
  hml_status st = gemm_from_blas(order, transA, transB, M, N, K, alpha, A, lda, B, ldb, beta, C,
                                 ldc, &p);
  if (st != HML_STATUS_SUCCESS) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (p.M == 0 || p.N == 0) return HML_STATUS_SUCCESS;
  if (p.K == 0 || p.alpha == 0.0f) return launch_scale(p.C, p.M, p.N, p.scm, p.scn, p.beta, s);
  GemvProblem g;
  if (as_gemv(p, &g)) return launch_gemv(g, kGemvTuned, s);
  hml_sgemm_config c;
  st = select_config(p, &c, s);
  if (st != HML_STATUS_SUCCESS) return st;
  return run_config(p, c, s, true);
}

hml_status hml_sgemm_ex_config(hml_order order, hml_op transA, hml_op transB, int M, int N,
                               int K, float alpha, const float *A, int lda, const float *B,
                               int ldb, float beta, float *C, int ldc,
                               const hml_sgemm_config *config, void *stream) {
  if (!config || config->algo == HML_ALGO_AUTO) return HML_STATUS_INVALID_VALUE;
  GemmProblem p;
  hml_status st = gemm_from_blas(order, transA, transB, M, N, K, alpha, A, lda, B, ldb, beta, C,
                                 ldc, &p);
  if (st != HML_STATUS_SUCCESS) return st;
  return run_config(p, *config, static_cast<cudaStream_t>(stream));
}

hml_status hml_sgemm_select(hml_order order, hml_op transA, hml_op transB, int M, int N, int K,
                            hml_sgemm_config *config) {
  if (!config) return HML_STATUS_INVALID_VALUE;
  GemmProblem p;
  // strides do not influence the choice beyond layout: use dense ones
  const bool cm = order == HML_COL_MAJOR;
  const int lda = std::max(1, cm ? (transA == HML_OP_N ? M : K) : (transA == HML_OP_N ? K : M));
  const int ldb = std::max(1, cm ? (transB == HML_OP_N ? K : N) : (transB == HML_OP_N ? N : K));
  const int ldc = std::max(1, cm ? M : N);
  alignas(16) static float dummy[4];
  hml_status st = gemm_from_blas(order, transA, transB, M, N, K, 1.0f, dummy, lda, dummy, ldb,
                                 0.0f, dummy, ldc, &p);
  if (st != HML_STATUS_SUCCESS) return st;
  return select_config(p, config);
}

hml_status hml_sgemm_select_algo(hml_order order, hml_op transA, hml_op transB, int M, int N,
                                 int K, int algo, hml_sgemm_config *config) {
  if (!config) return HML_STATUS_INVALID_VALUE;
  if (algo == HML_ALGO_AUTO) return hml_sgemm_select(order, transA, transB, M, N, K, config);
  if (algo != HML_ALGO_SIMT && algo != HML_ALGO_BF16X3 && algo != HML_ALGO_BF16X6 &&
      algo != HML_ALGO_TF32X3 && algo != HML_ALGO_FP16X3)
    return HML_STATUS_INVALID_VALUE;
  GemmProblem p;
  const bool cm = order == HML_COL_MAJOR;
  const int lda = std::max(1, cm ? (transA == HML_OP_N ? M : K) : (transA == HML_OP_N ? K : M));
  const int ldb = std::max(1, cm ? (transB == HML_OP_N ? K : N) : (transB == HML_OP_N ? N : K));
  const int ldc = std::max(1, cm ? M : N);
  alignas(16) static float dummy[4];
  hml_status st = gemm_from_blas(order, transA, transB, M, N, K, 1.0f, dummy, lda, dummy, ldb,
                                 0.0f, dummy, ldc, &p);
  if (st != HML_STATUS_SUCCESS) return st;
  *config = heuristic_config(p, algo);
  return check_config(p, *config);
}

hml_status hml_sgemm_config_check(hml_order order, hml_op transA, hml_op transB, int M, int N,
                                  int K, int lda, int ldb, int ldc,
                                  const hml_sgemm_config *config) {
  if (!config) return HML_STATUS_INVALID_VALUE;
  alignas(16) static float dummy[4];
  GemmProblem p;
  hml_status st = gemm_from_blas(order, transA, transB, M, N, K, 1.0f, dummy, lda, dummy, ldb,
                                 0.0f, dummy, ldc, &p);
  if (st != HML_STATUS_SUCCESS) return st;
  return check_config(p, *config);
}

int hml_sgemm_num_configs(void) { return static_cast<int>(space().size()); }

hml_status hml_sgemm_get_config(int index, hml_sgemm_config *config) {
  if (!config || index < 0 || index >= static_cast<int>(space().size()))
    return HML_STATUS_INVALID_VALUE;
  *config = space()[index];
  return HML_STATUS_SUCCESS;
}

int hml_sgemm_config_index(const hml_sgemm_config *config) {
  if (!config) return -1;
  const auto &s = space();
  for (size_t i = 0; i < s.size(); ++i)
    if (same_config(s[i], *config)) return static_cast<int>(i);
  return -1;
}

hml_status hml_sgemv_ex(hml_order order, hml_op trans, int M, int N, float alpha,
                        const float *A, int lda, const float *x, float beta, float *y,
                        void *stream) {
  GemvProblem g;
  hml_status st = gemv_from_blas(order, trans, M, N, alpha, A, lda, x, beta, y, &g);
  if (st != HML_STATUS_SUCCESS) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (g.P == 0) return HML_STATUS_SUCCESS;
  if (g.Q == 0 || g.alpha == 0.0f) return launch_scale(g.y, g.P, 1, g.incy, 0, g.beta, s);
  return launch_gemv(g, kGemvTuned, s);
}

hml_status hml_sgemv_select(hml_order order, hml_op trans, int M, int N, int lda, int *variant) {
  if (!variant) return HML_STATUS_INVALID_VALUE;
  GemvProblem g;
  float y = 0.0f;  // only the layout is read
  hml_status st = gemv_from_blas(order, trans, M, N, 0.0f, nullptr, lda, nullptr, 0.0f, &y, &g);
  if (st != HML_STATUS_SUCCESS) return st;
  int v = 0;
  *variant = g.P > 0 && g.Q > 0 && gemv_tuned_lookup(g, &v) &&
                     gemv_variant_valid(gemv_rows_layout(g), v)
                 ? v
                 : 0;
  return HML_STATUS_SUCCESS;
}

hml_status hml_sgemv_ex_variant(hml_order order, hml_op trans, int M, int N, float alpha,
                                const float *A, int lda, const float *x, float beta, float *y,
                                int variant, void *stream) {
  GemvProblem g;
  hml_status st = gemv_from_blas(order, trans, M, N, alpha, A, lda, x, beta, y, &g);
  if (st != HML_STATUS_SUCCESS) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (g.P == 0) return HML_STATUS_SUCCESS;
  if (g.Q == 0 || g.alpha == 0.0f) return launch_scale(g.y, g.P, 1, g.incy, 0, g.beta, s);
  if (variant < 0) return HML_STATUS_INVALID_VALUE;
  return launch_gemv(g, variant, s);
}

hml_status hml_fill_random(float *out, size_t n, uint64_t seed, uint64_t stream_id, int dist,
                           void *stream) {
  return fill_random(out, n, seed, stream_id, dist, static_cast<cudaStream_t>(stream));
}

hml_status hml_sgemm_error_fp64(hml_order order, hml_op transA, hml_op transB, int M, int N,
                                int K, float alpha, const float *A, int lda, const float *B,
                                int ldb, float beta, const float *C0, const float *C, int ldc,
                                double err[4], void *stream) {
  if (!err) return HML_STATUS_INVALID_VALUE;
  GemmProblem p;
  hml_status st = gemm_from_blas(order, transA, transB, M, N, K, alpha, A, lda, B, ldb, beta,
                                 const_cast<float *>(C), ldc, &p);
  if (st != HML_STATUS_SUCCESS) return st;
  return sgemm_error_fp64(p, C0, err, static_cast<cudaStream_t>(stream));
}

hml_status hml_device_error(int *code) {
  if (!code) return HML_STATUS_INVALID_VALUE;
  *code = 0;
  // the allocation-free entry point's own word first; it allocates nothing
  int na = 0;
  hml_status st = noalloc_take_error(&na);
  if (st != HML_STATUS_SUCCESS) return st;
  // the library's word exists once a kernel that records errors has run
  int *w = device_error_word_if_any();
  int h = 0;
  cudaError_t e = cudaSuccess;
  if (w) {
    e = cudaMemcpy(&h, w, sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && h != 0) e = cudaMemset(w, 0, sizeof(int));
    note_cuda_error(e, "device_error");
  }
  *code = h != 0 ? h : na;
  return cuda_status(e);
}

hml_status hml_check_wait_limit(void *stream) {
  return check_wait_limit(static_cast<cudaStream_t>(stream));
}

hml_status hml_release_resources(void) { return release_all(); }

uint64_t hml_launch_count(void) { return launch_count(); }

}  // extern "C"
