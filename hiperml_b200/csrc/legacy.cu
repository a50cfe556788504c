// legacy.cu -- the reference's public C++ entry points (same names,
// signatures and C++ linkage as include/hml_sgemm.h and include/hml_sgemv.h
// of the reference), as shims over the C ABI.
//
// hmlSgemm / hmlSgemv take HOST pointers (src/hml_sgemm.cu:120-211,
// src/hml_sgemv.cu:125-213).  Where the reference cudaMallocs and frees three
// buffers per call and copies synchronously, these keep grow-only device
// buffers per device and move the data on a library-owned stream:
// A is copied in row chunks while the chunks already on the device are
// multiplied, and each finished chunk of C is copied back while the next one
// runs (copy/compute overlap on two streams).  Host buffers that are pinned
// (cudaHostAlloc / cudaHostRegister) are copied by DMA directly.
#include <cstdio>
#include <cstring>
#include <mutex>
#include <map>
#include <string>

#include "../../include/hml_sgemm.h"
#include "../../include/hml_sgemv.h"
#include "hml_internal.h"
#include "hml_select.h"

namespace hml {

hml_status cfg_v1_load(int kind, const char *path, int *rules);
bool cfg_v1_sgemv_rule(int N, int *type, int *block_stops, int *row_stops);
hml_status tune_load(const char *path, int *records);
hml_status sgemv_variant(int order, int trans, int M, int N, float alpha, const float *A, int lda,
                         const float *x, float beta, float *y, int variant, cudaStream_t s);

namespace {

constexpr int kChunks = 4;

struct HostPath {
  cudaStream_t copy = nullptr, comp = nullptr;
  cudaEvent_t in_ready[kChunks] = {}, out_ready[kChunks] = {}, b_ready = nullptr;
  float *buf = nullptr;
  size_t cap = 0;  // floats
};

std::mutex g_mu;
std::map<int, HostPath> g_paths;

hml_status get_path(HostPath **out) {
  int d = 0;
  cudaGetDevice(&d);
  HostPath &h = g_paths[d];
  if (!h.copy) {
    cudaError_t e = cudaStreamCreateWithFlags(&h.copy, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h.comp, cudaStreamNonBlocking);
    for (int i = 0; i < kChunks && e == cudaSuccess; ++i) {
      e = cudaEventCreateWithFlags(&h.in_ready[i], cudaEventDisableTiming);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h.out_ready[i], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h.b_ready, cudaEventDisableTiming);
    if (e != cudaSuccess) {
      note_cuda_error(e, "host path setup");
      h.copy = nullptr;
      return HML_STATUS_CUDA_ERROR;
    }
  }
  *out = &h;
  return HML_STATUS_SUCCESS;
}

hml_status reserve(HostPath &h, size_t floats) {
  if (h.cap >= floats) return HML_STATUS_SUCCESS;
  if (h.buf) {
    cudaStreamSynchronize(h.copy);
    cudaStreamSynchronize(h.comp);
    cudaFree(h.buf);
    h.buf = nullptr;
    h.cap = 0;
  }
  cudaError_t e = cudaMalloc(&h.buf, floats * sizeof(float));
  if (e != cudaSuccess) {
    note_cuda_error(e, "host path buffers");
    h.buf = nullptr;
    return HML_STATUS_ALLOC_FAILED;
  }
  h.cap = floats;
  return HML_STATUS_SUCCESS;
}

void report(const char *fn, hml_status st) {
  if (st == HML_STATUS_SUCCESS) return;
  fprintf(stderr, "hml: %s: %s (%s)\n", fn, hml_status_string(st), last_error_text());
}

#define HML_TRY(expr)                                  \
  do {                                                 \
    cudaError_t e_ = (expr);                           \
    if (e_ != cudaSuccess) {                           \
      note_cuda_error(e_, #expr);                      \
      return HML_STATUS_CUDA_ERROR;                    \
    }                                                  \
  } while (0)

// Row-major C(MxN) = alpha A(MxK) B(KxN) + beta C on host pointers.
// `basic` forces the heuristic configuration (the reference's basic kernel
// is a fixed 6x6 var-K launch, src/hml_sgemm.cu:39-113).
hml_status host_sgemm(bool basic, float *C, const float *A, const float *B, int M, int N, int K,
                      float alpha, float beta) {
  if (M < 0 || N < 0 || K < 0) return HML_STATUS_INVALID_VALUE;
  if (M == 0 || N == 0) return HML_STATUS_SUCCESS;
  if (!C || (K > 0 && (!A || !B))) return HML_STATUS_INVALID_VALUE;
  std::lock_guard<std::mutex> lk(g_mu);
  HostPath *hp;
  hml_status st = get_path(&hp);
  if (st != HML_STATUS_SUCCESS) return st;
  HostPath &h = *hp;
  const size_t nA = static_cast<size_t>(M) * K, nB = static_cast<size_t>(K) * N,
               nC = static_cast<size_t>(M) * N;
  st = reserve(h, nA + nB + nC + 64);
  if (st != HML_STATUS_SUCCESS) return st;
  // sub-buffers start on 64-byte boundaries
  float *dA = h.buf;
  float *dB = reinterpret_cast<float *>((reinterpret_cast<uintptr_t>(dA + nA) + 63) & ~uintptr_t(63));
  float *dC = reinterpret_cast<float *>((reinterpret_cast<uintptr_t>(dB + nB) + 63) & ~uintptr_t(63));
  HML_TRY(cudaMemcpyAsync(dB, B, nB * sizeof(float), cudaMemcpyHostToDevice, h.copy));
  HML_TRY(cudaEventRecord(h.b_ready, h.copy));
  HML_TRY(cudaStreamWaitEvent(h.comp, h.b_ready, 0));
  // row chunks (whole problem when small)
  const int chunks = (nA * sizeof(float) >= (64u << 20) && M >= 4 * 1024) ? kChunks : 1;
  const int rows_per = (M + chunks - 1) / chunks;
  hml_sgemm_config cfg = {};
  for (int c = 0; c < chunks; ++c) {
    const int r0 = c * rows_per;
    const int rc = std::min(M, r0 + rows_per) - r0;
    if (rc <= 0) break;
    HML_TRY(cudaMemcpyAsync(dA + static_cast<size_t>(r0) * K, A + static_cast<size_t>(r0) * K,
                            static_cast<size_t>(rc) * K * sizeof(float), cudaMemcpyHostToDevice,
                            h.copy));
    if (beta != 0.0f)
      HML_TRY(cudaMemcpyAsync(dC + static_cast<size_t>(r0) * N, C + static_cast<size_t>(r0) * N,
                              static_cast<size_t>(rc) * N * sizeof(float),
                              cudaMemcpyHostToDevice, h.copy));
    HML_TRY(cudaEventRecord(h.in_ready[c], h.copy));
    HML_TRY(cudaStreamWaitEvent(h.comp, h.in_ready[c], 0));
    if (basic) {
      GemmProblem p;
      st = gemm_from_blas(HML_ROW_MAJOR, HML_OP_N, HML_OP_N, rc, N, K, alpha,
                          dA + static_cast<size_t>(r0) * K, K, dB, N, beta,
                          dC + static_cast<size_t>(r0) * N, N, &p);
      if (st != HML_STATUS_SUCCESS) return st;
      if (p.N == 1 || p.K == 0 || p.alpha == 0.0f) {
        st = hml_sgemm_ex(HML_ROW_MAJOR, HML_OP_N, HML_OP_N, rc, N, K, alpha,
                          dA + static_cast<size_t>(r0) * K, K, dB, N, beta,
                          dC + static_cast<size_t>(r0) * N, N, h.comp);
      } else {
        cfg = heuristic_config(p, HML_ALGO_SIMT);
        st = run_config(p, cfg, h.comp);
      }
    } else {
      // a loaded reference v1 rule decides, as in the reference's hmlSgemm
      // (src/hml_sgemm.cu:166-167); otherwise the library's own selection
      GemmProblem p;
      st = gemm_from_blas(HML_ROW_MAJOR, HML_OP_N, HML_OP_N, rc, N, K, alpha,
                          dA + static_cast<size_t>(r0) * K, K, dB, N, beta,
                          dC + static_cast<size_t>(r0) * N, N, &p);
      if (st != HML_STATUS_SUCCESS) return st;
      hml_sgemm_config v1;
      if (p.N > 1 && p.K > 0 && p.alpha != 0.0f && v1_rule_config(p, K, N, &v1))
        st = run_config(p, v1, h.comp);
      else
        st = hml_sgemm_ex(HML_ROW_MAJOR, HML_OP_N, HML_OP_N, rc, N, K, alpha,
                          dA + static_cast<size_t>(r0) * K, K, dB, N, beta,
                          dC + static_cast<size_t>(r0) * N, N, h.comp);
    }
    if (st != HML_STATUS_SUCCESS) return st;
    HML_TRY(cudaEventRecord(h.out_ready[c], h.comp));
    HML_TRY(cudaStreamWaitEvent(h.copy, h.out_ready[c], 0));
    HML_TRY(cudaMemcpyAsync(C + static_cast<size_t>(r0) * N, dC + static_cast<size_t>(r0) * N,
                            static_cast<size_t>(rc) * N * sizeof(float), cudaMemcpyDeviceToHost,
                            h.copy));
  }
  HML_TRY(cudaStreamSynchronize(h.copy));
  HML_TRY(cudaStreamSynchronize(h.comp));
  int code = 0;
  if (hml_device_error(&code) == HML_STATUS_SUCCESS && code != 0) return HML_STATUS_TIMEOUT;
  return HML_STATUS_SUCCESS;
}

// Row-major y(M) = alpha A(MxN) x(N) + beta y.
hml_status host_sgemv(int variant, float *y, const float *A, const float *x, int M, int N,
                      float alpha, float beta) {
  if (M < 0 || N < 0) return HML_STATUS_INVALID_VALUE;
  if (M == 0) return HML_STATUS_SUCCESS;
  if (!y || (N > 0 && (!A || !x))) return HML_STATUS_INVALID_VALUE;
  std::lock_guard<std::mutex> lk(g_mu);
  HostPath *hp;
  hml_status st = get_path(&hp);
  if (st != HML_STATUS_SUCCESS) return st;
  HostPath &h = *hp;
  const size_t nA = static_cast<size_t>(M) * N;
  st = reserve(h, nA + N + M + 64);
  if (st != HML_STATUS_SUCCESS) return st;
  float *dA = h.buf;
  float *dx = reinterpret_cast<float *>((reinterpret_cast<uintptr_t>(dA + nA) + 63) & ~uintptr_t(63));
  float *dy = reinterpret_cast<float *>((reinterpret_cast<uintptr_t>(dx + N) + 63) & ~uintptr_t(63));
  HML_TRY(cudaMemcpyAsync(dA, A, nA * sizeof(float), cudaMemcpyHostToDevice, h.comp));
  HML_TRY(cudaMemcpyAsync(dx, x, static_cast<size_t>(N) * sizeof(float), cudaMemcpyHostToDevice, h.comp));
  if (beta != 0.0f)
    HML_TRY(cudaMemcpyAsync(dy, y, static_cast<size_t>(M) * sizeof(float), cudaMemcpyHostToDevice, h.comp));
  st = sgemv_variant(HML_ROW_MAJOR, HML_OP_N, M, N, alpha, dA, std::max(1, N), dx, beta, dy,
                     variant, h.comp);
  if (st != HML_STATUS_SUCCESS) return st;
  HML_TRY(cudaMemcpyAsync(y, dy, static_cast<size_t>(M) * sizeof(float), cudaMemcpyDeviceToHost, h.comp));
  HML_TRY(cudaStreamSynchronize(h.comp));
  return HML_STATUS_SUCCESS;
}

// threads per row of the GEMV row kernel from a reference v1 SGEMV rule;
// without one, the measured table's variant (else the heuristic)
int sgemv_variant_for(int N) {
  int type, bs, rs;
  if (!cfg_v1_sgemv_rule(N, &type, &bs, &rs)) return kGemvTuned;
  int tpr = 4;
  while (tpr < 256 && tpr < 16 * bs) tpr <<= 1;
  return tpr;
}

}  // namespace

hml_status sgemv_variant(int order, int trans, int M, int N, float alpha, const float *A, int lda,
                         const float *x, float beta, float *y, int variant, cudaStream_t s) {
  GemvProblem g;
  hml_status st = gemv_from_blas(static_cast<hml_order>(order), static_cast<hml_op>(trans), M, N,
                                 alpha, A, lda, x, beta, y, &g);
  if (st != HML_STATUS_SUCCESS) return st;
  if (g.P == 0) return HML_STATUS_SUCCESS;
  if (g.Q == 0 || g.alpha == 0.0f) return launch_scale(g.y, g.P, 1, g.incy, 0, g.beta, s);
  return launch_gemv(g, variant, s);
}

hml_status host_sgemm_c(int basic, float *C, const float *A, const float *B, int M, int N, int K,
                        float alpha, float beta) {
  return host_sgemm(basic != 0, C, A, B, M, N, K, alpha, beta);
}

hml_status host_sgemv_c(int basic, float *y, const float *A, const float *x, int M, int N,
                        float alpha, float beta) {
  return host_sgemv(basic ? 0 : sgemv_variant_for(N), y, A, x, M, N, alpha, beta);
}

hml_status config_file(int kind, const char *path) {
  if (!path) return HML_STATUS_SUCCESS;
  FILE *f = fopen(path, "rb");
  if (!f) return HML_STATUS_IO_ERROR;
  char head[64] = {};
  const bool got = fgets(head, sizeof head, f) != nullptr;
  fclose(f);
  int n = 0;
  // this library's measured table holds SGEMM and SGEMV records alike
  if (got && strncmp(head, "#HML-B200 tuning v2", 19) == 0) return tune_load(path, &n);
  return cfg_v1_load(kind, path, &n);
}

}  // namespace hml

// ----------------------------------------------------- reference C++ ABI
void hmlSgemmKernelConfig(char *sgemmKernelConfigFileName) {
  hml::report("hmlSgemmKernelConfig", hml::config_file(0, sgemmKernelConfigFileName));
}

void hmlSgemmBasic(float *C, const float *A, const float *B, const int M, const int N, const int K,
                   const float alpha, const float beta) {
  hml::report("hmlSgemmBasic", hml::host_sgemm(true, C, A, B, M, N, K, alpha, beta));
}

void hmlSgemm(float *C, const float *A, const float *B, const int M, const int N, const int K,
              const float alpha, const float beta) {
  hml::report("hmlSgemm", hml::host_sgemm(false, C, A, B, M, N, K, alpha, beta));
}

void hmlSgemvKernelConfig(char *sgemvKernelConfigFileName) {
  hml::report("hmlSgemvKernelConfig", hml::config_file(1, sgemvKernelConfigFileName));
}

void hmlSgemvBasic(float *y, const float *A, const float *x, const int M, const int N,
                   const float alpha, const float beta) {
  hml::report("hmlSgemvBasic", hml::host_sgemv_c(1, y, A, x, M, N, alpha, beta));
}

void hmlSgemv(float *y, const float *A, const float *x, const int M, const int N,
              const float alpha, const float beta) {
  hml::report("hmlSgemv", hml::host_sgemv_c(0, y, A, x, M, N, alpha, beta));
}

// ------------------------------------------------- status-returning forms
extern "C" {

hml_status hml_host_sgemm(int basic, float *C, const float *A, const float *B, int M, int N, int K,
                          float alpha, float beta) {
  return hml::host_sgemm_c(basic, C, A, B, M, N, K, alpha, beta);
}

hml_status hml_host_sgemv(int basic, float *y, const float *A, const float *x, int M, int N,
                          float alpha, float beta) {
  return hml::host_sgemv_c(basic, y, A, x, M, N, alpha, beta);
}

hml_status hml_config_file(int kind, const char *path) { return hml::config_file(kind, path); }

hml_status hml_sgemm_v1_config(int M, int N, int K, hml_sgemm_config *config) {
  using namespace hml;
  if (!config) return HML_STATUS_INVALID_VALUE;
  if (M < 1 || N < 1 || K < 1) return HML_STATUS_INVALID_VALUE;
  // a dense row-major problem on aligned dummy pointers: only the layout and
  // the sizes matter to the choice
  alignas(16) static float dummy[4];
  GemmProblem p;
  hml_status st = gemm_from_blas(HML_ROW_MAJOR, HML_OP_N, HML_OP_N, M, N, K, 1.0f, dummy, K,
                                 dummy, N, 0.0f, dummy, N, &p);
  if (st != HML_STATUS_SUCCESS) return st;
  if (p.N <= 1) return HML_STATUS_CONFIG_ERROR;  // served by the GEMV kernels
  return v1_rule_config(p, K, N, config) ? HML_STATUS_SUCCESS : HML_STATUS_CONFIG_ERROR;
}

}  // extern "C"
