// predictor.cu -- the learned configuration predictor: a small MLP trained on
// the GPU, by the kernels in this file, on the times the autotuner measures.
//
// The reference picks a kernel from static per-GPU tables indexed by
// (min(K,96), ceil(min(N,96)/16)) (src/hml_sgemm_kernel.cu:189-237), filled
// by an online tuner that takes minutes per table
// (src/hml_sgemm_kernel.cu:356-555).  Here the autotuner's measurements over
// many shapes train a network that generalises to unseen shapes:
//
//   features f (5)  = log2(M)/16, log2(N)/8, log2(K)/14, A K-contiguous,
//                     B K-contiguous   (of the canonical long-M problem)
//   h1 = relu(W1 f + b1)      64
//   h2 = relu(W2 h1 + b2)     64
//   s  = W3 h2 + b3           one score per configuration of the space
//
// Training target: s_j ~ y_j = min(log(t_j / t_best), clip) for every
// configuration j measured on the shape (masked mean squared error), so the
// score ranks configurations by predicted time.  Prediction = argmin of s
// over the configurations that can run the problem and that the math mode
// allows.  Kernels: dense forward, masked-MSE gradient, dense backward (data
// and weights), AdamW update, row gather and a one-block-per-problem
// inference kernel.  All reductions run in a fixed order (no atomics), so
// training is deterministic for a given seed.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <dlfcn.h>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "hml_select.h"
#include "hml_tune.h"

namespace hml {
namespace {

constexpr int kIn = 5;
constexpr int kH = 64;
constexpr int kMaxDev = 64;

// parameter layout: W1[kH][kIn] b1[kH] W2[kH][kH] b2[kH] W3[C][kH] b3[C]
struct Layout {
  size_t w1, b1, w2, b2, w3, b3, total;
  __host__ __device__ explicit Layout(int C) {
    w1 = 0;
    b1 = w1 + kH * kIn;
    w2 = b1 + kH;
    b2 = w2 + kH * kH;
    w3 = b2 + kH;
    b3 = w3 + static_cast<size_t>(C) * kH;
    total = b3 + C;
  }
};

// ---------------------------------------------------------------- kernels
// Y[s][o] = act(sum_i X[s][i] W[o][i] + b[o])
__global__ void dense_fwd_kernel(const float *__restrict__ W, const float *__restrict__ b,
                                 const float *__restrict__ X, float *__restrict__ Y, int n,
                                 int in, int out, int relu) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n * out) return;
  const int s = idx / out, o = idx % out;
  const float *x = X + static_cast<size_t>(s) * in;
  const float *w = W + static_cast<size_t>(o) * in;
  float acc = b[o];
  for (int i = 0; i < in; ++i) acc = fmaf(x[i], w[i], acc);
  Y[idx] = relu ? fmaxf(acc, 0.0f) : acc;
}

// dY = 2 w (y - t) * scale;  row_loss[s] = scale * sum_j w (y - t)^2
__global__ void mse_grad_kernel(const float *__restrict__ Y, const float *__restrict__ T,
                                const float *__restrict__ Wt, int C, float scale,
                                float *__restrict__ dY, float *__restrict__ row_loss) {
  __shared__ float red[256];
  const int s = blockIdx.x;
  const size_t base = static_cast<size_t>(s) * C;
  float acc = 0.0f;
  for (int j = threadIdx.x; j < C; j += blockDim.x) {
    const float w = Wt[base + j];
    const float d = Y[base + j] - T[base + j];
    dY[base + j] = 2.0f * w * d * scale;
    acc = fmaf(w * d, d, acc);
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) row_loss[s] = red[0] * scale;
}

// dX[s][i] = (sum_o dY[s][o] W[o][i]) * (X[s][i] > 0)   (X = relu output)
__global__ void dense_bwd_data_kernel(const float *__restrict__ W, const float *__restrict__ dY,
                                      const float *__restrict__ X, float *__restrict__ dX, int n,
                                      int in, int out) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n * in) return;
  const int s = idx / in, i = idx % in;
  const float *dy = dY + static_cast<size_t>(s) * out;
  float acc = 0.0f;
  for (int o = 0; o < out; ++o) acc = fmaf(dy[o], W[static_cast<size_t>(o) * in + i], acc);
  dX[idx] = X[idx] > 0.0f ? acc : 0.0f;
}

// dW[o][i] = sum_s dY[s][o] X[s][i];  db[o] = sum_s dY[s][o]  (thread per
// weight, i == in is the bias; samples summed in order)
__global__ void dense_bwd_weight_kernel(const float *__restrict__ dY,
                                        const float *__restrict__ X, float *__restrict__ dW,
                                        float *__restrict__ db, int n, int in, int out) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= out * (in + 1)) return;
  const int o = idx / (in + 1), i = idx % (in + 1);
  float acc = 0.0f;
  if (i < in) {
    for (int s = 0; s < n; ++s)
      acc = fmaf(dY[static_cast<size_t>(s) * out + o], X[static_cast<size_t>(s) * in + i], acc);
    dW[static_cast<size_t>(o) * in + i] = acc;
  } else {
    for (int s = 0; s < n; ++s) acc += dY[static_cast<size_t>(s) * out + o];
    db[o] = acc;
  }
}

// AdamW: m = b1 m + (1-b1) g; v = b2 v + (1-b2) g^2;
// p -= lr (m / c1 / (sqrt(v / c2) + eps) + wd p)
__global__ void adamw_kernel(float *__restrict__ p, const float *__restrict__ g,
                             float *__restrict__ m, float *__restrict__ v, int np, float lr,
                             float b1, float b2, float eps, float c1, float c2, float wd) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.0f - b1) * gi;
  const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * ((mi / c1) / (sqrtf(vi / c2) + eps) + wd * p[i]);
}

__global__ void gather_rows_kernel(const float *__restrict__ src, const int *__restrict__ idx,
                                   float *__restrict__ dst, int rows, int cols) {
  const size_t e = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= static_cast<size_t>(rows) * cols) return;
  const int r = static_cast<int>(e / cols), c = static_cast<int>(e % cols);
  dst[e] = src[static_cast<size_t>(idx[r]) * cols + c];
}

__global__ void sum_into_kernel(const float *__restrict__ v, int n, float *__restrict__ out) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    float s = 0.0f;
    for (int i = 0; i < n; ++i) s += v[i];
    *out += s;
  }
}

// One block (kH threads) per problem: scores of every configuration, argmin
// over the allowed ones (lowest index on ties).  out_idx = -1 when none is
// allowed.
__global__ void __launch_bounds__(kH) predict_kernel(const float *__restrict__ P, int C,
                                                     const float *__restrict__ feats,
                                                     const uint32_t *__restrict__ allow,
                                                     int words, int *__restrict__ out_idx,
                                                     float *__restrict__ out_score) {
  const Layout L(C);
  __shared__ float f[kIn], h1[kH], h2[kH];
  __shared__ float best_s[kH];
  __shared__ int best_i[kH];
  const int s = blockIdx.x, t = threadIdx.x;
  if (t < kIn) f[t] = feats[s * kIn + t];
  __syncthreads();
  float a = P[L.b1 + t];
  for (int i = 0; i < kIn; ++i) a = fmaf(f[i], P[L.w1 + t * kIn + i], a);
  h1[t] = fmaxf(a, 0.0f);
  __syncthreads();
  a = P[L.b2 + t];
  for (int i = 0; i < kH; ++i) a = fmaf(h1[i], P[L.w2 + t * kH + i], a);
  h2[t] = fmaxf(a, 0.0f);
  __syncthreads();
  float bs = INFINITY;
  int bi = -1;
  const uint32_t *al = allow + static_cast<size_t>(s) * words;
  for (int o = t; o < C; o += kH) {
    if (!((al[o >> 5] >> (o & 31)) & 1u)) continue;
    float y = P[L.b3 + o];
    for (int i = 0; i < kH; ++i) y = fmaf(h2[i], P[L.w3 + static_cast<size_t>(o) * kH + i], y);
    if (y < bs) {  // o increases: strict < keeps the lowest index
      bs = y;
      bi = o;
    }
  }
  best_s[t] = bs;
  best_i[t] = bi;
  __syncthreads();
  for (int h = kH / 2; h > 0; h >>= 1) {
    if (t < h) {
      const float so = best_s[t + h];
      const int io = best_i[t + h];
      if (io >= 0 && (best_i[t] < 0 || so < best_s[t] || (so == best_s[t] && io < best_i[t]))) {
        best_s[t] = so;
        best_i[t] = io;
      }
    }
    __syncthreads();
  }
  if (t == 0) {
    out_idx[s] = best_i[0];
    if (out_score) out_score[s] = best_s[0];
  }
}

inline unsigned blocks_for(size_t n, int per) { return static_cast<unsigned>((n + per - 1) / per); }

// ---------------------------------------------------------- device buffers
struct DevBuf {
  std::vector<void *> ptrs;
  bool ok = true;
  template <typename T>
  T *get(size_t count) {
    void *p = nullptr;
    if (count == 0) count = 1;
    if (cudaMalloc(&p, count * sizeof(T)) != cudaSuccess) {
      ok = false;
      return nullptr;
    }
    ptrs.push_back(p);
    return static_cast<T *>(p);
  }
  ~DevBuf() {
    for (void *p : ptrs) cudaFree(p);
  }
};

// Forward + loss gradient + backward of one batch already on the device.
struct Net {
  int C;
  Layout L;
  explicit Net(int c) : C(c), L(c) {}
  void forward(const float *P, const float *X, float *H1, float *H2, float *Y, int n,
               cudaStream_t s) const {
    dense_fwd_kernel<<<blocks_for(size_t(n) * kH, 256), 256, 0, s>>>(P + L.w1, P + L.b1, X, H1,
                                                                     n, kIn, kH, 1);
    dense_fwd_kernel<<<blocks_for(size_t(n) * kH, 256), 256, 0, s>>>(P + L.w2, P + L.b2, H1, H2,
                                                                     n, kH, kH, 1);
    dense_fwd_kernel<<<blocks_for(size_t(n) * C, 256), 256, 0, s>>>(P + L.w3, P + L.b3, H2, Y, n,
                                                                    kH, C, 0);
    count_launch(3);
  }
  void backward(const float *P, const float *X, const float *H1, const float *H2,
                const float *dY, float *dH2, float *dH1, float *G, int n,
                cudaStream_t s) const {
    dense_bwd_weight_kernel<<<blocks_for(size_t(C) * (kH + 1), 128), 128, 0, s>>>(
        dY, H2, G + L.w3, G + L.b3, n, kH, C);
    dense_bwd_data_kernel<<<blocks_for(size_t(n) * kH, 256), 256, 0, s>>>(P + L.w3, dY, H2, dH2,
                                                                          n, kH, C);
    dense_bwd_weight_kernel<<<blocks_for(size_t(kH) * (kH + 1), 128), 128, 0, s>>>(
        dH2, H1, G + L.w2, G + L.b2, n, kH, kH);
    dense_bwd_data_kernel<<<blocks_for(size_t(n) * kH, 256), 256, 0, s>>>(P + L.w2, dH2, H1, dH1,
                                                                          n, kH, kH);
    dense_bwd_weight_kernel<<<blocks_for(size_t(kH) * (kIn + 1), 128), 128, 0, s>>>(
        dH1, X, G + L.w1, G + L.b1, n, kIn, kH);
    count_launch(5);
  }
};

// ------------------------------------------------------------------ model
struct Model {
  int C = 0;
  std::vector<hml_sgemm_config> cfgs;
  std::vector<float> params;
  float *dev_params[kMaxDev] = {};
  std::map<std::tuple<int, int, int, int, int, int, int>, int> memo;
  ~Model() {
    for (float *p : dev_params)
      if (p) cudaFree(p);
  }
};

std::mutex g_pmu;
Model *g_model = nullptr;
bool g_default_tried = false;
cudaStream_t g_pstream[kMaxDev] = {};

uint64_t splitmix(uint64_t *state) {
  uint64_t z = (*state += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
float uniform01(uint64_t *state) {
  return static_cast<float>((splitmix(state) >> 40) * (1.0 / 16777216.0));
}

// the canonical problem of a BLAS shape with 16-byte-rounded leading
// dimensions (the autotuner's layout) on 16-byte-aligned stand-in pointers
hml_status shape_problem(hml_order order, int ta, int tb, int M, int N, int K, GemmProblem *p) {
  if ((ta != 0 && ta != 1) || (tb != 0 && tb != 1)) return HML_STATUS_INVALID_VALUE;
  const bool cm = order == HML_COL_MAJOR;
  auto r4 = [](int x) { return (std::max(1, x) + 3) / 4 * 4; };
  const int lda = r4(cm ? (ta == 0 ? M : K) : (ta == 0 ? K : M));
  const int ldb = r4(cm ? (tb == 0 ? K : N) : (tb == 0 ? N : K));
  const int ldc = r4(cm ? M : N);
  alignas(16) static float stand_in[4];
  return gemm_from_blas(order, static_cast<hml_op>(ta), static_cast<hml_op>(tb), M, N, K, 1.0f,
                        stand_in, lda, stand_in, ldb, 0.0f, stand_in, ldc, p);
}

bool allowed_algo(int algo) { return algo != HML_ALGO_BF16X3 || math_mode() == HML_MATH_FAST; }

void allow_bits(const GemmProblem &p, const std::vector<hml_sgemm_config> &cfgs, uint32_t *bits) {
  const int words = (static_cast<int>(cfgs.size()) + 31) / 32;
  std::fill(bits, bits + words, 0u);
  for (size_t j = 0; j < cfgs.size(); ++j)
    if (allowed_algo(cfgs[j].algo) && check_config_ok(p, cfgs[j]))
      bits[j >> 5] |= 1u << (j & 31);
}

bool aligned16(const void *ptr) { return (reinterpret_cast<uintptr_t>(ptr) & 15u) == 0; }

hml_status dev_params(Model *m, float **out) {
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= kMaxDev) return HML_STATUS_NOT_SUPPORTED;
  if (!m->dev_params[dev]) {
    float *p = nullptr;
    cudaError_t e = cudaMalloc(&p, m->params.size() * sizeof(float));
    if (e == cudaSuccess)
      e = cudaMemcpy(p, m->params.data(), m->params.size() * sizeof(float),
                     cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      if (p) cudaFree(p);
      note_cuda_error(e, "predictor parameters");
      return HML_STATUS_CUDA_ERROR;
    }
    m->dev_params[dev] = p;
  }
  *out = m->dev_params[dev];
  return HML_STATUS_SUCCESS;
}

hml_status private_stream(cudaStream_t *s) {
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= kMaxDev) return HML_STATUS_NOT_SUPPORTED;
  if (!g_pstream[dev] &&
      cudaStreamCreateWithFlags(&g_pstream[dev], cudaStreamNonBlocking) != cudaSuccess)
    return HML_STATUS_CUDA_ERROR;
  *s = g_pstream[dev];
  return HML_STATUS_SUCCESS;
}

// Runs the inference kernel on n problems (features and allow bits on the
// host).  Caller holds g_pmu.
hml_status infer(Model *m, const std::vector<float> &feats, const std::vector<uint32_t> &bits,
                 int n, int *idx_out, float *score_out) {
  if (n == 0) return HML_STATUS_SUCCESS;
  // everything below runs on a private stream that no capture holds; relaxed
  // capture mode lets it proceed while another stream is being captured
  cudaStreamCaptureMode mode = cudaStreamCaptureModeRelaxed;
  cudaThreadExchangeStreamCaptureMode(&mode);
  hml_status st = HML_STATUS_SUCCESS;
  {
    float *P = nullptr;
    cudaStream_t s = nullptr;
    st = dev_params(m, &P);
    if (st == HML_STATUS_SUCCESS) st = private_stream(&s);
    if (st == HML_STATUS_SUCCESS) {
      const int words = (m->C + 31) / 32;
      DevBuf db;
      float *df = db.get<float>(feats.size());
      uint32_t *dbits = db.get<uint32_t>(bits.size());
      int *didx = db.get<int>(n);
      float *dsc = db.get<float>(n);
      cudaError_t e = db.ok ? cudaSuccess : cudaErrorMemoryAllocation;
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(df, feats.data(), feats.size() * sizeof(float), cudaMemcpyHostToDevice,
                            s);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(dbits, bits.data(), bits.size() * sizeof(uint32_t),
                            cudaMemcpyHostToDevice, s);
      if (e == cudaSuccess) {
        predict_kernel<<<n, kH, 0, s>>>(P, m->C, df, dbits, words, didx, dsc);
        count_launch();
        e = cudaGetLastError();
      }
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(idx_out, didx, n * sizeof(int), cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess && score_out)
        e = cudaMemcpyAsync(score_out, dsc, n * sizeof(float), cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      if (e != cudaSuccess) {
        note_cuda_error(e, "predictor inference");
        st = HML_STATUS_CUDA_ERROR;
      }
    }  // device buffers released here, still in relaxed mode
  }
  cudaThreadExchangeStreamCaptureMode(&mode);
  return st;
}

void features_of(const GemmProblem &p, float *f) {
  f[0] = static_cast<float>(std::log2(static_cast<double>(std::max(1, p.M))) / 16.0);
  f[1] = static_cast<float>(std::log2(static_cast<double>(std::max(1, p.N))) / 8.0);
  f[2] = static_cast<float>(std::log2(static_cast<double>(std::max(1, p.K))) / 14.0);
  f[3] = p.a_kcontig() ? 1.0f : 0.0f;
  f[4] = p.b_kcontig() ? 1.0f : 0.0f;
}

}  // namespace

// --------------------------------------------------------------- selection
namespace {
Model *parse_model(const char *path, hml_status *st);

// The network shipped beside the library (data/predictor_b200.txt next to
// libhml_b200.so), loaded on the first selection that finds no predictor.
// HML_PREDICTOR=<path> names another file, HML_PREDICTOR=none disables it.
// Caller holds g_pmu.
void load_default_locked() {
  if (g_default_tried) return;
  g_default_tried = true;
  std::string path;
  const char *env = getenv("HML_PREDICTOR");
  if (env && *env) {
    if (strcmp(env, "none") == 0) return;
    path = env;
  } else {
    Dl_info info;
    if (!dladdr(reinterpret_cast<void *>(&load_default_locked), &info) || !info.dli_fname) return;
    path = info.dli_fname;
    const size_t slash = path.rfind('/');
    path = (slash == std::string::npos ? std::string(".") : path.substr(0, slash)) +
           "/data/predictor_b200.txt";
  }
  hml_status st;
  Model *m = parse_model(path.c_str(), &st);
  if (m) g_model = m;
}
}  // namespace

bool predictor_lookup(const GemmProblem &p, hml_sgemm_config *c, cudaStream_t user_stream) {
  std::lock_guard<std::mutex> lk(g_pmu);
  if (!g_model) load_default_locked();
  Model *m = g_model;
  if (!m) return false;
  const int64_t sa = p.a_kcontig() ? p.sam : p.sak;
  const int tma = aligned16(p.A) && (sa * 4) % 16 == 0 ? 1 : 0;
  const auto key = std::make_tuple(p.a_kcontig() ? 1 : 0, p.b_kcontig() ? 1 : 0, p.M, p.N, p.K,
                                   tma, math_mode());
  auto it = m->memo.find(key);
  int idx;
  if (it != m->memo.end()) {
    idx = it->second;
  } else {
    // a stream under capture gets the heuristic rather than a synchronising
    // inference call; the answer is not memoised so a later call predicts
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (user_stream && cudaStreamIsCapturing(user_stream, &cs) == cudaSuccess &&
        cs != cudaStreamCaptureStatusNone)
      return false;
    std::vector<float> f(kIn);
    features_of(p, f.data());
    std::vector<uint32_t> bits((m->C + 31) / 32);
    allow_bits(p, m->cfgs, bits.data());
    if (infer(m, f, bits, 1, &idx, nullptr) != HML_STATUS_SUCCESS) return false;
    if (m->memo.size() > (1u << 16)) m->memo.clear();
    m->memo[key] = idx;
  }
  if (idx < 0) return false;
  *c = m->cfgs[idx];
  return true;
}

// ---------------------------------------------------------------- training
hml_status predictor_train(hml_order order, const int32_t *shapes, const float *times, int n,
                           const hml_sgemm_config *cfgs, int C,
                           const hml_predictor_options *opt, float *loss_history) {
  if (!shapes || !times || !cfgs || !opt || n < 1 || C < 1 || C > 4096)
    return HML_STATUS_INVALID_VALUE;
  if (opt->epochs < 1 || opt->batch < 1 || !(opt->lr > 0.0f) || !(opt->target_clip > 0.0f))
    return HML_STATUS_INVALID_VALUE;
  const Layout L(C);
  const size_t np = L.total;
  // ---- host data: features, targets, weights
  std::vector<float> X(static_cast<size_t>(n) * kIn), T(static_cast<size_t>(n) * C, 0.0f),
      W(static_cast<size_t>(n) * C, 0.0f), wsum(n, 0.0f);
  for (int i = 0; i < n; ++i) {
    const int32_t *sh = shapes + static_cast<size_t>(i) * 5;
    GemmProblem p;
    hml_status st = shape_problem(order, sh[3], sh[4], sh[0], sh[1], sh[2], &p);
    if (st != HML_STATUS_SUCCESS || p.M < 1 || p.N < 1 || p.K < 1) {
      note_text_error("predictor training: invalid shape");
      return HML_STATUS_INVALID_VALUE;
    }
    features_of(p, &X[static_cast<size_t>(i) * kIn]);
    const float *t = times + static_cast<size_t>(i) * C;
    float best = INFINITY;
    for (int j = 0; j < C; ++j)
      if (t[j] > 0.0f && std::isfinite(t[j])) best = std::min(best, t[j]);
    if (!std::isfinite(best)) continue;  // nothing measured: weight 0
    for (int j = 0; j < C; ++j) {
      if (!(t[j] > 0.0f) || !std::isfinite(t[j])) continue;
      T[static_cast<size_t>(i) * C + j] =
          std::min(static_cast<float>(std::log(static_cast<double>(t[j]) / best)), opt->target_clip);
      W[static_cast<size_t>(i) * C + j] = 1.0f;
      wsum[i] += 1.0f;
    }
  }
  // ---- parameters: He-uniform weights from SplitMix64, zero biases
  std::vector<float> P(np, 0.0f);
  uint64_t rs = opt->seed ^ 0x5DEECE66Dull;
  auto init = [&](size_t off, int fan_in, size_t count) {
    const float a = std::sqrt(6.0f / fan_in);
    for (size_t i = 0; i < count; ++i) P[off + i] = (2.0f * uniform01(&rs) - 1.0f) * a;
  };
  init(L.w1, kIn, kH * kIn);
  init(L.w2, kH, kH * kH);
  init(L.w3, kH, static_cast<size_t>(C) * kH);
  // ---- device
  const int B = std::min(opt->batch, n);
  DevBuf db;
  float *dX = db.get<float>(X.size()), *dT = db.get<float>(T.size()), *dW = db.get<float>(W.size());
  float *dP = db.get<float>(np), *dG = db.get<float>(np), *dm = db.get<float>(np),
        *dv = db.get<float>(np);
  float *bX = db.get<float>(size_t(B) * kIn), *bT = db.get<float>(size_t(B) * C),
        *bW = db.get<float>(size_t(B) * C);
  float *H1 = db.get<float>(size_t(B) * kH), *H2 = db.get<float>(size_t(B) * kH),
        *Y = db.get<float>(size_t(B) * C), *dY = db.get<float>(size_t(B) * C),
        *dH2 = db.get<float>(size_t(B) * kH), *dH1 = db.get<float>(size_t(B) * kH),
        *rl = db.get<float>(B), *eloss = db.get<float>(opt->epochs);
  int *didx = db.get<int>(n);
  if (!db.ok) {
    note_text_error("predictor training: device allocation failed");
    return HML_STATUS_ALLOC_FAILED;
  }
  cudaStream_t s = nullptr;
  cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  auto h2d = [&](void *d, const void *h, size_t bytes) {
    if (e == cudaSuccess) e = cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, s);
  };
  h2d(dX, X.data(), X.size() * 4);
  h2d(dT, T.data(), T.size() * 4);
  h2d(dW, W.data(), W.size() * 4);
  h2d(dP, P.data(), np * 4);
  if (e == cudaSuccess) e = cudaMemsetAsync(dm, 0, np * 4, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(dv, 0, np * 4, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(eloss, 0, size_t(opt->epochs) * 4, s);
  const Net net(C);
  std::vector<int> perm(n);
  for (int i = 0; i < n; ++i) perm[i] = i;
  const int steps_per_epoch = (n + B - 1) / B;
  const double total_steps = static_cast<double>(steps_per_epoch) * opt->epochs;
  int step = 0;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  for (int ep = 0; ep < opt->epochs && e == cudaSuccess; ++ep) {
    for (int i = n - 1; i > 0; --i) {  // Fisher-Yates with SplitMix64
      const int j = static_cast<int>(splitmix(&rs) % static_cast<uint64_t>(i + 1));
      std::swap(perm[i], perm[j]);
    }
    // the upload must finish before perm is reshuffled next epoch
    e = cudaMemcpyAsync(didx, perm.data(), n * sizeof(int), cudaMemcpyHostToDevice, s);
    for (int b0 = 0; b0 < n && e == cudaSuccess; b0 += B) {
      const int nb = std::min(B, n - b0);
      double ws = 0.0;
      for (int i = 0; i < nb; ++i) ws += wsum[perm[b0 + i]];
      const float scale = ws > 0.0 ? static_cast<float>(1.0 / ws) : 0.0f;
      gather_rows_kernel<<<blocks_for(size_t(nb) * kIn, 256), 256, 0, s>>>(dX, didx + b0, bX, nb,
                                                                           kIn);
      gather_rows_kernel<<<blocks_for(size_t(nb) * C, 256), 256, 0, s>>>(dT, didx + b0, bT, nb, C);
      gather_rows_kernel<<<blocks_for(size_t(nb) * C, 256), 256, 0, s>>>(dW, didx + b0, bW, nb, C);
      count_launch(3);
      net.forward(dP, bX, H1, H2, Y, nb, s);
      mse_grad_kernel<<<nb, 256, 0, s>>>(Y, bT, bW, C, scale, dY, rl);
      sum_into_kernel<<<1, 1, 0, s>>>(rl, nb, eloss + ep);
      count_launch(2);
      net.backward(dP, bX, H1, H2, dY, dH2, dH1, dG, nb, s);
      ++step;
      const double frac = (step - 1) / std::max(1.0, total_steps - 1);
      const float lr = static_cast<float>(opt->lr * (0.05 + 0.95 * 0.5 * (1.0 + std::cos(M_PI * frac))));
      const float c1 = 1.0f - std::pow(b1, static_cast<float>(step));
      const float c2 = 1.0f - std::pow(b2, static_cast<float>(step));
      adamw_kernel<<<blocks_for(np, 256), 256, 0, s>>>(dP, dG, dm, dv, static_cast<int>(np), lr, b1,
                                                       b2, eps, c1, c2, opt->weight_decay);
      count_launch();
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // perm is rewritten next epoch
  }
  std::vector<float> hist(opt->epochs);
  if (e == cudaSuccess) e = cudaMemcpyAsync(P.data(), dP, np * 4, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(hist.data(), eloss, hist.size() * 4, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (s) cudaStreamDestroy(s);
  if (e != cudaSuccess) {
    note_cuda_error(e, "predictor training");
    return HML_STATUS_CUDA_ERROR;
  }
  if (loss_history)
    for (int ep = 0; ep < opt->epochs; ++ep) loss_history[ep] = hist[ep] / steps_per_epoch;
  Model *m = new Model;
  m->C = C;
  m->cfgs.assign(cfgs, cfgs + C);
  m->params = P;
  std::lock_guard<std::mutex> lk(g_pmu);
  delete g_model;
  g_model = m;
  g_default_tried = true;
  return HML_STATUS_SUCCESS;
}

// Loss and gradient of the network on host data, through the training
// kernels (one forward, one loss gradient, one backward).
hml_status predictor_loss_grad(const float *params, int C, const float *feats,
                               const float *targets, const float *weights, int n, float *grad,
                               float *loss) {
  if (!params || !feats || !targets || !weights || n < 1 || C < 1 || C > 4096)
    return HML_STATUS_INVALID_VALUE;
  const Layout L(C);
  DevBuf db;
  float *dP = db.get<float>(L.total), *dG = db.get<float>(L.total);
  float *X = db.get<float>(size_t(n) * kIn), *T = db.get<float>(size_t(n) * C),
        *W = db.get<float>(size_t(n) * C);
  float *H1 = db.get<float>(size_t(n) * kH), *H2 = db.get<float>(size_t(n) * kH),
        *Y = db.get<float>(size_t(n) * C), *dY = db.get<float>(size_t(n) * C),
        *dH2 = db.get<float>(size_t(n) * kH), *dH1 = db.get<float>(size_t(n) * kH),
        *rl = db.get<float>(n), *ls = db.get<float>(1);
  if (!db.ok) return HML_STATUS_ALLOC_FAILED;
  double ws = 0.0;
  for (size_t i = 0; i < size_t(n) * C; ++i) ws += weights[i];
  const float scale = ws > 0.0 ? static_cast<float>(1.0 / ws) : 0.0f;
  cudaError_t e = cudaMemcpy(dP, params, L.total * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(X, feats, size_t(n) * kIn * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(T, targets, size_t(n) * C * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(W, weights, size_t(n) * C * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(ls, 0, 4);
  if (e == cudaSuccess) {
    const Net net(C);
    net.forward(dP, X, H1, H2, Y, n, nullptr);
    mse_grad_kernel<<<n, 256>>>(Y, T, W, C, scale, dY, rl);
    sum_into_kernel<<<1, 1>>>(rl, n, ls);
    count_launch(2);
    net.backward(dP, X, H1, H2, dY, dH2, dH1, dG, n, nullptr);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess && grad) e = cudaMemcpy(grad, dG, L.total * 4, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && loss) e = cudaMemcpy(loss, ls, 4, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    note_cuda_error(e, "predictor loss/gradient");
    return HML_STATUS_CUDA_ERROR;
  }
  return HML_STATUS_SUCCESS;
}

hml_status predictor_predict_batch(hml_order order, const int32_t *shapes, int n, int32_t *out) {
  if (!shapes || !out || n < 0) return HML_STATUS_INVALID_VALUE;
  std::lock_guard<std::mutex> lk(g_pmu);
  Model *m = g_model;
  if (!m) {
    note_text_error("no predictor loaded");
    return HML_STATUS_NOT_SUPPORTED;
  }
  const int words = (m->C + 31) / 32;
  std::vector<float> f(static_cast<size_t>(n) * kIn);
  std::vector<uint32_t> bits(static_cast<size_t>(n) * words);
  for (int i = 0; i < n; ++i) {
    const int32_t *sh = shapes + static_cast<size_t>(i) * 5;
    GemmProblem p;
    hml_status st = shape_problem(order, sh[3], sh[4], sh[0], sh[1], sh[2], &p);
    if (st != HML_STATUS_SUCCESS) return st;
    features_of(p, &f[static_cast<size_t>(i) * kIn]);
    allow_bits(p, m->cfgs, &bits[static_cast<size_t>(i) * words]);
  }
  std::vector<int> idx(n);
  hml_status st = infer(m, f, bits, n, idx.data(), nullptr);
  if (st != HML_STATUS_SUCCESS) return st;
  for (int i = 0; i < n; ++i) out[i] = idx[i];
  return HML_STATUS_SUCCESS;
}

// ------------------------------------------------------------------- files
hml_status predictor_save(const char *path) {
  std::lock_guard<std::mutex> lk(g_pmu);
  if (!g_model) return HML_STATUS_NOT_SUPPORTED;
  FILE *f = fopen(path, "w");
  if (!f) return HML_STATUS_IO_ERROR;
  const Model &m = *g_model;
  fprintf(f, "#HML-B200 predictor v1\n");
  fprintf(f, "inputs %d hidden %d %d outputs %d\n", kIn, kH, kH, m.C);
  for (const hml_sgemm_config &c : m.cfgs)
    fprintf(f, "config %d %d %d %d %d %d\n", c.algo, c.tile_m, c.tile_n, c.split_k, c.stages,
            c.variant);
  fprintf(f, "params %zu\n", m.params.size());
  for (size_t i = 0; i < m.params.size(); ++i)
    fprintf(f, "%.9g%c", m.params[i], (i % 8 == 7 || i + 1 == m.params.size()) ? '\n' : ' ');
  const bool ok = fflush(f) == 0;
  fclose(f);
  return ok ? HML_STATUS_SUCCESS : HML_STATUS_IO_ERROR;
}

namespace {

// Parses a predictor file; nullptr (and *st) on any error.
Model *parse_model(const char *path, hml_status *st) {
  *st = HML_STATUS_SUCCESS;
  FILE *f = fopen(path, "r");
  if (!f) {
    *st = HML_STATUS_IO_ERROR;
    return nullptr;
  }
  char line[256];
  auto fail = [&](const char *why) -> Model * {
    fclose(f);
    note_text_error(why);
    *st = HML_STATUS_CONFIG_ERROR;
    return nullptr;
  };
  if (!fgets(line, sizeof line, f) || strncmp(line, "#HML-B200 predictor v1", 22) != 0)
    return fail("predictor file: missing header");
  int in = 0, h1 = 0, h2 = 0, C = 0;
  if (fscanf(f, " inputs %d hidden %d %d outputs %d", &in, &h1, &h2, &C) != 4 || in != kIn ||
      h1 != kH || h2 != kH || C < 1 || C > 4096)
    return fail("predictor file: bad network dimensions");
  std::vector<hml_sgemm_config> cfgs(C);
  const auto &space = config_space();
  for (int j = 0; j < C; ++j) {
    hml_sgemm_config &c = cfgs[j];
    if (fscanf(f, " config %d %d %d %d %d %d", &c.algo, &c.tile_m, &c.tile_n, &c.split_k,
               &c.stages, &c.variant) != 6)
      return fail("predictor file: bad config line");
    bool known = false;
    for (const hml_sgemm_config &s : space)
      known = known || (s.algo == c.algo && s.tile_m == c.tile_m && s.tile_n == c.tile_n &&
                        s.split_k == c.split_k && s.stages == c.stages && s.variant == c.variant);
    if (!known) return fail("predictor file: configuration outside this library's space");
  }
  size_t np = 0;
  if (fscanf(f, " params %zu", &np) != 1 || np != Layout(C).total)
    return fail("predictor file: bad parameter count");
  std::vector<float> P(np);
  for (size_t i = 0; i < np; ++i)
    if (fscanf(f, " %f", &P[i]) != 1 || !std::isfinite(P[i]))
      return fail("predictor file: bad parameter value");
  fclose(f);
  Model *m = new Model;
  m->C = C;
  m->cfgs = cfgs;
  m->params = P;
  return m;
}

}  // namespace

hml_status predictor_load(const char *path) {
  hml_status st;
  Model *m = parse_model(path, &st);
  if (!m) return st;
  std::lock_guard<std::mutex> lk(g_pmu);
  delete g_model;
  g_model = m;
  g_default_tried = true;  // an explicit load replaces the shipped network
  return HML_STATUS_SUCCESS;
}

hml_status predictor_clear() {
  std::lock_guard<std::mutex> lk(g_pmu);
  delete g_model;
  g_model = nullptr;
  g_default_tried = true;  // cleared stays cleared
  return HML_STATUS_SUCCESS;
}

int predictor_outputs() {
  std::lock_guard<std::mutex> lk(g_pmu);
  return g_model ? g_model->C : 0;
}

hml_status predictor_params(float *out, size_t cap, size_t *count) {
  std::lock_guard<std::mutex> lk(g_pmu);
  if (!g_model) return HML_STATUS_NOT_SUPPORTED;
  if (count) *count = g_model->params.size();
  if (out) {
    if (cap < g_model->params.size()) return HML_STATUS_INVALID_VALUE;
    std::copy(g_model->params.begin(), g_model->params.end(), out);
  }
  return HML_STATUS_SUCCESS;
}

hml_status predictor_features(hml_order order, int ta, int tb, int M, int N, int K, float *f) {
  if (!f) return HML_STATUS_INVALID_VALUE;
  GemmProblem p;
  hml_status st = shape_problem(order, ta, tb, M, N, K, &p);
  if (st != HML_STATUS_SUCCESS) return st;
  features_of(p, f);
  return HML_STATUS_SUCCESS;
}

}  // namespace hml

extern "C" {

hml_status hml_predictor_train(hml_order order, const int32_t *shapes, const float *times_us,
                               int n, const hml_sgemm_config *configs, int n_configs,
                               const hml_predictor_options *options, float *loss_history) {
  return hml::predictor_train(order, shapes, times_us, n, configs, n_configs, options,
                              loss_history);
}

hml_status hml_predictor_loss_grad(const float *params, int n_configs, const float *features,
                                   const float *targets, const float *weights, int n,
                                   float *grad, float *loss) {
  return hml::predictor_loss_grad(params, n_configs, features, targets, weights, n, grad, loss);
}

hml_status hml_predictor_predict_batch(hml_order order, const int32_t *shapes, int n,
                                       int32_t *config_index) {
  return hml::predictor_predict_batch(order, shapes, n, config_index);
}

hml_status hml_predictor_save(const char *path) {
  return path ? hml::predictor_save(path) : HML_STATUS_INVALID_VALUE;
}

hml_status hml_predictor_load(const char *path) {
  return path ? hml::predictor_load(path) : HML_STATUS_INVALID_VALUE;
}

hml_status hml_predictor_clear(void) { return hml::predictor_clear(); }

int hml_predictor_outputs(void) { return hml::predictor_outputs(); }

hml_status hml_predictor_params(float *out, size_t capacity, size_t *count) {
  return hml::predictor_params(out, capacity, count);
}

hml_status hml_predictor_features(hml_order order, int transA, int transB, int M, int N, int K,
                                  float features[5]) {
  return hml::predictor_features(order, transA, transB, M, N, K, features);
}

}  // extern "C"
