// tune.cu -- the measuring autotuner and its table.
//
// Replaces the reference's online exhaustive tuner
// (src/hml_sgemm_kernel.cu:356-555), which timed 27 kernels per (K, colStops)
// class with the host wall clock around launch + cudaDeviceSynchronize on a
// fixed 1e6-row problem, kept only the argmax and aborted on any failed
// launch.  Here every configuration of the space that can run the given
// problem is timed with CUDA events on the stream, L2 flushed before every
// timed launch, median of `reps`; a configuration that fails is recorded with
// its status and skipped.  The full timing table is returned to the caller
// (it is the learned predictor's training data), and the fastest
// configuration allowed by the math mode is recorded in the tuned table that
// hml_sgemm_ex consults first.
//
// The GEMV half (hml_autotune_sgemv) replaces the reference's SGEMV tuner
// (hmlSgemvKernelConfigOnline, src/hml_sgemv_kernel.cu:391-633), which
// timed its kernel types per N class on the host clock: here every variant
// of the kernel that serves the problem's layout (threads per row, or CTAs
// per column tile) is timed the same way as the SGEMM configurations and the
// fastest is recorded in a second table that hml_sgemv_ex consults first.
//
// Tuned-table file, "#HML-B200 tuning v2":
//   # device <name> sms <n>
//   akc bkc M N K : algo tile_m tile_n split_k stages variant time_us
//   v cols P Q : variant time_us
// (akc/bkc: whether A / B are K-contiguous in the canonical long-M form;
// a "v" record is a GEMV: cols = 1 when the columns of A are contiguous,
// P = length of y, Q = length of x).
#include <dlfcn.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "hml_select.h"
#include "hml_tune.h"

namespace hml {

hml_status fill_random(float *out, size_t n, uint64_t seed, uint64_t stream_id, int dist,
                       cudaStream_t s);

namespace {

struct Key {
  int akc, bkc, M, N, K;
  bool operator<(const Key &o) const {
    return std::tie(akc, bkc, M, N, K) < std::tie(o.akc, o.bkc, o.M, o.N, o.K);
  }
};
struct Rec {
  hml_sgemm_config cfg;
  float us;
};

// GEMV records: layout (0 = rows of A contiguous, 1 = columns), P, Q
struct GKey {
  int cols, P, Q;
  bool operator<(const GKey &o) const {
    return std::tie(cols, P, Q) < std::tie(o.cols, o.P, o.Q);
  }
};
struct GRec {
  int variant;
  float us;
};

std::mutex g_mu;
std::map<Key, Rec> g_table;
std::map<GKey, GRec> g_gemv_table;
int g_math_mode = HML_MATH_FP32;
bool g_default_tried = false;  // the shipped table was loaded or ruled out

Key key_of(const GemmProblem &p) {
  return Key{p.a_kcontig() ? 1 : 0, p.b_kcontig() ? 1 : 0, p.M, p.N, p.K};
}

bool allowed(int algo) { return algo != HML_ALGO_BF16X3 || g_math_mode == HML_MATH_FAST; }

GKey gkey_of(const GemvProblem &p) { return GKey{gemv_rows_layout(p) ? 0 : 1, p.P, p.Q}; }

}  // namespace

int math_mode() { return g_math_mode; }

hml_status tune_load(const char *path, int *records);

namespace {
// The table shipped beside the library (data/tuned_b200.txt next to
// libhml_b200.so): the autotuner's measured best configurations on the B200
// for the library's reference workloads, in the role of the reference's
// per-GPU .cfg files.  It is loaded on the first selection when no table was
// loaded, measured or cleared before; HML_TUNED=<path> names another file,
// HML_TUNED=none disables it.
void load_default_table() {
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_default_tried) return;
    g_default_tried = true;
    if (!g_table.empty()) return;
  }
  std::string path;
  const char *env = getenv("HML_TUNED");
  if (env && *env) {
    if (strcmp(env, "none") == 0) return;
    path = env;
  } else {
    Dl_info info;
    if (!dladdr(reinterpret_cast<void *>(&load_default_table), &info) || !info.dli_fname) return;
    path = info.dli_fname;
    const size_t slash = path.rfind('/');
    path = (slash == std::string::npos ? std::string(".") : path.substr(0, slash)) +
           "/data/tuned_b200.txt";
  }
  int n = 0;
  tune_load(path.c_str(), &n);  // a missing file leaves the table empty
}
}  // namespace

bool tuned_lookup(const GemmProblem &p, hml_sgemm_config *c) {
  load_default_table();
  std::lock_guard<std::mutex> lk(g_mu);
  if (g_table.empty()) return false;
  const Key k = key_of(p);
  auto it = g_table.find(k);
  if (it != g_table.end() && allowed(it->second.cfg.algo)) {
    *c = it->second.cfg;
    return true;
  }
  // nearest measured class in log space with the same operand orders
  double best = 1e300;
  const Rec *pick = nullptr;
  for (const auto &kv : g_table) {
    if (kv.first.akc != k.akc || kv.first.bkc != k.bkc || !allowed(kv.second.cfg.algo)) continue;
    const double dm = std::log2(double(kv.first.M) / k.M);
    const double dn = std::log2(double(kv.first.N) / k.N);
    const double dk = std::log2(double(kv.first.K) / k.K);
    const double d = dm * dm + 4.0 * dn * dn + dk * dk;  // N decides the tile most
    if (d < best && check_config_ok(p, kv.second.cfg)) {
      best = d;
      pick = &kv.second;
    }
  }
  // only trust neighbours within a factor ~2 in every dimension
  if (!pick || best > 3.0) return false;
  *c = pick->cfg;
  return true;
}

bool gemv_tuned_lookup(const GemvProblem &p, int *variant) {
  load_default_table();
  std::lock_guard<std::mutex> lk(g_mu);
  if (g_gemv_table.empty()) return false;
  const GKey k = gkey_of(p);
  auto it = g_gemv_table.find(k);
  if (it != g_gemv_table.end()) {
    *variant = it->second.variant;
    return true;
  }
  // nearest measured shape of the same layout in log space, within about a
  // factor 2 in one dimension (the split of the column kernel follows the
  // number of row tiles, the row kernel's threads per row the row length)
  double best = 1e300;
  const GRec *pick = nullptr;
  for (const auto &kv : g_gemv_table) {
    if (kv.first.cols != k.cols) continue;
    const double dp = std::log2(double(kv.first.P) / k.P);
    const double dq = std::log2(double(kv.first.Q) / k.Q);
    const double d = dp * dp + dq * dq;
    if (d < best) {
      best = d;
      pick = &kv.second;
    }
  }
  if (!pick || best > 1.0) return false;
  *variant = pick->variant;
  return true;
}

hml_status tune_load(const char *path, int *records) {
  FILE *f = fopen(path, "rb");
  if (!f) return HML_STATUS_IO_ERROR;
  char line[512];
  std::map<Key, Rec> t;
  std::map<GKey, GRec> gt;
  int n = 0, lineno = 0;
  bool header = false;
  while (fgets(line, sizeof line, f)) {
    ++lineno;
    if (lineno == 1) {
      header = strncmp(line, "#HML-B200 tuning v2", 19) == 0;
      if (!header) break;
      continue;
    }
    if (line[0] == '#' || line[0] == '\n') continue;
    if (line[0] == 'v') {
      GKey g;
      GRec r;
      if (sscanf(line, "v %d %d %d : %d %f", &g.cols, &g.P, &g.Q, &r.variant, &r.us) != 5 ||
          g.cols < 0 || g.cols > 1 || g.P < 1 || g.Q < 1 ||
          !gemv_variant_valid(g.cols == 0, r.variant)) {
        fclose(f);
        fprintf(stderr, "hml: %s:%d: bad GEMV tuning record: %s", path, lineno, line);
        return HML_STATUS_CONFIG_ERROR;
      }
      gt[g] = r;
      ++n;
      continue;
    }
    Key k;
    hml_sgemm_config c;
    float us;
    if (sscanf(line, "%d %d %d %d %d : %d %d %d %d %d %d %f", &k.akc, &k.bkc, &k.M, &k.N, &k.K,
               &c.algo, &c.tile_m, &c.tile_n, &c.split_k, &c.stages, &c.variant, &us) != 12 ||
        k.M < 1 || k.N < 1 || k.K < 1 || k.N > k.M || k.akc < 0 || k.akc > 1 || k.bkc < 0 ||
        k.bkc > 1) {
      fclose(f);
      fprintf(stderr, "hml: %s:%d: bad tuning record: %s", path, lineno, line);
      return HML_STATUS_CONFIG_ERROR;
    }
    bool known = false;
    for (const auto &sc : config_space())
      if (sc.algo == c.algo && sc.tile_m == c.tile_m && sc.tile_n == c.tile_n &&
          sc.split_k == c.split_k && sc.stages == c.stages && sc.variant == c.variant)
        known = true;
    if (!known) {
      fclose(f);
      fprintf(stderr, "hml: %s:%d: configuration not in this build's space\n", path, lineno);
      return HML_STATUS_CONFIG_ERROR;
    }
    t[k] = Rec{c, us};
    ++n;
  }
  fclose(f);
  if (!header) return HML_STATUS_CONFIG_ERROR;
  std::lock_guard<std::mutex> lk(g_mu);
  g_default_tried = true;  // an explicit table replaces the shipped one
  for (auto &kv : t) g_table[kv.first] = kv.second;
  for (auto &kv : gt) g_gemv_table[kv.first] = kv.second;
  if (records) *records = n;
  return HML_STATUS_SUCCESS;
}

hml_status tune_save(const char *path) {
  FILE *f = fopen(path, "wb");
  if (!f) return HML_STATUS_IO_ERROR;
  cudaDeviceProp prop;
  int dev = 0;
  cudaGetDevice(&dev);
  std::string name = "unknown";
  int sms = 0;
  if (cudaGetDeviceProperties(&prop, dev) == cudaSuccess) {
    name = prop.name;
    sms = prop.multiProcessorCount;
  }
  for (auto &ch : name)
    if (ch == ' ') ch = '_';
  fprintf(f, "#HML-B200 tuning v2\n# device %s sms %d\n", name.c_str(), sms);
  fprintf(f, "# akc bkc M N K : algo tile_m tile_n split_k stages variant time_us\n");
  std::lock_guard<std::mutex> lk(g_mu);
  for (const auto &kv : g_table) {
    const Key &k = kv.first;
    const hml_sgemm_config &c = kv.second.cfg;
    fprintf(f, "%d %d %d %d %d : %d %d %d %d %d %d %.3f\n", k.akc, k.bkc, k.M, k.N, k.K, c.algo,
            c.tile_m, c.tile_n, c.split_k, c.stages, c.variant, kv.second.us);
  }
  if (!g_gemv_table.empty()) fprintf(f, "# v cols P Q : variant time_us\n");
  for (const auto &kv : g_gemv_table)
    fprintf(f, "v %d %d %d : %d %.3f\n", kv.first.cols, kv.first.P, kv.first.Q,
            kv.second.variant, kv.second.us);
  const bool ok = fflush(f) == 0;
  fclose(f);
  return ok ? HML_STATUS_SUCCESS : HML_STATUS_IO_ERROR;
}

namespace {

// Timing buffers kept across calls (operands at the largest size tuned so
// far, and a buffer larger than L2 that is rewritten before each timing).
struct TuneBufs {
  float *A = nullptr, *B = nullptr, *C = nullptr, *flush = nullptr;
  size_t nA = 0, nB = 0, nC = 0, nflush = 0;
  int dev = -1;
};
TuneBufs g_bufs;

hml_status grow(float **p, size_t *have, size_t want, cudaStream_t s, uint64_t seed) {
  if (*have >= want) return HML_STATUS_SUCCESS;
  if (*p) {
    cudaStreamSynchronize(s);
    cudaFree(*p);
    *p = nullptr;
    *have = 0;
  }
  cudaError_t e = cudaMalloc(p, want * sizeof(float));
  if (e != cudaSuccess) {
    note_cuda_error(e, "autotune buffers");
    *p = nullptr;
    return HML_STATUS_ALLOC_FAILED;
  }
  *have = want;
  return fill_random(*p, want, seed, 0, 0, s);
}

}  // namespace

hml_status autotune(hml_order order, hml_op ta, hml_op tb, int M, int N, int K,
                    uint32_t families, int reps, hml_tune_entry *entries, int max_entries,
                    int *n_entries, cudaStream_t s) {
  if (n_entries) *n_entries = 0;
  if (M < 1 || N < 1 || K < 1 || reps < 1 || reps > 50) return HML_STATUS_INVALID_VALUE;
  if (families == 0) families = (1u << HML_ALGO_SIMT) | (1u << HML_ALGO_BF16X3) | (1u << HML_ALGO_BF16X6);
  const bool cm = order == HML_COL_MAJOR;
  // leading dimensions rounded up to 16 bytes, the layout every kernel
  // family (TMA included) can address
  auto r4 = [](int x) { return (std::max(1, x) + 3) / 4 * 4; };
  const int lda = r4(cm ? (ta == HML_OP_N ? M : K) : (ta == HML_OP_N ? K : M));
  const int ldb = r4(cm ? (tb == HML_OP_N ? K : N) : (tb == HML_OP_N ? N : K));
  const int ldc = r4(cm ? M : N);
  // stored extents: ld x (number of ld-strided lines: columns in
  // column-major order, rows in row-major order)
  const size_t a_lines = cm ? (ta == HML_OP_N ? K : M) : (ta == HML_OP_N ? M : K);
  const size_t b_lines = cm ? (tb == HML_OP_N ? N : K) : (tb == HML_OP_N ? K : N);
  const size_t c_lines = cm ? N : M;
  std::lock_guard<std::mutex> lk(g_mu);  // one tuning at a time
  int dev = 0;
  cudaGetDevice(&dev);
  if (g_bufs.dev != dev) {
    // buffers belong to one device; start over on another
    g_bufs = TuneBufs();
    g_bufs.dev = dev;
  }
  hml_status st;
  if ((st = grow(&g_bufs.A, &g_bufs.nA, a_lines * lda, s, 101)) != HML_STATUS_SUCCESS ||
      (st = grow(&g_bufs.B, &g_bufs.nB, b_lines * ldb, s, 102)) != HML_STATUS_SUCCESS ||
      (st = grow(&g_bufs.C, &g_bufs.nC, c_lines * ldc, s, 103)) != HML_STATUS_SUCCESS ||
      (st = grow(&g_bufs.flush, &g_bufs.nflush, size_t(64) << 20, s, 104)) != HML_STATUS_SUCCESS)
    return st;
  GemmProblem p;
  st = gemm_from_blas(order, ta, tb, M, N, K, 1.0f, g_bufs.A, lda, g_bufs.B, ldb, 0.0f, g_bufs.C,
                      ldc, &p);
  if (st != HML_STATUS_SUCCESS) return st;
  if (p.N == 1) return HML_STATUS_NOT_SUPPORTED;  // routed to the GEMV kernels
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    return HML_STATUS_CUDA_ERROR;
  }
  const size_t flush_bytes = g_bufs.nflush * sizeof(float);
  // A resident in L2 would make small problems look faster than in use:
  // flush whenever the operands fit in L2
  const bool need_flush = (static_cast<size_t>(M) * K + static_cast<size_t>(K) * N) * 4 <
                          size_t(200) << 20;
  int count = 0;
  float best = 1e30f;
  hml_sgemm_config best_cfg = {};
  for (const hml_sgemm_config &c : config_space()) {
    if (!(families & (1u << c.algo))) continue;
    hml_tune_entry ent;
    ent.config = c;
    ent.time_us = -1.0f;
    ent.status = check_config(p, c);
    if (ent.status == HML_STATUS_SUCCESS) {
      // warm-up launch (also rejects configurations the driver refuses);
      // timed as hml_sgemm_ex runs a selected configuration (the tail-wave
      // split of the tensor-core forms included), since the table feeds it
      ent.status = run_config(p, c, s, true);
      std::vector<float> ts;
      for (int r = 0; r < reps && ent.status == HML_STATUS_SUCCESS; ++r) {
        if (need_flush) cudaMemsetAsync(g_bufs.flush, r & 0xff, flush_bytes, s);
        cudaEventRecord(e0, s);
        ent.status = run_config(p, c, s, true);
        cudaEventRecord(e1, s);
        if (cudaEventSynchronize(e1) != cudaSuccess) {
          ent.status = HML_STATUS_CUDA_ERROR;
          break;
        }
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        ts.push_back(ms * 1000.0f);
        // a configuration four times slower than the best needs no median
        if (ts.size() == 1 && ts[0] > 4.0f * best) break;
      }
      if (ent.status == HML_STATUS_SUCCESS && !ts.empty()) {
        std::sort(ts.begin(), ts.end());
        ent.time_us = ts[ts.size() / 2];
        if (ent.time_us < best && allowed(c.algo)) {
          best = ent.time_us;
          best_cfg = c;
        }
      } else if (ent.status == HML_STATUS_SUCCESS) {
        ent.status = HML_STATUS_CUDA_ERROR;
      }
      // a failed launch leaves a sticky error only if the context is lost;
      // clear the non-sticky ones so the next configuration starts clean
      cudaGetLastError();
    }
    if (entries && count < max_entries) entries[count] = ent;
    ++count;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (n_entries) *n_entries = std::min(count, max_entries);
  if (best < 1e30f) g_table[key_of(p)] = Rec{best_cfg, best};
  return best < 1e30f ? HML_STATUS_SUCCESS : HML_STATUS_NOT_SUPPORTED;
}

hml_status autotune_gemv(hml_order order, hml_op trans, int M, int N, int reps,
                         hml_sgemv_tune_entry *entries, int max_entries, int *n_entries,
                         cudaStream_t s) {
  if (n_entries) *n_entries = 0;
  if (M < 1 || N < 1 || reps < 1 || reps > 50 || (order != HML_ROW_MAJOR && order != HML_COL_MAJOR) ||
      (trans != HML_OP_N && trans != HML_OP_T))
    return HML_STATUS_INVALID_VALUE;
  const bool cm = order == HML_COL_MAJOR;
  // A stored M x N with its leading dimension rounded up to 16 bytes
  const int lda = (cm ? M : N) + 3 - ((cm ? M : N) + 3) % 4;
  const size_t a_lines = cm ? N : M;
  const size_t nx = trans == HML_OP_N ? N : M;
  const size_t ny = trans == HML_OP_N ? M : N;
  std::lock_guard<std::mutex> lk(g_mu);
  int dev = 0;
  cudaGetDevice(&dev);
  if (g_bufs.dev != dev) {
    g_bufs = TuneBufs();
    g_bufs.dev = dev;
  }
  hml_status st;
  if ((st = grow(&g_bufs.A, &g_bufs.nA, a_lines * lda, s, 101)) != HML_STATUS_SUCCESS ||
      (st = grow(&g_bufs.B, &g_bufs.nB, nx, s, 102)) != HML_STATUS_SUCCESS ||
      (st = grow(&g_bufs.C, &g_bufs.nC, ny, s, 103)) != HML_STATUS_SUCCESS ||
      (st = grow(&g_bufs.flush, &g_bufs.nflush, size_t(64) << 20, s, 104)) != HML_STATUS_SUCCESS)
    return st;
  GemvProblem g;
  st = gemv_from_blas(order, trans, M, N, 1.0f, g_bufs.A, lda, g_bufs.B, 0.0f, g_bufs.C, &g);
  if (st != HML_STATUS_SUCCESS) return st;
  const bool rows = gemv_rows_layout(g);
  std::vector<int> variants;
  if (rows)
    for (int v = 4; v <= 256; v <<= 1) variants.push_back(v);
  else
    for (int v : {1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 20, 24, 32, 48, 64, 96,
                  128, 192, 256})
      variants.push_back(v);
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
    return HML_STATUS_CUDA_ERROR;
  const size_t flush_bytes = g_bufs.nflush * sizeof(float);
  const bool need_flush = static_cast<size_t>(M) * N * 4 < size_t(200) << 20;
  int count = 0;
  float best = 1e30f;
  int best_v = 0;
  for (int v : variants) {
    hml_sgemv_tune_entry ent;
    ent.variant = v;
    ent.time_us = -1.0f;
    ent.status = launch_gemv(g, v, s);  // warm-up
    std::vector<float> ts;
    for (int r = 0; r < reps && ent.status == HML_STATUS_SUCCESS; ++r) {
      if (need_flush) cudaMemsetAsync(g_bufs.flush, r & 0xff, flush_bytes, s);
      cudaEventRecord(e0, s);
      ent.status = launch_gemv(g, v, s);
      cudaEventRecord(e1, s);
      if (cudaEventSynchronize(e1) != cudaSuccess) {
        ent.status = HML_STATUS_CUDA_ERROR;
        break;
      }
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, e0, e1);
      ts.push_back(ms * 1000.0f);
      if (ts.size() == 1 && ts[0] > 4.0f * best) break;
    }
    if (ent.status == HML_STATUS_SUCCESS && !ts.empty()) {
      std::sort(ts.begin(), ts.end());
      ent.time_us = ts[ts.size() / 2];
      if (ent.time_us < best) {
        best = ent.time_us;
        best_v = v;
      }
    } else if (ent.status == HML_STATUS_SUCCESS) {
      ent.status = HML_STATUS_CUDA_ERROR;
    }
    cudaGetLastError();
    if (entries && count < max_entries) entries[count] = ent;
    ++count;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (n_entries) *n_entries = std::min(count, max_entries);
  if (best < 1e30f) g_gemv_table[gkey_of(g)] = GRec{best_v, best};
  return best < 1e30f ? HML_STATUS_SUCCESS : HML_STATUS_CUDA_ERROR;
}

hml_status tune_clear() {
  std::lock_guard<std::mutex> lk(g_mu);
  g_table.clear();
  g_gemv_table.clear();
  g_default_tried = true;  // cleared means empty: the shipped table stays out
  return HML_STATUS_SUCCESS;
}

int tune_size() {
  std::lock_guard<std::mutex> lk(g_mu);
  return static_cast<int>(g_table.size() + g_gemv_table.size());
}

hml_status set_math_mode(int mode) {
  if (mode != HML_MATH_FP32 && mode != HML_MATH_FAST) return HML_STATUS_INVALID_VALUE;
  g_math_mode = mode;
  return HML_STATUS_SUCCESS;
}

}  // namespace hml

extern "C" {

hml_status hml_autotune_sgemm(hml_order order, hml_op transA, hml_op transB, int M, int N, int K,
                              uint32_t families, int reps, hml_tune_entry *entries,
                              int max_entries, int *n_entries, void *stream) {
  return hml::autotune(order, transA, transB, M, N, K, families, reps, entries, max_entries,
                       n_entries, static_cast<cudaStream_t>(stream));
}

hml_status hml_autotune_sgemv(hml_order order, hml_op trans, int M, int N, int reps,
                              hml_sgemv_tune_entry *entries, int max_entries, int *n_entries,
                              void *stream) {
  return hml::autotune_gemv(order, trans, M, N, reps, entries, max_entries, n_entries,
                            static_cast<cudaStream_t>(stream));
}

hml_status hml_tune_save(const char *path) {
  return path ? hml::tune_save(path) : HML_STATUS_INVALID_VALUE;
}

hml_status hml_tune_load(const char *path, int *records) {
  return path ? hml::tune_load(path, records) : HML_STATUS_INVALID_VALUE;
}

hml_status hml_tune_clear(void) { return hml::tune_clear(); }

int hml_tune_size(void) { return hml::tune_size(); }

hml_status hml_set_math_mode(int mode) { return hml::set_math_mode(mode); }

}  // extern "C"
