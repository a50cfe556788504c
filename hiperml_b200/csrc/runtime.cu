// runtime.cu -- per-device resources of the library: the device error word,
// stream-keyed workspaces, tensor-map encoding through the driver entry
// point (no link-time dependency on libcuda), and error bookkeeping.
#include <atomic>
#include <mutex>
#include <map>
#include <string>
#include <utility>
#include <cstdio>
#include <cstring>

#include "hml_internal.h"

namespace hml {
namespace {

std::mutex g_mu;
std::map<int, int *> g_err_words;  // device -> error word
struct Ws {
  void *ptr = nullptr;
  size_t bytes = 0;
};
std::map<std::pair<int, cudaStream_t>, Ws> g_ws;
std::map<std::pair<int, cudaStream_t>, Ws> g_ws1;  // a second buffer per stream (slot 1)
std::map<std::pair<int, cudaStream_t>, Ws> g_counters;
std::map<int, int> g_sms;
thread_local std::string t_last_error;

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                  const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                  const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn g_encode = nullptr;

int current_device() {
  int d = 0;
  cudaGetDevice(&d);
  return d;
}

}  // namespace

std::atomic<uint64_t> g_launches{0};

void count_launch(int n) { g_launches.fetch_add(static_cast<uint64_t>(n), std::memory_order_relaxed); }
uint64_t launch_count() { return g_launches.load(std::memory_order_relaxed); }

void note_cuda_error(cudaError_t e, const char *where) {
  if (e == cudaSuccess) return;
  t_last_error = std::string(where) + ": " + cudaGetErrorString(e);
}

const char *last_error_text() { return t_last_error.c_str(); }

void note_text_error(const char *text) { t_last_error = text; }

int sm_count() {
  const int d = current_device();
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_sms.find(d);
  if (it != g_sms.end()) return it->second;
  int n = 148;
  if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, d) != cudaSuccess) n = 148;
  g_sms[d] = n;
  return n;
}

int *device_error_word_if_any() {
  const int d = current_device();
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_err_words.find(d);
  return it != g_err_words.end() ? it->second : nullptr;
}

int *device_error_word() {
  const int d = current_device();
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_err_words.find(d);
  if (it != g_err_words.end()) return it->second;
  int *w = nullptr;
  if (cudaMalloc(&w, 256) != cudaSuccess) return nullptr;
  if (cudaMemset(w, 0, 256) != cudaSuccess) {
    cudaFree(w);
    return nullptr;
  }
  g_err_words[d] = w;
  return w;
}

hml_status workspace(size_t bytes, cudaStream_t s, void **ptr) { return workspace_slot(0, bytes, s, ptr); }

hml_status workspace_slot(int slot, size_t bytes, cudaStream_t s, void **ptr) {
  const int d = current_device();
  std::lock_guard<std::mutex> lk(g_mu);
  Ws &w = (slot == 0 ? g_ws : g_ws1)[std::make_pair(d, s)];
  if (w.bytes < bytes) {
    if (w.ptr) {
      // earlier work on this stream may still use the old buffer
      cudaStreamSynchronize(s);
      cudaFree(w.ptr);
      w.ptr = nullptr;
      w.bytes = 0;
    }
    size_t want = bytes < (1u << 20) ? (1u << 20) : bytes;
    cudaError_t e = cudaMalloc(&w.ptr, want);
    if (e != cudaSuccess) {
      note_cuda_error(e, "workspace");
      w.ptr = nullptr;
      return HML_STATUS_ALLOC_FAILED;
    }
    w.bytes = want;
  }
  *ptr = w.ptr;
  return HML_STATUS_SUCCESS;
}

bool tensor_map_2d(CUtensorMap *map, CUtensorMapDataType dtype, const void *base, uint64_t dim0,
                   uint64_t dim1, uint64_t stride1_bytes, uint32_t box0, uint32_t box1,
                   CUtensorMapSwizzle swizzle) {
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_encode) {
      void *fn = nullptr;
      cudaDriverEntryPointQueryResult q;
      if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) !=
              cudaSuccess ||
          q != cudaDriverEntryPointSuccess || !fn) {
        t_last_error = "cuTensorMapEncodeTiled unavailable";
        return false;
      }
      g_encode = reinterpret_cast<EncodeTiledFn>(fn);
    }
  }
  if (dim0 == 0 || dim1 == 0) {
    // a zero extent is not encodable; such problems never launch a load
    dim0 = dim0 ? dim0 : 1;
    dim1 = dim1 ? dim1 : 1;
  }
  cuuint64_t dims[2] = {dim0, dim1};
  cuuint64_t strides[1] = {stride1_bytes};
  cuuint32_t box[2] = {box0, box1};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = g_encode(map, dtype, 2, const_cast<void *>(base), dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    char buf[128];
    snprintf(buf, sizeof buf, "cuTensorMapEncodeTiled failed (%d)", static_cast<int>(r));
    t_last_error = buf;
    return false;
  }
  return true;
}

hml_status tile_counters(size_t n, cudaStream_t s, unsigned **ptr) {
  const int d = current_device();
  std::lock_guard<std::mutex> lk(g_mu);
  Ws &w = g_counters[std::make_pair(d, s)];
  const size_t bytes = n * sizeof(unsigned);
  if (w.bytes < bytes) {
    if (w.ptr) {
      cudaStreamSynchronize(s);
      cudaFree(w.ptr);
      w.ptr = nullptr;
      w.bytes = 0;
    }
    size_t want = bytes < 65536 ? 65536 : bytes;
    cudaError_t e = cudaMalloc(&w.ptr, want);
    if (e == cudaSuccess) e = cudaMemsetAsync(w.ptr, 0, want, s);
    if (e != cudaSuccess) {
      note_cuda_error(e, "tile counters");
      if (w.ptr) cudaFree(w.ptr);
      w.ptr = nullptr;
      return HML_STATUS_ALLOC_FAILED;
    }
    w.bytes = want;
  }
  *ptr = static_cast<unsigned *>(w.ptr);
  return HML_STATUS_SUCCESS;
}

hml_status release_all() {
  std::lock_guard<std::mutex> lk(g_mu);
  cudaDeviceSynchronize();
  for (auto &kv : g_ws)
    if (kv.second.ptr) cudaFree(kv.second.ptr);
  g_ws.clear();
  for (auto &kv : g_ws1)
    if (kv.second.ptr) cudaFree(kv.second.ptr);
  g_ws1.clear();
  for (auto &kv : g_counters)
    if (kv.second.ptr) cudaFree(kv.second.ptr);
  g_counters.clear();
  return HML_STATUS_SUCCESS;
}

}  // namespace hml
