// ref_gpu_registry.cu -- TEST INFRASTRUCTURE ONLY.  The host side of the
// texture stand-in of ref_gpu_compat.h: which texture object has which name,
// and the per-translation-unit device tables a binding updates.
#include <cuda_runtime.h>

#include <mutex>
#include <vector>

namespace {
struct Entry {
  const void *obj;
  int id;
};
std::mutex &mu() {
  static std::mutex m;
  return m;
}
std::vector<Entry> &textures() {
  static std::vector<Entry> v;
  return v;
}
std::vector<cudaError_t (*)(int, const void *, size_t)> &tables() {
  static std::vector<cudaError_t (*)(int, const void *, size_t)> v;
  return v;
}
}  // namespace

void hml_ref_register_texture(const void *host_obj, int id) {
  std::lock_guard<std::mutex> lk(mu());
  for (const Entry &e : textures())
    if (e.obj == host_obj) return;
  textures().push_back({host_obj, id});
}

void hml_ref_register_table(cudaError_t (*update)(int, const void *, size_t)) {
  std::lock_guard<std::mutex> lk(mu());
  tables().push_back(update);
}

cudaError_t hml_ref_bind(const void *host_obj, const void *ptr, size_t n) {
  std::lock_guard<std::mutex> lk(mu());
  int id = -1;
  for (const Entry &e : textures())
    if (e.obj == host_obj) id = e.id;
  if (id < 0) return cudaErrorInvalidValue;
  for (auto update : tables()) {
    cudaError_t err = update(id, ptr, n);
    if (err != cudaSuccess) return err;
  }
  return cudaSuccess;
}
