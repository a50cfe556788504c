// batched.cu -- many uneven SGEMMs in one persistent launch with a device work
// queue (hml_batch_plan_*, hml_sgemm_batched).
//
// The reference runs one problem per call: every hmlSgemm copies, launches a
// grid sized to that problem and synchronises (src/hml_sgemm.cu:120-211), so
// a stream of small skinny problems leaves most of the GPU idle between and
// inside calls.  Here a plan turns a whole batch into one list of tile work
// items and a single launch of 2 CTAs per SM drains it:
//
//   * host side (once per plan): each problem is normalised to the canonical
//     long-M form, given the narrowest 128-row FP32 SIMT tile that covers its
//     N, and cut into 128 x BN tiles.  The tiles of all problems are sorted
//     by estimated duration, longest first (longest-processing-time order),
//     so the queue ends with short tiles and the machine drains evenly.
//   * device side: every CTA repeatedly takes the next item from a global
//     atomic counter, computes that tile with the same staged-slab arithmetic
//     as the single-problem SIMT kernel (simt_tile.cuh) -- a 16-byte
//     cp.async ring when the problem's base and leading dimension allow it,
//     4-byte copies otherwise -- and writes its C tile.  No CTA ever waits
//     for another: the counter is the only shared state, so the launch needs
//     no co-residency and cannot deadlock.  The last CTA to finish resets the
//     counter, which makes the launch replayable from a CUDA graph
//     (hml_batch_plan_graph_launch captures it once and replays the graph).
//
// Problems the tensor cores can take (N > 8, A addressable by TMA, a real
// product) go to the split-BF16 part of the plan instead (sgemm_tc.cu,
// tc_batch_*): one B-splitting launch and one persistent launch per tile
// width class, whose CTAs work through host-balanced item lists.  Both parts
// are captured in the plan's graph.
//
// Each tile's result equals, bit for bit, the single-problem kernel's result
// for the configuration hml_batch_problem_config reports (the SIMT tile, or
// BF16X6 with the class's tile width, split_k = 1).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <numeric>
#include <vector>

#include "hml_internal.h"
#include "simt_tile.cuh"

namespace hml {
namespace {

// Tile shapes of the batched kernel: SIMT variants with 128-row tiles (4 x 16
// micro-tiles or narrower), small enough in registers and shared memory for
// 2 CTAs per SM.  Slot s covers N up to kSlotN[s].
constexpr int kSlotVariant[] = {1, 0, 2, 7, 8};
constexpr int kSlotN[] = {8, 16, 32, 64, 128};
constexpr int kNumSlots = 5;
constexpr int kBatchThreads = 256;
constexpr int kBatchRingBytes = 110 * 1024;  // per CTA, 2 CTAs per SM
constexpr int kBatchSmem = kBatchRingBytes + 1024;  // + alignment slack
constexpr int kBatchMaxStages = 6;

struct BatchProblem {
  const float *A;
  const float *B;
  float *C;
  int64_t sam, sak, sbk, sbn, scm, scn;
  int M, N, K;
  float alpha, beta;
  int kind;  // slot * 4 + a_kcontig * 2 + b_kcontig
  int vec;   // bit 0: A is read in 16-byte granules, bit 1: B
  int pad_;
};

struct BatchItem {
  int prob;
  int mt;  // row tile (units of 128 rows)
  int nt;  // column tile (units of the slot's BN)
  int pad_;
};

struct BatchArgs {
  const BatchProblem *probs;
  const BatchItem *items;
  int nitems;
  unsigned *queue;  // [0] next item, [1] CTAs finished
};

template <int V, bool AK, bool BK_>
__device__ __noinline__ void batch_tile(const BatchProblem &p, int64_t m0, int n0,
                                           uint8_t *smem) {
  constexpr SimtShape sh = kSimtShapes[V];
  using T = SimtTile<sh.tm, sh.tn, sh.wm, sh.wn, sh.wk, AK, BK_>;
  constexpr int BM = T::BM, BN = T::BN, NT = T::NT;
  static_assert(BM == 128, "batched tiles are 128 rows");
  constexpr int A_BYTES = T::A_BYTES, STAGE_BYTES = T::STAGE_BYTES;
  constexpr int ST = kBatchRingBytes / STAGE_BYTES < kBatchMaxStages
                         ? kBatchRingBytes / STAGE_BYTES
                         : kBatchMaxStages;
  static_assert(ST >= 2 && T::RED_BYTES <= kBatchRingBytes, "ring");

  const int tid = threadIdx.x;
  const int M = p.M, N = p.N, K = p.K;
  const float *A = p.A;
  const float *B = p.B;
  const int64_t sam = p.sam, sak = p.sak, sbk = p.sbk, sbn = p.sbn;
  const bool va = p.vec & 1, vb = (p.vec >> 1) & 1;
  const int nk = (K + kBK - 1) / kBK;

  auto issue = [&](int it) {
    const int s = it % ST;
    const int k0 = it * kBK;
    const uint32_t ua = smem_u32(smem + s * STAGE_BYTES);
    const uint32_t ub = ua + A_BYTES;
    if (va) {
      for (int e = tid; e < BM * kBK / 4; e += NT) {
        const int m = AK ? e / (kBK / 4) : 4 * (e % (BM / 4));
        const int k = AK ? 4 * (e % (kBK / 4)) : e / (BM / 4);
        const int64_t gm = m0 + m;
        const int gk = k0 + k;
        const int64_t rem = AK ? (gm < M ? K - gk : 0) : (gk < K ? M - gm : 0);
        const int bytes = rem <= 0 ? 0 : rem >= 4 ? 16 : static_cast<int>(rem) * 4;
        const float *src = bytes ? A + gm * sam + static_cast<int64_t>(gk) * sak : A;
        cp_async16(ua + T::a_off(m, k), src, bytes);
      }
    } else {
      for (int e = tid; e < BM * kBK; e += NT) {
        const int m = AK ? e / kBK : e % BM;
        const int k = AK ? e % kBK : e / BM;
        const int64_t gm = m0 + m;
        const int gk = k0 + k;
        const bool ok = gm < M && gk < K;
        cp_async4(ua + T::a_off(m, k), ok ? A + gm * sam + static_cast<int64_t>(gk) * sak : A, ok);
      }
    }
    if (vb) {
      for (int e = tid; e < BN * kBK / 4; e += NT) {
        const int n = BK_ ? e / (kBK / 4) : 4 * (e % (BN / 4));
        const int k = BK_ ? 4 * (e % (kBK / 4)) : e / (BN / 4);
        const int gn = n0 + n;
        const int gk = k0 + k;
        const int64_t rem = BK_ ? (gn < N ? K - gk : 0) : (gk < K ? N - gn : 0);
        const int bytes = rem <= 0 ? 0 : rem >= 4 ? 16 : static_cast<int>(rem) * 4;
        const float *src = bytes ? B + static_cast<int64_t>(gk) * sbk + static_cast<int64_t>(gn) * sbn : B;
        cp_async16(ub + T::b_off(n, k), src, bytes);
      }
    } else {
      for (int e = tid; e < BN * kBK; e += NT) {
        const int n = BK_ ? e / kBK : e % BN;
        const int k = BK_ ? e % kBK : e / BN;
        const int gn = n0 + n;
        const int gk = k0 + k;
        const bool ok = gn < N && gk < K;
        cp_async4(ub + T::b_off(n, k),
                  ok ? B + static_cast<int64_t>(gk) * sbk + static_cast<int64_t>(gn) * sbn : B, ok);
      }
    }
  };

  float acc[sh.tm][sh.tn];
  T::zero(acc);
  for (int it = 0; it < ST - 1; ++it) {
    if (it < nk) issue(it);
    cp_async_commit();
  }
  const typename T::Coord co = T::coord(tid);
  for (int it = 0; it < nk; ++it) {
    const int s = it % ST;
    cp_async_wait_ring(ST);
    __syncthreads();
    if (it + ST - 1 < nk) issue(it + ST - 1);
    cp_async_commit();
    T::slab(reinterpret_cast<const float *>(smem + s * STAGE_BYTES),
            reinterpret_cast<const float *>(smem + s * STAGE_BYTES + A_BYTES), acc, co);
  }
  asm volatile("cp.async.wait_all;" ::: "memory");
  __syncthreads();  // every slab consumed: the ring becomes the reduction buffer
  float *red = reinterpret_cast<float *>(smem);
  T::stash(red, acc, co);
  __syncthreads();
  T::reduce_wk(red, tid);
  __syncthreads();
  T::store_c(red, tid, m0, n0, M, N, p.C, p.scm, p.scn, p.alpha, p.beta);
  __syncthreads();  // the reduction buffer is read before the next tile's copies land
}

template <int SLOT>
__device__ __forceinline__ void batch_slot(const BatchProblem &p, int lay, int64_t m0, int nt,
                                           uint8_t *smem) {
  constexpr int V = kSlotVariant[SLOT];
  constexpr int BN = kSimtShapes[V].bn();
  static_assert(BN == kSlotN[SLOT], "slot width");
  const int n0 = nt * BN;
  switch (lay) {
    case 0: batch_tile<V, false, false>(p, m0, n0, smem); break;
    case 1: batch_tile<V, false, true>(p, m0, n0, smem); break;
    case 2: batch_tile<V, true, false>(p, m0, n0, smem); break;
    default: batch_tile<V, true, true>(p, m0, n0, smem); break;
  }
}

__global__ void __launch_bounds__(kBatchThreads, 2) batched_kernel(BatchArgs a) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = align_shared(smem_raw, 1024);
  __shared__ int s_item;
  const int tid = threadIdx.x;
  for (;;) {
    if (tid == 0) s_item = static_cast<int>(atomicAdd(&a.queue[0], 1u));
    __syncthreads();
    const int it = s_item;
    __syncthreads();  // s_item is read by all before thread 0 may overwrite it
    if (it >= a.nitems) break;
    const BatchItem w = a.items[it];
    const BatchProblem &p = a.probs[w.prob];
    const int kind = p.kind;
    const int64_t m0 = static_cast<int64_t>(w.mt) * 128;
    const int lay = kind & 3;
    switch (kind >> 2) {
      case 0: batch_slot<0>(p, lay, m0, w.nt, smem); break;
      case 1: batch_slot<1>(p, lay, m0, w.nt, smem); break;
      case 2: batch_slot<2>(p, lay, m0, w.nt, smem); break;
      case 3: batch_slot<3>(p, lay, m0, w.nt, smem); break;
      default: batch_slot<4>(p, lay, m0, w.nt, smem); break;
    }
  }
  // the last CTA out resets the queue for the next launch of the plan
  if (tid == 0) {
    __threadfence();
    const unsigned done = atomicAdd(&a.queue[1], 1u);
    if (done == gridDim.x - 1) {
      atomicExch(&a.queue[0], 0u);
      atomicExch(&a.queue[1], 0u);
      __threadfence();
    }
  }
}

int slot_for(int N) {
  for (int s = 0; s < kNumSlots; ++s)
    if (N <= kSlotN[s]) return s;
  return kNumSlots - 1;
}

bool aligned16(const void *ptr) { return (reinterpret_cast<uintptr_t>(ptr) & 15u) == 0; }

// Estimated seconds of one tile on one CTA (2 CTAs per SM share the SM's
// FP32 rate and its share of HBM bandwidth); only the order matters.
double tile_cost(int bn, int K) {
  const double flops = 2.0 * 128.0 * bn * K, bytes = 4.0 * (128.0 + bn) * K;
  return std::max(flops / 120e9, bytes / 20e9) + 2e-6;
}

}  // namespace

// Host-side plan (opaque to callers).
struct BatchPlan {
  int device = -1;
  int count = 0;
  int nitems = 0;
  int ctas = 0;
  double flops = 0.0, bytes = 0.0;
  void *dev = nullptr;  // [queue 256 B][problems][items]
  BatchArgs args = {};
  TcBatch *tc = nullptr;  // the split-BF16 part
  cudaStream_t capture_stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

namespace {

hml_status build_host(hml_order order, const hml_gemm_desc *descs, int count,
                      std::vector<BatchProblem> *probs, std::vector<BatchItem> *items,
                      std::vector<GemmProblem> *tc_probs, double *flops, double *bytes) {
  if (count < 0 || (count > 0 && !descs)) return HML_STATUS_INVALID_VALUE;
  std::vector<double> cost;
  *flops = 0.0;
  *bytes = 0.0;
  for (int i = 0; i < count; ++i) {
    const hml_gemm_desc &d = descs[i];
    GemmProblem g;
    hml_status st = gemm_from_blas(order, static_cast<hml_op>(d.transA),
                                   static_cast<hml_op>(d.transB), d.M, d.N, d.K, d.alpha, d.A,
                                   d.lda, d.B, d.ldb, d.beta, d.C, d.ldc, &g);
    if (st != HML_STATUS_SUCCESS) {
      char msg[96];
      snprintf(msg, sizeof msg, "batch problem %d: invalid arguments", i);
      note_text_error(msg);
      return st;
    }
    if (g.M == 0 || g.N == 0) continue;
    if (tc_probs && tc_batch_eligible(g)) {
      tc_probs->push_back(g);
      *flops += 2.0 * g.M * g.N * static_cast<double>(g.K);
      *bytes += 4.0 * (static_cast<double>(g.M) * g.K + static_cast<double>(g.K) * g.N +
                       static_cast<double>(g.M) * g.N * (g.beta != 0.0f ? 2 : 1));
      continue;
    }
    BatchProblem b;
    memset(&b, 0, sizeof b);
    b.A = g.A; b.B = g.B; b.C = g.C;
    b.sam = g.sam; b.sak = g.sak; b.sbk = g.sbk; b.sbn = g.sbn; b.scm = g.scm; b.scn = g.scn;
    b.M = g.M; b.N = g.N; b.K = g.K;
    b.alpha = g.alpha; b.beta = g.beta;
    if (g.K == 0 || g.alpha == 0.0f) {
      // no product: the tile arithmetic runs on zero operands
      b.K = 0;
      b.alpha = 0.0f;
      b.A = nullptr;
      b.B = nullptr;
    }
    const bool ak = g.a_kcontig(), bk = g.b_kcontig();
    const int slot = slot_for(g.N);
    b.kind = slot * 4 + (ak ? 2 : 0) + (bk ? 1 : 0);
    const int64_t sa = ak ? g.sam : g.sak;  // the non-unit stride of A
    const int64_t sb = bk ? g.sbn : g.sbk;
    b.vec = (b.A && aligned16(g.A) && sa % 4 == 0 ? 1 : 0) |
            (b.B && aligned16(g.B) && sb % 4 == 0 ? 2 : 0);
    const int bn = kSlotN[slot];
    const int64_t mt = (static_cast<int64_t>(g.M) + 127) / 128;
    const int64_t nt = (static_cast<int64_t>(g.N) + bn - 1) / bn;
    if (static_cast<int64_t>(items->size()) + mt * nt > 0x7fffffff) return HML_STATUS_NOT_SUPPORTED;
    const int pi = static_cast<int>(probs->size());
    probs->push_back(b);
    const double c = tile_cost(bn, b.K);
    for (int64_t x = 0; x < mt; ++x)
      for (int64_t y = 0; y < nt; ++y) {
        items->push_back(BatchItem{pi, static_cast<int>(x), static_cast<int>(y), 0});
        cost.push_back(c);
      }
    *flops += 2.0 * g.M * g.N * static_cast<double>(b.K);
    *bytes += 4.0 * (static_cast<double>(g.M) * b.K + static_cast<double>(b.K) * g.N +
                     static_cast<double>(g.M) * g.N * (g.beta != 0.0f ? 2 : 1));
  }
  // longest first; ties keep problem and tile order
  std::vector<int> order_idx(items->size());
  std::iota(order_idx.begin(), order_idx.end(), 0);
  std::stable_sort(order_idx.begin(), order_idx.end(),
                   [&](int x, int y) { return cost[x] > cost[y]; });
  std::vector<BatchItem> sorted(items->size());
  for (size_t i = 0; i < order_idx.size(); ++i) sorted[i] = (*items)[order_idx[i]];
  items->swap(sorted);
  return HML_STATUS_SUCCESS;
}

size_t layout_bytes(size_t nprob, size_t nitems, size_t *off_prob, size_t *off_items) {
  *off_prob = 256;
  *off_items = *off_prob + ((nprob * sizeof(BatchProblem) + 255) & ~size_t(255));
  return *off_items + nitems * sizeof(BatchItem);
}

hml_status kernel_attributes() {
  static int done[64] = {0};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 64 && done[dev]) return HML_STATUS_SUCCESS;
  cudaError_t e = cudaFuncSetAttribute(batched_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       kBatchSmem);
  if (e != cudaSuccess) {
    note_cuda_error(e, "batched attributes");
    return HML_STATUS_CUDA_ERROR;
  }
  if (dev >= 0 && dev < 64) done[dev] = 1;
  return HML_STATUS_SUCCESS;
}

cudaError_t launch_batched(const BatchArgs &args, int ctas, cudaStream_t s) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(static_cast<unsigned>(ctas));
  cfg.blockDim = dim3(kBatchThreads);
  cfg.dynamicSmemBytes = kBatchSmem;
  cfg.stream = s;
  return cudaLaunchKernelEx(&cfg, batched_kernel, args);
}

int grid_for(int nitems) {
  return std::max(1, std::min(nitems, 2 * sm_count()));
}

}  // namespace

// ----------------------------------------------------------- plan objects
hml_status batch_plan_create(hml_order order, const hml_gemm_desc *descs, int count,
                             BatchPlan **out) {
  if (!out) return HML_STATUS_INVALID_VALUE;
  *out = nullptr;
  std::vector<BatchProblem> probs;
  std::vector<BatchItem> items;
  std::vector<GemmProblem> tc_probs;
  double flops, bytes;
  hml_status st = build_host(order, descs, count, &probs, &items, &tc_probs, &flops, &bytes);
  if (st != HML_STATUS_SUCCESS) return st;
  st = kernel_attributes();
  if (st != HML_STATUS_SUCCESS) return st;
  TcBatch *tc = nullptr;
  st = tc_batch_create(tc_probs.data(), static_cast<int>(tc_probs.size()), nullptr, &tc);
  if (st != HML_STATUS_SUCCESS) return st;
  BatchPlan *pl = new (std::nothrow) BatchPlan;
  if (!pl) {
    tc_batch_destroy(tc);
    return HML_STATUS_ALLOC_FAILED;
  }
  pl->tc = tc;
  cudaGetDevice(&pl->device);
  pl->count = count;
  pl->nitems = static_cast<int>(items.size());
  pl->ctas = grid_for(pl->nitems);
  pl->flops = flops;
  pl->bytes = bytes;
  size_t op, oi;
  const size_t total = layout_bytes(probs.size(), items.size(), &op, &oi);
  cudaError_t e = cudaMalloc(&pl->dev, total);
  if (e != cudaSuccess) {
    note_cuda_error(e, "batch plan allocation");
    tc_batch_destroy(pl->tc);
    delete pl;
    return HML_STATUS_ALLOC_FAILED;
  }
  uint8_t *base = static_cast<uint8_t *>(pl->dev);
  e = cudaMemset(base, 0, 256);
  if (e == cudaSuccess && !probs.empty())
    e = cudaMemcpy(base + op, probs.data(), probs.size() * sizeof(BatchProblem),
                   cudaMemcpyHostToDevice);
  if (e == cudaSuccess && !items.empty())
    e = cudaMemcpy(base + oi, items.data(), items.size() * sizeof(BatchItem),
                   cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    note_cuda_error(e, "batch plan upload");
    cudaFree(pl->dev);
    tc_batch_destroy(pl->tc);
    delete pl;
    return HML_STATUS_CUDA_ERROR;
  }
  pl->args.queue = reinterpret_cast<unsigned *>(base);
  pl->args.probs = reinterpret_cast<const BatchProblem *>(base + op);
  pl->args.items = reinterpret_cast<const BatchItem *>(base + oi);
  pl->args.nitems = pl->nitems;
  *out = pl;
  return HML_STATUS_SUCCESS;
}

// The plan's launches: the SIMT queue, then the split-BF16 part.
hml_status launch_plan(BatchPlan *pl, cudaStream_t s) {
  if (pl->nitems > 0) {
    count_launch();
    const cudaError_t e = launch_batched(pl->args, pl->ctas, s);
    note_cuda_error(e, "batched launch");
    if (e != cudaSuccess) return HML_STATUS_CUDA_ERROR;
  }
  return tc_batch_launch(pl->tc, s);
}

bool plan_empty(const BatchPlan *pl) { return pl->nitems == 0 && tc_batch_items(pl->tc) == 0; }

hml_status batch_plan_run(BatchPlan *pl, cudaStream_t s) {
  if (!pl) return HML_STATUS_INVALID_VALUE;
  if (plan_empty(pl)) return HML_STATUS_SUCCESS;
  return launch_plan(pl, s);
}

hml_status batch_plan_graph_launch(BatchPlan *pl, cudaStream_t s) {
  if (!pl) return HML_STATUS_INVALID_VALUE;
  if (plan_empty(pl)) return HML_STATUS_SUCCESS;
  cudaError_t e = cudaSuccess;
  if (!pl->exec) {
    // capture the plan's launches once on a private stream
    e = cudaStreamCreateWithFlags(&pl->capture_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess)
      e = cudaStreamBeginCapture(pl->capture_stream, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      const hml_status sl = launch_plan(pl, pl->capture_stream);
      e = cudaStreamEndCapture(pl->capture_stream, &pl->graph);
      if (e == cudaSuccess && sl != HML_STATUS_SUCCESS) e = cudaErrorLaunchFailure;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&pl->exec, pl->graph, 0);
    if (e != cudaSuccess) {
      note_cuda_error(e, "batched graph capture");
      if (pl->graph) cudaGraphDestroy(pl->graph);
      pl->graph = nullptr;
      pl->exec = nullptr;
      return HML_STATUS_CUDA_ERROR;
    }
  }
  count_launch();
  e = cudaGraphLaunch(pl->exec, s);
  note_cuda_error(e, "batched graph launch");
  return cuda_status(e);
}

void batch_plan_destroy(BatchPlan *pl) {
  if (!pl) return;
  if (pl->exec) cudaGraphExecDestroy(pl->exec);
  if (pl->graph) cudaGraphDestroy(pl->graph);
  if (pl->capture_stream) cudaStreamDestroy(pl->capture_stream);
  if (pl->dev) cudaFree(pl->dev);
  tc_batch_destroy(pl->tc);
  delete pl;
}

// One-shot batch: the plan lives in stream-ordered memory for one launch.
hml_status sgemm_batched(hml_order order, const hml_gemm_desc *descs, int count, cudaStream_t s) {
  std::vector<BatchProblem> probs;
  std::vector<BatchItem> items;
  std::vector<GemmProblem> tc_probs;
  double flops, bytes;
  hml_status st = build_host(order, descs, count, &probs, &items, &tc_probs, &flops, &bytes);
  if (st != HML_STATUS_SUCCESS) return st;
  if (!tc_probs.empty()) {
    // the split-BF16 part in stream-ordered memory, released after its launches
    TcBatch *tc = nullptr;
    st = tc_batch_create(tc_probs.data(), static_cast<int>(tc_probs.size()), s, &tc);
    if (st != HML_STATUS_SUCCESS) return st;
    st = tc_batch_launch(tc, s);
    tc_batch_destroy(tc);
    if (st != HML_STATUS_SUCCESS) return st;
  }
  if (items.empty()) return HML_STATUS_SUCCESS;
  st = kernel_attributes();
  if (st != HML_STATUS_SUCCESS) return st;
  size_t op, oi;
  const size_t total = layout_bytes(probs.size(), items.size(), &op, &oi);
  void *dev = nullptr;
  cudaError_t e = cudaMallocAsync(&dev, total, s);
  if (e != cudaSuccess) {
    note_cuda_error(e, "batch allocation");
    return HML_STATUS_ALLOC_FAILED;
  }
  uint8_t *base = static_cast<uint8_t *>(dev);
  e = cudaMemsetAsync(base, 0, 256, s);
  // pageable sources: each copy has left the host buffer when it returns
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(base + op, probs.data(), probs.size() * sizeof(BatchProblem),
                        cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(base + oi, items.data(), items.size() * sizeof(BatchItem),
                        cudaMemcpyHostToDevice, s);
  BatchArgs args;
  args.queue = reinterpret_cast<unsigned *>(base);
  args.probs = reinterpret_cast<const BatchProblem *>(base + op);
  args.items = reinterpret_cast<const BatchItem *>(base + oi);
  args.nitems = static_cast<int>(items.size());
  if (e == cudaSuccess) {
    count_launch();
    e = launch_batched(args, grid_for(args.nitems), s);
  }
  const cudaError_t ef = cudaFreeAsync(dev, s);
  if (e == cudaSuccess) e = ef;
  note_cuda_error(e, "batched launch");
  return cuda_status(e);
}

}  // namespace hml

// ------------------------------------------------------------------ C ABI
struct hml_batch_plan_s {
  hml::BatchPlan *impl;
};

extern "C" {

hml_status hml_batch_plan_create(hml_order order, const hml_gemm_desc *descs, int count,
                                 hml_batch_plan *plan) {
  if (!plan) return HML_STATUS_INVALID_VALUE;
  *plan = nullptr;
  hml::BatchPlan *impl = nullptr;
  const hml_status st = hml::batch_plan_create(order, descs, count, &impl);
  if (st != HML_STATUS_SUCCESS) return st;
  hml_batch_plan h = new (std::nothrow) hml_batch_plan_s;
  if (!h) {
    hml::batch_plan_destroy(impl);
    return HML_STATUS_ALLOC_FAILED;
  }
  h->impl = impl;
  *plan = h;
  return HML_STATUS_SUCCESS;
}

hml_status hml_batch_plan_run(hml_batch_plan plan, void *stream) {
  if (!plan) return HML_STATUS_INVALID_VALUE;
  return hml::batch_plan_run(plan->impl, static_cast<cudaStream_t>(stream));
}

hml_status hml_batch_plan_graph_launch(hml_batch_plan plan, void *stream) {
  if (!plan) return HML_STATUS_INVALID_VALUE;
  return hml::batch_plan_graph_launch(plan->impl, static_cast<cudaStream_t>(stream));
}

hml_status hml_batch_plan_info(hml_batch_plan plan, int *tiles, int *ctas, double *flops,
                               double *bytes) {
  if (!plan) return HML_STATUS_INVALID_VALUE;
  if (tiles) *tiles = plan->impl->nitems + hml::tc_batch_items(plan->impl->tc);
  if (ctas) *ctas = std::max(plan->impl->nitems > 0 ? plan->impl->ctas : 0,
                             hml::tc_batch_ctas(plan->impl->tc));
  if (flops) *flops = plan->impl->flops;
  if (bytes) *bytes = plan->impl->bytes;
  return HML_STATUS_SUCCESS;
}

hml_status hml_batch_plan_destroy(hml_batch_plan plan) {
  if (!plan) return HML_STATUS_SUCCESS;
  hml::batch_plan_destroy(plan->impl);
  delete plan;
  return HML_STATUS_SUCCESS;
}

hml_status hml_sgemm_batched(hml_order order, const hml_gemm_desc *descs, int count,
                             void *stream) {
  return hml::sgemm_batched(order, descs, count, static_cast<cudaStream_t>(stream));
}

hml_status hml_batch_problem_config(hml_order order, const hml_gemm_desc *desc,
                                    hml_sgemm_config *config) {
  using namespace hml;
  if (!desc || !config) return HML_STATUS_INVALID_VALUE;
  GemmProblem g;
  hml_status st = gemm_from_blas(order, static_cast<hml_op>(desc->transA),
                                 static_cast<hml_op>(desc->transB), desc->M, desc->N, desc->K,
                                 desc->alpha, desc->A, desc->lda, desc->B, desc->ldb, desc->beta,
                                 desc->C, desc->ldc, &g);
  if (st != HML_STATUS_SUCCESS) return st;
  if (g.M > 0 && g.N > 0 && tc_batch_eligible(g)) {
    *config = tc_batch_config(g);
    return HML_STATUS_SUCCESS;
  }
  const int slot = slot_for(g.N);
  *config = hml_sgemm_config{HML_ALGO_SIMT, 128, kSlotN[slot], 1, 3, kSlotVariant[slot]};
  return HML_STATUS_SUCCESS;
}

}  // extern "C"
