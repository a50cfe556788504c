// select.cu -- which configuration hml_sgemm_ex runs.
//
// Order of precedence (replacing the reference's static table lookup
// cfg[min(K,96)][ceil(min(N,96)/16)], src/hml_sgemm_kernel.cu:189-237):
//   1. the measured table of the autotuner (exact shape class, else the
//      nearest measured class in log space), when one is loaded;
//   2. the learned predictor, when one is loaded;
//   3. the heuristic below.
#include <algorithm>
#include <cmath>

#include "hml_select.h"
#include "hml_tune.h"

namespace hml {

int simt_num_shapes();
void simt_shape(int v, int *bm, int *bn, int *wk);
int tc_num_shapes();
void tc_shape(int v, int *bm, int *bn);
bool tc_config_fits(int bn, int ns, int stages);
int tc_ns(int algo);

namespace {

int pow2_at_least(int64_t x, int cap) {
  int s = 1;
  while (s < cap && s < x) s <<= 1;
  return s;
}

// pick split_k so the grid covers the machine about `waves` times while each
// CTA keeps at least `min_k` of K
int choose_split(int64_t tiles, int K, int ctas_per_sm, int min_k) {
  const int64_t want = static_cast<int64_t>(sm_count()) * ctas_per_sm;
  int split = tiles >= want ? 1 : pow2_at_least((want + tiles - 1) / tiles, 16);
  while (split > 1 && K / split < min_k) split >>= 1;
  return split;
}

}  // namespace

hml_sgemm_config heuristic_config(const GemmProblem &p, int algo) {
  hml_sgemm_config c = {};
  if (algo == HML_ALGO_BF16X3 || algo == HML_ALGO_BF16X6 || algo == HML_ALGO_TF32X3) {
    int best = -1;
    // the narrowest single-CTA (128-row) tile that holds N
    for (int v = 0; v < tc_num_shapes(); ++v) {
      int bm, bn;
      tc_shape(v, &bm, &bn);
      if (bm != 128) continue;
      best = v;
      if (bn >= p.N) break;
    }
    if (best >= 0) {
      int bm, bn;
      tc_shape(best, &bm, &bn);
      const int64_t tiles = ((p.M + bm - 1) / bm) * static_cast<int64_t>((p.N + bn - 1) / bn);
      int stages = 2;
      for (int st : {4, 6, 8})
        if (tc_config_fits(bn, tc_ns(algo), st)) stages = st;
      c = {algo, bm, bn, choose_split(tiles, p.K, 1, 256), stages, best};
      return c;
    }
  }
  // SIMT, N <= 8 with contiguous columns of A: the stream-K kernel with the
  // narrowest NB that holds N and its deepest ring (measured on B200,
  // 65536 x 8 x 4096: 6.5 TB/s against 4.8 for the tiled kernel)
  for (int i = 0; i < stream_num_variants(); ++i) {
    const int nb = stream_tile_n(i);
    if (nb < p.N) continue;
    const hml_sgemm_config sc = {HML_ALGO_SIMT, 128, nb, 1, stream_max_stages(nb),
                                 simt_num_shapes() + i};
    if (check_stream(p, sc) == HML_STATUS_SUCCESS) return sc;
    break;
  }
  // SIMT: the narrowest tile that holds N, wider rows when M is large
  int var;
  if (p.N <= 8) var = 1;
  else if (p.N <= 16) var = 0;
  else if (p.N <= 32) var = (p.M >= 256 * 2 * sm_count()) ? 3 : 2;
  else if (p.N <= 64) var = (p.M >= 256 * sm_count()) ? 4 : 7;
  else var = (p.M >= 256 * sm_count()) ? 5 : 8;
  int bm, bn, wk;
  simt_shape(var, &bm, &bn, &wk);
  const int per_sm = (bm * bn <= 128 * 16 * 2) ? 2 : 1;
  const int64_t tiles = ((p.M + bm - 1) / bm) * static_cast<int64_t>((p.N + bn - 1) / bn);
  const int split = choose_split(tiles, p.K, per_sm, 128);
  // deepest ring that fits the per-CTA share of shared memory
  const size_t budget = (227 * 1024) / per_sm - 2048;
  int stages = 2;
  for (int s : {3, 4, 6})
    if (static_cast<size_t>(bm + bn) * 128 * s <= budget) stages = s;
  c = {HML_ALGO_SIMT, bm, bn, split, stages, var};
  return c;
}

hml_status select_config(const GemmProblem &p, hml_sgemm_config *c, cudaStream_t s) {
  if (tuned_lookup(p, c) && check_config_ok(p, *c)) return HML_STATUS_SUCCESS;
  if (predictor_lookup(p, c, s) && check_config_ok(p, *c)) return HML_STATUS_SUCCESS;
  // Measured on B200 (M = 65536, K = 4096): FP32 SIMT wins at N <= 16 (the
  // HBM-bound GEMV-like shapes); the split-BF16 tensor-core forms win from
  // N = 32 on.  BF16X6 keeps FP32-level accuracy; BF16X3 (faster, ~2**-17)
  // only in the fast math mode.
  if (p.N > 16 && p.M >= 1024 && p.K >= 64) {
    const int algo = math_mode() == HML_MATH_FAST ? HML_ALGO_BF16X3 : HML_ALGO_BF16X6;
    const hml_sgemm_config tc = heuristic_config(p, algo);
    if (check_config_ok(p, tc)) {
      *c = tc;
      return HML_STATUS_SUCCESS;
    }
  }
  *c = heuristic_config(p, HML_ALGO_SIMT);
  return HML_STATUS_SUCCESS;
}

}  // namespace hml
