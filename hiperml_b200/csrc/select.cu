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
int simt_ctas_per_sm(int v);
int tc_num_shapes();
void tc_shape(int v, int *bm, int *bn);
bool tc_config_fits(int bn, int ns, int stages);
int tc_ns(int algo);
bool cfg_v1_sgemm_rule(int K, int N, int *type, int *row_stops);

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
  if (algo == HML_ALGO_BF16X3 || algo == HML_ALGO_BF16X6 || algo == HML_ALGO_TF32X3 ||
      algo == HML_ALGO_FP16X3) {
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
  // SIMT, measured on B200 (M = 1024 to 65536, K = 4096, and squares to
  // 8192): 128-row tiles 8, 16, 32 and 64 wide up to those N, except 256 x 64
  // tiles of 4-row micro-tiles from N = 33 once M gives them 64 row tiles
  // (16384 x 64: 208 us against 228); above N = 64 those 256 x 64 tiles (52
  // TFLOP/s at N = 128) unless 32-wide tiles, at about 42 TFLOP/s, leave
  // enough fewer columns idle (N = 96: 1.27 ms against 1.31)
  int var;
  if (p.N <= 8) var = 1;
  else if (p.N <= 16) var = 0;
  else if (p.N <= 32) var = 2;
  else if (p.N <= 64) var = p.M >= 64 * 256 ? 6 : 7;
  else {
    const int64_t cols32 = (p.N + 31) / 32 * 32, cols64 = (p.N + 63) / 64 * 64;
    var = cols32 * 52 < cols64 * 42 ? 2 : 6;
  }
  return simt_config(p, var);
}

// The tiled SIMT configuration of micro-tile shape `var` for this problem.
// split_k so the grid covers every CTA slot of the machine, at most 8 (4096
// x 32 x 4096: 41 us against 68 at 16), and 2 for tiles
// of two CTAs an SM where the grid is under two waves and K is long (65536
// x 128 x 4096 on 256 x 64 tiles: 1.31 ms; one CTA an SM measured slower
// split); a 3-deep ring where both CTAs of an SM fit with it, else 2
// (deeper rings measured no faster and cost the second CTA).
hml_sgemm_config simt_config(const GemmProblem &p, int var) {
  int bm, bn, wk;
  simt_shape(var, &bm, &bn, &wk);
  const int per_sm = simt_ctas_per_sm(var);
  const int64_t tiles = ((p.M + bm - 1) / bm) * static_cast<int64_t>((p.N + bn - 1) / bn);
  int split = std::min(choose_split(tiles, p.K, per_sm, 128), 8);
  if (split == 1 && per_sm == 2 && tiles < 2LL * sm_count() * per_sm && p.K >= 2048) split = 2;
  // the per-CTA share of shared memory, less barriers and alignment slack
  const size_t budget = (227 * 1024) / per_sm - 2048;
  const int stages = static_cast<size_t>(bm + bn) * 128 * 3 <= budget ? 3 : 2;
  return hml_sgemm_config{HML_ALGO_SIMT, bm, bn, split, stages, var};
}

// A reference v1 SGEMM rule (src/hml_sgemm_kernel.cu:189-237: kernel type
// and rowStops for the class K' = min(K, 96), colStops = ceil(min(N, 96) /
// 16) of a row-major M x N x K problem) mapped onto the tiled SIMT family,
// the counterpart of the reference's tiled SIMT kernels: a tile of
// 16 * rowStops rows (basic kernel: 6 x 6 stops) becomes the 128- or
// 256-row SIMT tile nearest to it, its 16 * colStops columns the narrowest
// SIMT tile width that holds min(N, 16 * colStops) of the problem's columns.
// False when no rule applies or the mapped configuration cannot run.
bool v1_rule_config(const GemmProblem &p, int K_row, int N_row, hml_sgemm_config *c) {
  int type = 0, row_stops = 0;
  if (!cfg_v1_sgemm_rule(K_row, N_row, &type, &row_stops)) return false;
  const int col_stops = type == 0 ? 6 : (std::min(N_row, 96) + 15) / 16;
  const int rows = 16 * (type == 0 ? 6 : row_stops);
  const int want_m = rows >= 192 ? 256 : 128;
  const int want_n = std::min(p.N, 16 * col_stops);
  int best = -1, best_bn = 0, widest = -1, widest_bn = 0;
  for (int v = 0; v < simt_num_shapes(); ++v) {
    int bm, bn, wk;
    simt_shape(v, &bm, &bn, &wk);
    if (bm != want_m) continue;
    if (bn >= want_n && (best < 0 || bn < best_bn)) {
      best = v;
      best_bn = bn;
    }
    if (bn > widest_bn) {
      widest = v;
      widest_bn = bn;
    }
  }
  if (best < 0) best = widest;
  if (best < 0) return false;
  const hml_sgemm_config cand = simt_config(p, best);
  if (!check_config_ok(p, cand)) return false;
  *c = cand;
  return true;
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
