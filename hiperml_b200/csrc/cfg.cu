// cfg.cu -- the reference's v1 tuning-file grammar.
//
// SGEMM v1 (src/hml_sgemm_kernel.cu:18-36, reader :573-602):
//     "K colStops : kernelType rowStops", K 2..96, colStops 1..6 in the
//     shipped files, kernelType {0 basic, 1 var-K, 2 const-K}.
// SGEMV v1 (src/hml_sgemv_kernel.cu:19-37, reader :650-679):
//     "N : kernelType blockStops rowStops", N 0..1024 (row 0 serves N>1024).
// Lines starting with '#' are comments; the last duplicate rule wins.  Unlike
// the reference reader, every field is range-checked against the table
// bounds (cHmlMaxSkinnyK = 96, cHmlMaxStops = 16, cHmlMaxSkinnyN = 1024,
// cHmlMaxBlockStops = 16) and a malformed or out-of-range line rejects the
// whole file with HML_STATUS_CONFIG_ERROR instead of writing out of bounds.
//
// The rules name Fermi/Kepler kernels that do not exist here.  They steer
// the reference-facing host calls, as in the reference: hmlSgemm runs a
// problem a rule covers on the tiled SIMT kernel with the tile nearest to the
// rule's (16*rowStops rows, 16*colStops columns; select.cu v1_rule_config),
// hmlSgemv on the row kernel with 16*blockStops threads per row.  The
// device-pointer ABI (hml_sgemm_ex, hml_sgemv_ex) ignores them and keeps the
// measured B200 table.
//
// cfg_v1_save writes the loaded rules back in the same grammar and in the
// order of the reference's printers (src/hml_sgemm_kernel.cu:557-568,
// src/hml_sgemv_kernel.cu:634-645): SGEMM for K = 2..96 and colStops =
// 1..16, SGEMV for N = 0..1024, each rule whose rowStops is positive.
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "hml_internal.h"

namespace hml {
namespace {

constexpr int kMaxK = 96, kMaxStops = 16, kMaxN = 1024, kMaxBlockStops = 16;

struct SgemmRule {
  int type = -1, row_stops = 0;
};
struct SgemvRule {
  int type = -1, block_stops = 0, row_stops = 0;
};

std::mutex g_mu;
bool g_sgemm_loaded = false, g_sgemv_loaded = false;
SgemmRule g_sgemm[kMaxK + 1][kMaxStops + 1];
SgemvRule g_sgemv[kMaxN + 1];

bool comment_or_blank(const char *s) {
  while (*s == ' ' || *s == '\t' || *s == '\r' || *s == '\n') ++s;
  return *s == '#' || *s == '\0';
}

}  // namespace

hml_status cfg_v1_load(int kind, const char *path, int *rules) {
  if (!path || (kind != 0 && kind != 1)) return HML_STATUS_INVALID_VALUE;
  FILE *f = fopen(path, "rb");
  if (!f) return HML_STATUS_IO_ERROR;
  std::vector<SgemmRule> gm((kMaxK + 1) * (kMaxStops + 1));
  std::vector<SgemvRule> gv(kMaxN + 1);
  char line[1024];
  int n = 0, lineno = 0;
  hml_status st = HML_STATUS_SUCCESS;
  while (fgets(line, sizeof line, f)) {
    ++lineno;
    if (comment_or_blank(line)) continue;
    if (kind == 0) {
      int K, cs, type, rs;
      char tail;
      if (sscanf(line, "%d %d : %d %d %c", &K, &cs, &type, &rs, &tail) != 4 || K < 0 ||
          K > kMaxK || cs < 0 || cs > kMaxStops || type < 0 || type > 2 || rs < 0 ||
          rs > kMaxStops) {
        fprintf(stderr, "hml: %s:%d: bad SGEMM v1 rule: %s", path, lineno, line);
        st = HML_STATUS_CONFIG_ERROR;
        break;
      }
      gm[K * (kMaxStops + 1) + cs] = {type, rs};
    } else {
      int N, type, bs, rs;
      char tail;
      if (sscanf(line, "%d : %d %d %d %c", &N, &type, &bs, &rs, &tail) != 4 || N < 0 ||
          N > kMaxN || type < 0 || type > 2 || bs < 0 || bs > kMaxBlockStops || rs < 0 ||
          rs > kMaxStops) {
        fprintf(stderr, "hml: %s:%d: bad SGEMV v1 rule: %s", path, lineno, line);
        st = HML_STATUS_CONFIG_ERROR;
        break;
      }
      gv[N] = {type, bs, rs};
    }
    ++n;
  }
  fclose(f);
  if (st != HML_STATUS_SUCCESS) return st;
  std::lock_guard<std::mutex> lk(g_mu);
  if (kind == 0) {
    for (int K = 0; K <= kMaxK; ++K)
      for (int c = 0; c <= kMaxStops; ++c) g_sgemm[K][c] = gm[K * (kMaxStops + 1) + c];
    g_sgemm_loaded = true;
  } else {
    for (int N = 0; N <= kMaxN; ++N) g_sgemv[N] = gv[N];
    g_sgemv_loaded = true;
  }
  if (rules) *rules = n;
  if (kind == 0)
    fprintf(stderr,
            "hml: %d SGEMM v1 rules from %s: hmlSgemm maps them onto FP32 SIMT tiles; "
            "hml_sgemm_ex keeps the measured B200 table\n",
            n, path);
  return HML_STATUS_SUCCESS;
}

hml_status cfg_v1_save(int kind, const char *path) {
  if (!path || (kind != 0 && kind != 1)) return HML_STATUS_INVALID_VALUE;
  std::vector<SgemmRule> gm;
  std::vector<SgemvRule> gv;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (kind == 0 ? !g_sgemm_loaded : !g_sgemv_loaded) return HML_STATUS_CONFIG_ERROR;
    if (kind == 0) {
      for (int K = 0; K <= kMaxK; ++K)
        for (int c = 0; c <= kMaxStops; ++c) gm.push_back(g_sgemm[K][c]);
    } else {
      gv.assign(g_sgemv, g_sgemv + kMaxN + 1);
    }
  }
  FILE *f = fopen(path, "wb");
  if (!f) return HML_STATUS_IO_ERROR;
  bool ok = true;
  if (kind == 0) {
    ok = fprintf(f,
                 "#SGEMM smart kernel config file v1.0\n"
                 "#written by hml-b200 from the rules it loaded\n"
                 "#rule: K colStops : kernelType rowStops  (kernelType 0 basic, 1 var-K, "
                 "2 const-K; colStops = (N + 15) / 16)\n") > 0;
    for (int K = 2; ok && K <= kMaxK; ++K)
      for (int c = 1; ok && c <= kMaxStops; ++c) {
        const SgemmRule &r = gm[K * (kMaxStops + 1) + c];
        if (r.row_stops > 0) ok = fprintf(f, "%d %d : %d %d\n", K, c, r.type, r.row_stops) > 0;
      }
  } else {
    ok = fprintf(f,
                 "#SGEMV smart kernel config file v1.0\n"
                 "#written by hml-b200 from the rules it loaded\n"
                 "#rule: N : kernelType blockStops rowStops  (N 0 serves N > 1024)\n") > 0;
    for (int N = 0; ok && N <= kMaxN; ++N) {
      const SgemvRule &r = gv[N];
      if (r.row_stops > 0)
        ok = fprintf(f, "%d : %d %d %d\n", N, r.type, r.block_stops, r.row_stops) > 0;
    }
  }
  if (fclose(f) != 0) ok = false;
  return ok ? HML_STATUS_SUCCESS : HML_STATUS_IO_ERROR;
}

// The reference's keying: K' = min(K, 96), colStops = ceil(min(N, 96) / 16)
// (src/hml_sgemm_kernel.cu:198-213).  False when no valid rule applies.
bool cfg_v1_sgemm_rule(int K, int N, int *type, int *row_stops) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_sgemm_loaded) return false;
  const int cs = (std::min(N, 96) + 15) / 16;
  const int k = std::min(K, kMaxK);
  const SgemmRule &r = g_sgemm[k][cs];
  if (r.type < 0 || r.row_stops <= 0) return false;
  *type = r.type;
  *row_stops = r.row_stops;
  return true;
}

// Keying cfg[N <= 1024 ? N : 0] (src/hml_sgemv_kernel.cu:323-332).
bool cfg_v1_sgemv_rule(int N, int *type, int *block_stops, int *row_stops) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_sgemv_loaded) return false;
  const SgemvRule &r = g_sgemv[N <= kMaxN ? N : 0];
  if (r.type < 0 || r.block_stops <= 0 || r.row_stops <= 0) return false;
  *type = r.type;
  *block_stops = r.block_stops;
  *row_stops = r.row_stops;
  return true;
}

void cfg_v1_clear() {
  std::lock_guard<std::mutex> lk(g_mu);
  g_sgemm_loaded = g_sgemv_loaded = false;
}

}  // namespace hml

extern "C" {

hml_status hml_cfg_v1_load(int kind, const char *path, int *rules) {
  return hml::cfg_v1_load(kind, path, rules);
}

hml_status hml_cfg_v1_sgemm_rule(int K, int N, int *type, int *row_stops) {
  if (!type || !row_stops) return HML_STATUS_INVALID_VALUE;
  return hml::cfg_v1_sgemm_rule(K, N, type, row_stops) ? HML_STATUS_SUCCESS
                                                       : HML_STATUS_CONFIG_ERROR;
}

hml_status hml_cfg_v1_sgemv_rule(int N, int *type, int *block_stops, int *row_stops) {
  if (!type || !block_stops || !row_stops) return HML_STATUS_INVALID_VALUE;
  return hml::cfg_v1_sgemv_rule(N, type, block_stops, row_stops) ? HML_STATUS_SUCCESS
                                                                  : HML_STATUS_CONFIG_ERROR;
}

hml_status hml_cfg_v1_save(int kind, const char *path) { return hml::cfg_v1_save(kind, path); }

void hml_cfg_v1_clear(void) { hml::cfg_v1_clear(); }

}  // extern "C"
