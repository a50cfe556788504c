// hml_select.h -- configuration selection for hml_sgemm_ex: the measured
// table (autotuner), then the learned predictor, then a heuristic.
#pragma once
#include <vector>

#include "hml_internal.h"

namespace hml {
hml_status select_config(const GemmProblem &p, hml_sgemm_config *c, cudaStream_t s = nullptr);
hml_sgemm_config heuristic_config(const GemmProblem &p, int algo);
hml_sgemm_config simt_config(const GemmProblem &p, int var);
// A loaded reference v1 SGEMM rule for the row-major K x N class, mapped onto
// the SIMT family (false when none applies).
bool v1_rule_config(const GemmProblem &p, int K_row, int N_row, hml_sgemm_config *c);
const std::vector<hml_sgemm_config> &config_space();
// auto_choice: the configuration came from select_config, so the launch may
// add the tail-wave split of launch_tc.
hml_status run_config(const GemmProblem &p, const hml_sgemm_config &c, cudaStream_t s,
                      bool auto_choice = false);
}  // namespace hml
