// hml_select.h -- configuration selection for hml_sgemm_ex: the measured
// table (autotuner), then the learned predictor, then a heuristic.
#pragma once
#include <vector>

#include "hml_internal.h"

namespace hml {
hml_status select_config(const GemmProblem &p, hml_sgemm_config *c, cudaStream_t s = nullptr);
hml_sgemm_config heuristic_config(const GemmProblem &p, int algo);
const std::vector<hml_sgemm_config> &config_space();
hml_status run_config(const GemmProblem &p, const hml_sgemm_config &c, cudaStream_t s);
}  // namespace hml
