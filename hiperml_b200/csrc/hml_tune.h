// hml_tune.h -- the autotuner's measured table and the learned predictor, as
// seen by configuration selection.
#pragma once
#include "hml_internal.h"

namespace hml {
hml_status check_config(const GemmProblem &p, const hml_sgemm_config &c);
bool check_config_ok(const GemmProblem &p, const hml_sgemm_config &c);
// Fill *c from the measured table / the predictor; false when neither holds
// an answer for this problem.
bool tuned_lookup(const GemmProblem &p, hml_sgemm_config *c);
bool predictor_lookup(const GemmProblem &p, hml_sgemm_config *c);
int math_mode();
}  // namespace hml
