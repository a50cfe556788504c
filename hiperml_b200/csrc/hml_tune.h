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
// The predictor runs its inference kernel on a private stream the first
// time it sees a shape class; `s` is the caller's stream, checked so that a
// stream under capture is not made to wait.
bool predictor_lookup(const GemmProblem &p, hml_sgemm_config *c, cudaStream_t s);
int math_mode();
// The GEMV variant the measured table holds for this problem (its shape or
// a neighbour within about a factor 2 with the same layout); false when none.
bool gemv_tuned_lookup(const GemvProblem &p, int *variant);
}  // namespace hml
