// predictor.cu -- the learned configuration predictor (placeholder).
#include "hml_tune.h"

namespace hml {
bool predictor_lookup(const GemmProblem &, hml_sgemm_config *) { return false; }
}  // namespace hml
