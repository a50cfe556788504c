// tune.cu -- measured configuration table (filled by the autotuner).
#include "hml_tune.h"

namespace hml {
bool tuned_lookup(const GemmProblem &, hml_sgemm_config *) { return false; }
bool predictor_lookup(const GemmProblem &, hml_sgemm_config *) { return false; }
hml_status tune_load(const char *, int *) { return HML_STATUS_NOT_SUPPORTED; }
}  // namespace hml
