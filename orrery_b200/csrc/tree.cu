// Barnes-Hut pipeline (under construction).
#include "tree.hpp"

namespace ob {

TreePipeline::TreePipeline(const ob_solver_params &params) : params_(params) {}
TreePipeline::~TreePipeline() = default;

void TreePipeline::evaluate(uint32_t, const double *, const double *, const double *,
                            const double *, double *, double *, double *, unsigned *,
                            cudaEvent_t, cudaEvent_t, bool, cudaStream_t) {
    throw Error(OB_ERROR_UNSUPPORTED, "the tree solver is not built yet");
}

ob_counts TreePipeline::device_counts() { return ob_counts{}; }
void TreePipeline::reset_counts() {}

} // namespace ob
