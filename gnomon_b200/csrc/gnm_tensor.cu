// gnm_tensor.cu — placeholder until the tcgen05 engine lands.
#include "gnm_plan.h"
#include "gnm_tensor.h"

namespace gnm {
void tensor_plan_create(gnm_plan*) { fail(GNM_ERR_COMPUTE, "tensor engine not built"); }
void tensor_plan_destroy(gnm_plan*) {}
void tensor_reset(gnm_plan*, cudaStream_t) {}
void tensor_accumulate(gnm_plan*, const uint8_t*, uint64_t, uint64_t, uint64_t, cudaStream_t) {}
void tensor_finalize(gnm_plan*, double*, uint32_t*, bool, cudaStream_t) {}
void backward_dw(gnm_plan*, const uint8_t*, uint64_t, const float*, float*, float*, cudaStream_t) {
  fail(GNM_ERR_COMPUTE, "backward not built");
}
}  // namespace gnm
