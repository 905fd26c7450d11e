// Tensor-core (tcgen05, BF16) coherence Gram. Placeholder until the sm_100a kernel lands.
#include "common.cuh"

namespace mr {
int gram_tc(const float2*, int, int, int, const int32_t*, int64_t, const uint8_t*, int, int, int, float2*, int,
            cudaStream_t) {
  return fail(MR_ERR_UNSUPPORTED, "emperical_co_pc: tensor-core precision not available in this build");
}
}  // namespace mr
