// eb2_stage_mixed.cu -- mixed-precision fused stage (placeholder until the
// FP32 reconstruction kernel lands).
#include "eb2_kernels.h"

namespace eb2 {
cudaError_t launch_stage_mixed(const StageArgs& a, cudaStream_t s) {
    (void)a;
    (void)s;
    return cudaErrorNotSupported;
}
}  // namespace eb2
