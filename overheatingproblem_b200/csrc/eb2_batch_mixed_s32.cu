// eb2_batch_mixed_s32.cu -- the batched mixed stage kernels in the
// 32 x 32-cell, 512-thread tile shape (a candidate of the server's autotuner).
#include "eb2_batch_mixed.cuh"

namespace eb2 {

cudaError_t launch_stage_batch_mixed_s32(const BatchLaunch& b, const Numerics& num, int stage,
                                        cudaStream_t s) {
    return batchmixed::launch<mixstage::Shape32>(b, num, stage, s);
}

cudaError_t launch_stage_slot_mixed_s32(const StageArgs& a, const Numerics& num,
                                       cudaStream_t s) {
    return batchmixed::launch_slot<mixstage::Shape32>(a, num, s);
}

}  // namespace eb2
