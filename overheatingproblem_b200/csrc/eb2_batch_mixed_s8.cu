// eb2_batch_mixed_s8.cu -- the batched mixed stage kernels in the
// 8 x 32-cell, 128-thread tile shape (a candidate of the server's autotuner).
#include "eb2_batch_mixed.cuh"

namespace eb2 {

cudaError_t launch_stage_batch_mixed_s8(const BatchLaunch& b, const Numerics& num, int stage,
                                        cudaStream_t s) {
    return batchmixed::launch<mixstage::Shape8>(b, num, stage, s);
}

cudaError_t launch_stage_slot_mixed_s8(const StageArgs& a, const Numerics& num,
                                       cudaStream_t s) {
    return batchmixed::launch_slot<mixstage::Shape8>(a, num, s);
}

}  // namespace eb2
