// eb2_batch_mixed.cu -- the batched mixed stage kernels in the default tile
// shape (16 x 32 cells, 256 threads), and the dispatch over the shapes the
// server's autotuner chooses from.
#include "eb2_batch_mixed.cuh"

namespace eb2 {

cudaError_t launch_stage_batch_mixed_s8(const BatchLaunch& b, const Numerics& num, int stage,
                                        cudaStream_t s);
cudaError_t launch_stage_batch_mixed_s32(const BatchLaunch& b, const Numerics& num, int stage,
                                         cudaStream_t s);

cudaError_t launch_stage_slot_mixed_s8(const StageArgs& a, const Numerics& num,
                                       cudaStream_t s);
cudaError_t launch_stage_slot_mixed_s32(const StageArgs& a, const Numerics& num,
                                        cudaStream_t s);

cudaError_t launch_stage_slot_mixed(const StageArgs& a, const Numerics& num, int shape,
                                    cudaStream_t s) {
    switch (shape) {
        case 0: return batchmixed::launch_slot<mixstage::Shape16>(a, num, s);
        case 1: return launch_stage_slot_mixed_s8(a, num, s);
        case 2: return launch_stage_slot_mixed_s32(a, num, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_stage_batch_mixed(const BatchLaunch& b, const Numerics& num, int stage,
                                     cudaStream_t s) {
    switch (b.shape) {
        case 0: return batchmixed::launch<mixstage::Shape16>(b, num, stage, s);
        case 1: return launch_stage_batch_mixed_s8(b, num, stage, s);
        case 2: return launch_stage_batch_mixed_s32(b, num, stage, s);
        default: return cudaErrorInvalidValue;
    }
}

// Tile rows, threads and resident CTAs per SM of each batched shape (index 0
// is the FP64 form's tile for an FP64 server).
int batch_shape_tile_x(int precision, int shape) {
    if (precision == 0) return FP64_TILE_X;
    return shape == 1 ? mixstage::Shape8::TX : shape == 2 ? mixstage::Shape32::TX
                                                           : mixstage::Shape16::TX;
}

int stage_batch_max_blocks_per_sm(int precision, int shape) {
    if (precision == 0) return 2;
    return shape == 1 ? mixstage::Shape8::CTAS : shape == 2 ? mixstage::Shape32::CTAS
                                                             : mixstage::Shape16::CTAS;
}

int batch_shapes(int precision) { return precision == 0 ? 1 : kMixedShapes; }

}  // namespace eb2
