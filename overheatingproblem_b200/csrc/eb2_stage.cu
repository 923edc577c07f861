// eb2_stage.cu -- dispatch of the fused stage kernels by reconstruction.
#include "eb2_kernels.h"

namespace eb2 {

cudaError_t launch_stage_fp64_w5(const StageArgs& a, cudaStream_t s);
cudaError_t launch_stage_fp64_tvd(const StageArgs& a, cudaStream_t s);
cudaError_t launch_stage_fp64_g1(const StageArgs& a, cudaStream_t s);
cudaError_t launch_stage_fp64_w3(const StageArgs& a, cudaStream_t s);
cudaError_t launch_stage_fp64_hc(const StageArgs& a, cudaStream_t s);

cudaError_t launch_stage_fp64(const StageArgs& a, cudaStream_t s) {
    if (a.num.flux >= FLUX_HLLHC) return launch_stage_fp64_hc(a, s);
    switch (a.num.recon) {
        case 5: return launch_stage_fp64_w5(a, s);
        case 3: return launch_stage_fp64_w3(a, s);
        case 2: return launch_stage_fp64_tvd(a, s);
        case 1: return launch_stage_fp64_g1(a, s);
        default: return cudaErrorInvalidValue;
    }
}

int stage_blocks(const Grid& g, bool mixed) {
    const int tx = mixed ? MIXED_PARTIAL_ROWS : FP64_TILE_X;
    return ((g.ny + STAGE_TILE_Y - 1) / STAGE_TILE_Y) * ((g.nx + tx - 1) / tx);
}

int stage_blocks_max(const Grid& g) {
    const int a = stage_blocks(g, false), b = stage_blocks(g, true);
    return a > b ? a : b;
}

}  // namespace eb2
