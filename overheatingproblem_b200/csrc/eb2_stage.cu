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

// Upper bound of the block count of any stage kernel (partials buffer size):
// both forms tile the interior with at least 16 x 32 cells per block.
int stage_blocks(const Grid& g) { return ((g.ny + 31) / 32) * ((g.nx + 15) / 16); }

}  // namespace eb2
