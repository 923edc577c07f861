// TVD instantiations of the FP64 fused stage: component minmod and
// characteristic van Leer (include/Reconstruction.h:314-315, 418-419 of the
// reference).  Built with -fmad=false: see eb2_point_fp64.cuh.
#include "eb2_stage_fp64.cuh"

namespace eb2 {
cudaError_t launch_stage_fp64_tvd(const StageArgs& a, cudaStream_t s) {
    if (a.num.characteristic) return fp64stage::launch_flux<2, true, false>(a, s);
    return fp64stage::launch_flux<2, false, false>(a, s);
}
}  // namespace eb2
