// WENO5 instantiations of the FP64 fused stage (component WENO5-JS, and
// characteristic WENO5 with Jiang-Shu or WENO-Z weights).  Built with
// -fmad=false: see eb2_point_fp64.cuh.
#include "eb2_stage_fp64.cuh"

namespace eb2 {
cudaError_t launch_stage_fp64_w5(const StageArgs& a, cudaStream_t s) {
    if (!a.num.characteristic) return fp64stage::launch_flux<5, false, false>(a, s);
    if (a.num.weno_z) return fp64stage::launch_flux<5, true, true>(a, s);
    return fp64stage::launch_flux<5, true, false>(a, s);
}
}  // namespace eb2
