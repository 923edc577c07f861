// WENO3 instantiations of the FP64 fused stage, component and characteristic
// (WENO3_Reconstruction, include/Reconstruction.h:684-870 of the reference).
// Built with -fmad=false: see eb2_point_fp64.cuh.
#include "eb2_stage_fp64.cuh"

namespace eb2 {
cudaError_t launch_stage_fp64_w3(const StageArgs& a, cudaStream_t s) {
    if (a.num.characteristic) return fp64stage::launch_flux<3, true, false>(a, s);
    return fp64stage::launch_flux<3, false, false>(a, s);
}
}  // namespace eb2
