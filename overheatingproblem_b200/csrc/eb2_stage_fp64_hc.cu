// Heat-conduction flux instantiations of the FP64 fused stage (AR_scheme
// 11/22/33: HLLHC, HLLCHC, RoeHC, include/scheme.h:1860-3109 of the reference)
// for every reconstruction.  Built with -fmad=false: see eb2_point_fp64.cuh.
#include "eb2_stage_fp64.cuh"

namespace eb2 {
namespace {
template <int RECON, bool CHAR, bool WZ>
cudaError_t hc(const StageArgs& a, cudaStream_t s) {
    switch (a.num.flux) {
        case FLUX_HLLHC: return fp64stage::launch_one<RECON, CHAR, WZ, FLUX_HLLHC>(a, s);
        case FLUX_HLLCHC: return fp64stage::launch_one<RECON, CHAR, WZ, FLUX_HLLCHC>(a, s);
        case FLUX_ROEHC: return fp64stage::launch_one<RECON, CHAR, WZ, FLUX_ROEHC>(a, s);
        default: return cudaErrorInvalidValue;
    }
}
}  // namespace

cudaError_t launch_stage_fp64_hc(const StageArgs& a, cudaStream_t s) {
    const bool ch = a.num.characteristic;
    switch (a.num.recon) {
        case 5:
            if (!ch) return hc<5, false, false>(a, s);
            return a.num.weno_z ? hc<5, true, true>(a, s) : hc<5, true, false>(a, s);
        case 3: return ch ? hc<3, true, false>(a, s) : hc<3, false, false>(a, s);
        case 2: return ch ? hc<2, true, false>(a, s) : hc<2, false, false>(a, s);
        case 1: return ch ? hc<1, true, false>(a, s) : hc<1, false, false>(a, s);
        default: return cudaErrorInvalidValue;
    }
}
}  // namespace eb2
