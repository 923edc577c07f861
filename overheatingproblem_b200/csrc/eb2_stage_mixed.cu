// eb2_stage_mixed.cu -- instantiations and dispatch of the mixed-precision
// fused stage (characteristic WENO5 with Jiang-Shu or WENO-Z weights x four
// Riemann solvers).  Built with FMA contraction on.
#include "eb2_stage_mixed.cuh"

namespace eb2 {

template <bool WZ>
static cudaError_t by_flux(const StageArgs& a, cudaStream_t s) {
    switch (a.num.flux) {
        case FLUX_HLL: return mixstage::launch_one<WZ, FLUX_HLL>(a, s);
        case FLUX_HLLC: return mixstage::launch_one<WZ, FLUX_HLLC>(a, s);
        case FLUX_ROE: return mixstage::launch_one<WZ, FLUX_ROE>(a, s);
        case FLUX_LLF: return mixstage::launch_one<WZ, FLUX_LLF>(a, s);
        case FLUX_HLLHC: return mixstage::launch_one<WZ, FLUX_HLLHC>(a, s);
        case FLUX_HLLCHC: return mixstage::launch_one<WZ, FLUX_HLLCHC>(a, s);
        case FLUX_ROEHC: return mixstage::launch_one<WZ, FLUX_ROEHC>(a, s);
        default: return cudaErrorNotSupported;
    }
}

// Tile rows of the single-solve mixed stage (its partials hold one triple per
// tile).

cudaError_t launch_stage_mixed(const StageArgs& a, cudaStream_t s) {
    // the mixed form implements the characteristic WENO5 reconstruction only
    if (a.num.recon != 5 || !a.num.characteristic) return cudaErrorNotSupported;
    return a.num.weno_z ? by_flux<true>(a, s) : by_flux<false>(a, s);
}

}  // namespace eb2
