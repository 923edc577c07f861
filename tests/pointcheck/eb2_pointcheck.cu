// eb2_pointcheck.cu -- CPU access to the per-interface routines of both
// stage kernels, for tests that compare the mixed-precision face arithmetic
// with the FP64 face arithmetic without a GPU.  Host code only: the routines
// are the same host+device templates the kernels instantiate, fed from arrays
// laid out with the kernels' shared-memory strides.
#include "eb2_stage_fp64.cuh"
#include "eb2_stage_mixed.cuh"

using namespace eb2;

namespace {

template <int DIR, int RECON, bool CH, bool WZ, int FLUX>
unsigned fp64_face(const double* cells, double delta, const Gas& g, int pos, double* F) {
    static double sU[4 * fp64stage::FS], sP[5 * fp64stage::PS];
    for (int n = 0; n < 6; n++)
        for (int k = 0; k < 4; k++) sU[k * fp64stage::FS + n] = cells[4 * n + k];
    double w[5];
    for (int c = 0; c < 2; c++) {
        const double* q = cells + 4 * (2 + c);
        x64::primitive5(q[0], q[1], q[2], q[3], g, w);
        for (int k = 0; k < 5; k++) sP[k * fp64stage::PS + c] = w[k];
    }
    return fp64stage::interface_flux<false, DIR, RECON, CH, WZ, FLUX>(sU, 1, sP, sP + 1, delta, g, pos,
                                                               F, 1);
}

template <int DIR, bool WZ, int FLUX>
unsigned mixed_face(const double* cells, double pthr, const Gas& g, int pos, double* F) {
    float4 sU[6];
    for (int n = 0; n < 6; n++)
        sU[n] = make_float4((float)cells[4 * n], (float)cells[4 * n + 1], (float)cells[4 * n + 2],
                            (float)cells[4 * n + 3]);
    // the six cells in FP64 as the kernel's near-vacuum path reads them from
    // the stage input: field planes of 6 values, cell i at index 2
    double u[24];
    for (int n = 0; n < 6; n++)
        for (int k = 0; k < 4; k++) u[n + 6 * k] = cells[4 * n + k];
    float4 P[2];
    float2 H[2];
    for (int c = 0; c < 2; c++) {
        float qf[4];
        for (int k = 0; k < 4; k++) qf[k] = (float)cells[4 * (2 + c) + k];
        f32::cell_prims(cells + 4 * (2 + c), qf, g, P + c, H + c);
    }
    float4 Ff;
    unsigned st = mixstage::interface_flux<DIR, WZ, FLUX>(sU, 1, P, H, P + 1, H + 1, u, 2, 3, 6,
                                                          (float)pthr, g, pos, &Ff);
    F[0] = Ff.x;
    F[1] = Ff.y;
    F[2] = Ff.z;
    F[3] = Ff.w;
    return st;
}

template <int DIR, int RECON, bool CH, bool WZ>
unsigned fp64_by_flux(int flux, const double* c, double d, const Gas& g, int pos, double* F) {
    switch (flux) {
        case FLUX_HLL: return fp64_face<DIR, RECON, CH, WZ, FLUX_HLL>(c, d, g, pos, F);
        case FLUX_HLLC: return fp64_face<DIR, RECON, CH, WZ, FLUX_HLLC>(c, d, g, pos, F);
        case FLUX_ROE: return fp64_face<DIR, RECON, CH, WZ, FLUX_ROE>(c, d, g, pos, F);
        case FLUX_HLLHC: return fp64_face<DIR, RECON, CH, WZ, FLUX_HLLHC>(c, d, g, pos, F);
        case FLUX_HLLCHC: return fp64_face<DIR, RECON, CH, WZ, FLUX_HLLCHC>(c, d, g, pos, F);
        case FLUX_ROEHC: return fp64_face<DIR, RECON, CH, WZ, FLUX_ROEHC>(c, d, g, pos, F);
        default: return fp64_face<DIR, RECON, CH, WZ, FLUX_LLF>(c, d, g, pos, F);
    }
}

template <int DIR, bool WZ>
unsigned mixed_by_flux(int flux, const double* c, double pthr, const Gas& g, int pos, double* F) {
    switch (flux) {
        case FLUX_HLL: return mixed_face<DIR, WZ, FLUX_HLL>(c, pthr, g, pos, F);
        case FLUX_HLLC: return mixed_face<DIR, WZ, FLUX_HLLC>(c, pthr, g, pos, F);
        case FLUX_ROE: return mixed_face<DIR, WZ, FLUX_ROE>(c, pthr, g, pos, F);
        case FLUX_HLLHC: return mixed_face<DIR, WZ, FLUX_HLLHC>(c, pthr, g, pos, F);
        case FLUX_HLLCHC: return mixed_face<DIR, WZ, FLUX_HLLCHC>(c, pthr, g, pos, F);
        case FLUX_ROEHC: return mixed_face<DIR, WZ, FLUX_ROEHC>(c, pthr, g, pos, F);
        default: return mixed_face<DIR, WZ, FLUX_LLF>(c, pthr, g, pos, F);
    }
}

Gas gas_of(double gamma) { return Gas{gamma, gamma - 1.0, gamma / (gamma - 1.0)}; }

}  // namespace

// cells: 6 conserved states (rho, rho u, rho v, rho E) of cells i-2..i+3 along
// the sweep; F: the flux at face i+1/2.  Characteristic WENO5 only.
extern "C" unsigned pc_face_fp64(int dir, int weno_z, int flux, double gamma, const double* cells,
                                 double delta, int positivity, double* F) {
    Gas g = gas_of(gamma);
    if (dir == 1)
        return weno_z ? fp64_by_flux<1, 5, true, true>(flux, cells, delta, g, positivity, F)
                      : fp64_by_flux<1, 5, true, false>(flux, cells, delta, g, positivity, F);
    return weno_z ? fp64_by_flux<2, 5, true, true>(flux, cells, delta, g, positivity, F)
                  : fp64_by_flux<2, 5, true, false>(flux, cells, delta, g, positivity, F);
}

extern "C" unsigned pc_face_mixed(int dir, int weno_z, int flux, double gamma,
                                  const double* cells, double pthr, int positivity, double* F) {
    Gas g = gas_of(gamma);
    if (dir == 1)
        return weno_z ? mixed_by_flux<1, true>(flux, cells, pthr, g, positivity, F)
                      : mixed_by_flux<1, false>(flux, cells, pthr, g, positivity, F);
    return weno_z ? mixed_by_flux<2, true>(flux, cells, pthr, g, positivity, F)
                  : mixed_by_flux<2, false>(flux, cells, pthr, g, positivity, F);
}
