/* CFD_convection.h -- drop-in for the reference's include/CFD_convection.h:
 * the interface fluxes of the state in both directions, on the GPU. */
#ifndef CFD_CONVECTION_H
#define CFD_CONVECTION_H

#include "rpf_glue.h"
#include "Reconstruction.h"
#include "scheme.h"
#include "function.h"

/* Flux_Reconstruction_RP (include/CFD_convection.h:38-200): reconstruction of
 * Recon_Accur (characteristic per Characteriz) and Riemann solver AR_scheme
 * (1 HLL, 2 HLLC, 3 Roe, 11/22/33 the heat-conduction variants, anything
 * else LLF) along x into f and along y into g. */
static inline void Flux_Reconstruction_RP(int AR_scheme, int var_, int rows, int cols, int GC,
                                          double (*y)[rows][cols], double (*f)[rows][cols],
                                          double (*g)[rows][cols], double dt, double dx,
                                          double dy) {
    rpf_globals gl = rpf_collect();
    (void)var_;
    (void)GC;
    (void)dt;
    rpf_check(rpf_flux_reconstruction(AR_scheme, rows, cols, &y[0][0][0], &f[0][0][0],
                                      &g[0][0][0], dx, dy, &gl),
              "Flux_Reconstruction_RP");
}

#endif
