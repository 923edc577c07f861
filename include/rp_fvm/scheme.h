/* scheme.h -- drop-in for the reference's include/scheme.h: the Riemann
 * fluxes at the interfaces of given left/right states, and the flux
 * difference, on the GPU. */
#ifndef SCHEME_H
#define SCHEME_H

#include "rpf_glue.h"
#include "Characteriz.h"
#include "function.h"

static inline void rpf_flux_call(int scheme, int dir, int rows, int cols, double *ql,
                                 double *qr, double *flux, const char *who) {
    rpf_globals g = rpf_collect();
    rpf_check(rpf_riemann(scheme, dir, rows, cols, ql, qr, flux, &g), who);
}

/* LLF_Flux (include/scheme.h:229-386), AR_scheme's default. */
static inline void LLF_Flux(int dir, int var_, int rows, int cols, int GC,
                            double (*L_state)[rows][cols], double (*R_state)[rows][cols],
                            double (*Flux)[rows][cols]) {
    (void)var_;
    (void)GC;
    rpf_flux_call(0, dir, rows, cols, &L_state[0][0][0], &R_state[0][0][0], &Flux[0][0][0],
                  "LLF_Flux");
}

/* HLL_Flux (include/scheme.h:400-674); interfaces the reference skips
 * (non-physical states) keep their previous Flux entries. */
static inline void HLL_Flux(int dir, int var_, int rows, int cols, int GC,
                            double (*L_state)[rows][cols], double (*R_state)[rows][cols],
                            double (*Flux)[rows][cols]) {
    (void)var_;
    (void)GC;
    rpf_flux_call(1, dir, rows, cols, &L_state[0][0][0], &R_state[0][0][0], &Flux[0][0][0],
                  "HLL_Flux");
}

/* HLLC_Flux (include/scheme.h:690-1001). */
static inline void HLLC_Flux(int dir, int var_, int rows, int cols, int GC,
                             double (*L_state)[rows][cols], double (*R_state)[rows][cols],
                             double (*Flux)[rows][cols]) {
    (void)var_;
    (void)GC;
    rpf_flux_call(2, dir, rows, cols, &L_state[0][0][0], &R_state[0][0][0], &Flux[0][0][0],
                  "HLLC_Flux");
}

/* Roe_Flux (include/scheme.h:1018-1322). */
static inline void Roe_Flux(int dir, int var_, int rows, int cols, int GC,
                            double (*L_state)[rows][cols], double (*R_state)[rows][cols],
                            double (*flux)[rows][cols]) {
    (void)var_;
    (void)GC;
    rpf_flux_call(3, dir, rows, cols, &L_state[0][0][0], &R_state[0][0][0], &flux[0][0][0],
                  "Roe_Flux");
}

/* Space_Discrete_Item (include/scheme.h:3758-3777): the residual
 * -(f_i - f_{i-1})/dx - (g_j - g_{j-1})/dy + s on the interior. */
static inline void Space_Discrete_Item(int var_, int rows, int cols, int GC, double delta_x,
                                       double delta_y, double (*f)[rows][cols],
                                       double (*g)[rows][cols], double (*s)[rows][cols],
                                       double (*resid)[rows][cols]) {
    rpf_globals gl = rpf_collect();
    (void)var_;
    (void)GC;
    rpf_check(rpf_space_discrete(rows, cols, delta_x, delta_y, &f[0][0][0], &g[0][0][0],
                                 &s[0][0][0], &resid[0][0][0], &gl),
              "Space_Discrete_Item");
}

#endif
