/* time_advance.h -- drop-in for the reference's include/time_advance.h: one
 * SSP Runge-Kutta step of the state on the GPU (boundary fill, fluxes, flux
 * difference and stage combination per stage, all in one device pass). */
#ifndef TIME_ADVANCE_H
#define TIME_ADVANCE_H

#include "rpf_glue.h"
#include "mesh.h"
#include "initialize.h"
#include "CFD_convection.h"

static inline void rpf_rk_call(int order, int AR_scheme, int rows, int cols, double *y,
                               double dt, double dx, double dy, const char *who) {
    rpf_globals g = rpf_collect();
    rpf_check(rpf_rk(order, AR_scheme, rows, cols, y, dt, dx, dy, &g), who);
}

/* RK1_TimeAd (include/time_advance.h:643-708). */
static inline void RK1_TimeAd(int AR_scheme, int var_, int rows, int cols, int GC,
                              double (*y)[rows][cols], double dt, double dx, double dy) {
    (void)var_;
    (void)GC;
    rpf_rk_call(1, AR_scheme, rows, cols, &y[0][0][0], dt, dx, dy, "RK1_TimeAd");
}

/* RK2_TimeAd (include/time_advance.h:711-785). */
static inline void RK2_TimeAd(int AR_scheme, int var_, int rows, int cols, int GC,
                              double (*y)[rows][cols], double dt, double dx, double dy) {
    (void)var_;
    (void)GC;
    rpf_rk_call(2, AR_scheme, rows, cols, &y[0][0][0], dt, dx, dy, "RK2_TimeAd");
}

/* RK3_TimeAd (include/time_advance.h:788-882). */
static inline void RK3_TimeAd(int AR_scheme, int var_, int rows, int cols, int GC,
                              double (*y)[rows][cols], double dt, double dx, double dy) {
    (void)var_;
    (void)GC;
    rpf_rk_call(3, AR_scheme, rows, cols, &y[0][0][0], dt, dx, dy, "RK3_TimeAd");
}

/* RK1_TimeAd_BS (include/time_advance.h:886-1025): the backward-step flow on
 * two blocks (the channel above the step, the inlet section beside it). */
static inline void RK1_TimeAd_BS(int AR_scheme, int var_, int rows, int cols, int GC,
                                 double (*y)[rows][cols], double dt, double dx, double dy) {
    (void)var_;
    (void)GC;
    rpf_globals g = rpf_collect();
    rpf_check(rpf_rk1_bs(AR_scheme, rows, cols, &y[0][0][0], dt, dx, dy, &g), "RK1_TimeAd_BS");
}

#endif
