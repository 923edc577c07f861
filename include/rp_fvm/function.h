/* function.h -- drop-in for the reference's include/function.h: the CFL time
 * step of the state on the GPU, and the accuracy test's fixed step. */
#ifndef FUNCTION_H
#define FUNCTION_H

#include "rpf_glue.h"

/* min_of_two (include/function.h:58-63). */
static inline double min_of_two(double a, double b) { return a < b ? a : b; }

/* Get_Delta_T_2D (include/function.h:144-175): CFL * min(dx, dy) over the
 * sum of the two wave-speed maxima of the interior.  Called as the
 * reference's main does, with (var, rows, cols, U). */
static inline double Get_Delta_T_2D(int var_, int rows, int cols, double (*x)[rows][cols],
                                    double dx, double dy) {
    rpf_globals g = rpf_collect();
    double dt = 0.0;
    (void)var_;
    rpf_check(rpf_delta_t(rows, cols, &x[0][0][0], dx, dy, &dt, &g), "Get_Delta_T_2D");
    return dt;
}

/* Precision_Get_Delta_T_2D (include/function.h:239-241): the accuracy test's
 * step 0.5 dx^(5/3), independent of the state. */
static inline double Precision_Get_Delta_T_2D(int var_, int rows, int cols,
                                              double (*x)[rows][cols], double dx, double dy) {
    (void)var_;
    (void)rows;
    (void)cols;
    (void)x;
    (void)dy;
    return 0.5 * pow(dx, 5.0 / 3);
}

#endif
