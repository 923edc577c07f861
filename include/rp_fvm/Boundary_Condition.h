/* Boundary_Condition.h -- drop-in for the reference's
 * include/Boundary_Condition.h: Boundary_Conditions on the GPU copy of the
 * state, with the boundary kinds of bc_config and the inflow / fixed-value
 * states of the globals below. */
#ifndef BOUNDARY_CONDITION_H
#define BOUNDARY_CONDITION_H

#include <ctype.h>
#include "rpf_glue.h"
#include "mesh.h"
#include "initialize.h"
#include "scheme.h"
#include "function.h"

/* Side names the reference defines here (include/Boundary_Condition.h:15-18);
 * kept for source compatibility: any later identifier L, R, T or B in the
 * caller's code is replaced by these strings, as with the reference. */
#define L "left"
#define R "right"
#define T "top"
#define B "bottom"

/* include/Boundary_Condition.h:49, same default (a Mach-3 stream of rho 1.4). */
double inflow_state[4] = {1.4, 1.4 * 3.0, 0.0, 1.0 / 0.4 + 0.5 * 1.4 * 3.0 * 3.0};

/* Boundary_Conditions (include/Boundary_Condition.h:963-980): the four sides
 * of the state y in the order left, right, bottom, top. */
static inline void Boundary_Conditions(int var_, int rows, int cols, double (*y)[rows][cols],
                                       int GC) {
    rpf_globals g = rpf_collect();
    (void)var_;
    (void)GC;
    rpf_check(rpf_boundary(rows, cols, &y[0][0][0], &g), "Boundary_Conditions");
}

#endif
