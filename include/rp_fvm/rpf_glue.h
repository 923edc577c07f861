/* rpf_glue.h -- shared part of the drop-in header set: the boundary types
 * the settings refer to (include/Boundary_Condition.h:21-49 of the
 * reference, same names and values), the collection of the calling
 * translation unit's settings, and the error policy. */
#ifndef RPF_GLUE_H
#define RPF_GLUE_H

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "Golbal.h"
#include "../euler_b200.h"
#include "rpf_runtime.h"

typedef enum {
    BC_OUTFLOW = 0,
    BC_REFLECTION = 1,
    BC_PERIODICITY = 2,
    BC_INFLOW = 3,
    BC_FIXED_VALUE = 4
} BC_Type;

typedef struct {
    BC_Type left;
    BC_Type right;
    BC_Type bottom;
    BC_Type top;
} BoundaryConfig;

extern BoundaryConfig bc_config;         /* defined by the caller (src/RP_FVM.c:88) */
extern double inflow_state[4];           /* defined in Boundary_Condition.h       */
extern double L_fixed_value_state[4];    /* defined in initialize.h               */
extern double R_fixed_value_state[4];
extern double B_fixed_value_state[4];
extern double T_fixed_value_state[4];

/* The settings the reference's functions read from globals. */
static inline rpf_globals rpf_collect(void) {
    rpf_globals g;
    memset(&g, 0, sizeof g);
    g.gamma = M_gamma;
    g.cfl = CFL;
    g.gravity = Gravity;
    g.time = Time;
    g.source = Source ? 1 : 0;
    g.recon = Recon_Accur;
    g.characteristic = Characteriz ? 1 : 0;
    g.bc[0] = (int)bc_config.left;
    g.bc[1] = (int)bc_config.right;
    g.bc[2] = (int)bc_config.bottom;
    g.bc[3] = (int)bc_config.top;
    memcpy(g.inflow, inflow_state, sizeof g.inflow);
    memcpy(g.fixed, L_fixed_value_state, 4 * sizeof(double));
    memcpy(g.fixed + 4, R_fixed_value_state, 4 * sizeof(double));
    memcpy(g.fixed + 8, B_fixed_value_state, 4 * sizeof(double));
    memcpy(g.fixed + 12, T_fixed_value_state, 4 * sizeof(double));
    return g;
}

/* A non-physical state is reported once and the run goes on (the reference
 * runs on into NaNs); any other failure ends the program, as the reference's
 * own fatal errors do. */
static inline void rpf_check(int rc, const char *where) {
    static int warned;
    if (rc == 0) return;
    if (rc == EB2_ENONPHYS) {
        if (!warned) fprintf(stderr, "Warning: %s: %s\n", where, rpf_last_error());
        warned = 1;
        return;
    }
    fprintf(stderr, "Error: %s: %s\n", where, rpf_last_error());
    exit(1);
}

#endif
