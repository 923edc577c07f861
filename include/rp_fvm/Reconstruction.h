/* Reconstruction.h -- drop-in for the reference's include/Reconstruction.h:
 * interface states of the state y along one direction, on the GPU, with the
 * branch (characteristic or component) of the global Characteriz. */
#ifndef RECONSTRUCTION_H
#define RECONSTRUCTION_H

#include "rpf_glue.h"
#include "function.h"
#include "Characteriz.h"

/* WENO5_Reconstruction (include/Reconstruction.h:887-1074): WENO-Z weights
 * in the characteristic branch, Jiang-Shu in the component branch.  dir 1 =
 * x, 2 = y; conserl / conserr receive the states left / right of each
 * interface, other entries are left as they were. */
static inline void WENO5_Reconstruction(int dir, int var_, int rows, int cols, int GC,
                                        double (*y)[rows][cols], double (*conserl)[rows][cols],
                                        double (*conserr)[rows][cols]) {
    rpf_globals g = rpf_collect();
    (void)var_;
    (void)GC;
    /* the spacing does not enter the WENO5 states */
    rpf_check(rpf_reconstruct(5, dir, rows, cols, &y[0][0][0], &conserl[0][0][0],
                              &conserr[0][0][0], 1.0, 1.0, &g),
              "WENO5_Reconstruction");
}

/* TVD_Reconstruction (include/Reconstruction.h:260-446): van Leer on
 * characteristic variables, minmod on conserved variables. */
static inline void TVD_Reconstruction(int dir, int var_, int rows, int cols, int GC,
                                      double (*y)[rows][cols], double (*conserl)[rows][cols],
                                      double (*conserr)[rows][cols], double delta_x,
                                      double delta_y) {
    rpf_globals g = rpf_collect();
    (void)var_;
    (void)GC;
    rpf_check(rpf_reconstruct(2, dir, rows, cols, &y[0][0][0], &conserl[0][0][0],
                              &conserr[0][0][0], delta_x, delta_y, &g),
              "TVD_Reconstruction");
}

#endif
