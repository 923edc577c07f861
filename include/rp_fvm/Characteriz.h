/* Characteriz.h -- drop-in for the reference's include/Characteriz.h: the
 * Roe-averaged eigenvector matrices on the GPU. */
#ifndef CHARACTERIZ_H
#define CHARACTERIZ_H

#include "rpf_glue.h"

/* Compute_Eigen_2DX / _2DY (include/Characteriz.h:300-500): from the
 * primitives Pri, eigen_l[k][m] = row k of L and eigen_r[m][k] = column k of
 * R at each x (y) interface. */
static inline void Compute_Eigen_2DX(int var_, int rows, int cols, double (*Pri)[rows][cols],
                                     double (*eigen_l)[var_][rows][cols],
                                     double (*eigen_r)[var_][rows][cols]) {
    rpf_globals g = rpf_collect();
    rpf_check(rpf_eigen(1, rows, cols, &Pri[0][0][0], &eigen_l[0][0][0][0],
                        &eigen_r[0][0][0][0], &g),
              "Compute_Eigen_2DX");
}

static inline void Compute_Eigen_2DY(int var_, int rows, int cols, double (*Pri)[rows][cols],
                                     double (*eigen_l)[var_][rows][cols],
                                     double (*eigen_r)[var_][rows][cols]) {
    rpf_globals g = rpf_collect();
    rpf_check(rpf_eigen(2, rows, cols, &Pri[0][0][0], &eigen_l[0][0][0][0],
                        &eigen_r[0][0][0][0], &g),
              "Compute_Eigen_2DY");
}

#endif
