/* mesh.h -- drop-in for the reference's include/mesh.h: cell centres. */
#ifndef MESH_H
#define MESH_H

#include "rpf_glue.h"
#include "initialize.h"

/* Mesh_2D (include/mesh.h:151-160): centres (k + 1/2) * delta of the
 * interior cells, computed as delta * k + 0.5 * delta like the reference so
 * that written coordinates agree to the bit. */
static inline void Mesh_2D(int rows, int cols, double *mesh_x, double *mesh_y, double deltax,
                           double deltay) {
    for (int k = 0; k < rows; k++) mesh_x[k] = deltax * k + 0.5 * deltax;
    for (int k = 0; k < cols; k++) mesh_y[k] = deltay * k + 0.5 * deltay;
}

#endif
