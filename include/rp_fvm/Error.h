/* Error.h -- drop-in for the reference's include/Error.h: density error norms
 * of the accuracy test against the exact solution rho = 1 + 0.2 sin(x - t),
 * the convergence orders and their table.  These read the state on the host,
 * so each first brings the caller's copy up to date.  The norms, the order
 * formula and the printed lines are the reference's (Error.h:129-329): the
 * accuracy test's output is compared line by line. */
#ifndef ERROR_H
#define ERROR_H

#include "rpf_glue.h"
#include "Reconstruction.h"
#include "function.h"

typedef struct {
    int grid_points;
    double delta_x;
    double L1_error;
    double L2_error;
    double Linf_error;
    double L1_order;
    double L2_order;
    double Linf_order;
} ErrorData;

ErrorData error_table[100];
int error_count = 0;

/* |exact - rho| at the interior cells of the first interior column. */
static inline double rpf_density_error(int rows, int cols, int GC, double (*Conser)[rows][cols],
                                       int i, double Delta, double t) {
    double xc = (i - GC + 0.5) * Delta;
    return (1.0 + 0.2 * sin(xc - t)) - Conser[0][i][GC];
}

/* TEST_Scheme_Error_L1 (Error.h:129-160): dx * sum |exact - rho|. */
static inline void TEST_Scheme_Error_L1(int var_, int rows, int cols, int GC,
                                        double (*Conser)[rows][cols], double Delta,
                                        double Time_, int grid_points, int store_index) {
    (void)var_;
    rpf_check(rpf_sync_host(&Conser[0][0][0]), "TEST_Scheme_Error_L1");
    double e = 0.0;
    for (int i = GC; i < rows - GC; i++)
        e += fabs(rpf_density_error(rows, cols, GC, Conser, i, Delta, Time_)) * Delta;
    error_table[store_index].grid_points = grid_points;
    error_table[store_index].delta_x = Delta;
    error_table[store_index].L1_error = e;
    printf("L1 Error = %.10e \n", e);
}

/* TEST_Scheme_Error_L2 (Error.h:171-200): sqrt(dx * sum (exact - rho)^2). */
static inline void TEST_Scheme_Error_L2(int var_, int rows, int cols, int GC,
                                        double (*Conser)[rows][cols], double Delta,
                                        double Time_, int store_index) {
    (void)var_;
    rpf_check(rpf_sync_host(&Conser[0][0][0]), "TEST_Scheme_Error_L2");
    double e = 0.0;
    for (int i = GC; i < rows - GC; i++) {
        double d = rpf_density_error(rows, cols, GC, Conser, i, Delta, Time_);
        e += d * d * Delta;
    }
    e = sqrt(e);
    error_table[store_index].L2_error = e;
    printf("L2 Error = %.10e \n", e);
}

/* TEST_Scheme_Error_Linf (Error.h:214-245): max |exact - rho|. */
static inline void TEST_Scheme_Error_Linf(int var_, int rows, int cols, int GC,
                                          double (*Conser)[rows][cols], double Delta,
                                          double Time_, int store_index) {
    (void)var_;
    rpf_check(rpf_sync_host(&Conser[0][0][0]), "TEST_Scheme_Error_Linf");
    double e = 0.0;
    for (int i = GC; i < rows - GC; i++) {
        double d = fabs(rpf_density_error(rows, cols, GC, Conser, i, Delta, Time_));
        if (d > e) e = d;
    }
    error_table[store_index].Linf_error = e;
    printf("L∞ Error = %.10e \n", e);
}

/* calculate_orders (Error.h:259-295): log(e_coarse / e_fine) / log(N_fine /
 * N_coarse) for each norm, 0 where an error is not positive. */
static inline double rpf_order(double coarse, double fine, double ratio) {
    return (coarse > 0 && fine > 0) ? log(coarse / fine) / log(ratio) : 0.0;
}

static inline void calculate_orders(void) {
    for (int i = 1; i < error_count; i++) {
        ErrorData *a = &error_table[i - 1], *b = &error_table[i];
        double ratio = (double)b->grid_points / (double)a->grid_points;
        b->L1_order = rpf_order(a->L1_error, b->L1_error, ratio);
        b->L2_order = rpf_order(a->L2_error, b->L2_error, ratio);
        b->Linf_order = rpf_order(a->Linf_error, b->Linf_error, ratio);
        printf("Order calculation for grid %d (N=%d) to %d (N=%d): h_ratio = %.4f, L1_order = %.4f\n",
               i - 1, a->grid_points, i, b->grid_points, ratio, b->L1_order);
    }
}

/* print_error_table (Error.h:303-329). */
static inline void print_error_table(void) {
    printf("\n\n");
    printf("===============================================================================\n");
    printf("Table 3.3: Errors and numerical orders of accuracy of the density\n");
    printf("===============================================================================\n");
    printf("Grid points  Δx        L1 error    Order     L2 error    Order     L∞ error    Order\n");
    printf("------------------------------------------------------------------------------\n");
    printf("%-11d  %-9.6f  %-10.2e  %-8s  %-10.2e  %-8s  %-10.2e  %-8s\n",
           error_table[0].grid_points, error_table[0].delta_x, error_table[0].L1_error, "---",
           error_table[0].L2_error, "---", error_table[0].Linf_error, "---");
    for (int i = 1; i < error_count; i++)
        printf("%-11d  %-9.6f  %-10.2e  %-8.2f  %-10.2e  %-8.2f  %-10.2e  %-8.2f\n",
               error_table[i].grid_points, error_table[i].delta_x, error_table[i].L1_error,
               error_table[i].L1_order, error_table[i].L2_error, error_table[i].L2_order,
               error_table[i].Linf_error, error_table[i].Linf_order);
    printf("===============================================================================\n");
}

#endif
