/*
 * ref_harness.c -- thin C-ABI wrapper around the reference solver itself.
 *
 * TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file together with
 * the reference's own src/RP_FVM.c (its main() renamed) and headers, exactly
 * as they lie in the reference tree, into oracle/_ref/libref.so.  A second
 * build, oracle/_ref/libref_wjs.so, uses a copy of the headers in which the
 * characteristic WENO5 branch calls the Jiang-Shu weights WENO5_L/R instead
 * of WENO5Z_L/R (include/Reconstruction.h:941-942, 997-998): the
 * "characteristic WENO5-JS" combination the reference never runs as shipped.
 * Nothing here is product code.  Every entry point forwards to the reference
 * function named in its comment; the only composed routine is ref_rk_dmr,
 * which runs the RK stages of include/time_advance.h with the exact
 * double-Mach boundary BC_DoubleMach_2D (include/Boundary_Condition.h:480),
 * whose call sites are commented out in the reference.  A third build,
 * oracle/_ref/libref_wjs_dmr.so, switches those commented-out calls on inside
 * the reference's own RK1/RK2/RK3_TimeAd (time_advance.h:591-862), so that
 * ref_rk there is the reference's own double-Mach step; tests check that
 * ref_rk_dmr gives the same bits.
 */
#define main rp_fvm_main
#include "RP_FVM.c"
#undef main

/* The reference's TU-static globals (include/Golbal.h:45-70) */
void ref_set_params(double gamma, double cfl, int recon, int characteriz,
                    int source, double gravity) {
    M_gamma = gamma;
    CFL = cfl;
    Recon_Accur = recon;
    Characteriz = characteriz ? true : false;
    Source = source ? true : false;
    Gravity = gravity;
}

void ref_set_bc(int left, int right, int bottom, int top) {
    bc_config.left = (BC_Type)left;
    bc_config.right = (BC_Type)right;
    bc_config.bottom = (BC_Type)bottom;
    bc_config.top = (BC_Type)top;
}

void ref_get_bc(int *out4) {
    out4[0] = bc_config.left;
    out4[1] = bc_config.right;
    out4[2] = bc_config.bottom;
    out4[3] = bc_config.top;
}

/* Init_Euler_2D, include/initialize.h:1558 */
void ref_init(int test_case, int rows, int cols, double *pri, double *U, double *F,
              double *G, double *lx, double *ly, double *tmax) {
    Init_Euler_2D((TestCase2D)test_case, var, rows, cols, GhostCell,
                  (double (*)[rows][cols])pri, (double (*)[rows][cols])U,
                  (double (*)[rows][cols])F, (double (*)[rows][cols])G, lx, ly, tmax);
}

/* Con_to_Pri_2D, include/initialize.h:1437 */
void ref_con_to_pri(int rows, int cols, double *pri, double *U) {
    Con_to_Pri_2D(var, rows, cols, (double (*)[rows][cols])pri, (double (*)[rows][cols])U);
}

/* Compute_Eigen_2DX / _2DY, include/Characteriz.h:300, 402 */
void ref_eigen(int dir, int rows, int cols, double *pri, double *el, double *er) {
    if (dir == 1)
        Compute_Eigen_2DX(var, rows, cols, (double (*)[rows][cols])pri,
                          (double (*)[var][rows][cols])el, (double (*)[var][rows][cols])er);
    else
        Compute_Eigen_2DY(var, rows, cols, (double (*)[rows][cols])pri,
                          (double (*)[var][rows][cols])el, (double (*)[var][rows][cols])er);
}

/* the reconstruction switch of Flux_Reconstruction_RP (CFD_convection.h:67-85) */
void ref_recon(int dir, int rows, int cols, double *U, double *ql, double *qr,
               double dx, double dy) {
    double (*y)[rows][cols] = (double (*)[rows][cols])U;
    double (*a)[rows][cols] = (double (*)[rows][cols])ql;
    double (*b)[rows][cols] = (double (*)[rows][cols])qr;
    switch (Recon_Accur) {
        case 1: Reconstruction_Godunov(dir, var, rows, cols, GhostCell, y, a, b, dx); break;
        case 2: TVD_Reconstruction(dir, var, rows, cols, GhostCell, y, a, b, dx, dy); break;
        case 3: WENO3_Reconstruction(dir, var, rows, cols, GhostCell, y, a, b); break;
        case 5: WENO5_Reconstruction(dir, var, rows, cols, GhostCell, y, a, b); break;
        default: break;
    }
}

/* HLL_Flux / HLLC_Flux / Roe_Flux / LLF_Flux, include/scheme.h */
void ref_riemann(int scheme, int dir, int rows, int cols, double *ql, double *qr,
                 double *flux) {
    double (*a)[rows][cols] = (double (*)[rows][cols])ql;
    double (*b)[rows][cols] = (double (*)[rows][cols])qr;
    double (*f)[rows][cols] = (double (*)[rows][cols])flux;
    switch (scheme) {
        case 1: HLL_Flux(dir, var, rows, cols, GhostCell, a, b, f); break;
        case 2: HLLC_Flux(dir, var, rows, cols, GhostCell, a, b, f); break;
        case 3: Roe_Flux(dir, var, rows, cols, GhostCell, a, b, f); break;
        case 11: HLLHC_Flux(dir, var, rows, cols, GhostCell, a, b, f); break;
        case 22: HLLCHC_Flux(dir, var, rows, cols, GhostCell, a, b, f); break;
        case 33: RoeHC_Flux(dir, var, rows, cols, GhostCell, a, b, f); break;
        default: LLF_Flux(dir, var, rows, cols, GhostCell, a, b, f); break;
    }
}

/* Flux_Reconstruction_RP, include/CFD_convection.h:38 */
void ref_flux_recon(int scheme, int rows, int cols, double *U, double *f, double *g,
                    double dt, double dx, double dy) {
    Flux_Reconstruction_RP(scheme, var, rows, cols, GhostCell, (double (*)[rows][cols])U,
                           (double (*)[rows][cols])f, (double (*)[rows][cols])g, dt, dx, dy);
}

/* Space_Discrete_Item, include/scheme.h:3758 */
void ref_space_item(int rows, int cols, double dx, double dy, double *f, double *g,
                    double *s, double *Lt) {
    Space_Discrete_Item(var, rows, cols, GhostCell, dx, dy, (double (*)[rows][cols])f,
                        (double (*)[rows][cols])g, (double (*)[rows][cols])s,
                        (double (*)[rows][cols])Lt);
}

/* Boundary_Conditions, include/Boundary_Condition.h:963 */
void ref_bc(int rows, int cols, double *U) {
    Boundary_Conditions(var, rows, cols, (double (*)[rows][cols])U, GhostCell);
}

/* BC_DoubleMach_2D, include/Boundary_Condition.h:480 */
void ref_bc_dmr(int rows, int cols, double *U, double t) {
    BC_DoubleMach_2D(var, rows, cols, (double (*)[rows][cols])U, GhostCell, t);
}

/* Source_Gravity, include/scheme.h:3723 */
void ref_source(int rows, int cols, double *U, double *s) {
    Source_Gravity(var, rows, cols, GhostCell, (double (*)[rows][cols])U,
                   (double (*)[rows][cols])s);
}

/* RK1/RK2/RK3_TimeAd, include/time_advance.h:643, 711, 788 */
void ref_rk(int order, int scheme, int rows, int cols, double *U, double dt, double dx,
            double dy) {
    double (*y)[rows][cols] = (double (*)[rows][cols])U;
    if (order == 1) RK1_TimeAd(scheme, var, rows, cols, GhostCell, y, dt, dx, dy);
    else if (order == 2) RK2_TimeAd(scheme, var, rows, cols, GhostCell, y, dt, dx, dy);
    else RK3_TimeAd(scheme, var, rows, cols, GhostCell, y, dt, dx, dy);
}

/* RK stages of include/time_advance.h:711-882 with BC_DoubleMach_2D applied to
 * each stage input at the step's start time, as the commented-out call sites
 * (time_advance.h:747, 765, 826, 843, 861) would. */
void ref_rk_dmr(int order, int scheme, int rows, int cols, double *U, double dt,
                double dx, double dy, double t) {
    double (*y)[rows][cols] = (double (*)[rows][cols])U;
    size_t bytes = (size_t)var * rows * cols * sizeof(double);
    double (*Lt)[rows][cols] = calloc(1, bytes);
    double (*U1)[rows][cols] = calloc(1, bytes);
    double (*U2)[rows][cols] = calloc(1, bytes);
    double (*f)[rows][cols] = calloc(1, bytes);
    double (*g)[rows][cols] = calloc(1, bytes);
    double (*s)[rows][cols] = calloc(1, bytes);
    double (*in[3])[rows][cols] = {y, U1, U2};
    for (int st = 0; st < order; st++) {
        double (*x)[rows][cols] = in[st];
        if (Source) Source_Gravity(var, rows, cols, GhostCell, x, s);
        BC_DoubleMach_2D(var, rows, cols, x, GhostCell, t);
        Flux_Reconstruction_RP(scheme, var, rows, cols, GhostCell, x, f, g, dt, dx, dy);
        Space_Discrete_Item(var, rows, cols, GhostCell, dx, dy, f, g, s, Lt);
        for (int k = 0; k < var; k++)
            for (int i = GhostCell; i <= rows - GhostCell - 1; i++)
                for (int j = GhostCell; j <= cols - GhostCell - 1; j++) {
                    if (order == 1) y[k][i][j] = y[k][i][j] + dt * Lt[k][i][j];
                    else if (st == 0) U1[k][i][j] = y[k][i][j] + dt * Lt[k][i][j];
                    else if (order == 2)
                        y[k][i][j] = 0.5 * y[k][i][j] + 0.5 * (U1[k][i][j] + dt * Lt[k][i][j]);
                    else if (st == 1)
                        U2[k][i][j] = (3.0 / 4.0) * y[k][i][j] +
                                      (1.0 / 4.0) * (U1[k][i][j] + dt * Lt[k][i][j]);
                    else
                        y[k][i][j] = (1.0 / 3.0) * y[k][i][j] +
                                     (2.0 / 3.0) * (U2[k][i][j] + dt * Lt[k][i][j]);
                }
    }
    free(Lt); free(U1); free(U2); free(f); free(g); free(s);
}

/* The reference's global Time (include/Golbal.h:45): the time BC_DoubleMach_2D
 * reads in the libref_wjs_dmr.so build, whose RK stages call it. */
void ref_set_time(double t) { Time = t; }

/* Get_Delta_T_2D, include/function.h:144 */
double ref_dt(int rows, int cols, double *U, double dx, double dy) {
    return Get_Delta_T_2D(var, rows, cols, (double (*)[rows][cols])U, dx, dy);
}

/* Mesh_2D, include/mesh.h:151 */
void ref_mesh(int nx, int ny, double *mx, double *my, double dx, double dy) {
    Mesh_2D(nx, ny, mx, my, dx, dy);
}

/* ReadControlFile, src/RP_FVM.c:382: parse, then copy ctrl_params out.
 * ints: test_case, L_nx, L_ny, Time_ADM, scheme, Source, Control_Compution,
 *       Control_output, Recon_Accur, Characteriz
 * dbls: M_gamma, Gravity, CFL, Tmax */
void ref_read_control(const char *path, int *ints, double *dbls, char *outdir, int n) {
    ReadControlFile(path);
    ints[0] = ctrl_params.test_case;
    ints[1] = ctrl_params.L_nx;
    ints[2] = ctrl_params.L_ny;
    ints[3] = ctrl_params.Time_ADM;
    ints[4] = ctrl_params.scheme;
    ints[5] = ctrl_params.Source;
    ints[6] = ctrl_params.Control_Compution;
    ints[7] = ctrl_params.Control_output;
    ints[8] = ctrl_params.Recon_Accur;
    ints[9] = ctrl_params.Characteriz;
    dbls[0] = ctrl_params.M_gamma;
    dbls[1] = ctrl_params.Gravity;
    dbls[2] = ctrl_params.CFL;
    dbls[3] = ctrl_params.Tmax;
    snprintf(outdir, (size_t)n, "%s", ctrl_params.output_dir);
}

/* the time loop of src/RP_FVM.c:179-267 (Control_Compution = 0) without its
 * progress output; dmr selects BC_DoubleMach_2D for the stage inputs */
long ref_run(int order, int scheme, int rows, int cols, double *U, double dx, double dy,
             double tmax, int n_out, int dmr, double *t_final) {
    double out_dt = tmax / n_out, next_out = out_dt, dt = 0.0;
    long ite = 0;
    for (Time = 0.0; Time < tmax; Time = Time + dt) {
        dt = Get_Delta_T_2D(var, rows, cols, (double (*)[rows][cols])U, dx, dy);
        if (Time + dt > next_out) dt = next_out - Time;
        if (Time + dt >= tmax) dt = tmax - Time;
        if (dmr) ref_rk_dmr(order, scheme, rows, cols, U, dt, dx, dy, Time);
        else ref_rk(order, scheme, rows, cols, U, dt, dx, dy);
        double now = Time + dt;
        if (fabs(now - next_out) < 1e-10 * out_dt) next_out += out_dt;
        ite++;
    }
    if (t_final) *t_final = Time;
    return ite;
}

int ref_num_threads(void) { return omp_get_max_threads(); }
void ref_set_threads(int n) { omp_set_num_threads(n); }

/* RK1_TimeAd_BS, include/time_advance.h:886: the two-block backward-step step */
void ref_rk1_bs(int scheme, int rows, int cols, double *U, double dt, double dx, double dy) {
    RK1_TimeAd_BS(scheme, var, rows, cols, GhostCell, (double (*)[rows][cols])U, dt, dx, dy);
}
