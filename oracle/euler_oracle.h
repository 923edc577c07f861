/*
 * euler_oracle.h -- CPU oracle for the 2D Euler finite-volume step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * solver's hot path (xujf520/OverheatingProblem, src/RP_FVM.c and the headers
 * it includes) used as the parity checker for the CUDA product.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it.  The
 * product library never links or calls it.
 *
 * Parity status: pinned.  tests/test_oracle_pin.py compares every entry point
 * below bit-for-bit against the reference itself, compiled from its own
 * sources by oracle/Makefile into oracle/_ref/, and against the golden vectors
 * in tests/golden/ that tests/golden/make_golden.py produced from that build.
 *
 * State layout is the reference's: double U[4][rows][cols], rows = nx + 2*gc
 * is the x index i, cols = ny + 2*gc is the y index j (unit stride), gc = 4
 * (include/Golbal.h:49).  Floating-point expressions keep the reference's
 * evaluation order exactly, because the checker compares bits.
 */
#ifndef EULER_ORACLE_H
#define EULER_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Boundary kinds, numbered as BC_Type in include/Boundary_Condition.h:21-27. */
enum { ORC_BC_OUTFLOW = 0, ORC_BC_REFLECT = 1, ORC_BC_PERIODIC = 2,
       ORC_BC_INFLOW = 3, ORC_BC_FIXED = 4 };

typedef struct {
    int nx, ny, gc;        /* interior cells along x and y, ghost layers       */
    double gamma;          /* M_gamma                                          */
    double cfl;            /* CFL                                              */
    int recon;             /* Recon_Accur: 1 Godunov, 2 TVD, 5 WENO5           */
    int characteristic;    /* Characteriz                                      */
    int weno_z;            /* characteristic WENO5 uses WENO-Z weights (1, the
                              reference as shipped) or Jiang-Shu weights (0)   */
    int source;            /* Source: gravity source on                        */
    double gravity;        /* Gravity                                          */
    int bc[4];             /* left, right, bottom, top  (ORC_BC_*)             */
    int dmr;               /* 1: use the exact double-Mach boundary instead     */
    double inflow[4];      /* inflow_state                                     */
    double fixed[4][4];    /* L/R/B/T_fixed_value_state                        */
} orc_params;

/* Fill p with the reference's defaults for an nx x ny grid. */
void orc_defaults(orc_params *p, int nx, int ny);

/* Con_to_Pri_2D (include/initialize.h:1437-1454): box [gc-1, rows-gc]^2. */
void orc_con_to_pri(const orc_params *p, const double *U, double *pri);

/* Compute_Eigen_2DX / _2DY (include/Characteriz.h:300-398, 402-500).
 * Writes eig_l[k][m][rows][cols] and eig_r[m][k][rows][cols] on the
 * reference's interface ranges. */
void orc_eigen(const orc_params *p, int dir, const double *pri,
               double *eig_l, double *eig_r);

/* Reconstruction dispatch of Flux_Reconstruction_RP
 * (include/CFD_convection.h:67-85): conserl/conserr on the sweep's range. */
int orc_recon(const orc_params *p, int dir, const double *U,
              double *conserl, double *conserr, double dx, double dy);

/* Riemann flux dispatch (include/CFD_convection.h:89-117). */
void orc_riemann(const orc_params *p, int scheme, int dir,
                 const double *ql, const double *qr, double *flux);

/* Flux_Reconstruction_RP (include/CFD_convection.h:38-200). f and g get the
 * interface fluxes on [gc-1, rows-gc) x [gc, cols-gc) and
 * [gc, rows-gc) x [gc-1, cols-gc) respectively. */
int orc_flux_recon(const orc_params *p, int scheme, const double *U,
                   double *f, double *g, double dx, double dy);

/* Space_Discrete_Item (include/scheme.h:3758-3777). */
void orc_space_item(const orc_params *p, double dx, double dy, const double *f,
                    const double *g, const double *s, double *Lout);

/* Boundary_Conditions (include/Boundary_Condition.h:963-980), or
 * BC_DoubleMach_2D (:480-692) when p->dmr is set. */
void orc_bc(const orc_params *p, double *U, double time);

/* Source_Gravity (include/scheme.h:3723-3751). */
void orc_source(const orc_params *p, const double *U, double *s);

/* RK1/RK2/RK3_TimeAd (include/time_advance.h:643-882). time is only read by
 * the double-Mach boundary. Returns 0, or -1 on a bad argument. */
int orc_rk(const orc_params *p, int order, int scheme, double *U, double dt,
           double dx, double dy, double time);

/* Get_Delta_T_2D (include/function.h:144-175). */
double orc_dt(const orc_params *p, const double *U, double dx, double dy);

/* The two wave-speed maxima that Get_Delta_T_2D combines. */
void orc_wave_speeds(const orc_params *p, const double *U, double *sx,
                     double *sy);

/* Mesh_2D (include/mesh.h:151-160). */
void orc_mesh(int nx, int ny, double *mx, double *my, double dx, double dy);

/* Initial states.  Each writes primitive (rho,u,v,p) into the interior, zero
 * elsewhere, then the conserved U; sets the boundary kinds in p and returns
 * the domain lengths and final time. */
enum { ORC_CASE_FOUR_QUADRANT = 1, ORC_CASE_WALL_HEATING = 2,
       ORC_CASE_DOUBLE_MACH = 3, ORC_CASE_PRECISION = 4, ORC_CASE_NOH_1D = 5,
       ORC_CASE_SOD_1D = 6 };
int orc_init_case(orc_params *p, int which, const double *qstate, double *U,
                  double *lx, double *ly, double *tmax);

/* The host time loop of src/RP_FVM.c:179-267 with Control_Compution = 0:
 * runs until tmax with the CFL dt, clipping at output times (n_out outputs).
 * Returns the number of steps. */
long orc_run(const orc_params *p, int order, int scheme, double *U, double dx,
             double dy, double tmax, int n_out, double *t_final);

#ifdef __cplusplus
}
#endif
#endif
