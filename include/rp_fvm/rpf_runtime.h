/*
 * rpf_runtime.h -- runtime behind the drop-in header set in this directory.
 *
 * The headers next to this file carry the names of the reference solver's
 * headers (the include/ directory of xujf520/OverheatingProblem) and declare its entry
 * points with the same names and signatures, as static inline functions
 * that forward here; src/RP_FVM.c compiles against them unchanged and runs
 * its step on the GPU through libeuler_b200.so.  No counterpart in the
 * reference: this is the glue between its header API and the C ABI of
 * euler_b200.h.
 *
 * State.  Each host state array U[4][rows][cols] the caller passes is bound
 * to a GPU context (eb2_ctx) on first use; the step runs on the device copy.
 * In the default RESIDENT mode the state stays on the device between calls:
 * it is uploaded when first seen (or after rpf_host_modified) and downloaded
 * when a call reads it on the host (Con_to_Pri_2D, the error norms,
 * rpf_sync_host).  The reference's own main loop only touches U through
 * those calls.  STRICT mode (rpf_set_coherence, or RPF_COHERENCE=strict in
 * the environment) copies the state both ways around every call instead.
 *
 * Settings.  The reference keeps its settings in file-static globals of the
 * calling translation unit (include/Golbal.h:45-70, Boundary_Condition.h:30-49,
 * initialize.h:1298-1301); the headers pass them by value in rpf_globals on
 * every call.
 *
 * Errors.  The reference's functions return void; these return 0 or an
 * EB2_E* code and print a message.  The headers stop the program (exit 1)
 * on codes other than EB2_ENONPHYS, as the reference does on its own fatal
 * errors: there is no CPU path to fall back to.
 */
#ifndef RPF_RUNTIME_H
#define RPF_RUNTIME_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct rpf_globals {
    double gamma;          /* M_gamma                                          */
    double cfl;            /* CFL                                              */
    double gravity;        /* Gravity                                          */
    double time;           /* Time (read by time-dependent boundaries)         */
    int source;            /* Source                                           */
    int recon;             /* Recon_Accur                                      */
    int characteristic;    /* Characteriz                                      */
    int bc[4];             /* bc_config: left, right, bottom, top              */
    int reserved;          /* zero (keeps the struct free of padding)          */
    double inflow[4];      /* inflow_state                                     */
    double fixed[16];      /* L_, R_, B_, T_fixed_value_state                  */
} rpf_globals;

enum { RPF_RESIDENT = 0, RPF_STRICT = 1 };

/* Library-level options (no reference counterpart). */
int rpf_set_coherence(int mode);
int rpf_set_device(int device);
/* EB2_FP64 (default: bit-identical to the reference) or EB2_MIXED. */
int rpf_set_precision(int precision);
/* WENO weights of the characteristic branch: -1 as the reference (WENO-Z),
 * 0 Jiang-Shu, 1 WENO-Z.  The component branch always uses Jiang-Shu. */
int rpf_set_char_weno(int weno_z);

/* Coherence of a bound state array. */
int rpf_host_modified(const double *U);  /* the caller wrote U on the host  */
int rpf_sync_host(double *U);            /* bring the host copy up to date  */
int rpf_release(const double *U);        /* drop U's device copy            */
int rpf_release_all(void);
/* Status bits (EB2_ST_*) the kernels raised since the last call of this. */
unsigned rpf_take_status(void);

/* Entry points; the header functions named in each comment forward here.
 * rows, cols include 4 ghost layers on each side. */

/* Init_Euler_2D / Init_Precision (include/initialize.h:1558, 1609); writes
 * pri, U, F, G, the domain lengths, the final time and the case's boundary
 * kinds into bc_out[4]. */
int rpf_init(int test_case, int rows, int cols, double *pri, double *U, double *F, double *G,
             double *Lx, double *Ly, double *Tmax, int *bc_out, const rpf_globals *g);
/* Con_to_Pri_2D (include/initialize.h:1437); also brings U up to date. */
int rpf_con_to_pri(int rows, int cols, double *pri, double *U, const rpf_globals *g);
/* Boundary_Conditions (include/Boundary_Condition.h:963). */
int rpf_boundary(int rows, int cols, double *U, const rpf_globals *g);
/* Get_Delta_T_2D (include/function.h:144). */
int rpf_delta_t(int rows, int cols, double *U, double dx, double dy, double *dt,
                const rpf_globals *g);
/* RK1_TimeAd / RK2_TimeAd / RK3_TimeAd (include/time_advance.h:643, 711, 788). */
int rpf_rk(int order, int scheme, int rows, int cols, double *U, double dt, double dx,
           double dy, const rpf_globals *g);
/* WENO5_Reconstruction (recon 5) / TVD_Reconstruction (recon 2)
 * (include/Reconstruction.h:887, 260). */
int rpf_reconstruct(int recon, int dir, int rows, int cols, double *U, double *conserl,
                    double *conserr, double dx, double dy, const rpf_globals *g);
/* Compute_Eigen_2DX / _2DY (include/Characteriz.h:300, 402). */
int rpf_eigen(int dir, int rows, int cols, const double *pri, double *eig_l, double *eig_r,
              const rpf_globals *g);
/* HLL_Flux / HLLC_Flux / Roe_Flux (include/scheme.h:400, 690, 1018). */
int rpf_riemann(int scheme, int dir, int rows, int cols, const double *conserl,
                const double *conserr, double *flux, const rpf_globals *g);
/* Flux_Reconstruction_RP (include/CFD_convection.h:38). */
int rpf_flux_reconstruction(int scheme, int rows, int cols, double *U, double *f, double *gf,
                            double dx, double dy, const rpf_globals *g);
/* Space_Discrete_Item (include/scheme.h:3758). */
int rpf_space_discrete(int rows, int cols, double dx, double dy, const double *f,
                       const double *gf, const double *s, double *lout, const rpf_globals *g);

/* RK1_TimeAd_BS (include/time_advance.h:886): one forward-Euler step of the
 * backward-step flow on its two blocks, the channel above the step and the
 * inlet section beside it, with BC_BackwardStep_2D's boundaries. */
int rpf_rk1_bs(int scheme, int rows, int cols, double *U, double dt, double dx, double dy,
               const rpf_globals *g);

/* Message of the last failure (thread-local). */
const char *rpf_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
