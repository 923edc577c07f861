/*
 * euler_b200.h -- C ABI of libeuler_b200.so, the B200 (sm_100a) 2D Euler
 * finite-volume step.
 *
 * The entry points replace the operator API of the reference solver
 * (xujf520/OverheatingProblem): the static inline C functions of its headers
 * that src/RP_FVM.c calls, plus the control file reader.  Each declaration
 * cites the reference function it stands in for.  Plain pointers and sizes
 * only; no CUDA or C++ types cross this boundary.
 *
 * Model.  A context (eb2_ctx) owns one solve: its conserved state
 * double U[4][nx+8][ny+8] (the reference's layout: x index i = row, y index j
 * = unit stride, 4 ghost layers) lives in GPU memory, together with every
 * temporary the step needs, allocated once at creation.  The reference's
 * mutable globals (M_gamma, CFL, Recon_Accur, Characteriz, Source, Gravity,
 * bc_config) become per-context settings.  Calls on one context are ordered
 * on its CUDA stream and return after the result is complete; contexts are
 * independent of one another.
 *
 * Arrays passed by the host are full [4][rows][cols] (or [4][4][rows][cols])
 * double arrays in host memory, rows = nx + 8, cols = ny + 8.
 *
 * Return values: EB2_OK (0) or one of the EB2_E* codes; eb2_last_error()
 * gives the message of the calling thread's last failure.
 */
#ifndef EULER_B200_H
#define EULER_B200_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct eb2_ctx eb2_ctx;

enum {
    EB2_OK = 0,
    EB2_EARG = 1,         /* invalid argument                                     */
    EB2_ENOMEM = 2,       /* device or host allocation failed                     */
    EB2_ECUDA = 3,        /* CUDA error, or no CUDA device (there is no CPU path) */
    EB2_ENONPHYS = 4,     /* non-physical state met (see eb2_status)              */
    EB2_EUNSUPPORTED = 5, /* option the library does not implement               */
    EB2_EBUSY = 6         /* server: no free slot or HBM budget for the request   */
};

/* Status bits accumulated by the kernels of a context. */
enum {
    EB2_ST_NONPHYSICAL = 1, /* reconstructed rho<=0, p<=0 or NaN at an interface  */
    EB2_ST_NAN_STATE = 2,   /* NaN in an updated conserved state                  */
    EB2_ST_BAD_DT = 4       /* non-finite or non-positive CFL time step            */
};

/* Boundary kinds: BC_Type, include/Boundary_Condition.h:21-27. */
enum { EB2_BC_OUTFLOW = 0, EB2_BC_REFLECTION = 1, EB2_BC_PERIODICITY = 2,
       EB2_BC_INFLOW = 3, EB2_BC_FIXED_VALUE = 4 };

/* Arithmetic of the step. */
enum { EB2_FP64 = 0,      /* plain drop-in: bit-identical to the reference        */
       EB2_MIXED = 1 };   /* FP32 reconstruction/fluxes, FP64 state and RK sums   */

/* Initial states for eb2_init_case: the reference's TestCase2D values
 * (include/Golbal.h:8-30) that the library implements, plus two cases that
 * take their parameters from `q`. */
enum {
    EB2_CASE_PRECISION = 0,          /* TEST_PRECISION                           */
    EB2_CASE_SOD_1D = 1,             /* TEST_1D_SHOCKTUBE                        */
    EB2_CASE_CONTACT_1D = 2,         /* TEST_1D_CONTACTWAVE                      */
    EB2_CASE_SHOCK_IMPACT_1D = 3,    /* TEST_1D_SHOCKIMPACT                      */
    EB2_CASE_DOUBLE_RARE_1D = 5,     /* TEST_1D_DOUBLERARE                       */
    EB2_CASE_IMPACT_WALL_1D = 4,     /* TEST_1D_IMPACTWALL                       */
    EB2_CASE_NOH_1D = 6,             /* TEST_1D_NOHPROBLEM                       */
    EB2_CASE_RIEMANN_1 = 7,          /* TEST_2D_SHOCKTUBE_CASE1 .. CASE5 = 7..11 */
    EB2_CASE_TAYLOR_GREEN = 12,      /* TEST_TAYLOR_GREEN_VORTEX                 */
    EB2_CASE_GAUSSIAN_PULSE = 13,    /* TEST_GAUSSIAN_PULSE                      */
    EB2_CASE_KELVIN_HELMHOLTZ = 14,  /* TEST_KELVIN_HELMHOLTZ                    */
    EB2_CASE_RAYLEIGH_TAYLOR = 15,   /* TEST_RAYLEIGH_TAYLOR                     */
    EB2_CASE_DOUBLE_MACH = 16,       /* TEST_DOUBLE_MACH_REFLECTION              */
    EB2_CASE_BLAST_WAVE = 17,        /* TEST_BLAST_WAVE                          */
    EB2_CASE_NOH_2D = 18,            /* TEST_NOH_PROBLEM: rand() perturbations in
                                        the order of a one-thread run           */
    EB2_CASE_ODD_EVEN = 19,          /* TEST_OddEven_Decoupling                  */
    EB2_CASE_BACKWARD_STEP = 20,     /* TEST_BACKWARD_STEP: the initial stream
                                        (the step is the multi-block path)      */
    EB2_CASE_FOUR_QUADRANT = 100,    /* q[16] = (rho,u,v,p) of the upper-right,
                                        upper-left, lower-left, lower-right
                                        quadrants of [0,1]^2; q == NULL gives
                                        the 1.5/0.5323/0.138/0.5323 states     */
    EB2_CASE_WALL_HEATING = 101      /* [0,1]x[0,0.02], rho=1, u=-q[0] (q==NULL:
                                        q[0]=1), v=0, p=1e-4, reflecting x=0,
                                        outflow x=1, periodic in y, t=0.6      */
};

/* --- context --------------------------------------------------------------- */

/* One solve of nx x ny interior cells on CUDA device `device`.  Allocates all
 * device memory the step needs.  Fails with EB2_ECUDA when no GPU is usable. */
int eb2_ctx_create(eb2_ctx **out, int nx, int ny, int device);
int eb2_ctx_destroy(eb2_ctx *ctx);

/* Use a caller-owned cudaStream_t (passed as void*); NULL restores the
 * context's own stream. */
int eb2_set_stream(eb2_ctx *ctx, void *cuda_stream);

/* set_material_parameters (src/RP_FVM.c:600-605): M_gamma, Source, Gravity, CFL. */
int eb2_set_material(eb2_ctx *ctx, double gamma, int source, double gravity, double cfl);

/* Recon_Accur and Characteriz (include/Golbal.h:58-60): recon 1 (first
 * order), 2 (TVD: minmod on conserved, van Leer on characteristic variables)
 * or 5 (WENO5).  weno_z selects the WENO-Z weights the reference's
 * characteristic branch uses (include/Reconstruction.h:941-942); 0 gives
 * Jiang-Shu weights there.  The component branch always uses Jiang-Shu. */
int eb2_set_reconstruction(eb2_ctx *ctx, int recon, int characteristic, int weno_z);

/* EB2_FP64 or EB2_MIXED. */
int eb2_set_precision(eb2_ctx *ctx, int precision);

/* Opt-in, not in the reference: at an interface whose reconstructed states
 * have rho<=0 or p<=0, use the two adjacent cell averages instead. */
int eb2_set_positivity_fallback(eb2_ctx *ctx, int on);

/* bc_config (include/Boundary_Condition.h:30-38). */
int eb2_set_bc(eb2_ctx *ctx, int left, int right, int bottom, int top);
/* The context's boundary kinds (left, right, bottom, top), e.g. as set by
 * eb2_init_case the way Init_Euler_2D sets bc_config. */
int eb2_get_bc(eb2_ctx *ctx, int *kinds4);
/* inflow_state (Boundary_Condition.h:41,49) and L/R/B/T_fixed_value_state
 * (include/initialize.h:1298-1301), conserved variables; NULL keeps a value. */
int eb2_set_bc_states(eb2_ctx *ctx, const double *inflow4, const double *fixed16);
/* Use BC_DoubleMach_2D (Boundary_Condition.h:480-692) for all four sides. */
int eb2_set_double_mach(eb2_ctx *ctx, int on);

/* --- state ------------------------------------------------------------------- */

/* Init_Euler_2D (include/initialize.h:1558-1606): writes the initial conserved
 * state of case `test_case` on the device, sets the case's boundary kinds and
 * returns its domain lengths and final time. */
int eb2_init_case(eb2_ctx *ctx, int test_case, const double *q, double *lx, double *ly,
                  double *tmax);

/* Init_Euler_2D in full: eb2_init_case, plus the case's primitive state
 * (initEulerTestCase), and the physical fluxes of the initial state
 * (initEulerflux2D, include/initialize.h:1409-1434) into host arrays
 * pri, F, G [4][rows][cols]; any of them may be NULL. */
int eb2_init_case_fields(eb2_ctx *ctx, int test_case, const double *q, double *pri,
                         double *F, double *G, double *lx, double *ly, double *tmax);

/* Copy the full state (ghosts included) between host and device. */
int eb2_upload(eb2_ctx *ctx, const double *U);
int eb2_download(eb2_ctx *ctx, double *U);

/* Device address of the state, for callers that manage device memory. */
int eb2_state_device_ptr(eb2_ctx *ctx, double **dptr);

/* --- operators (each replaces the reference function named) --------------- */

/* Boundary_Conditions (include/Boundary_Condition.h:963-980) on the state;
 * `time` is read only by the double-Mach boundary. */
int eb2_bc_apply(eb2_ctx *ctx, double time);

/* Con_to_Pri_2D (include/initialize.h:1437-1454): primitives of the state on
 * the box [3, rows-4]^2 into pri[4][rows][cols]. */
int eb2_con_to_pri(eb2_ctx *ctx, double *pri);

/* Compute_Eigen_2DX / _2DY (include/Characteriz.h:300-500): from pri
 * [4][rows][cols] into eig_l[4][4][rows][cols] (eig_l[k][m]: row k of L) and
 * eig_r[4][4][rows][cols] (eig_r[m][k]). */
int eb2_eigen(eb2_ctx *ctx, int dir, const double *pri, double *eig_l, double *eig_r);

/* WENO5_Reconstruction / TVD_Reconstruction / Reconstruction_Godunov
 * (include/Reconstruction.h:887, 260, 51) of the state along dir (1 = x,
 * 2 = y) into conserl / conserr [4][rows][cols]. */
int eb2_reconstruct(eb2_ctx *ctx, int dir, double dx, double dy, double *conserl,
                    double *conserr);

/* HLL_Flux / HLLC_Flux / Roe_Flux / LLF_Flux (include/scheme.h:400, 690, 1018,
 * 229) for AR_scheme `scheme` along dir; entries the reference's HLL skips are
 * left as they were in `flux`. */
int eb2_riemann(eb2_ctx *ctx, int scheme, int dir, const double *conserl,
                const double *conserr, double *flux);

/* Flux_Reconstruction_RP (include/CFD_convection.h:38-200) of the state. */
int eb2_flux_reconstruction(eb2_ctx *ctx, int scheme, double dx, double dy, double *f,
                            double *g);

/* Space_Discrete_Item (include/scheme.h:3758-3777): L = -(f_i - f_{i-1})/dx
 * - (g_j - g_{j-1})/dy + s on the interior.  s == NULL takes the gravity
 * source of the state (Source_Gravity, :3723) when Source is on, else zero. */
int eb2_space_discrete(eb2_ctx *ctx, double dx, double dy, const double *f, const double *g,
                       const double *s, double *L);

/* Get_Delta_T_2D (include/function.h:144-175). */
int eb2_delta_t(eb2_ctx *ctx, double dx, double dy, double *dt);
/* The two maxima it combines: max(|u|+a), max(|v|+a) over the interior. */
int eb2_wave_speeds(eb2_ctx *ctx, double *sx, double *sy);

/* RK1_TimeAd / RK2_TimeAd / RK3_TimeAd (include/time_advance.h:643, 711, 788):
 * one step of `order` with Riemann solver `scheme`; `time` is read only by
 * the double-Mach boundary.  Returns EB2_ENONPHYS when a kernel met a
 * non-physical state (the step still completes, as the reference's does). */
int eb2_rk_step(eb2_ctx *ctx, int order, int scheme, double dt, double dx, double dy,
                double time);

/* The time loop of src/RP_FVM.c:179-267 (Control_Compution = 0) run on the
 * device: CFL time step, clipping at the n_out output times and at tmax,
 * `order`-stage SSP-RK steps.  Steps are issued in CUDA graphs of a few steps
 * without host round trips.  At each output time the loop pauses and calls
 * on_output(user, time, step) (may be NULL), from which the caller may read
 * the state.  Returns the step count and the final time. */
/* RK1_TimeAd_BS (include/time_advance.h:886-1025): one forward-Euler step of the
 * backward-step flow on the context's state.  Block 1 (the channel above the
 * step: all nx rows, int(0.8 ny) columns from column int(0.2 ny)) and block 2
 * (the inlet section beside the step: int(0.2 nx) x int(0.2 ny) at the lower
 * left) are advanced with their own ghost layers, filled by the rules of
 * BC_BackwardStep_2D (include/Boundary_Condition.h:696-850); the rest of the
 * lower strip is the step and keeps its values.  The context's
 * reconstruction, gas and gravity source apply; the step runs in the FP64
 * form whatever the context's precision (the reference's bits).  Returns
 * EB2_ENONPHYS if a non-physical state was met. */
int eb2_rk1_backward_step(eb2_ctx *ctx, int scheme, double dt, double dx, double dy);

typedef void (*eb2_output_fn)(void *user, double time, long long step);
int eb2_run(eb2_ctx *ctx, int order, int scheme, double dx, double dy, double t0,
            double tmax, int n_out, eb2_output_fn on_output, void *user, long long *steps,
            double *t_final);

/* No reference counterpart: advance exactly `nsteps` steps of the device time
 * loop (CFL time step from the device reduction, no output or tmax clipping),
 * issued as CUDA graphs.  Used for fixed-length runs and benchmarks. */
int eb2_advance(eb2_ctx *ctx, int order, int scheme, double dx, double dy, int nsteps);

/* No reference counterpart: benchmark helper.  Runs `nsteps` steps as
 * eb2_advance does, but launched one by one with CUDA events around each step
 * and around each stage kernel, and a write of `flush_bytes` bytes between
 * steps (outside the timed intervals) to evict the L2 cache.  step_ms[s]
 * receives the device time of step s; *stage_ms the summed device time of the
 * fused stage kernels and *stage_launches their count; *launches the number of
 * library kernels launched inside the timed intervals. */
int eb2_bench_steps(eb2_ctx *ctx, int order, int scheme, double dx, double dy, int nsteps,
                    unsigned long long flush_bytes, float *step_ms, float *stage_ms,
                    int *stage_launches, long long *launches);

/* --- solve server (no counterpart in the reference) -------------------------- */

/* Many independent solves on one GPU with continuous batching.  Each request
 * is one eb2_run-style solve (SSP-RK3, WENO5, CFL time step, its own final
 * time) of an EB2_CASE_* initial state.  Admitted requests keep their state on
 * the device and advance together: a batch step is one CUDA graph whose
 * stage kernels walk a device work list of (solve, tile) pairs with a
 * persistent grid (sized per batch shape by timing, the autotuner).  Requests
 * are admitted while a slot is free and the HBM budget allows, and retired as
 * they finish; a solve's result does not depend on what else is in the batch
 * (the same bits as alone, and as eb2_run on a context). */
typedef struct eb2_server eb2_server;

typedef struct {
    int test_case;        /* EB2_CASE_*                                         */
    int nx, ny;           /* interior cells                                     */
    int has_q;            /* q holds case parameters (see eb2_init_case)        */
    double q[16];
    double lx, ly;        /* domain lengths; <= 0 keeps the case's              */
    double tmax;          /* final time; <= 0 keeps the case's                  */
    double cfl;           /* CFL number; <= 0 gives 0.5                         */
} eb2_request;

/* scheme as AR_scheme (1/2/3/11/22/33, anything else LLF); recon must be 5;
 * the mixed form needs characteristic. */
int eb2_server_create(eb2_server **out, int device, int max_slots,
                      unsigned long long hbm_budget_bytes, int precision, int recon,
                      int characteristic, int weno_z, int scheme, double gamma);
int eb2_server_destroy(eb2_server *srv);
/* Admit a request (EB2_EBUSY: no slot or budget now). */
int eb2_server_submit(eb2_server *srv, const eb2_request *req, long long *id);
/* Advance all admitted solves by `ngraphs` batch graphs (4 steps each); the
 * number of solves that finished is returned in *nfinished. */
int eb2_server_step(eb2_server *srv, int ngraphs, int *nfinished);
/* Finished solves awaiting eb2_server_fetch: ids, final times, step counts. */
int eb2_server_poll(eb2_server *srv, long long *ids, double *t_final, long long *steps,
                    unsigned *status, int max, int *n);
/* Copy a finished solve's state to U (may be NULL) and free its slot. */
int eb2_server_fetch(eb2_server *srv, long long id, double *U);
/* Device time of every batch step run so far (CUDA events around the graphs
 * of each eb2_server_step; set against a replay's wall time it is the share of
 * the time the GPU spent stepping solves), and the host seconds spent in the
 * autotuner's trials and in admission, work-list rebuilds and retirement.
 * Any output pointer may be NULL. */
int eb2_server_timing(eb2_server *srv, double *busy_ms, double *tune_s, double *admin_s);
int eb2_server_stats(eb2_server *srv, unsigned long long *hbm_used, int *active,
                     long long *graph_launches);
/* The request loop: replay n requests arriving arrival_s[i] seconds after the
 * call in real time (FIFO admission by slot and budget, batch steps, retire as
 * finished).  Per request: admission and finish times in seconds since the
 * start, step counts and status bits (EB2_ST_*; any of these arrays may be
 * NULL) and, when results != NULL and results[i] != NULL, the final state. */
int eb2_server_run_trace(eb2_server *srv, const eb2_request *reqs, const double *arrival_s,
                         int n, double *admit_s, double *finish_s, long long *steps,
                         unsigned *status, double **results, double *makespan_s);

/* --- step without allocation ------------------------------------------------ */

/* No counterpart in the reference.  Some callers cannot call cudaMalloc at
 * all: a host application whose own pool owns all device memory, a real-time
 * loop that forbids allocation after start-up, a plug-in that is only handed
 * device pointers.  eb2_rk_step_noalloc runs one RK1/RK2/RK3 step of the FP64
 * form (the same kernels as eb2_rk_step, the same bits) on a state U that the
 * caller holds in device memory, [4][nx+8][ny+8] in the layout above, updated
 * in place, and allocates nothing: its scratch (two stage states and a control
 * block) lives in one static __device__ array of the library, about 16 MiB,
 * that every GPU which loads the library keeps until the process exits.
 *
 * Limits: (nx+8)*(ny+8) <= EB2_NOALLOC_MAX_CELLS, else EB2_EARG.  All calls
 * share the one array: calls that overlap on the GPU (other streams, other
 * host threads) race and must not be issued.  Each call looks up the array's
 * device address in the calling thread's current context (cudaGetSymbolAddress,
 * not a stream operation), so callers on a context of their own get that
 * context's copy; the first call in a context also loads the library's device
 * code there, so make that first call before any stream capture.  Every
 * reconstruction (recon 1/2/3/5) and every AR_scheme of eb2_rk_step (HLL, HLLC,
 * Roe, the heat-conduction fluxes 11/22/33, LLF) is accepted.  The call enqueues
 * on `cuda_stream` (NULL: the legacy default stream) and returns after the
 * step, with EB2_ENONPHYS if a non-physical state was met.  Nothing in the
 * array has to start at zero: each call clears the control block itself, and
 * every stage-buffer value a call reads was written earlier in that call.
 * Boundary kinds use the reference's default inflow and fixed states. */
#define EB2_NOALLOC_MAX_CELLS 262144
typedef struct {
    double gamma;
    int recon, characteristic, weno_z;               /* as eb2_set_reconstruction */
    int bc_left, bc_right, bc_bottom, bc_top;        /* EB2_BC_*                  */
    int source;
    double gravity;
} eb2_noalloc_config;
int eb2_rk_step_noalloc(double *U_device, int nx, int ny, const eb2_noalloc_config *cfg,
                        int order, int scheme, double dt, double dx, double dy, double time,
                        void *cuda_stream);

/* --- diagnostics ------------------------------------------------------------- */

int eb2_status(eb2_ctx *ctx, unsigned *flags);
int eb2_clear_status(eb2_ctx *ctx);
int eb2_synchronize(eb2_ctx *ctx);
const char *eb2_last_error(void);
const char *eb2_version(void);

/* --- control file -------------------------------------------------------------- */

/* ControlParams (src/RP_FVM.c:66-82). */
typedef struct {
    int test_case;
    int L_nx, L_ny;
    int Time_ADM;
    int scheme;
    double M_gamma;
    int Source;
    double Gravity;
    double CFL;
    double Tmax;
    int Control_Compution;
    int Control_output;
    int Recon_Accur;
    int Characteriz;
    char output_dir[256];
} eb2_control;

/* ReadControlFile (src/RP_FVM.c:382-589): the reference's defaults, then the
 * `key: value` lines of the file ('#' comments), with its test-case names and
 * its warnings on stderr.  Returns EB2_EARG when the file cannot be opened
 * (the reference exits instead). */
int eb2_read_control_file(const char *path, eb2_control *out);

#ifdef __cplusplus
}
#endif
#endif /* EULER_B200_H */
