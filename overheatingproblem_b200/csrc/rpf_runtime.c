/* rpf_runtime.c -- runtime of the drop-in header set (include/rp_fvm/):
 * binds the caller's host state arrays to GPU contexts, keeps the host and
 * device copies coherent, applies the caller's global settings, and forwards
 * each reference entry point to the C ABI of euler_b200.h.
 *
 * Single-threaded, as the reference is: calls must not overlap. */
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "euler_b200.h"
#include "rp_fvm/rpf_runtime.h"

enum { SYNCED = 0, HOST_NEWER = 1, DEVICE_NEWER = 2 };
enum { MAX_BINDINGS = 64 };

typedef struct binding {
    const double *host; /* NULL: a scratch context of this shape           */
    int rows, cols;
    eb2_ctx *ctx;
    int state;
    unsigned long long used; /* last use, for eviction                      */
    int configured;
    rpf_globals cfg;         /* settings last applied to ctx                */
    int precision, weno_z, recon;
} binding;

static binding g_bind[MAX_BINDINGS];
static unsigned long long g_clock;
static int g_mode = -1;
static int g_device;
static int g_precision = EB2_FP64;
static int g_char_weno = -1;
static unsigned g_status;
static _Thread_local char g_err[512];

static int fail(int code, const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
    return code;
}

/* A failed library call: keep its code and message. */
static int lib_fail(int code, const char *what) {
    fail(code, "%s: %s", what, eb2_last_error());
    return code;
}

#define LIB(call, what)                          \
    do {                                         \
        int rc_ = (call);                        \
        if (rc_) return lib_fail(rc_, (what));   \
    } while (0)

const char *rpf_last_error(void) { return g_err; }

static int mode(void) {
    if (g_mode < 0) {
        const char *e = getenv("RPF_COHERENCE");
        g_mode = (e && strcmp(e, "strict") == 0) ? RPF_STRICT : RPF_RESIDENT;
    }
    return g_mode;
}

int rpf_set_coherence(int m) {
    if (m != RPF_RESIDENT && m != RPF_STRICT) return fail(EB2_EARG, "coherence mode %d", m);
    g_mode = m;
    return EB2_OK;
}

int rpf_set_device(int device) {
    if (device < 0) return fail(EB2_EARG, "device %d", device);
    g_device = device;
    return EB2_OK;
}

int rpf_set_precision(int precision) {
    if (precision != EB2_FP64 && precision != EB2_MIXED)
        return fail(EB2_EARG, "precision %d", precision);
    g_precision = precision;
    return EB2_OK;
}

int rpf_set_char_weno(int weno_z) {
    if (weno_z < -1 || weno_z > 1) return fail(EB2_EARG, "weno_z %d", weno_z);
    g_char_weno = weno_z;
    return EB2_OK;
}

unsigned rpf_take_status(void) {
    unsigned s = g_status;
    g_status = 0;
    return s;
}

/* --- bindings ------------------------------------------------------------ */

static int pull(binding *b) {
    if (b->state != DEVICE_NEWER) return EB2_OK;
    LIB(eb2_download(b->ctx, (double *)b->host), "download");
    b->state = SYNCED;
    return EB2_OK;
}

static int push(binding *b) {
    if (b->state != HOST_NEWER) return EB2_OK;
    LIB(eb2_upload(b->ctx, b->host), "upload");
    b->state = SYNCED;
    return EB2_OK;
}

static void drop(binding *b) {
    if (b->ctx) eb2_ctx_destroy(b->ctx);
    memset(b, 0, sizeof *b);
}

/* After a call changed the device copy. */
static int device_wrote(binding *b) {
    if (!b->host) return EB2_OK;
    b->state = DEVICE_NEWER;
    return mode() == RPF_STRICT ? pull(b) : EB2_OK;
}

/* The binding of host array U (NULL: any context of this shape), created on
 * first use with the host copy marked newer.  An address seen before with
 * another shape is another array.  When every slot is taken the least
 * recently used binding is written back to its host array and dropped. */
static int bind(const double *U, int rows, int cols, binding **out) {
    if (rows < 9 || cols < 9) return fail(EB2_EARG, "grid %d x %d has no interior", rows, cols);
    binding *hit = NULL, *lru = NULL, *slot = NULL;
    for (int k = 0; k < MAX_BINDINGS && !hit; k++) {
        binding *b = &g_bind[k];
        if (!b->ctx) {
            if (!slot) slot = b;
            continue;
        }
        int same = U ? b->host == U : (!b->host && b->rows == rows && b->cols == cols);
        if (same && b->rows == rows && b->cols == cols) {
            hit = b;
        } else if (same) {
            drop(b);
            if (!slot) slot = b;
        } else if (!lru || b->used < lru->used) {
            lru = b;
        }
    }
    if (!hit) {
        if (!slot) {
            if (lru->host) {
                int rc = pull(lru);
                if (rc) return rc;
            }
            drop(lru);
            slot = lru;
        }
        eb2_ctx *c = NULL;
        LIB(eb2_ctx_create(&c, rows - 8, cols - 8, g_device), "context");
        slot->host = U;
        slot->rows = rows;
        slot->cols = cols;
        slot->ctx = c;
        slot->state = U ? HOST_NEWER : SYNCED;
        slot->configured = 0;
        hit = slot;
    }
    hit->used = ++g_clock;
    *out = hit;
    return EB2_OK;
}

/* Apply the caller's settings; `recon` > 0 overrides Recon_Accur. */
static int configure(binding *b, const rpf_globals *g, int recon) {
    int r = recon > 0 ? recon : g->recon;
    int wz = g_char_weno < 0 ? 1 : g_char_weno;
    if (b->configured && b->precision == g_precision && b->weno_z == wz && b->recon == r &&
        memcmp(&b->cfg, g, sizeof *g) == 0)
        return EB2_OK;
    eb2_ctx *c = b->ctx;
    LIB(eb2_set_material(c, g->gamma, g->source, g->gravity, g->cfl), "set_material_parameters");
    LIB(eb2_set_reconstruction(c, r, g->characteristic, wz), "Recon_Accur/Characteriz");
    LIB(eb2_set_precision(c, g_precision), "precision");
    LIB(eb2_set_bc(c, g->bc[0], g->bc[1], g->bc[2], g->bc[3]), "bc_config");
    LIB(eb2_set_bc_states(c, g->inflow, g->fixed), "boundary states");
    b->cfg = *g;
    b->precision = g_precision;
    b->weno_z = wz;
    b->recon = r;
    b->configured = 1;
    return EB2_OK;
}

static int note_status(int rc) {
    if (rc == EB2_ENONPHYS) {
        g_status |= EB2_ST_NONPHYSICAL;
        fail(rc, "non-physical state met: %s", eb2_last_error());
    }
    return rc;
}

#define TRY(expr)              \
    do {                       \
        int rc_ = (expr);      \
        if (rc_) return rc_;   \
    } while (0)

int rpf_host_modified(const double *U) {
    for (int k = 0; k < MAX_BINDINGS; k++)
        if (g_bind[k].ctx && g_bind[k].host == U) g_bind[k].state = HOST_NEWER;
    return EB2_OK;
}

int rpf_sync_host(double *U) {
    for (int k = 0; k < MAX_BINDINGS; k++)
        if (g_bind[k].ctx && g_bind[k].host == U) return pull(&g_bind[k]);
    return EB2_OK;
}

int rpf_release(const double *U) {
    for (int k = 0; k < MAX_BINDINGS; k++)
        if (g_bind[k].ctx && g_bind[k].host == U) {
            TRY(pull(&g_bind[k]));
            drop(&g_bind[k]);
        }
    return EB2_OK;
}

int rpf_release_all(void) {
    for (int k = 0; k < MAX_BINDINGS; k++)
        if (g_bind[k].ctx) {
            if (g_bind[k].host) TRY(pull(&g_bind[k]));
            drop(&g_bind[k]);
        }
    return EB2_OK;
}

/* --- entry points ---------------------------------------------------------- */

int rpf_init(int test_case, int rows, int cols, double *pri, double *U, double *F, double *G,
             double *Lx, double *Ly, double *Tmax, int *bc_out, const rpf_globals *g) {
    binding *b;
    TRY(bind(U, rows, cols, &b));
    TRY(configure(b, g, 0));
    LIB(eb2_init_case_fields(b->ctx, test_case, NULL, pri, F, G, Lx, Ly, Tmax),
        "Init_Euler_2D");
    LIB(eb2_download(b->ctx, U), "download");
    b->state = SYNCED;
    int bc[4];
    LIB(eb2_get_bc(b->ctx, bc), "bc_config");
    memcpy(b->cfg.bc, bc, sizeof bc);
    if (bc_out) memcpy(bc_out, bc, sizeof bc);
    return EB2_OK;
}

int rpf_con_to_pri(int rows, int cols, double *pri, double *U, const rpf_globals *g) {
    binding *b;
    TRY(bind(U, rows, cols, &b));
    TRY(configure(b, g, 0));
    TRY(push(b));
    LIB(eb2_con_to_pri(b->ctx, pri), "Con_to_Pri_2D");
    return pull(b);
}

int rpf_boundary(int rows, int cols, double *U, const rpf_globals *g) {
    binding *b;
    TRY(bind(U, rows, cols, &b));
    TRY(configure(b, g, 0));
    TRY(push(b));
    LIB(eb2_bc_apply(b->ctx, g->time), "Boundary_Conditions");
    return device_wrote(b);
}

int rpf_delta_t(int rows, int cols, double *U, double dx, double dy, double *dt,
                const rpf_globals *g) {
    binding *b;
    TRY(bind(U, rows, cols, &b));
    TRY(configure(b, g, 0));
    TRY(push(b));
    LIB(eb2_delta_t(b->ctx, dx, dy, dt), "Get_Delta_T_2D");
    return EB2_OK;
}

int rpf_rk(int order, int scheme, int rows, int cols, double *U, double dt, double dx,
           double dy, const rpf_globals *g) {
    binding *b;
    TRY(bind(U, rows, cols, &b));
    TRY(configure(b, g, 0));
    TRY(push(b));
    int rc = eb2_rk_step(b->ctx, order, scheme, dt, dx, dy, g->time);
    if (rc && rc != EB2_ENONPHYS) return lib_fail(rc, "RK_TimeAd");
    TRY(device_wrote(b));
    return note_status(rc);
}

int rpf_reconstruct(int recon, int dir, int rows, int cols, double *U, double *conserl,
                    double *conserr, double dx, double dy, const rpf_globals *g) {
    binding *b;
    TRY(bind(U, rows, cols, &b));
    TRY(configure(b, g, recon));
    TRY(push(b));
    LIB(eb2_reconstruct(b->ctx, dir, dx, dy, conserl, conserr), "Reconstruction");
    return EB2_OK;
}

int rpf_eigen(int dir, int rows, int cols, const double *pri, double *eig_l, double *eig_r,
              const rpf_globals *g) {
    binding *b;
    TRY(bind(NULL, rows, cols, &b));
    TRY(configure(b, g, 0));
    LIB(eb2_eigen(b->ctx, dir, pri, eig_l, eig_r), "Compute_Eigen_2D");
    return EB2_OK;
}

int rpf_riemann(int scheme, int dir, int rows, int cols, const double *conserl,
                const double *conserr, double *flux, const rpf_globals *g) {
    binding *b;
    TRY(bind(NULL, rows, cols, &b));
    TRY(configure(b, g, 0));
    LIB(eb2_riemann(b->ctx, scheme, dir, conserl, conserr, flux), "Riemann flux");
    return EB2_OK;
}

int rpf_flux_reconstruction(int scheme, int rows, int cols, double *U, double *f, double *gf,
                            double dx, double dy, const rpf_globals *g) {
    binding *b;
    TRY(bind(U, rows, cols, &b));
    TRY(configure(b, g, 0));
    TRY(push(b));
    LIB(eb2_flux_reconstruction(b->ctx, scheme, dx, dy, f, gf), "Flux_Reconstruction_RP");
    return EB2_OK;
}

int rpf_space_discrete(int rows, int cols, double dx, double dy, const double *f,
                       const double *gf, const double *s, double *lout, const rpf_globals *g) {
    binding *b;
    TRY(bind(NULL, rows, cols, &b));
    TRY(configure(b, g, 0));
    LIB(eb2_space_discrete(b->ctx, dx, dy, f, gf, s, lout), "Space_Discrete_Item");
    return EB2_OK;
}

/* --- RK1_TimeAd_BS (include/time_advance.h:886-1025) ---------------------
 * One forward-Euler step of the backward-step flow on two blocks: block 1 is
 * the channel above the step (the whole length, the upper part of the height,
 * int(0.8 ny) cells), block 2 the inlet section beside the step (int(0.2 nx)
 * by int(0.2 ny) cells at the lower left).  The rest of the lower strip is
 * the step and is not advanced.  The whole step runs on the GPU
 * (eb2_rk1_backward_step): block gather, the ghost layers of
 * BC_BackwardStep_2D, the gravity source, flux reconstruction, flux
 * difference and Euler update of each block, and the scatter back into U. */
int rpf_rk1_bs(int scheme, int rows, int cols, double *U, double dt, double dx, double dy,
               const rpf_globals *g) {
    binding *b;
    TRY(bind(U, rows, cols, &b));
    TRY(configure(b, g, 0));
    TRY(push(b));
    int rc = eb2_rk1_backward_step(b->ctx, scheme, dt, dx, dy);
    if (rc && rc != EB2_ENONPHYS) return lib_fail(rc, "RK1_TimeAd_BS");
    TRY(device_wrote(b));
    return note_status(rc);
}
