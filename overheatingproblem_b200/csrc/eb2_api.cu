// eb2_api.cu -- host runtime and C ABI of libeuler_b200 (include/euler_b200.h).
//
// A context owns one solve on one CUDA stream: the state and two stage
// buffers (the reference's Conser_U1 / Conser_U2, allocated once instead of
// per call), granular-API temporaries allocated on first use, the reduction
// partials and the device control block.  There is no CPU path: every entry
// point that computes runs a kernel, and creation fails without a GPU.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <climits>
#include <cstdlib>
#include <cstring>
#include <new>

#include "../../include/euler_b200.h"
#include "eb2_kernels.h"

using namespace eb2;

namespace {
thread_local char g_err[512] = "";

int fail(int code, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
    return code;
}

#define CK(expr)                                                                         \
    do {                                                                                 \
        cudaError_t e_ = (expr);                                                         \
        if (e_ != cudaSuccess)                                                           \
            return fail(EB2_ECUDA, "%s: %s (%s:%d)", #expr, cudaGetErrorString(e_),      \
                        __FILE__, __LINE__);                                             \
    } while (0)

int map_scheme(int scheme, int* flux) {
    switch (scheme) {
        case 1: *flux = FLUX_HLL; return EB2_OK;
        case 2: *flux = FLUX_HLLC; return EB2_OK;
        case 3: *flux = FLUX_ROE; return EB2_OK;
        case 11: *flux = FLUX_HLLHC; return EB2_OK;
        case 22: *flux = FLUX_HLLCHC; return EB2_OK;
        case 33: *flux = FLUX_ROEHC; return EB2_OK;
        default: *flux = FLUX_LLF; return EB2_OK;  // CFD_convection.h:111-116
    }
}

__global__ void k_set_step(Ctrl* c, double t, double dt) {
    c->t = t;
    c->dt = dt;
    c->active = 1;
    c->host_dt = 1;
}

__global__ void k_set_loop(Ctrl* c, double t0, double tmax, double out_dt, double cfl,
                           double dmin, long long max_step) {
    c->max_step = max_step;
    c->t = t0;
    c->dt = 0.0;
    c->tmax = tmax;
    c->out_dt = out_dt;
    c->next_out = out_dt;
    c->cfl = cfl;
    c->dmin = dmin;
    c->step = 0;
    c->active = 1;
    c->out_pending = 0;
    c->host_dt = 0;
}

__global__ void k_set_cfl(Ctrl* c, double cfl, double dmin) {
    c->cfl = cfl;
    c->dmin = dmin;
}

__global__ void k_resume(Ctrl* c) {
    c->out_pending = 0;
    c->active = (c->t < c->tmax) && !(c->status & ST_BAD_DT) && c->step < c->max_step;
}

__global__ void k_clear_status(Ctrl* c) { c->status = 0; }
}  // namespace

struct eb2_ctx {
    int device = 0;
    cudaStream_t own = nullptr, stream = nullptr;
    Grid grid{};
    Gas gas{};
    Numerics num{};
    Boundary bnd{};
    double cfl = 0.5;
    int precision = EB2_FP64;
    size_t nstate = 0;             // doubles in one [4][rows][cols] array
    double *u = nullptr, *u1 = nullptr, *u2 = nullptr;
    double* tmp[4] = {nullptr, nullptr, nullptr, nullptr};  // granular temporaries
    double* partials = nullptr;
    int npartials = 0;
    Ctrl* ctrl = nullptr;
    Ctrl* hctrl = nullptr;         // pinned mirror
    long long launches = 0;        // library kernels launched so far
    // cached CUDA graph of `per_graph` device-loop steps
    cudaGraphExec_t gexec = nullptr;
    unsigned char gkey[sizeof(Numerics) + sizeof(Boundary) + sizeof(Grid) + 4 * sizeof(int)] = {};
};

namespace {
int check(eb2_ctx* c) {
    if (!c) return fail(EB2_EARG, "null context");
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return fail(EB2_ECUDA, "cudaSetDevice: %s", cudaGetErrorString(e));
    return EB2_OK;
}

void set_spacing(eb2_ctx* c, double dx, double dy) {
    c->grid.dx = dx;
    c->grid.dy = dy;
    c->grid.inv_dx = 1.0 / dx;  // Space_Discrete_Item's inv_dx (scheme.h:3762)
    c->grid.inv_dy = 1.0 / dy;
}

// The mixed form implements characteristic WENO5 with the four classical
// fluxes only.
int check_precision_flux(const eb2_ctx* c, int flux) {
    (void)flux;
    if (c->precision != EB2_MIXED) return EB2_OK;
    if (c->num.recon != 5 || !c->num.characteristic)
        return fail(EB2_EUNSUPPORTED,
                    "the mixed form reconstructs with characteristic WENO5 only");
    return EB2_OK;
}

int ensure_tmp(eb2_ctx* c, int n) {
    for (int q = 0; q < n; q++)
        if (!c->tmp[q]) {
            CK(cudaMalloc(&c->tmp[q], c->nstate * sizeof(double)));
            CK(cudaMemsetAsync(c->tmp[q], 0, c->nstate * sizeof(double), c->stream));
        }
    return EB2_OK;
}

cudaError_t stage(eb2_ctx* c, const double* uin, const double* un, double* uout, int comb,
                  bool partials) {
    StageArgs a;
    a.uin = uin;
    a.un = un;
    a.uout = uout;
    a.grid = c->grid;
    a.gas = c->gas;
    a.num = c->num;
    a.combine = comb;
    a.ctrl = c->ctrl;
    a.partials = partials ? c->partials : nullptr;
    return c->precision == EB2_MIXED ? launch_stage_mixed(a, c->stream)
                                     : launch_stage_fp64(a, c->stream);
}

// The stages of RK1/RK2/RK3_TimeAd (include/time_advance.h:643-882): the
// boundary fill of each stage input, then the fused sweep/combine kernel.
// The last stage writes the wave-speed partials of the new state.
cudaError_t enqueue_step(eb2_ctx* c, int order, cudaEvent_t* ev = nullptr) {
    cudaError_t e;
    const Ctrl* ct = c->ctrl;
    // stage inputs, outputs and combinations of each order
    double* in[3] = {c->u, c->u1, c->u2};
    double* out1[1] = {c->u1};
    double* out2[2] = {c->u1, c->u};
    double* out3[3] = {c->u1, c->u2, c->u};
    const int comb2[2] = {COMB_EULER, COMB_RK2};
    const int comb3[3] = {COMB_EULER, COMB_RK3_2, COMB_RK3_3};
    for (int st = 0; st < order; st++) {
        if ((e = launch_bc(in[st], c->grid, c->bnd, ct, 0.0, c->stream))) return e;
        c->launches++;
        double* o = order == 1 ? out1[st] : (order == 2 ? out2[st] : out3[st]);
        int comb = order == 1 ? COMB_EULER : (order == 2 ? comb2[st] : comb3[st]);
        if (ev && (e = cudaEventRecord(ev[2 * st], c->stream))) return e;
        if ((e = stage(c, in[st], c->u, o, comb, st == order - 1))) return e;
        c->launches++;
        if (ev && (e = cudaEventRecord(ev[2 * st + 1], c->stream))) return e;
    }
    if (order == 1) {
        c->launches++;
        return launch_copy_interior(c->u, c->u1, c->grid, c->stream);
    }
    return cudaSuccess;
}

int read_status(eb2_ctx* c, unsigned* st) {
    CK(cudaMemcpyAsync(&c->hctrl->status, &c->ctrl->status, sizeof(unsigned),
                       cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    *st = c->hctrl->status;
    return EB2_OK;
}
}  // namespace

void eb2::set_last_error(const char* msg) { snprintf(g_err, sizeof g_err, "%s", msg); }

void eb2::set_loop_ctrl(Ctrl* c, double t0, double tmax, double out_dt, double cfl, double dmin,
                        long long max_step, cudaStream_t s) {
    k_set_loop<<<1, 1, 0, s>>>(c, t0, tmax, out_dt, cfl, dmin, max_step);
}

extern "C" {

const char* eb2_last_error(void) { return g_err; }
const char* eb2_version(void) { return "euler_b200 0.1 (sm_100a)"; }

int eb2_ctx_create(eb2_ctx** out, int nx, int ny, int device) {
    if (!out) return fail(EB2_EARG, "null output pointer");
    *out = nullptr;
    if (nx < 1 || ny < 1) return fail(EB2_EARG, "grid %d x %d is empty", nx, ny);
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0)
        return fail(EB2_ECUDA, "no CUDA device available (%s); libeuler_b200 has no CPU path",
                    e != cudaSuccess ? cudaGetErrorString(e) : "0 devices");
    if (device < 0 || device >= ndev) return fail(EB2_EARG, "device %d out of range", device);
    CK(cudaSetDevice(device));
    eb2_ctx* c = new (std::nothrow) eb2_ctx();
    if (!c) return fail(EB2_ENOMEM, "host allocation failed");
    c->device = device;
    c->grid.nx = nx;
    c->grid.ny = ny;
    c->grid.rows = nx + 2 * GC;
    c->grid.cols = ny + 2 * GC;
    set_spacing(c, 1.0 / nx, 1.0 / ny);
    eb2_set_material(c, 1.4, 0, 1.0, 0.5);
    c->num.recon = 5;            // Recon_Accur = 5 (include/Golbal.h:58)
    c->num.characteristic = 0;   // Characteriz = false (include/Golbal.h:60)
    c->num.weno_z = 1;
    c->num.flux = FLUX_HLLC;
    for (int s = 0; s < 4; s++) c->bnd.kind[s] = BC_OUTFLOW;
    const double mach3[4] = {1.4, 1.4 * 3.0, 0.0, 1.0 / 0.4 + 0.5 * 1.4 * 3.0 * 3.0};
    for (int k = 0; k < 4; k++) {
        c->bnd.inflow[k] = mach3[k];
        for (int s = 0; s < 4; s++) c->bnd.fixed[s][k] = mach3[k];
    }
    c->nstate = (size_t)4 * c->grid.rows * c->grid.cols;
    size_t bytes = c->nstate * sizeof(double);
    int rc = EB2_OK;
    auto bail = [&](int code) {
        eb2_ctx_destroy(c);
        return code;
    };
    if ((e = cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking)))
        return bail(fail(EB2_ECUDA, "stream: %s", cudaGetErrorString(e)));
    c->stream = c->own;
    if (cudaMalloc(&c->u, bytes) || cudaMalloc(&c->u1, bytes) || cudaMalloc(&c->u2, bytes))
        return bail(fail(EB2_ENOMEM, "device allocation of 3 x %zu bytes failed", bytes));
    c->npartials = stage_blocks_max(c->grid);
    if (c->npartials < 296) c->npartials = 296;
    if (cudaMalloc(&c->partials, 3 * sizeof(double) * c->npartials) ||
        cudaMalloc(&c->ctrl, sizeof(Ctrl)) || cudaMallocHost(&c->hctrl, sizeof(Ctrl)))
        return bail(fail(EB2_ENOMEM, "device allocation failed"));
    if (cudaMemsetAsync(c->u, 0, bytes, c->stream) || cudaMemsetAsync(c->u1, 0, bytes, c->stream) ||
        cudaMemsetAsync(c->u2, 0, bytes, c->stream) ||
        cudaMemsetAsync(c->ctrl, 0, sizeof(Ctrl), c->stream) ||
        cudaStreamSynchronize(c->stream))
        return bail(fail(EB2_ECUDA, "initialisation failed"));
    (void)rc;
    *out = c;
    return EB2_OK;
}

int eb2_ctx_destroy(eb2_ctx* c) {
    if (!c) return EB2_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    cudaFree(c->u);
    cudaFree(c->u1);
    cudaFree(c->u2);
    for (auto& t : c->tmp) cudaFree(t);
    cudaFree(c->partials);
    cudaFree(c->ctrl);
    cudaFreeHost(c->hctrl);
    if (c->gexec) cudaGraphExecDestroy(c->gexec);
    if (c->own) cudaStreamDestroy(c->own);
    delete c;
    return EB2_OK;
}

int eb2_set_stream(eb2_ctx* c, void* s) {
    if (int r = check(c)) return r;
    CK(cudaStreamSynchronize(c->stream));
    c->stream = s ? (cudaStream_t)s : c->own;
    return EB2_OK;
}

int eb2_set_material(eb2_ctx* c, double gamma, int source, double gravity, double cfl) {
    if (!c) return fail(EB2_EARG, "null context");
    if (!(gamma > 1.0)) return fail(EB2_EARG, "gamma must exceed 1");
    c->gas.gamma = gamma;
    c->gas.gm1 = gamma - 1.0;
    c->gas.gr = gamma / (gamma - 1.0);
    c->num.source = source ? 1 : 0;
    c->num.gravity = gravity;
    c->cfl = cfl;
    return EB2_OK;
}

int eb2_set_reconstruction(eb2_ctx* c, int recon, int characteristic, int weno_z) {
    if (!c) return fail(EB2_EARG, "null context");
    if (recon != 1 && recon != 2 && recon != 3 && recon != 5)
        return fail(EB2_EARG,
                    "The reconstruction program with the %d-th order has not been implemented.",
                    recon);
    c->num.recon = recon;
    c->num.characteristic = characteristic ? 1 : 0;
    c->num.weno_z = weno_z ? 1 : 0;
    return EB2_OK;
}

int eb2_set_precision(eb2_ctx* c, int precision) {
    if (!c) return fail(EB2_EARG, "null context");
    if (precision != EB2_FP64 && precision != EB2_MIXED)
        return fail(EB2_EARG, "precision %d unknown", precision);
    c->precision = precision;
    return EB2_OK;
}

int eb2_set_positivity_fallback(eb2_ctx* c, int on) {
    if (!c) return fail(EB2_EARG, "null context");
    c->num.positivity = on ? 1 : 0;
    return EB2_OK;
}

int eb2_set_bc(eb2_ctx* c, int left, int right, int bottom, int top) {
    if (!c) return fail(EB2_EARG, "null context");
    int k[4] = {left, right, bottom, top};
    int n[4] = {c->grid.nx, c->grid.nx, c->grid.ny, c->grid.ny};
    for (int s = 0; s < 4; s++) {
        if (k[s] < BC_OUTFLOW || k[s] > BC_FIXED) return fail(EB2_EARG, "bc kind %d", k[s]);
        if ((k[s] == BC_PERIODIC || (k[s] == BC_REFLECT && (s == 0 || s == 3))) && n[s] < GC)
            return fail(EB2_EUNSUPPORTED,
                        "a mirrored or periodic side needs at least %d interior cells", GC);
    }
    for (int s = 0; s < 4; s++) c->bnd.kind[s] = k[s];
    return EB2_OK;
}

int eb2_get_bc(eb2_ctx* c, int* kinds4) {
    if (!c || !kinds4) return fail(EB2_EARG, "null argument");
    for (int s = 0; s < 4; s++) kinds4[s] = c->bnd.kind[s];
    return EB2_OK;
}

int eb2_set_bc_states(eb2_ctx* c, const double* inflow4, const double* fixed16) {
    if (!c) return fail(EB2_EARG, "null context");
    if (inflow4) memcpy(c->bnd.inflow, inflow4, sizeof c->bnd.inflow);
    if (fixed16) memcpy(c->bnd.fixed, fixed16, sizeof c->bnd.fixed);
    return EB2_OK;
}

int eb2_set_double_mach(eb2_ctx* c, int on) {
    if (!c) return fail(EB2_EARG, "null context");
    if (on && c->grid.ny < GC) return fail(EB2_EUNSUPPORTED, "double-Mach wall needs ny >= 4");
    c->bnd.dmr = on ? 1 : 0;
    return EB2_OK;
}

}  // extern "C"

// Initial-state descriptor, domain lengths, final time and boundary kinds of
// test case tc (shared by eb2_init_case and the solve server).
int eb2::case_setup(int tc, const double* q, InitDesc& d, double* L, double& T, int* bc) {
    memset(&d, 0, sizeof d);
    L[0] = L[1] = 1.0;
    T = 0.0;
    for (int s = 0; s < 4; s++) bc[s] = BC_OUTFLOW;
    auto put = [&](int s, double r, double u, double v, double p) {
        d.st[s][0] = r; d.st[s][1] = u; d.st[s][2] = v; d.st[s][3] = p;
    };
    // initial states of include/initialize.h, primitive (rho, u, v, p)
    static const double riemann[5][4][4] = {
        // quadrants in the if-chain order (i<,j<), (i<,j>=), (i>=,j<), (i>=,j>=)
        {{2, -0.75, 0.5, 1}, {1, -0.75, -0.5, 1}, {1, 0.75, 0.5, 1}, {3, 0.75, -0.5, 1}},
        {{2, 0, -0.3, 1}, {1, 0, -0.4, 1}, {1.0625, 0, 0.2145, 0.4}, {0.5197, 0, -1.125, 0.4}},
        {{0.5065, 0.8939, 0, 0.35}, {1.5, 0, 0, 1.5}, {1.1, 0.8939, 0.8939, 1.1},
         {0.5065, 0, 0.8939, 0.35}},
        {{2, 0.75, 0.5, 1}, {1, 0.75, -0.5, 1}, {1, -0.75, 0.5, 1}, {3, -0.75, -0.5, 1}},
        {{1, -0.6259, 0.1, 1}, {0.5197, 0.1, 0.1, 0.4}, {0.8, 0.1, 0.1, 1}, {1, 0.1, -0.6259, 1}},
    };
    static const double riemann_t[5] = {0.23, 0.30, 0.25, 0.30, 0.25};
    switch (tc) {
        case EB2_CASE_PRECISION:  // initialize.h:36-60
            d.kind = INIT_SINE;
            L[0] = 2.0 * M_PI;
            T = 2.0;
            bc[0] = bc[1] = BC_PERIODIC;
            break;
        case EB2_CASE_SOD_1D:  // :70-110
            d.kind = INIT_HALF_X; d.full = 1;
            put(0, 1.0, 0.0, 0.0, 1.0);
            put(1, 0.125, 0.0, 0.0, 0.1);
            T = 0.2;
            break;
        case EB2_CASE_CONTACT_1D:  // :121-168
            d.kind = INIT_HALF_X; d.full = 1;
            put(0, 1.0, 0.0, 0.0, 1.0);
            put(1, 0.125, 0.0, 0.0, 1.0);
            T = 0.2;
            break;
        case EB2_CASE_SHOCK_IMPACT_1D:  // :172-219
            d.kind = INIT_HALF_X; d.full = 1;
            put(0, 1.0, 4.0, 0.0, 1.0);
            put(1, 1.0, -4.0, 0.0, 1.0);
            T = 0.2;
            break;
        case EB2_CASE_DOUBLE_RARE_1D:  // :223-269
            d.kind = INIT_HALF_X; d.full = 1;
            put(0, 1.0, -2.0, 0.0, 1.0);
            put(1, 1.0, 2.0, 0.0, 1.0);
            T = 0.15;
            break;
        case EB2_CASE_IMPACT_WALL_1D:  // :273-305
            d.kind = INIT_UNIFORM; d.full = 1;
            put(0, 1.0, 1.0, 0.0, 1.0);
            bc[1] = BC_REFLECT;
            T = 0.6;
            break;
        case EB2_CASE_NOH_1D:  // :315-347
            d.kind = INIT_UNIFORM; d.full = 1;
            put(0, 1.0, -1.0, 0.0, 1e-6);
            bc[0] = BC_REFLECT;
            T = 0.6;
            break;
        case 7: case 8: case 9: case 10: case 11: {  // :351-622
            d.kind = INIT_QUADRANT; d.full = 1;
            for (int s = 0; s < 4; s++)
                put(s, riemann[tc - 7][s][0], riemann[tc - 7][s][1], riemann[tc - 7][s][2],
                    riemann[tc - 7][s][3]);
            T = riemann_t[tc - 7];
            break;
        }
        case EB2_CASE_TAYLOR_GREEN:  // :626-683
            d.kind = INIT_FIELD;
            L[0] = L[1] = 2.0 * M_PI;
            T = 5.0;
            for (int s = 0; s < 4; s++) bc[s] = BC_PERIODIC;
            break;
        case EB2_CASE_GAUSSIAN_PULSE:  // :684-736
            d.kind = INIT_FIELD;
            L[0] = L[1] = 10.0;
            T = 4.0;
            break;
        case EB2_CASE_KELVIN_HELMHOLTZ:  // :737-835
            d.kind = INIT_FIELD;
            T = 2.0;
            for (int s = 0; s < 4; s++) bc[s] = BC_PERIODIC;
            break;
        case EB2_CASE_RAYLEIGH_TAYLOR:  // :836-889
            d.kind = INIT_FIELD;
            L[0] = 0.25;
            T = 1.95;
            bc[0] = bc[1] = BC_REFLECT;
            bc[2] = bc[3] = BC_FIXED;
            break;
        case EB2_CASE_BLAST_WAVE:  // :967-1060
            d.kind = INIT_FIELD;
            T = 0.01;
            for (int s = 0; s < 4; s++) bc[s] = BC_REFLECT;
            break;
        case EB2_CASE_NOH_2D:  // :1061-1185
            d.kind = INIT_FIELD;
            T = 0.6;
            for (int s = 0; s < 4; s++) bc[s] = BC_REFLECT;
            break;
        case EB2_CASE_ODD_EVEN:  // :1186-1296
            d.kind = INIT_FIELD;
            L[0] = 20.0;
            T = 2.0;
            bc[2] = bc[3] = BC_REFLECT;
            break;
        case EB2_CASE_BACKWARD_STEP:  // :1302-1388
            d.kind = INIT_FIELD;
            L[0] = 3.0;
            T = 4.0;
            bc[0] = BC_FIXED;
            bc[2] = bc[3] = BC_REFLECT;
            break;
        case EB2_CASE_DOUBLE_MACH:  // :890-952, boundary kinds :900-903
            d.kind = INIT_DMR;
            put(0, 8.0, 7.1447, -4.125, 116.5);
            put(1, 1.4, 0.0, 0.0, 1.0);
            L[0] = 4.0;
            T = 0.2;
            bc[0] = BC_INFLOW; bc[2] = BC_REFLECT; bc[3] = BC_REFLECT;
            break;
        case EB2_CASE_FOUR_QUADRANT: {
            static const double base[16] = {1.5, 0.0, 0.0, 1.5,     0.5323, 1.206, 0.0, 0.3,
                                             0.138, 1.206, 1.206, 0.029, 0.5323, 0.0, 1.206, 0.3};
            const double* s = q ? q : base;  // upper-right, upper-left, lower-left, lower-right
            d.kind = INIT_QUADRANT;
            const int map[4] = {2, 1, 3, 0};  // (x<,y<)=LL, (x<,y>=)=UL, (x>=,y<)=LR, (x>=,y>=)=UR
            for (int k = 0; k < 4; k++)
                put(k, s[4 * map[k]], s[4 * map[k] + 1], s[4 * map[k] + 2], s[4 * map[k] + 3]);
            T = 0.3;
            break;
        }
        case EB2_CASE_WALL_HEATING:
            d.kind = INIT_UNIFORM;
            put(0, 1.0, -(q ? q[0] : 1.0), 0.0, 1.0e-4);
            L[1] = 0.02;
            T = 0.6;
            bc[0] = BC_REFLECT; bc[2] = bc[3] = BC_PERIODIC;
            break;
        default:
            return fail(EB2_EUNSUPPORTED, "test case %d is not implemented", tc);
    }
    d.lx = L[0];
    d.ly = L[1];
    d.field_case = tc;
    return EB2_OK;
}

extern "C" {

int eb2_init_case(eb2_ctx* c, int tc, const double* q, double* lx, double* ly, double* tmax) {
    if (int r = check(c)) return r;
    InitDesc d;
    double L[2], T;
    int bc[4];
    if (int r = case_setup(tc, q, d, L, T, bc)) return r;
    if (int r = eb2_set_bc(c, bc[0], bc[1], bc[2], bc[3])) return r;
    c->bnd.dmr = 0;
    CK(launch_init(c->u, c->grid, c->gas, d, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (lx) *lx = L[0];
    if (ly) *ly = L[1];
    if (tmax) *tmax = T;
    return EB2_OK;
}

int eb2_init_case_fields(eb2_ctx* c, int tc, const double* q, double* pri, double* F,
                         double* G, double* lx, double* ly, double* tmax) {
    if (int r = check(c)) return r;
    InitDesc d;
    double L[2], T;
    int bc[4];
    if (int r = case_setup(tc, q, d, L, T, bc)) return r;
    if (int r = eb2_set_bc(c, bc[0], bc[1], bc[2], bc[3])) return r;
    if (int r = ensure_tmp(c, 3)) return r;
    c->bnd.dmr = 0;
    CK(launch_init(c->u, c->grid, c->gas, d, c->stream, c->tmp[0], c->tmp[1], c->tmp[2]));
    size_t b = c->nstate * sizeof(double);
    double* out[3] = {pri, F, G};
    for (int k = 0; k < 3; k++)
        if (out[k]) CK(cudaMemcpyAsync(out[k], c->tmp[k], b, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (lx) *lx = L[0];
    if (ly) *ly = L[1];
    if (tmax) *tmax = T;
    return EB2_OK;
}

int eb2_upload(eb2_ctx* c, const double* U) {
    if (int r = check(c)) return r;
    if (!U) return fail(EB2_EARG, "null host array");
    CK(cudaMemcpyAsync(c->u, U, c->nstate * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return EB2_OK;
}

int eb2_download(eb2_ctx* c, double* U) {
    if (int r = check(c)) return r;
    if (!U) return fail(EB2_EARG, "null host array");
    CK(cudaMemcpyAsync(U, c->u, c->nstate * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return EB2_OK;
}

int eb2_state_device_ptr(eb2_ctx* c, double** p) {
    if (!c || !p) return fail(EB2_EARG, "null argument");
    *p = c->u;
    return EB2_OK;
}

int eb2_bc_apply(eb2_ctx* c, double time) {
    if (int r = check(c)) return r;
    CK(launch_bc(c->u, c->grid, c->bnd, nullptr, time, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return EB2_OK;
}

int eb2_con_to_pri(eb2_ctx* c, double* pri) {
    if (int r = check(c)) return r;
    if (!pri) return fail(EB2_EARG, "null host array");
    if (int r = ensure_tmp(c, 1)) return r;
    CK(cudaMemcpyAsync(c->tmp[0], pri, c->nstate * sizeof(double), cudaMemcpyHostToDevice,
                       c->stream));
    CK(launch_con_to_pri(c->u, c->tmp[0], c->grid, c->gas, c->stream));
    CK(cudaMemcpyAsync(pri, c->tmp[0], c->nstate * sizeof(double), cudaMemcpyDeviceToHost,
                       c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return EB2_OK;
}

int eb2_eigen(eb2_ctx* c, int dir, const double* pri, double* el, double* er) {
    if (int r = check(c)) return r;
    if (dir != 1 && dir != 2) return fail(EB2_EARG, "dir must be 1 or 2");
    if (!pri || !el || !er) return fail(EB2_EARG, "null host array");
    size_t b4 = c->nstate * sizeof(double);
    double *dp = nullptr, *dl = nullptr, *dr = nullptr;
    CK(cudaMallocAsync(&dp, b4, c->stream));
    CK(cudaMallocAsync(&dl, 4 * b4, c->stream));
    CK(cudaMallocAsync(&dr, 4 * b4, c->stream));
    CK(cudaMemcpyAsync(dp, pri, b4, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(dl, el, 4 * b4, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(dr, er, 4 * b4, cudaMemcpyHostToDevice, c->stream));
    CK(launch_eigen(dir, dp, dl, dr, c->grid, c->gas, c->stream));
    CK(cudaMemcpyAsync(el, dl, 4 * b4, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(er, dr, 4 * b4, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaFreeAsync(dp, c->stream));
    CK(cudaFreeAsync(dl, c->stream));
    CK(cudaFreeAsync(dr, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return EB2_OK;
}

int eb2_reconstruct(eb2_ctx* c, int dir, double dx, double dy, double* ql, double* qr) {
    if (int r = check(c)) return r;
    if (dir != 1 && dir != 2) return fail(EB2_EARG, "dir must be 1 or 2");
    if (!ql || !qr) return fail(EB2_EARG, "null host array");
    if (int r = ensure_tmp(c, 2)) return r;
    set_spacing(c, dx, dy);
    size_t b = c->nstate * sizeof(double);
    CK(cudaMemcpyAsync(c->tmp[0], ql, b, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->tmp[1], qr, b, cudaMemcpyHostToDevice, c->stream));
    CK(launch_recon(dir, c->u, c->tmp[0], c->tmp[1], c->grid, c->gas, c->num, nullptr, c->stream));
    CK(cudaMemcpyAsync(ql, c->tmp[0], b, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(qr, c->tmp[1], b, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return EB2_OK;
}

int eb2_riemann(eb2_ctx* c, int scheme, int dir, const double* ql, const double* qr, double* f) {
    if (int r = check(c)) return r;
    if (dir != 1 && dir != 2) return fail(EB2_EARG, "dir must be 1 or 2");
    if (!ql || !qr || !f) return fail(EB2_EARG, "null host array");
    int flux;
    if (int r = map_scheme(scheme, &flux)) return r;
    if (int r = ensure_tmp(c, 3)) return r;
    size_t b = c->nstate * sizeof(double);
    CK(cudaMemcpyAsync(c->tmp[0], ql, b, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->tmp[1], qr, b, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->tmp[2], f, b, cudaMemcpyHostToDevice, c->stream));
    CK(launch_riemann(dir, c->tmp[0], c->tmp[1], c->tmp[2], c->grid, c->gas, flux,
                      &c->ctrl->status, c->stream));
    CK(cudaMemcpyAsync(f, c->tmp[2], b, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return EB2_OK;
}

int eb2_flux_reconstruction(eb2_ctx* c, int scheme, double dx, double dy, double* f, double* g) {
    if (int r = check(c)) return r;
    if (!f || !g) return fail(EB2_EARG, "null host array");
    int flux;
    if (int r = map_scheme(scheme, &flux)) return r;
    if (int r = ensure_tmp(c, 4)) return r;
    set_spacing(c, dx, dy);
    size_t b = c->nstate * sizeof(double);
    CK(cudaMemcpyAsync(c->tmp[2], f, b, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->tmp[3], g, b, cudaMemcpyHostToDevice, c->stream));
    CK(launch_recon(1, c->u, c->tmp[0], c->tmp[1], c->grid, c->gas, c->num, nullptr, c->stream));
    CK(launch_riemann(1, c->tmp[0], c->tmp[1], c->tmp[2], c->grid, c->gas, flux, &c->ctrl->status,
                      c->stream));
    CK(launch_recon(2, c->u, c->tmp[0], c->tmp[1], c->grid, c->gas, c->num, nullptr, c->stream));
    CK(launch_riemann(2, c->tmp[0], c->tmp[1], c->tmp[3], c->grid, c->gas, flux, &c->ctrl->status,
                      c->stream));
    CK(cudaMemcpyAsync(f, c->tmp[2], b, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(g, c->tmp[3], b, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return EB2_OK;
}

int eb2_space_discrete(eb2_ctx* c, double dx, double dy, const double* f, const double* g,
                       const double* s, double* L) {
    if (int r = check(c)) return r;
    if (!f || !g || !L) return fail(EB2_EARG, "null host array");
    if (int r = ensure_tmp(c, 4)) return r;
    set_spacing(c, dx, dy);
    size_t b = c->nstate * sizeof(double);
    CK(cudaMemcpyAsync(c->tmp[0], f, b, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->tmp[1], g, b, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->tmp[2], L, b, cudaMemcpyHostToDevice, c->stream));
    if (s) CK(cudaMemcpyAsync(c->tmp[3], s, b, cudaMemcpyHostToDevice, c->stream));
    CK(launch_space_item(c->tmp[0], c->tmp[1], s ? c->tmp[3] : nullptr, c->u, c->tmp[2], c->grid,
                         c->num, c->stream));
    CK(cudaMemcpyAsync(L, c->tmp[2], b, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return EB2_OK;
}

int eb2_wave_speeds(eb2_ctx* c, double* sx, double* sy) {
    if (int r = check(c)) return r;
    int nb = 0;
    CK(launch_wave_partials(c->u, c->grid, c->gas, c->partials, &nb, c->stream));
    CK(launch_finalize(c->ctrl, c->partials, nb, c->grid.nx * c->grid.ny, 0, c->stream));
    CK(cudaMemcpyAsync(c->hctrl, c->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (sx) *sx = c->hctrl->sx;
    if (sy) *sy = c->hctrl->sy;
    return EB2_OK;
}

int eb2_delta_t(eb2_ctx* c, double dx, double dy, double* dt) {
    if (int r = check(c)) return r;
    if (!dt) return fail(EB2_EARG, "null output");
    double dmin = dx > dy ? dy : dx;  // min_of_two (include/function.h:58-63)
    k_set_cfl<<<1, 1, 0, c->stream>>>(c->ctrl, c->cfl, dmin);
    CK(cudaGetLastError());
    if (int r = eb2_wave_speeds(c, nullptr, nullptr)) return r;
    *dt = c->hctrl->dt;
    return EB2_OK;
}

int eb2_rk_step(eb2_ctx* c, int order, int scheme, double dt, double dx, double dy,
                double time) {
    if (int r = check(c)) return r;
    if (order < 1 || order > 3) return fail(EB2_EARG, "Error: Invalid time advancement method");
    int flux;
    if (int r = map_scheme(scheme, &flux)) return r;
    if (int r = check_precision_flux(c, flux)) return r;
    c->num.flux = flux;
    set_spacing(c, dx, dy);
    unsigned before = 0, after = 0;
    if (int r = read_status(c, &before)) return r;
    if (c->precision == EB2_MIXED) {
        // the near-vacuum threshold of the mixed form needs the mean pressure
        int nb = 0;
        CK(launch_wave_partials(c->u, c->grid, c->gas, c->partials, &nb, c->stream));
        CK(launch_finalize(c->ctrl, c->partials, nb, c->grid.nx * c->grid.ny, 0, c->stream));
        c->launches += 2;
    }
    k_set_step<<<1, 1, 0, c->stream>>>(c->ctrl, time, dt);
    CK(cudaGetLastError());
    CK(enqueue_step(c, order));
    if (int r = read_status(c, &after)) return r;
    if ((after & ~before) & (ST_NONPHYSICAL | ST_NAN_STATE))
        return fail(EB2_ENONPHYS, "non-physical state met (status 0x%x)", after);
    return EB2_OK;
}

// RK1_TimeAd_BS (include/time_advance.h:886-1025): one forward-Euler step of
// the backward-step flow on two blocks, every part on the GPU.  Block 1 is
// the channel above the step (all nx rows, int(0.8 ny) columns starting
// int(0.2 ny) in), block 2 the inlet section beside the step (int(0.2 nx) x
// int(0.2 ny) at the lower left); the rest of the lower strip is the step and
// is not advanced.  Each block is gathered out of the state into a stage
// buffer of its own, its ghost layers are filled by BC_BackwardStep_2D's rules,
// the fused FP64 stage (flux reconstruction, flux difference, gravity source,
// Euler update) runs on it, and the block interiors are scattered back.  The
// FP64 stage runs whatever the context's precision: the reference's bits.
int eb2_rk1_backward_step(eb2_ctx* c, int scheme, double dt, double dx, double dy) {
    if (int r = check(c)) return r;
    const int G = GC;
    const int LNX = c->grid.nx, LNY = c->grid.ny;
    const int off = (int)(LNY * 0.2);
    Grid g1 = c->grid, g2 = c->grid;
    g1.rows = LNX + 2 * G;
    g1.cols = (int)(LNY * 0.8 + 2 * G);
    g2.rows = (int)(LNX * 0.2 + 2 * G);
    g2.cols = (int)(LNY * 0.2 + 2 * G);
    if (g2.rows < 2 * G + 1 || g2.cols < 2 * G + 1 || g1.cols < 2 * G + 1)
        return fail(EB2_EARG, "RK1_TimeAd_BS: grid %d x %d too small for the two blocks", LNX,
                    LNY);
    g1.nx = g1.rows - 2 * G;
    g1.ny = g1.cols - 2 * G;
    g2.nx = g2.rows - 2 * G;
    g2.ny = g2.cols - 2 * G;
    int flux;
    if (int r = map_scheme(scheme, &flux)) return r;
    c->num.flux = flux;
    set_spacing(c, dx, dy);
    g1.dx = g2.dx = c->grid.dx;
    g1.dy = g2.dy = c->grid.dy;
    g1.inv_dx = g2.inv_dx = c->grid.inv_dx;
    g1.inv_dy = g2.inv_dy = c->grid.inv_dy;
    if (int r = ensure_tmp(c, 2)) return r;
    // block 1 in u1 -> u2, block 2 in tmp[0] -> tmp[1] (each fits a state array)
    double *b1 = c->u1, *o1 = c->u2, *b2 = c->tmp[0], *o2 = c->tmp[1];
    Boundary in{};
    const double gm = c->gas.gamma;
    in.inflow[0] = 1.4;
    in.inflow[1] = 1.4 * 3.0;
    in.inflow[2] = 0.0;
    in.inflow[3] = 1.0 / (gm - 1) + 0.5 * 1.4 * 3 * 3;
    unsigned before = 0, after = 0;
    if (int r = read_status(c, &before)) return r;
    k_set_step<<<1, 1, 0, c->stream>>>(c->ctrl, 0.0, dt);
    CK(cudaGetLastError());
    CK(launch_bs_gather(c->u, c->grid, b1, g1, b2, g2, off, c->stream));
    CK(launch_bs_boundary(b1, g1, b2, g2, in, c->stream));
    double* ins[2] = {b1, b2};
    double* outs[2] = {o1, o2};
    const Grid* gs[2] = {&g1, &g2};
    for (int q = 0; q < 2; q++) {
        StageArgs a;
        a.uin = ins[q];
        a.un = ins[q];
        a.uout = outs[q];
        a.grid = *gs[q];
        a.gas = c->gas;
        a.num = c->num;
        a.combine = COMB_EULER;
        a.ctrl = c->ctrl;
        a.partials = nullptr;
        CK(launch_stage_fp64(a, c->stream));
    }
    CK(launch_bs_scatter(c->u, c->grid, o1, g1, o2, g2, off, c->stream));
    c->launches += 6;
    if (int r = read_status(c, &after)) return r;
    if ((after & ~before) & (ST_NONPHYSICAL | ST_NAN_STATE))
        return fail(EB2_ENONPHYS, "non-physical state met (status 0x%x)", after);
    return EB2_OK;
}

}  // extern "C"

namespace {
// Common set-up of a device time loop: numerics, spacing, control block and
// the first CFL time step.
int loop_setup(eb2_ctx* c, int order, int scheme, double dx, double dy, double t0, double tmax,
               double out_dt, long long max_step) {
    if (order < 1 || order > 3) return fail(EB2_EARG, "Error: Invalid time advancement method");
    int flux;
    if (int r = map_scheme(scheme, &flux)) return r;
    if (int r = check_precision_flux(c, flux)) return r;
    c->num.flux = flux;
    set_spacing(c, dx, dy);
    double dmin = dx > dy ? dy : dx;  // min_of_two (include/function.h:58-63)
    k_set_loop<<<1, 1, 0, c->stream>>>(c->ctrl, t0, tmax, out_dt, c->cfl, dmin, max_step);
    CK(cudaGetLastError());
    int nb = 0;
    CK(launch_wave_partials(c->u, c->grid, c->gas, c->partials, &nb, c->stream));
    CK(launch_finalize(c->ctrl, c->partials, nb, c->grid.nx * c->grid.ny, 1, c->stream));
    c->launches += 3;
    // set kernel attributes outside any capture
    StageArgs a{};
    a.grid = c->grid;
    a.num = c->num;
    CK(c->precision == EB2_MIXED ? launch_stage_mixed(a, c->stream)
                                 : launch_stage_fp64(a, c->stream));
    return EB2_OK;
}

// A CUDA graph of `per_graph` steps of the device loop, rebuilt only when the
// numerics, boundaries, spacing, order or length change.
int loop_graph(eb2_ctx* c, int order, int per_graph, cudaGraphExec_t* out) {
    unsigned char key[sizeof c->gkey];
    unsigned char* k = key;
    memcpy(k, &c->num, sizeof(Numerics)); k += sizeof(Numerics);
    memcpy(k, &c->bnd, sizeof(Boundary)); k += sizeof(Boundary);
    memcpy(k, &c->grid, sizeof(Grid)); k += sizeof(Grid);
    int tail[4] = {order, per_graph, c->precision, 0};
    memcpy(k, tail, sizeof tail);
    if (c->gexec && memcmp(key, c->gkey, sizeof key) == 0) {
        *out = c->gexec;
        return EB2_OK;
    }
    if (c->gexec) {
        cudaGraphExecDestroy(c->gexec);
        c->gexec = nullptr;
    }
    const int nstage = stage_blocks(c->grid, c->precision == EB2_MIXED);
    const long long cells = (long long)c->grid.nx * c->grid.ny;
    cudaGraph_t graph = nullptr;
    long long launches0 = c->launches;
    CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t ce = cudaSuccess;
    for (int s = 0; s < per_graph && ce == cudaSuccess; s++) {
        ce = enqueue_step(c, order);
        if (ce == cudaSuccess)
            ce = launch_finalize(c->ctrl, c->partials, nstage, (int)cells, 2, c->stream);
    }
    cudaError_t ee = cudaStreamEndCapture(c->stream, &graph);
    c->launches = launches0;  // captured launches are counted when the graph runs
    if (ce != cudaSuccess || ee != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        return fail(EB2_ECUDA, "graph capture: %s",
                    cudaGetErrorString(ce != cudaSuccess ? ce : ee));
    }
    ce = cudaGraphInstantiate(&c->gexec, graph, 0);
    cudaGraphDestroy(graph);
    if (ce != cudaSuccess) {
        c->gexec = nullptr;
        return fail(EB2_ECUDA, "graph instantiate: %s", cudaGetErrorString(ce));
    }
    memcpy(c->gkey, key, sizeof key);
    *out = c->gexec;
    return EB2_OK;
}

int steps_per_graph(const eb2_ctx* c) {
    long long cells = (long long)c->grid.nx * c->grid.ny;
    return cells >= (1LL << 22) ? 4 : (cells >= (1LL << 18) ? 8 : 32);
}

int launches_per_step(int order) { return 2 * order + 1 + (order == 1 ? 1 : 0); }

// Launch graphs until the loop stops; service output pauses.
int loop_drive(eb2_ctx* c, int order, eb2_output_fn cb, void* user) {
    const int per = steps_per_graph(c);
    cudaGraphExec_t exec = nullptr;
    if (int r = loop_graph(c, order, per, &exec)) return r;
    long long prev_step = 0;
    for (;;) {
        cudaError_t ce = cudaGraphLaunch(exec, c->stream);
        if (ce == cudaSuccess)
            ce = cudaMemcpyAsync(c->hctrl, c->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost,
                                 c->stream);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(c->stream);
        if (ce != cudaSuccess) return fail(EB2_ECUDA, "time loop: %s", cudaGetErrorString(ce));
        c->launches += (c->hctrl->step - prev_step) * launches_per_step(order);
        prev_step = c->hctrl->step;
        if (c->hctrl->out_pending) {
            if (cb) cb(user, c->hctrl->t, c->hctrl->step);
            k_resume<<<1, 1, 0, c->stream>>>(c->ctrl);
            CK(cudaGetLastError());
            continue;
        }
        if (!c->hctrl->active) break;
    }
    if (c->hctrl->status & ST_BAD_DT) return fail(EB2_ENONPHYS, "time step became invalid");
    return EB2_OK;
}

}  // namespace

extern "C" {

int eb2_run(eb2_ctx* c, int order, int scheme, double dx, double dy, double t0, double tmax,
            int n_out, eb2_output_fn cb, void* user, long long* steps, double* t_final) {
    if (int r = check(c)) return r;
    if (n_out < 1) return fail(EB2_EARG, "n_out must be >= 1");
    if (int r = loop_setup(c, order, scheme, dx, dy, t0, tmax, tmax / n_out, LLONG_MAX)) return r;
    int rc = loop_drive(c, order, cb, user);
    if (steps) *steps = c->hctrl->step;
    if (t_final) *t_final = c->hctrl->t;
    return rc;
}

int eb2_advance(eb2_ctx* c, int order, int scheme, double dx, double dy, int nsteps) {
    if (int r = check(c)) return r;
    if (nsteps < 0) return fail(EB2_EARG, "nsteps must be >= 0");
    if (nsteps == 0) return EB2_OK;
    const double inf = HUGE_VAL;
    if (int r = loop_setup(c, order, scheme, dx, dy, 0.0, inf, inf, nsteps)) return r;
    return loop_drive(c, order, nullptr, nullptr);
}

int eb2_bench_steps(eb2_ctx* c, int order, int scheme, double dx, double dy, int nsteps,
                    unsigned long long flush_bytes, float* step_ms, float* stage_ms,
                    int* stage_launches, long long* launches) {
    if (int r = check(c)) return r;
    if (nsteps < 1 || !step_ms) return fail(EB2_EARG, "need nsteps >= 1 and step_ms");
    const double inf = HUGE_VAL;
    if (int r = loop_setup(c, order, scheme, dx, dy, 0.0, inf, inf, nsteps)) return r;
    void* flush = nullptr;
    if (flush_bytes) CK(cudaMalloc(&flush, flush_bytes));
    const int nev = 2 * nsteps + 2 * order * nsteps;
    cudaEvent_t* ev = (cudaEvent_t*)calloc(nev, sizeof(cudaEvent_t));
    if (!ev) return fail(EB2_ENOMEM, "host allocation failed");
    int rc = EB2_OK;
    for (int q = 0; q < nev && rc == EB2_OK; q++)
        if (cudaEventCreate(&ev[q]) != cudaSuccess) rc = fail(EB2_ECUDA, "cudaEventCreate");
    const int nstage = stage_blocks(c->grid, c->precision == EB2_MIXED);
    const long long cells = (long long)c->grid.nx * c->grid.ny;
    long long l0 = c->launches;
    for (int s = 0; s < nsteps && rc == EB2_OK; s++) {
        cudaError_t e = cudaSuccess;
        if (flush) e = cudaMemsetAsync(flush, s & 0xff, flush_bytes, c->stream);
        if (!e) e = cudaEventRecord(ev[2 * s], c->stream);
        if (!e) e = enqueue_step(c, order, ev + 2 * nsteps + 2 * order * s);
        if (!e) e = launch_finalize(c->ctrl, c->partials, nstage, (int)cells, 2, c->stream);
        c->launches++;
        if (!e) e = cudaEventRecord(ev[2 * s + 1], c->stream);
        if (e) rc = fail(EB2_ECUDA, "bench step %d: %s", s, cudaGetErrorString(e));
    }
    if (rc == EB2_OK) {
        cudaError_t e = cudaStreamSynchronize(c->stream);
        if (e) rc = fail(EB2_ECUDA, "bench: %s", cudaGetErrorString(e));
    }
    float tot = 0.0f;
    for (int s = 0; s < nsteps && rc == EB2_OK; s++) {
        cudaEventElapsedTime(&step_ms[s], ev[2 * s], ev[2 * s + 1]);
        for (int st = 0; st < order; st++) {
            float ms = 0.0f;
            cudaEvent_t* q = ev + 2 * nsteps + 2 * order * s + 2 * st;
            cudaEventElapsedTime(&ms, q[0], q[1]);
            tot += ms;
        }
    }
    if (stage_ms) *stage_ms = tot;
    if (stage_launches) *stage_launches = order * nsteps;
    if (launches) *launches = c->launches - l0;
    for (int q = 0; q < nev; q++)
        if (ev[q]) cudaEventDestroy(ev[q]);
    free(ev);
    if (flush) cudaFree(flush);
    return rc;
}

int eb2_status(eb2_ctx* c, unsigned* flags) {
    if (int r = check(c)) return r;
    if (!flags) return fail(EB2_EARG, "null output");
    return read_status(c, flags);
}

int eb2_clear_status(eb2_ctx* c) {
    if (int r = check(c)) return r;
    k_clear_status<<<1, 1, 0, c->stream>>>(c->ctrl);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(c->stream));
    return EB2_OK;
}

int eb2_synchronize(eb2_ctx* c) {
    if (int r = check(c)) return r;
    CK(cudaStreamSynchronize(c->stream));
    return EB2_OK;
}

}  // extern "C"
