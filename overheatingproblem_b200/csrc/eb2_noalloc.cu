// eb2_noalloc.cu -- one SSP-RK step that allocates no memory.
//
// Some callers cannot call cudaMalloc: code that runs while another framework
// owns every byte of device memory through its own pool, real-time loops where
// allocation after start-up is forbidden because it can block or fail, and
// plug-ins that only ever see device pointers handed to them.  For them this
// file keeps the step's scratch -- the two RK stage states and the device
// control block -- in one statically sized __device__ array, so that the
// caller supplies only the state, in and out.  The array is part of the
// library image: every GPU that loads the library holds it until the process
// exits.
//
// The host-side name g_scratch is only a stand-in for the device array: a
// kernel handed it would fault or read the wrong memory.  Every call asks
// cudaGetSymbolAddress for the array's address in the calling thread's current
// context, with the target device current, and hands that address to the
// kernels.  A module-scope __device__ array has one copy per CUDA context, so
// an address remembered from an earlier call could belong to another context
// (one the caller created with the driver API, or a primary context that
// cudaDeviceReset has since replaced); the lookup is not a stream operation and
// costs far less than the step.
#include <cstdio>
#include <cstring>

#include "../../include/euler_b200.h"
#include "eb2_kernels.h"

using namespace eb2;

namespace {

constexpr size_t kCtrlBytes = 256;
constexpr size_t kScratchBytes =
    kCtrlBytes + 2 * 4 * sizeof(double) * (size_t)EB2_NOALLOC_MAX_CELLS;

// The scratch array.  All calls share it and it keeps the last call's contents.
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

__global__ void k_noalloc_begin(Ctrl* c, double t, double dt) {
    // the control block must start from zero on every call
    memset(c, 0, sizeof(Ctrl));
    c->t = t;
    c->dt = dt;
    c->active = 1;
    c->host_dt = 1;
}

// failures are reported through eb2_last_error() like every other entry point
int fail(int code, const char* msg, cudaError_t e = cudaSuccess) {
    char buf[256];
    snprintf(buf, sizeof buf, "%s%s%s", msg, e ? ": " : "", e ? cudaGetErrorString(e) : "");
    eb2::set_last_error(buf);
    return code;
}

}  // namespace

extern "C" int eb2_rk_step_noalloc(double* U, int nx, int ny, const eb2_noalloc_config* cfg,
                                   int order, int scheme, double dt, double dx, double dy,
                                   double time, void* cuda_stream) {
    if (!U || !cfg) return fail(EB2_EARG, "null argument");
    if (nx < 1 || ny < 1) return fail(EB2_EARG, "empty grid");
    if (order < 1 || order > 3) return fail(EB2_EARG, "order must be 1, 2 or 3");
    const long long rows = nx + 2LL * GC, cols = ny + 2LL * GC;
    if (rows * cols > (long long)EB2_NOALLOC_MAX_CELLS)
        return fail(EB2_EARG, "grid exceeds EB2_NOALLOC_MAX_CELLS (rows*cols incl. ghosts)");
    if (cfg->recon != 1 && cfg->recon != 2 && cfg->recon != 3 && cfg->recon != 5)
        return fail(EB2_EARG, "recon must be 1, 2, 3 or 5");
    if (!(cfg->gamma > 1.0)) return fail(EB2_EARG, "gamma must exceed 1");
    int kind[4] = {cfg->bc_left, cfg->bc_right, cfg->bc_bottom, cfg->bc_top};
    for (int s = 0; s < 4; s++) {
        if (kind[s] < BC_OUTFLOW || kind[s] > BC_FIXED) return fail(EB2_EARG, "bad bc kind");
        int n = s < 2 ? nx : ny;
        if ((kind[s] == BC_PERIODIC || (kind[s] == BC_REFLECT && (s == 0 || s == 3))) && n < GC)
            return fail(EB2_EUNSUPPORTED, "mirrored or periodic side needs 4 interior cells");
    }
    // the device address of the scratch array in the current context (the
    // first call in a context also loads the library's module there)
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
    if (e) return fail(EB2_ECUDA, "cudaGetSymbolAddress", e);
    unsigned char* base = (unsigned char*)p;
    Ctrl* ctrl = (Ctrl*)base;
    const size_t nstate = (size_t)4 * rows * cols;
    double* u1 = (double*)(base + kCtrlBytes);
    double* u2 = u1 + nstate;
    cudaStream_t s = (cudaStream_t)cuda_stream;

    Grid g{};
    g.nx = nx;
    g.ny = ny;
    g.rows = (int)rows;
    g.cols = (int)cols;
    g.dx = dx;
    g.dy = dy;
    g.inv_dx = 1.0 / dx;
    g.inv_dy = 1.0 / dy;
    Gas gas{cfg->gamma, cfg->gamma - 1.0, cfg->gamma / (cfg->gamma - 1.0)};
    Numerics num{};
    num.recon = cfg->recon;
    num.characteristic = cfg->characteristic ? 1 : 0;
    num.weno_z = cfg->weno_z ? 1 : 0;
    // AR_scheme numbering of Flux_Reconstruction_RP (include/CFD_convection.h:334-362)
    num.flux = scheme == 1    ? FLUX_HLL
               : scheme == 2  ? FLUX_HLLC
               : scheme == 3  ? FLUX_ROE
               : scheme == 11 ? FLUX_HLLHC
               : scheme == 22 ? FLUX_HLLCHC
               : scheme == 33 ? FLUX_ROEHC
                              : FLUX_LLF;
    num.source = cfg->source ? 1 : 0;
    num.gravity = cfg->gravity;
    Boundary b{};
    const double mach3[4] = {1.4, 1.4 * 3.0, 0.0, 1.0 / 0.4 + 0.5 * 1.4 * 3.0 * 3.0};
    for (int k = 0; k < 4; k++) {
        b.kind[k] = kind[k];
        b.inflow[k] = mach3[k];
        for (int q = 0; q < 4; q++) b.fixed[q][k] = mach3[k];
    }

    k_noalloc_begin<<<1, 1, 0, s>>>(ctrl, time, dt);
    if ((e = cudaGetLastError())) return fail(EB2_ECUDA, "launch", e);
    double* in[3] = {U, u1, u2};
    double* out[3][3] = {{U, nullptr, nullptr}, {u1, U, nullptr}, {u1, u2, U}};
    const int comb[3][3] = {{COMB_EULER, 0, 0}, {COMB_EULER, COMB_RK2, 0},
                            {COMB_EULER, COMB_RK3_2, COMB_RK3_3}};
    for (int st = 0; st < order; st++) {
        if ((e = launch_bc(in[st], g, b, ctrl, 0.0, s))) return fail(EB2_ECUDA, "bc", e);
        StageArgs a{};
        a.uin = in[st];
        a.un = U;
        // first-order steps write into the first stage buffer, then copy back
        a.uout = order == 1 ? u1 : out[order - 1][st];
        a.grid = g;
        a.gas = gas;
        a.num = num;
        a.combine = comb[order - 1][st];
        a.ctrl = ctrl;
        a.partials = nullptr;
        if ((e = launch_stage_fp64(a, s))) return fail(EB2_ECUDA, "stage", e);
    }
    if (order == 1 && (e = launch_copy_interior(U, u1, g, s))) return fail(EB2_ECUDA, "copy", e);
    unsigned status = 0;
    if ((e = cudaMemcpyAsync(&status, &ctrl->status, sizeof status, cudaMemcpyDeviceToHost, s)))
        return fail(EB2_ECUDA, "status read", e);
    if ((e = cudaStreamSynchronize(s))) return fail(EB2_ECUDA, "synchronize", e);
    if (status & (ST_NONPHYSICAL | ST_NAN_STATE))
        return fail(EB2_ENONPHYS, "non-physical state met");
    return EB2_OK;
}
