// eb2_kernels.h -- launch interface between the host runtime (eb2_api.cu)
// and the kernel translation units.
#pragma once

#include "eb2_common.cuh"

namespace eb2 {

// How a stage combines its flux difference L with the step's start state y
// and the stage input x (include/time_advance.h:694-701, 753-777, 831-872).
enum : int {
    COMB_EULER = 0,   // out = y + dt*L           (RK1; stage 1 of RK2/RK3, x == y)
    COMB_RK2 = 1,     // out = 0.5*y + 0.5*(x + dt*L)
    COMB_RK3_2 = 2,   // out = 3/4*y + 1/4*(x + dt*L)
    COMB_RK3_3 = 3,   // out = 1/3*y + 2/3*(x + dt*L)
};

struct StageArgs {
    const double* uin;    // stage input, ghosts filled
    const double* un;     // state at the start of the step
    double* uout;         // stage output (interior only)
    Grid grid;
    Gas gas;
    Numerics num;
    int combine;          // COMB_*
    Ctrl* ctrl;           // dt, active flag, status
    double* partials;     // per-block {max|u|+a, max|v|+a, sum p} of uout, or null
};

// Message returned by eb2_last_error() for the calling thread (not exported).
void set_last_error(const char* msg);

// Fused x+y sweep + RK combine, FP64 bit-parity form.
cudaError_t launch_stage_fp64(const StageArgs& a, cudaStream_t s);
// Same contract, mixed precision (FP32 reconstruction and fluxes).
cudaError_t launch_stage_mixed(const StageArgs& a, cudaStream_t s);
// Tile of one stage block (x rows by y columns).  FP64 form: 15 x 32 cells, so
// that its 16 x 32 x faces and 15 x 33 y faces (1007) fill four passes of
// 256 threads; mixed form: 16 x 32.
constexpr int FP64_TILE_X = 15, MIXED_TILE_X = 16, STAGE_TILE_Y = 32;
// The mixed stage kernels write one CFL partial triple per 8-row x 32-column
// block, whatever their tile shape (each tile shape's rows are a multiple of 8).
constexpr int MIXED_PARTIAL_ROWS = 8;
// Threads of the end-of-step reduction block (single solves and the server
// alike, so that both sum the partials in the same order).
constexpr int FINALIZE_THREADS = 1024;
// Blocks of one stage launch of the given form, and the most of either form
// (the size of a partials buffer).
int stage_blocks(const Grid& g, bool mixed);
int stage_blocks_max(const Grid& g);

// Ghost-cell fill of one state at the time held in ctrl->t (or `time` when
// ctrl is null).
cudaError_t launch_bc(double* u, const Grid& g, const Boundary& b, const Ctrl* ctrl,
                      double time, cudaStream_t s);

// Wave-speed partials of the interior of u (the reduction of Get_Delta_T_2D).
cudaError_t launch_wave_partials(const double* u, const Grid& g, const Gas& gas,
                                 double* partials, int* nblocks, cudaStream_t s);
// Reduce partials into ctrl: mode 0 = plain dt (granular API), mode 1 = start
// of a device time loop, mode 2 = end of a step of the device time loop.
cudaError_t launch_finalize(Ctrl* ctrl, const double* partials, int nblocks, int ncells,
                            int mode, cudaStream_t s);

// Interior copy src -> dst (RK1 writes its stage into scratch first).
cudaError_t launch_copy_interior(double* dst, const double* src, const Grid& g,
                                 cudaStream_t s);

// The backward-step flow's two-block step (RK1_TimeAd_BS): block interiors
// out of U (block 1 starting `off` columns in), the ghost layers of both
// blocks (Boundary::inflow holds the inflow state), block interiors back.
cudaError_t launch_bs_gather(const double* u, const Grid& g, double* b1, const Grid& g1,
                             double* b2, const Grid& g2, int off, cudaStream_t s);
cudaError_t launch_bs_boundary(double* b1, const Grid& g1, double* b2, const Grid& g2,
                               const Boundary& inflow, cudaStream_t s);
cudaError_t launch_bs_scatter(double* u, const Grid& g, const double* b1, const Grid& g1,
                              const double* b2, const Grid& g2, int off, cudaStream_t s);

// Granular reference entry points (one thread per interface or cell).
cudaError_t launch_con_to_pri(const double* u, double* pri, const Grid& g, const Gas& gas,
                              cudaStream_t s);
cudaError_t launch_eigen(int dir, const double* pri, double* el, double* er, const Grid& g,
                         const Gas& gas, cudaStream_t s);
cudaError_t launch_recon(int dir, const double* u, double* ql, double* qr, const Grid& g,
                         const Gas& gas, const Numerics& n, unsigned* status, cudaStream_t s);
cudaError_t launch_riemann(int dir, const double* ql, const double* qr, double* f,
                           const Grid& g, const Gas& gas, int flux, unsigned* status,
                           cudaStream_t s);
cudaError_t launch_space_item(const double* f, const double* gflux, const double* src,
                              const double* u,
                              double* lout, const Grid& g, const Numerics& n, cudaStream_t s);

// Initial states.
struct InitDesc {
    int kind;             // INIT_*
    int full;             // fill ghosts too (the reference's 1D/Riemann cases)
    double st[4][4];      // primitive states (rho, u, v, p)
    double lx, ly;
    int field_case;       // INIT_FIELD: the test case host_case_field evaluates
};
enum : int { INIT_UNIFORM = 0, INIT_HALF_X = 1, INIT_QUADRANT = 2, INIT_DMR = 3, INIT_SINE = 4,
             INIT_FIELD = 5 };

// Host evaluation of the primitive field of the test cases whose reference
// initialisers call libm or rand() (eb2_cases.cu): w[4][rows][cols], zeroed by
// the caller.  Returns false for any other case.
bool host_case_field(int tc, int rows, int cols, double gamma, double lx, double ly, double* w);

// Initial state, domain lengths L[2], final time and boundary kinds bc[4] of
// an EB2_CASE_* test case (eb2_api.cu).  Returns EB2_OK or an EB2_E* code.
int case_setup(int tc, const double* q, InitDesc& d, double* L, double& T, int* bc);

// Context-free pieces of the device loop (eb2_api.cu).
void set_loop_ctrl(Ctrl* c, double t0, double tmax, double out_dt, double cfl, double dmin,
                   long long max_step, cudaStream_t s);
// Writes the conserved state; pri (the case's primitives) and the initial
// physical fluxes fx, gy (initEulerflux2D) too when not null.
cudaError_t launch_init(double* u, const Grid& g, const Gas& gas, const InitDesc& d,
                        cudaStream_t s, double* pri = nullptr, double* fx = nullptr,
                        double* gy = nullptr);

}  // namespace eb2
