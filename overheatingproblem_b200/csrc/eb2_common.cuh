// eb2_common.cuh -- layout, constants and the device control block shared by
// every kernel of libeuler_b200.
//
// HBM layout of one solve's state is the reference's own: double
// U[4][rows][cols], rows = nx + 2*GC (x, index i), cols = ny + 2*GC (y, index
// j, unit stride), GC = 4 ghost layers (include/Golbal.h:49 of the reference).
// Keeping it lets host buffers of the reference API be copied in and out with
// one memcpy per field plane set.
#pragma once

#include <cstdint>
#include <cstring>
#include <cuda_runtime.h>

// Point arithmetic is host-and-device so that it can also be exercised on the
// CPU (eb2_pointcheck.cu).
#define EB2_HD __host__ __device__ __forceinline__

namespace eb2 {

constexpr int GC = 4;      // ghost layers
constexpr int NV = 4;      // conserved fields: rho, rho*u, rho*v, rho*E

// Status bits raised by kernels (atomicOr into Ctrl::status).
enum : unsigned {
    ST_NONPHYSICAL = 1u << 0,   // reconstructed rho<=0, p<=0 or NaN at an interface
    ST_NAN_STATE = 1u << 1,     // NaN in an updated conserved state
    ST_BAD_DT = 1u << 2,        // non-finite or non-positive CFL time step
};

// Boundary kinds, numbered as BC_Type (include/Boundary_Condition.h:21-27).
enum : int { BC_OUTFLOW = 0, BC_REFLECT = 1, BC_PERIODIC = 2, BC_INFLOW = 3, BC_FIXED = 4 };

// Riemann solvers, numbered as AR_scheme (include/CFD_convection.h:89-117).
// Every value other than 1/2/3/11/22/33 selects the local Lax-Friedrichs flux.
enum : int { FLUX_LLF = 0, FLUX_HLL = 1, FLUX_HLLC = 2, FLUX_ROE = 3,
             FLUX_HLLHC = 4, FLUX_HLLCHC = 5, FLUX_ROEHC = 6 };  // 11, 22, 33

// Ideal-gas constants as the reference forms them at run time:
// gm1 = M_gamma - 1.0, gr = M_gamma / (M_gamma - 1.0).
struct Gas {
    double gamma, gm1, gr;
};

// Device-resident solve control block: the host time loop of src/RP_FVM.c
// (:179-267) moved onto the GPU so that whole step sequences can run as one
// CUDA graph without host round trips.
struct Ctrl {
    double t;          // time at the start of the current step (global Time)
    double dt;         // time step of the current step
    double tmax;       // final time
    double out_dt;     // output interval Tmax / Control_output
    double next_out;   // next output time
    double cfl;        // CFL number
    double dmin;       // min(dx, dy)
    double sx, sy;     // last wave-speed maxima
    double pmean;      // mean interior pressure of the last reduced state
    long long step;    // completed steps (Ite)
    long long max_step;  // the loop also stops after this many steps
    int active;        // 1 while t < tmax and no output is pending
    int out_pending;   // an output time was reached at the end of the last step
    int host_dt;       // 1: dt is supplied by the host, no clipping
    unsigned status;   // ST_* bits
};

// Per-solve geometry and numerics passed by value to kernels.
struct Grid {
    int nx, ny, rows, cols;
    double dx, dy, inv_dx, inv_dy;
};

struct Numerics {
    int recon;            // 1 Godunov, 2 TVD, 5 WENO5
    int characteristic;   // reconstruct in characteristic variables
    int weno_z;           // characteristic WENO5 with WENO-Z weights
    int flux;             // FLUX_*
    int source;           // gravity source term
    double gravity;
    int positivity;       // first-order fallback at interfaces with rho<=0/p<=0
};

struct Boundary {
    int kind[4];          // left, right, bottom, top (BC_*)
    int dmr;              // exact double-Mach boundary (BC_DoubleMach_2D)
    double inflow[4];     // conserved inflow state
    double fixed[4][4];   // conserved fixed states per side
};

__host__ __device__ inline size_t at(int k, int i, int j, int rows, int cols) {
    return ((size_t)k * rows + (size_t)i) * (size_t)cols + (size_t)j;
}

}  // namespace eb2
