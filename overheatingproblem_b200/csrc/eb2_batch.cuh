// eb2_batch.cuh -- batched kernels of the solve server: many independent
// solves of different sizes advanced together, each with its own time step.
//
// Every solve ("slot") has a descriptor in device memory.  A device-resident
// work list holds one (slot, tile) pair per tile of every active slot; the
// stage kernels run a persistent grid whose CTAs walk that list, so one launch
// advances a stage of all slots and small solves share the GPU with large ones.
// Boundary fill and the end-of-step reduction run one block row per slot.
// The per-tile work is the single-solve kernels' own stage_tile, so a slot
// evolves bit for bit as the same solve run alone.
#pragma once

#include "eb2_kernels.h"

namespace eb2 {

// Tile shapes the batched mixed kernels come in (eb2_stage_mixed.cuh: 16 x 32
// cells and 256 threads, 8 x 32 and 128, 32 x 32 and 512); an FP64 server has
// one, the FP64 form's 15 x 32.
constexpr int kMixedShapes = 3;

struct SlotDesc {
    double* u;            // state
    double* u1;           // stage 1 output
    double* u2;           // stage 2 output
    double* partials;     // CFL partials (npartials triples)
    Ctrl* ctrl;           // control block of this solve
    Grid grid;
    Gas gas;
    Numerics num;
    Boundary bnd;
    int tiles_x;          // tiles along y (32 columns in every shape)
    int ntiles[kMixedShapes];  // tiles of the slot in each tile shape
    int ncells;
    int npartials;        // CFL partial triples its stage kernels write (mixed: per
                          // 8 x 32 block in every tile shape; FP64: per tile)
    int bc_blocks;        // ghost-fill blocks of this slot (its entries in the bc work list)
};

// Stage buffers of SSP-RK3 (the server runs third-order steps only).
__host__ __device__ __forceinline__ void rk3_buffers(const SlotDesc& s, int stage, const double*& in,
                                            double*& out, int& comb) {
    if (stage == 0) { in = s.u; out = s.u1; comb = COMB_EULER; }
    else if (stage == 1) { in = s.u1; out = s.u2; comb = COMB_RK3_2; }
    else { in = s.u2; out = s.u; comb = COMB_RK3_3; }
}

// (on the host too: the stage arguments of a slot with a launch of its own)
__host__ __device__ __forceinline__ StageArgs slot_args(const SlotDesc& s, int stage) {
    StageArgs a;
    rk3_buffers(s, stage, a.uin, a.uout, a.combine);
    a.un = s.u;
    a.grid = s.grid;
    a.gas = s.gas;
    a.num = s.num;
    a.ctrl = s.ctrl;
    a.partials = stage == 2 ? s.partials : nullptr;
    return a;
}

// Host-side launch interface (eb2_batch_fp64.cu / eb2_batch_mixed.cu).  The
// three work lists are rewritten on admission and retirement only; the
// kernels read their lengths from device memory, so that a captured launch
// stays valid while its grid covers the list (grids are sized to powers of two).
struct BatchLaunch {
    const SlotDesc* slots;   // device array of nslots descriptors
    int nslots;
    const int2* work;        // device work list of the stage kernels: (slot, tile)
    const int* nwork;        // device: its length
    int grid;                // CTAs of the stage kernels
    const int2* bc_work;     // device work list of the ghost fill: (slot, block of the slot)
    const int* nbc;          // device: its length
    int bc_grid;             // blocks of the ghost fill (>= *nbc)
    const int* active;       // device list of the active slots (end-of-step reduction)
    const int* nactive;      // device: its length
    int active_grid;         // blocks of the end-of-step reduction (>= *nactive)
    int each = 0;            // 1: one CTA per work item (grid >= every work-list
                             // length it is used with), 0: persistent CTAs that loop
    int shape = 0;           // tile shape of the stage kernels (index into the shapes)
};
cudaError_t launch_stage_batch_fp64(const BatchLaunch& b, const Numerics& num, int stage,
                                    cudaStream_t s);
cudaError_t launch_stage_batch_mixed(const BatchLaunch& b, const Numerics& num, int stage,
                                     cudaStream_t s);
// One stage of one slot as a launch of its own (the single-solve grid of tiles
// in batched tile shape `shape`, the arguments in the kernel's parameter
// block): the server gives this to slots that fill the GPU by themselves.
cudaError_t launch_stage_slot_mixed(const StageArgs& a, const Numerics& num, int shape,
                                    cudaStream_t s);
cudaError_t launch_bc_batch(const BatchLaunch& b, int stage, cudaStream_t s);
cudaError_t launch_finalize_batch(const BatchLaunch& b, cudaStream_t s);
// Tile shapes of a server's stage kernels (1 for FP64, kMixedShapes for the
// mixed form), their tile rows, and their resident CTAs per SM.
int batch_shapes(int precision);
int batch_shape_tile_x(int precision, int shape);
int stage_batch_max_blocks_per_sm(int precision, int shape);

}  // namespace eb2
