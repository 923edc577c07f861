// eb2_batch_fp64.cu -- batched stage (FP64 form), boundary and end-of-step
// kernels of the solve server.  Built with -fmad=false like the single-solve
// FP64 kernels, whose per-tile body it reuses.
#include "eb2_batch.cuh"
#include "eb2_loop.cuh"
#include "eb2_stage_fp64.cuh"

namespace eb2 {

template <int RECON, bool CHAR, bool WZ, int FLUX>
__global__ void __launch_bounds__(fp64stage::NT, 2)
    k_stage_batch(const SlotDesc* __restrict__ slots, const int2* __restrict__ work,
                  const int* __restrict__ nwork, int stage) {
    const int n = *nwork;
    for (int w = blockIdx.x; w < n; w += gridDim.x) {
        const int2 it = work[w];
        const SlotDesc& sd = slots[it.x];
        const StageArgs a = slot_args(sd, stage);
        const int ti = it.y / sd.tiles_x, tj = it.y - ti * sd.tiles_x;
        fp64stage::stage_tile<RECON, CHAR, WZ, FLUX>(a, ti, tj, sd.tiles_x);
        __syncthreads();  // shared memory is reused by the next tile
    }
}

// One CTA per work item, the stage arguments in shared memory (as in the
// mixed form's k_stage_batch_mixed_each).
template <int RECON, bool CHAR, bool WZ, int FLUX>
__global__ void __launch_bounds__(fp64stage::NT, 2)
    k_stage_batch_each(const SlotDesc* __restrict__ slots, const int2* __restrict__ work,
                       const int* __restrict__ nwork, int stage) {
    __shared__ StageArgs sa;
    __shared__ int3 tile;
    if ((int)blockIdx.x >= *nwork) return;
    if (threadIdx.x == 0) {
        const int2 it = work[blockIdx.x];
        const SlotDesc& sd = slots[it.x];
        sa = slot_args(sd, stage);
        const int ti = it.y / sd.tiles_x;
        tile = make_int3(ti, it.y - ti * sd.tiles_x, sd.tiles_x);
    }
    __syncthreads();
    fp64stage::stage_tile<RECON, CHAR, WZ, FLUX>(sa, tile.x, tile.y, tile.z);
}

template <int RECON, bool CHAR, bool WZ, int FLUX>
static cudaError_t one(const BatchLaunch& b, int stage, cudaStream_t s) {
    constexpr size_t bytes = fp64stage::smem_bytes<CHAR>();
    auto kern = k_stage_batch<RECON, CHAR, WZ, FLUX>;
    auto kern_each = k_stage_batch_each<RECON, CHAR, WZ, FLUX>;
    static bool configured[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!configured[dev]) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)bytes);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(kern_each, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)bytes);
        if (e != cudaSuccess) return e;
        configured[dev] = true;
    }
    if (b.grid <= 0) return cudaSuccess;  // configuration only
    if (b.each)
        kern_each<<<b.grid, fp64stage::NT, bytes, s>>>(b.slots, b.work, b.nwork, stage);
    else
        kern<<<b.grid, fp64stage::NT, bytes, s>>>(b.slots, b.work, b.nwork, stage);
    return cudaGetLastError();
}

template <int RECON, bool CHAR, bool WZ>
static cudaError_t by_flux(const BatchLaunch& b, int flux, int stage, cudaStream_t s) {
    switch (flux) {
        case FLUX_HLL: return one<RECON, CHAR, WZ, FLUX_HLL>(b, stage, s);
        case FLUX_HLLC: return one<RECON, CHAR, WZ, FLUX_HLLC>(b, stage, s);
        case FLUX_ROE: return one<RECON, CHAR, WZ, FLUX_ROE>(b, stage, s);
        case FLUX_HLLHC: return one<RECON, CHAR, WZ, FLUX_HLLHC>(b, stage, s);
        case FLUX_HLLCHC: return one<RECON, CHAR, WZ, FLUX_HLLCHC>(b, stage, s);
        case FLUX_ROEHC: return one<RECON, CHAR, WZ, FLUX_ROEHC>(b, stage, s);
        default: return one<RECON, CHAR, WZ, FLUX_LLF>(b, stage, s);
    }
}

cudaError_t launch_stage_batch_fp64(const BatchLaunch& b, const Numerics& num, int stage,
                                    cudaStream_t s) {
    // the server instantiates the characteristic and component WENO5 forms
    if (num.recon != 5) return cudaErrorNotSupported;
    if (!num.characteristic) return by_flux<5, false, false>(b, num.flux, stage, s);
    return num.weno_z ? by_flux<5, true, true>(b, num.flux, stage, s)
                      : by_flux<5, true, false>(b, num.flux, stage, s);
}

// Boundary fill of stage `stage`'s input for every active slot: each block
// of the bc work list fills its share of one slot's ghost layers.
__global__ void k_bc_batch(const SlotDesc* __restrict__ slots, const int2* __restrict__ work,
                           const int* __restrict__ nwork, int stage) {
    if ((int)blockIdx.x >= *nwork) return;
    const int2 it = work[blockIdx.x];
    const SlotDesc& sd = slots[it.x];
    if (!sd.ctrl || !sd.ctrl->active) return;
    double* u = stage == 0 ? sd.u : (stage == 1 ? sd.u1 : sd.u2);
    bc_fill(u, sd.grid, sd.bnd, sd.ctrl->t, it.y * (long long)blockDim.x + threadIdx.x,
            (long long)sd.bc_blocks * blockDim.x);
}

cudaError_t launch_bc_batch(const BatchLaunch& b, int stage, cudaStream_t s) {
    k_bc_batch<<<b.bc_grid, 256, 0, s>>>(b.slots, b.bc_work, b.nbc, stage);
    return cudaGetLastError();
}

// End of a step for every active slot: one block per slot.
__global__ void __launch_bounds__(FINALIZE_THREADS) k_finalize_batch(const SlotDesc* __restrict__ slots, const int* __restrict__ act,
                                 const int* __restrict__ nact) {
    __shared__ double red[96];
    if ((int)blockIdx.x >= *nact) return;
    const SlotDesc& sd = slots[act[blockIdx.x]];
    if (!sd.ctrl) return;
    finalize_body(sd.ctrl, sd.partials, sd.npartials, sd.ncells, 2, red);
}

cudaError_t launch_finalize_batch(const BatchLaunch& b, cudaStream_t s) {
    k_finalize_batch<<<b.active_grid, FINALIZE_THREADS, 0, s>>>(b.slots, b.active, b.nactive);
    return cudaGetLastError();
}

}  // namespace eb2
