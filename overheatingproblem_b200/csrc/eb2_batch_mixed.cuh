// eb2_batch_mixed.cuh -- batched stage kernels of the solve server, mixed
// precision (FMA contraction on), reusing the single-solve per-tile body, for
// any tile shape of eb2_stage_mixed.cuh; each shape is instantiated in a
// translation unit of its own (eb2_batch_mixed*.cu).
#pragma once

#include "eb2_batch.cuh"
#include "eb2_stage_mixed.cuh"

namespace eb2 {
namespace batchmixed {

template <class S, bool WZ, int FLUX>
__global__ void __launch_bounds__(S::NT, S::CTAS)
    k_stage_batch_mixed(const SlotDesc* __restrict__ slots, const int2* __restrict__ work,
                        const int* __restrict__ nwork, int stage) {
    const int n = *nwork;
    for (int w = blockIdx.x; w < n; w += gridDim.x) {
        const int2 it = work[w];
        const SlotDesc& sd = slots[it.x];
        const StageArgs a = slot_args(sd, stage);
        const int ti = it.y / sd.tiles_x, tj = it.y - ti * sd.tiles_x;
        mixstage::stage_tile<S, WZ, FLUX>(a, ti, tj, sd.tiles_x);
        __syncthreads();  // shared memory is reused by the next tile
    }
}

// One CTA per work item.  With no loop around the tile body, and the stage
// arguments in shared memory (read there as the single-solve kernel reads its
// parameter block), nothing but the tile's own values needs registers: the
// looping kernel spills 20-50 bytes per thread, this one none.
template <class S, bool WZ, int FLUX>
__global__ void __launch_bounds__(S::NT, S::CTAS)
    k_stage_batch_mixed_each(const SlotDesc* __restrict__ slots, const int2* __restrict__ work,
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
    mixstage::stage_tile<S, WZ, FLUX>(sa, tile.x, tile.y, tile.z);
}

// One slot's stage as a launch of its own: a CTA per tile, as the
// single-solve kernel, with the stage arguments in the parameter block.
template <class S, bool WZ, int FLUX>
__global__ void __launch_bounds__(S::NT, S::CTAS) k_stage_slot_mixed(StageArgs a) {
    mixstage::stage_tile<S, WZ, FLUX>(a, blockIdx.y, blockIdx.x, gridDim.x);
}

template <class S, bool WZ, int FLUX>
cudaError_t one_slot(const StageArgs& a, cudaStream_t s) {
    auto kern = k_stage_slot_mixed<S, WZ, FLUX>;
    static bool configured[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!configured[dev]) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)S::SMEM);
        if (e != cudaSuccess) return e;
        configured[dev] = true;
    }
    if (!a.uout) return cudaSuccess;  // configuration only
    dim3 grid((a.grid.ny + S::TY - 1) / S::TY, (a.grid.nx + S::TX - 1) / S::TX);
    kern<<<grid, S::NT, S::SMEM, s>>>(a);
    return cudaGetLastError();
}

template <class S, bool WZ>
cudaError_t slot_by_flux(const StageArgs& a, int flux, cudaStream_t s) {
    switch (flux) {
        case FLUX_HLL: return one_slot<S, WZ, FLUX_HLL>(a, s);
        case FLUX_HLLC: return one_slot<S, WZ, FLUX_HLLC>(a, s);
        case FLUX_ROE: return one_slot<S, WZ, FLUX_ROE>(a, s);
        case FLUX_HLLHC: return one_slot<S, WZ, FLUX_HLLHC>(a, s);
        case FLUX_HLLCHC: return one_slot<S, WZ, FLUX_HLLCHC>(a, s);
        case FLUX_ROEHC: return one_slot<S, WZ, FLUX_ROEHC>(a, s);
        default: return one_slot<S, WZ, FLUX_LLF>(a, s);
    }
}

template <class S>
cudaError_t launch_slot(const StageArgs& a, const Numerics& num, cudaStream_t s) {
    if (num.recon != 5 || !num.characteristic) return cudaErrorNotSupported;
    return num.weno_z ? slot_by_flux<S, true>(a, num.flux, s)
                      : slot_by_flux<S, false>(a, num.flux, s);
}

template <class S, bool WZ, int FLUX>
cudaError_t one(const BatchLaunch& b, int stage, cudaStream_t s) {
    auto kern = k_stage_batch_mixed<S, WZ, FLUX>;
    auto kern_each = k_stage_batch_mixed_each<S, WZ, FLUX>;
    static bool configured[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!configured[dev]) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)S::SMEM);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(kern_each, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)S::SMEM);
        if (e != cudaSuccess) return e;
        configured[dev] = true;
    }
    if (b.grid <= 0) return cudaSuccess;  // configuration only
    if (b.each)
        kern_each<<<b.grid, S::NT, S::SMEM, s>>>(b.slots, b.work, b.nwork, stage);
    else
        kern<<<b.grid, S::NT, S::SMEM, s>>>(b.slots, b.work, b.nwork, stage);
    return cudaGetLastError();
}

template <class S, bool WZ>
cudaError_t by_flux(const BatchLaunch& b, int flux, int stage, cudaStream_t s) {
    switch (flux) {
        case FLUX_HLL: return one<S, WZ, FLUX_HLL>(b, stage, s);
        case FLUX_HLLC: return one<S, WZ, FLUX_HLLC>(b, stage, s);
        case FLUX_ROE: return one<S, WZ, FLUX_ROE>(b, stage, s);
        case FLUX_HLLHC: return one<S, WZ, FLUX_HLLHC>(b, stage, s);
        case FLUX_HLLCHC: return one<S, WZ, FLUX_HLLCHC>(b, stage, s);
        case FLUX_ROEHC: return one<S, WZ, FLUX_ROEHC>(b, stage, s);
        default: return one<S, WZ, FLUX_LLF>(b, stage, s);
    }
}

template <class S>
cudaError_t launch(const BatchLaunch& b, const Numerics& num, int stage, cudaStream_t s) {
    if (num.recon != 5 || !num.characteristic) return cudaErrorNotSupported;
    return num.weno_z ? by_flux<S, true>(b, num.flux, stage, s)
                      : by_flux<S, false>(b, num.flux, stage, s);
}

}  // namespace batchmixed
}  // namespace eb2
