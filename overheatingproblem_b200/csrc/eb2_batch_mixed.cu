// eb2_batch_mixed.cu -- batched stage kernel of the solve server, mixed
// precision (FMA contraction on), reusing the single-solve per-tile body.
#include "eb2_batch.cuh"
#include "eb2_stage_mixed.cuh"

namespace eb2 {

template <bool WZ, int FLUX>
__global__ void __launch_bounds__(mixstage::NT, mixstage::CTAS)
    k_stage_batch_mixed(const SlotDesc* __restrict__ slots, const int2* __restrict__ work,
                        const int* __restrict__ nwork, int stage) {
    const int n = *nwork;
    for (int w = blockIdx.x; w < n; w += gridDim.x) {
        const int2 it = work[w];
        const SlotDesc& sd = slots[it.x];
        const StageArgs a = slot_args(sd, stage);
        const int ti = it.y / sd.tiles_x, tj = it.y - ti * sd.tiles_x;
        mixstage::stage_tile<WZ, FLUX>(a, ti, tj, sd.tiles_x);
        __syncthreads();  // shared memory is reused by the next tile
    }
}

// One CTA per work item.  With no loop around the tile body, and the stage
// arguments in shared memory (read there as the single-solve kernel reads its
// parameter block), nothing but the tile's own values needs registers: the
// looping kernel spills 20-50 bytes per thread, this one none.
template <bool WZ, int FLUX>
__global__ void __launch_bounds__(mixstage::NT, mixstage::CTAS)
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
    mixstage::stage_tile<WZ, FLUX>(sa, tile.x, tile.y, tile.z);
}

template <bool WZ, int FLUX>
static cudaError_t one(const BatchLaunch& b, int stage, cudaStream_t s) {
    auto kern = k_stage_batch_mixed<WZ, FLUX>;
    auto kern_each = k_stage_batch_mixed_each<WZ, FLUX>;
    static bool configured[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!configured[dev]) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)mixstage::SMEM);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(kern_each, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)mixstage::SMEM);
        if (e != cudaSuccess) return e;
        configured[dev] = true;
    }
    if (b.grid <= 0) return cudaSuccess;  // configuration only
    if (b.each)
        kern_each<<<b.grid, mixstage::NT, mixstage::SMEM, s>>>(b.slots, b.work, b.nwork, stage);
    else
        kern<<<b.grid, mixstage::NT, mixstage::SMEM, s>>>(b.slots, b.work, b.nwork, stage);
    return cudaGetLastError();
}

template <bool WZ>
static cudaError_t by_flux(const BatchLaunch& b, int flux, int stage, cudaStream_t s) {
    switch (flux) {
        case FLUX_HLL: return one<WZ, FLUX_HLL>(b, stage, s);
        case FLUX_HLLC: return one<WZ, FLUX_HLLC>(b, stage, s);
        case FLUX_ROE: return one<WZ, FLUX_ROE>(b, stage, s);
        case FLUX_HLLHC: return one<WZ, FLUX_HLLHC>(b, stage, s);
        case FLUX_HLLCHC: return one<WZ, FLUX_HLLCHC>(b, stage, s);
        case FLUX_ROEHC: return one<WZ, FLUX_ROEHC>(b, stage, s);
        default: return one<WZ, FLUX_LLF>(b, stage, s);
    }
}

cudaError_t launch_stage_batch_mixed(const BatchLaunch& b, const Numerics& num, int stage,
                                     cudaStream_t s) {
    if (num.recon != 5 || !num.characteristic) return cudaErrorNotSupported;
    return num.weno_z ? by_flux<true>(b, num.flux, stage, s) : by_flux<false>(b, num.flux, stage, s);
}

// Resident CTAs per SM of the batched stage kernels: the persistent-grid
// candidates of the server's autotuner go up to this many per SM.
int stage_batch_max_blocks_per_sm(int precision) { return precision == 0 ? 2 : mixstage::CTAS; }

}  // namespace eb2
