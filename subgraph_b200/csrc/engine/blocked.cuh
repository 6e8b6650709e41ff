// K2 with the register-blocked eMA (FP32; 256- or 512-thread CTAs), one
// kernel per blocked shape (|s|, |main|): each kernel's register allocation
// is that of its own schedule, so shapes with few held values and
// accumulators run two CTAs per SM.  Gather and main-row phases are those of
// fused_tile.  The shapes are instantiated in five translation units
// (blocked_a.cu ... blocked_e.cu) that compile in parallel.
#pragma once
#include "kernels.cuh"
#include "tile.cuh"

namespace sg {

// two CTAs per SM (64 registers a thread at 512 threads) when the schedule
// keeps at most 40 values (held operands + accumulators) live
template <int N, int P> constexpr int blk_min_blocks()
{
    return blk::Shape<N, P>::NH + blk::Shape<N, P>::NO <= 40 ? 2 : 1;
}

template <int NT, int Q, int N, int P>
__global__ void __launch_bounds__(NT, (NT == 512 ? blk_min_blocks<N, P>() : 2 * blk_min_blocks<N, P>()))
    k_fused_blk(StageDesc d)
{
    extern __shared__ __align__(32) unsigned char smem_raw[];
    if (d.ticket) {   // dynamic tiles, as k_fused
        __shared__ int s_tile;
        for (;;) {
            if (threadIdx.x == 0) s_tile = d.tile_begin + atomicAdd(d.ticket, 1);
            __syncthreads();
            const int tile = s_tile;
            if (tile >= d.ntiles) break;
            fused_tile<float, NT, Q, false, false, true, N, P>(d, tile, smem_raw);
        }
        return;
    }
    for (int tile = d.tile_begin + blockIdx.x; tile < d.ntiles; tile += gridDim.x)
        fused_tile<float, NT, Q, false, false, true, N, P>(d, tile, smem_raw);
}

template <int NT, int N, int P>
static void launch_blk_q(const StageDesc &d, const FusedConfig &cfg, cudaStream_t st)
{
    auto go = [&](auto kern) {
        if (cfg.smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cfg.smem);
        int per_sm = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, cfg.smem) != cudaSuccess || per_sm < 1)
            per_sm = 1;
        const int grid = std::max(1, std::min(d.ntiles - d.tile_begin, cfg.grid * per_sm));
        if (d.ticket) cudaMemsetAsync(d.ticket, 0, sizeof(int32_t), st);
        kern<<<grid, NT, cfg.smem, st>>>(d);
    };
    switch (d.gather_q) {
    case 1: go(k_fused_blk<NT, 1, N, P>); break;
    case 2: go(k_fused_blk<NT, 2, N, P>); break;
    default: go(k_fused_blk<NT, 4, N, P>); break;
    }
}

template <int N, int P>
static void launch_blk_shape(const StageDesc &d, const FusedConfig &cfg, cudaStream_t st)
{
    if (d.nthreads == 512) launch_blk_q<512, N, P>(d, cfg, st);
    else launch_blk_q<256, N, P>(d, cfg, st);
}

}  // namespace sg
