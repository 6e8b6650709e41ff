// K2 with the register-blocked eMA (FP32; 256- or 512-thread CTAs, which
// leave each thread the registers for a block's held values and
// accumulators).  Gather and main-row phases are those of fused_tile.
#include "kernels.cuh"
#include "tile.cuh"

namespace sg {

template <int NT, int Q>
__global__ void __launch_bounds__(NT) k_fused_blk(StageDesc d)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    for (int tile = blockIdx.x; tile < d.ntiles; tile += gridDim.x)
        fused_tile<float, NT, Q, false, false, true>(d, tile, smem_raw);
}

template <int NT>
static void launch_blk_q(const StageDesc &d, const FusedConfig &cfg, cudaStream_t st)
{
    auto go = [&](auto kern) {
        if (cfg.smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cfg.smem);
        int per_sm = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, cfg.smem) != cudaSuccess || per_sm < 1)
            per_sm = 1;
        const int grid = std::max(1, std::min(d.ntiles, cfg.grid * per_sm));
        kern<<<grid, NT, cfg.smem, st>>>(d);
    };
    switch (d.gather_q) {
    case 1: go(k_fused_blk<NT, 1>); break;
    case 2: go(k_fused_blk<NT, 2>); break;
    default: go(k_fused_blk<NT, 4>); break;
    }
}

void launch_fused_blk(const StageDesc &d, const FusedConfig &cfg, cudaStream_t st)
{
    if (d.nthreads == 512) launch_blk_q<512>(d, cfg, st);
    else launch_blk_q<256>(d, cfg, st);
}

}  // namespace sg
