// Dispatch of the register-blocked K2 to the translation unit holding the
// stage's shape.
#include "kernels.cuh"

namespace sg {

bool launch_fused_blk_a(const StageDesc &d, const FusedConfig &cfg, cudaStream_t st);
bool launch_fused_blk_b(const StageDesc &d, const FusedConfig &cfg, cudaStream_t st);
bool launch_fused_blk_c(const StageDesc &d, const FusedConfig &cfg, cudaStream_t st);
bool launch_fused_blk_d(const StageDesc &d, const FusedConfig &cfg, cudaStream_t st);
bool launch_fused_blk_e(const StageDesc &d, const FusedConfig &cfg, cudaStream_t st);

void launch_fused_blk(const StageDesc &d, const FusedConfig &cfg, cudaStream_t st)
{
    if (launch_fused_blk_a(d, cfg, st) || launch_fused_blk_b(d, cfg, st) || launch_fused_blk_c(d, cfg, st) ||
        launch_fused_blk_d(d, cfg, st))
        return;
    launch_fused_blk_e(d, cfg, st);
}

}  // namespace sg
