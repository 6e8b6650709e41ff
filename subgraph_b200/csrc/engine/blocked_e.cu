// Blocked-eMA kernels of the shapes in SG_BLK_SHAPES_E.
#include "blocked.cuh"

namespace sg {

bool launch_fused_blk_e(const StageDesc &d, const FusedConfig &cfg, cudaStream_t st)
{
#define SG_BLK_LAUNCH(NN, PP) \
    if (d.blk_shape == blk::shape_id(NN, PP)) { launch_blk_shape<NN, PP>(d, cfg, st); return true; }
    SG_BLK_SHAPES_E(SG_BLK_LAUNCH)
#undef SG_BLK_LAUNCH
    return false;
}

}  // namespace sg
