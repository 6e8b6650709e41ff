// Descriptors shared by the host engine and the device kernels.
#pragma once
#include <cstdint>

namespace sg {

enum CountMode : int32_t {
    kModeReference = 0,  // FP32 tables, the reference's arithmetic (isPruned=1)
    kModeFP64 = 1,       // FP64 tables, no scaling (the high-precision oracle mode)
    kModeOriginal = 2,   // FP32 tables, isPruned=0 arithmetic (no scale, FP32 root)
};

// One sub-template step of one coloring: the fused aggregation + eMA over all
// vertices.  Tables are vertex-major: row v holds the v-th vertex's L columns
// with a row pitch that is a multiple of 4 elements (16 B for FP32).
struct StageDesc {
    int32_t V;
    int32_t L_s, S, L_m, L_a;          // L_m / L_a = k when that child is a leaf
    int32_t out_pitch, main_pitch, aux_pitch;
    int32_t k;
    int32_t main_leaf, aux_leaf;       // child of size 1: one-hot colors
    int32_t is_root;                   // sub 0: per-vertex root values, no table
    int32_t scaled;                    // first non-bottom sub: x 1e-12 through FP64
    int32_t root_float;                // isPruned=0: root accumulated in FP32
    int32_t gather_group;              // lanes per vertex in the gather (power of 2)
    int32_t tile_v;                    // vertices per tile
    int32_t ntiles;
    int32_t out_chunk;                 // outputs staged in shared memory per pass
    int32_t hub_count;                 // vertices [0, hub_count) read hub_agg
    int32_t hub_pitch;                 // row pitch of hub_agg
    const void *main;
    const void *aux;
    void *out;
    const uint32_t *split;             // [L_s][S] (main col | aux col << 16), by output column
    const int16_t *rem;                // [L_s][k] main-leaf: aux column of set\{c}, or -1
    const uint8_t *color;              // [V] internal order
    const int32_t *off;                // [V+1]
    const int32_t *adj;                // [nnz]
    const void *hub_agg;               // [hub_count][aux_pitch] precomputed aggregation
    double *root_partial;              // [ntiles]
    double *root_vertex;               // [V] optional (internal order)
};

}  // namespace sg
