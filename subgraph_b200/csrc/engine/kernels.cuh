// Device kernels of the counting path (sm_100a):
//   k_color      bit-exact glibc rand() coloring by jump-ahead
//   k_remap      degree-ordered relabelling of the adjacency
//   k_fused      fused neighbour aggregation + eMA over one sub-template step
//   k_hub_partial / k_hub_combine  chunked aggregation of very-high-degree vertices
//   k_root_reduce deterministic FP64 (Kahan) reduction of the root partials
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "stage.cuh"

namespace sg {

constexpr int kColorBlock = 1024;      // values per coloring block (jump-ahead stride)
constexpr int kFusedThreads = 256;

struct ColorArgs {
    int32_t V;
    int32_t k;
    int32_t nblocks;
    const uint32_t *jump;      // [nblocks][31] coefficients of x^(341 + b*1024) mod P
    const uint32_t *coef;      // [31][1024] coefficients of x^t mod P
    const uint32_t *window;    // [ncolorings][31] initial window per coloring
    const int32_t *perm;       // original -> internal vertex id
    uint8_t *color;            // [ncolorings][V], internal order
    int64_t color_stride;
};

void launch_color(const ColorArgs &a, int ncolorings, cudaStream_t st);
void launch_remap(int32_t V, const int32_t *old_off, const int32_t *old_adj, const int32_t *new_off,
                  const int32_t *iperm, const int32_t *perm, int32_t *new_adj, cudaStream_t st);

struct FusedConfig {
    int tile_v;      // 32, 16 or 8
    int q;           // register chunks per lane in the gather: 1, 2, 4 or 8
    size_t smem;     // dynamic shared memory bytes
    int grid;        // CTAs
};

// Chooses tile size, gather grouping and shared memory for a stage (fills the
// stage's tile_v, gather_group, ntiles and out_chunk).  Returns false when no
// tiling fits in shared memory.
bool plan_fused(StageDesc &d, bool fp64, int sm_count, FusedConfig &cfg);
void launch_fused(const StageDesc &d, bool fp64, const FusedConfig &cfg, cudaStream_t st);

// Aggregation of the vertices [0, hub_count) split into neighbour chunks of
// `chunk` entries: every chunk sums sequentially into partial rows, then the
// partial rows of a vertex are added in chunk order into hub_agg.
struct HubArgs {
    int32_t hub_count;
    int32_t chunk;
    int32_t L_a, aux_pitch;      // aux row width / pitch (elements)
    int32_t row_pitch;           // pitch of partial and hub_agg rows
    int32_t k_leaf;              // > 0: the aux child is one-hot, count colors (k)
    const uint8_t *color;        // [V] internal order (k_leaf only)
    int32_t total_chunks;
    const int32_t *chunk_start;  // [hub_count+1] first chunk index of each hub
    const int32_t *off;
    const int32_t *adj;
    const void *aux;
    void *partial;               // [total_chunks][aux_pitch]
    void *hub_agg;               // [hub_count][aux_pitch]
};
void launch_hub(const HubArgs &h, bool fp64, int sm_count, cudaStream_t st);

void launch_root_reduce(const double *partial, int32_t n, double scale, double *out, cudaStream_t st);

}  // namespace sg
