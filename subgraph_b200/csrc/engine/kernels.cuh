// Device kernels of the counting path (sm_100a):
//   k_color      bit-exact glibc rand() coloring by jump-ahead
//   k_remap      degree-ordered relabelling of the adjacency
//   k_fused      fused neighbour aggregation + eMA over one sub-template step
//   k_hub_partial / k_hub_combine  chunked aggregation of very-high-degree vertices
//   k_root_reduce deterministic FP64 (Kahan) reduction of the root partials
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include <utility>
#include <vector>

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
    uint8_t *color;            // internal order: coloring c, vertex v at c * color_stride + v * vertex_stride
    int64_t color_stride;
    int64_t vertex_stride;     // 1: [ncolorings][V]; ncolorings: interleaved [V][ncolorings]
};

void launch_color(const ColorArgs &a, int ncolorings, cudaStream_t st);
// adjc[e] = adj[e] | color[adj[e] * cstride] << 28 (ids below 2^28, colors below 16)
void launch_color_adj(const int32_t *adj, int64_t nnz, const uint8_t *color, int64_t cstride, int32_t *adjc,
                      cudaStream_t st);
// relabelled adjacency; a neighbour id outside [0, V) is not followed: the
// first such entry's index is kept in *bad (atomicMin; the caller starts it
// at INT32_MAX) and a 0 is written in its place
void launch_remap(int32_t V, const int32_t *old_off, const int32_t *old_adj, const int32_t *new_off,
                  const int32_t *iperm, const int32_t *perm, int32_t *new_adj, int32_t *bad, cudaStream_t st);

struct FusedConfig {
    int tile_v;      // vertices per tile
    int q;           // 32-byte chunks per gather thread
    size_t smem;     // dynamic shared memory bytes
    int grid;        // CTAs per SM unit (scaled by the occupancy at launch)
};

// Chooses the tile size, CTA size, gather grouping and shared memory of a
// stage (fills tile_v, nthreads, gather_group, gather_q, ntiles, out_chunk,
// smem).  Returns false when no tiling fits in shared memory.
bool plan_fused(StageDesc &d, bool fp64, int sm_count, FusedConfig &cfg);
struct TileShape {
    int tile_v;      // vertices per tile
    int threads;     // CTA size
    int packed;      // eMA form: 0 per-output loop, 1 packed FP32x2 (32-vertex tiles), 2 register-blocked
    int q = 0;       // 32-byte column chunks per aggregation thread (1, 2, 4); 0: the fewest that keep
                     // nine in ten threads busy
    int nomask = 0;  // 1: read every column chunk (no chunk masks)
    int rooted = 0;  // register-blocked eMA in the rooted form (StageDesc::rooted)
    int flat = 0;    // 1: flat aggregation over each vertex's active chunks (StageDesc::cact)
};
// Sets an explicit shape (the autotuner's candidates); false when it does not fit.
bool set_shape(StageDesc &d, bool fp64, const TileShape &shape);
// The shapes the autotuner times for a stage.
std::vector<TileShape> candidate_shapes(const StageDesc &d, bool fp64);
void launch_fused(const StageDesc &d, bool fp64, const FusedConfig &cfg, cudaStream_t st);
// variant: the exact-order hub kernel's (threads, ring depth) pair, 0 .. hub_variants()-1
void launch_hub(const HubArgs &h, bool fp64, int sm_count, cudaStream_t st, int variant = 0);
int hub_variants();

// K2 with the register-blocked eMA (StageDesc::packed == 2)
void launch_fused_blk(const StageDesc &d, const FusedConfig &cfg, cudaStream_t st);
void launch_root_reduce(const double *partial, int32_t n, double scale, double *out, cudaStream_t st);

// isPruned=0 on a CSC graph: one sub-template step, one thread per vertex,
// with the running aggregation buffer carried in buf[V] (internal order)
constexpr int kOriginalThreads = 256;
struct OriginalArgs {
    int32_t V, L_s, S, split_stride;
    const uint32_t *split;     // [S][split_stride] main col | aux col << 16, per output column
    const int32_t *c2c;        // [L_s] output column of the i-th color set in lexicographic order
    int32_t main_leaf, aux_leaf, is_root;
    const float *main;
    int32_t main_pitch;
    const float *aux;
    int32_t aux_pitch;
    float *out;
    int32_t out_pitch;
    const uint8_t *color;      // [V] internal order
    const int32_t *off, *adj;
    float *buf;                // [V] CountMat::_bufVec, internal order
    double *partial;           // root: [blocks] per-block sums
    double *root_vertex;       // root: [V] optional
};
// returns the number of blocks (= root partials written)
int launch_original(const OriginalArgs &a, cudaStream_t st);

// the batched form (batch.cu)
// stage_end (optional): [nstages] %globaltimer when each stage's last item
// completed, ctl->t0 when item 0 was claimed
cudaError_t launch_persistent(const BatchStage *stages, int nstages, int total_items, int *done, BatchCtl *ctl,
                              long long wait_cycles, size_t smem, bool fp64, int sm_count, cudaStream_t st,
                              unsigned long long *stage_end = nullptr);
// n_slot (optional): per-slot partial counts (jobs of different templates)
void launch_root_reduce_slots(const double *partial, int64_t slot_stride, int32_t n, double scale, double *out,
                              int nslots, cudaStream_t st, const int32_t *n_slot = nullptr);

}  // namespace sg
