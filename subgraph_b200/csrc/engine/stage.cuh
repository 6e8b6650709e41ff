// Descriptors shared by the host engine and the device kernels.
#pragma once
#include <cstdint>

namespace sg {

enum CountMode : int32_t {
    kModeReference = 0,  // FP32 tables, the reference's arithmetic (isPruned=1)
    kModeFP64 = 1,       // FP64 tables, no scaling (the high-precision oracle mode)
    kModeOriginal = 2,   // isPruned=0 on a CSC graph: FP32, no scale, FP32 root, and the SpMV
                         // buffer accumulating over every split, sub and coloring (k_original)
    kModeOriginalCSR = 3,  // isPruned=0 on a CSR graph: the same, with a fresh aggregation per
                           // split (CSRGraph::SpMVNaiveFull overwrites its output)
};

// One sub-template step of nb colorings: the fused aggregation + eMA over all
// vertices.  Tables are vertex-major: row v holds the v-th vertex's L columns
// with a pitch that is a multiple of 8 elements (32-byte rows).  A batch of
// B colorings interleaves them per vertex: row v = [B][pitch] (row stride
// B*pitch), colors [V][B]; a launch handles colorings [b0, b0 + nb) of it
// (the table and color pointers are offset to b0).  The plain form is
// B = nb = 1.
struct StageDesc {
    int32_t V;
    int32_t L_s, S, L_m, L_a;          // L_m / L_a = k when that child is a leaf
    int32_t out_pitch, main_pitch, aux_pitch;   // row strides (elements)
    int32_t k;
    int32_t nb;                        // colorings of this launch
    int32_t cstride;                   // color of (v, b) at color[v * cstride + b]
    int32_t aux_cols, a_cstride;       // aux columns gathered per row; agg rows per coloring
    int32_t main_cols, m_cstride;      // main columns loaded per row; main rows per coloring
    int32_t out_w, s_cstride;          // columns written per row; output columns per coloring
    int32_t rp_stride;                 // root partials per coloring
    int32_t main_leaf, aux_leaf;       // child of size 1: one-hot colors
    int32_t is_root;                   // sub 0: per-vertex root values, no table
    int32_t scaled;                    // first non-bottom sub: x 1e-12 through FP64
    int32_t root_float;                // isPruned=0: root accumulated in FP32
    // launch shape (filled by plan_fused / the autotuner)
    int32_t tile_v;                    // vertices per tile
    int32_t nthreads;                  // CTA size (256 or 512)
    int32_t gather_group;              // threads per vertex in the aggregation
    int32_t gather_q;                  // 32-byte column chunks per thread (1, 2 or 4)
    int32_t ntiles;
    int32_t tile_begin;                // a launch covers tiles [tile_begin, ntiles)
    int32_t *ticket;                   // non-null: CTAs take tiles from this counter (zeroed before the
                                       // launch), else tile_begin + blockIdx.x, stride gridDim.x
    int32_t out_chunk;                 // outputs staged in shared memory per pass
    size_t smem;                       // dynamic shared memory bytes
    // vertices [0, hub_count) are aggregated by the hub kernel in neighbour
    // chunks; their partial rows are added here in chunk order
    int32_t hub_count;
    int32_t hub_pitch;                 // row pitch of hub_partial
    const int32_t *hub_chunk_start;    // [hub_count+1]
    const void *hub_partial;           // [chunks][hub_pitch]
    const void *main;
    const void *aux;
    void *out;
    const uint32_t *split;             // [S][split_stride] (main col | aux col << 16) per (split, output column)
    int32_t split_stride;              // L_s rounded up to a multiple of 4
    // eMA form: 0 per-output loop; 1 packed (FP32, 32-vertex tiles, two
    // vertices per lane: shared rows of kPackedRow floats and the split table
    // as byte offsets into shared memory); 2 register-blocked (FP32, the
    // outputs grouped by (|s|+1)-color supersets, blk_sched.hpp)
    int32_t packed;
    const uint32_t *aoff;              // [S][split_stride] aggregate row byte offset
    const uint32_t *moff;              // [S][split_stride] main row byte offset
    const int32_t *blk;                // [blk_nblocks][row] held / streamed / output columns per block
    int32_t blk_shape;                 // blk::shape_id of (|s|, |main|), 0 = no blocked form
    int32_t blk_nblocks;
    const int16_t *rem;                // [L_s][k] main-leaf: aux column of set\{c}, or -1
    // One coloring at a time: adjc[e] = neighbour id | its color << 28.  A
    // vertex of color c only reads aggregate columns without c (the others
    // meet a main entry that is an exact zero, or no output at all), and a
    // neighbour of color c_u only adds to sets containing c_u (its other
    // entries are exact zeros): cmask[c][chunk] has bit c_u set when the
    // 32-byte column chunk holds such a set; other chunks are skipped.
    // Rooted form (register-blocked eMA, one coloring per launch).  A vertex
    // of color c has non-zero outputs only for sets holding c, and in those
    // only the splits whose main set holds c give non-zero products; over the
    // other k-1 colors they form a stage of shape (|s|-1, |main|-1), whose
    // index tables are the same for every vertex.  The tile then keeps the
    // aggregate columns lacking c and the main columns holding c, compacted in
    // that numbering (agg_chunk, main_full), runs the rooted block tables, and
    // expands the outputs back to the table's columns (out_rank).  Skipped
    // products are exact zeros: the sums are those of the full loop.
    int32_t rooted;
    int32_t r_Ls, r_La, r_Lm;          // rooted output / aggregate / main columns
    const uint32_t *agg_chunk;         // [k][aux chunks of 8]: rank of the chunk's first column lacking c
                                       //   | mask of its columns lacking c << 16
    const int16_t *main_full;          // [k][r_Lm] table column of each rooted main set
    const int16_t *out_rank;           // [k][L_s] rooted output of each table column, -1: lacks c
    const int32_t *ublk, *rblk;        // block tables of the two forms (set_shape picks one into blk)
    int32_t ublk_shape, ublk_nblocks, rblk_shape, rblk_nblocks;
    const int32_t *adjc;               // [nnz], or null (adj)
    const uint16_t *cmask;             // [k][cmask_stride] (with adjc, non-leaf aux), or null: every chunk read
    int32_t cmask_stride;
    // Flat aggregation (with cmask, when only the aggregate columns lacking the
    // vertex's color are read: rooted eMA or one-hot main): row c of cact is
    // the count of the chunks that hold a set lacking c, then those chunks.
    // The tile's (vertex, chunk group) pairs over those lists are spread over
    // all threads instead of a fixed group of threads a vertex that also walks
    // the chunks no output reads.  ucact: the table, cact: set when in use.
    const uint16_t *cact, *ucact;      // [k][cact_stride]
    int32_t cact_stride;
    const uint8_t *color;              // [V] internal order
    const int32_t *off;                // [V+1]
    const int32_t *adj;                // [nnz]
    double *root_partial;              // [ntiles]
    double *root_vertex;               // [V] optional (internal order)
};

// Aggregation of the vertices [0, hub_count) in neighbour chunks of `chunk`
// entries; one item per (vertex, chunk) writes a partial row.
struct HubArgs {
    int32_t hub_count;
    int32_t chunk;
    int32_t L_a, aux_pitch;      // aux columns summed per row / row stride (elements)
    int32_t row_pitch;           // pitch of the partial rows
    int32_t k_leaf;              // > 0: the aux child is one-hot, count colors (k) of nb colorings
    int32_t nb, cstride;         // k_leaf: colorings, color layout (color[v * cstride + b])
    int32_t total_chunks;
    const uint8_t *color;        // [V] internal order (k_leaf, gmask)
    const int32_t *adjc;         // one coloring: neighbour ids tagged with their colour, or null (k_leaf, gmask)
    const int32_t *chunk_start;  // [hub_count+1] first chunk index of each hub
    const int32_t *off;
    const int32_t *adj;
    const void *aux;
    void *partial;               // [total_chunks][row_pitch]
    // exact order: every hub is one chunk (all its neighbours) and its columns
    // are split among lanes, each lane summing its columns over the whole
    // neighbour list in order -- the reference's summation order
    int32_t exact_order;
    int32_t *ticket;             // exact order: the next item to take (zeroed before each launch)
    // exact order, colour-tagged ids (adjc): gmask[c][g] has bit c_u set when
    // the 32-column group g holds a set with c_u and without c.  A hub of
    // colour c copies group g of a neighbour of colour c_u only then (else a
    // zero slice): the neighbour's other entries of the group are exact zeros
    // or lie in columns holding c, which no reader of the hub row uses (they
    // meet main entries that are exact zeros, or no output).  Null: every slice.
    const uint16_t *gmask;
    int32_t gmask_stride;
};

// ---------------------------------------------------------------------------
// The batched form's work queue: one entry per (coloring slot, sub-template)
// stage, hub chunks and fused tile groups as items.
// ---------------------------------------------------------------------------
constexpr int kBatchThreads = 512;    // persistent CTAs of 512 threads, two per SM when shared memory allows
// producers (main, aux, hub chunks) plus the readers of earlier tables whose
// arena range a stage overwrites; trees of up to 16 vertices need at most 9
constexpr int kBatchMaxDeps = 12;
constexpr int kStageHub = 0, kStageFused = 1;
constexpr int kHubItemChunks = 8;     // hub neighbour chunks per queue item

struct BatchStage {
    int32_t kind;            // kStageHub or kStageFused
    int32_t first_item;      // items [first_item, first_item + nitems)
    int32_t nitems;
    int32_t tiles_per_item;  // fused: consecutive tiles per item
    int32_t ndeps;
    int32_t deps[kBatchMaxDeps];   // stages that must be complete (all their items)
    StageDesc d;
    HubArgs h;
};

struct BatchCtl {
    int32_t next_item;       // the queue head
    int32_t error;           // set when a dependency wait ran out of time
    int32_t error_stage;
    int32_t pad;
    unsigned long long t0;   // %globaltimer when item 0 was claimed (job latencies)
};

}  // namespace sg
