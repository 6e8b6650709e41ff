// Device kernels of the color-coding counting path, written for sm_100a.
//
// The count tables are vertex-major (row v = the v-th vertex's color-set
// columns), so the neighbour aggregation reads whole contiguous rows with
// 128-bit loads.  Every aggregated column is summed by one lane in the order
// of the vertex's neighbour list, and every eMA product is accumulated in the
// order of the split table with separately rounded multiply and add: for
// vertices below the hub threshold the FP32 results equal the reference's
// CPU arithmetic (CSCGraph.hpp:242-307, DataTableColMajor.cpp:346-400) bit
// for bit.
#include "kernels.cuh"

#include <algorithm>
#include <cstdio>
#include <vector>

#include "tile.cuh"

namespace sg {

// ---------------------------------------------------------------------------
// K1: coloring.  The glibc TYPE_3 stream after srand(seed) is the lag-31
// recurrence s_m = s_{m-3} + s_{m-31} (mod 2^32) started from a 31-word
// window; rand() number v is s_{341+v} >> 1 (CountMat.cpp:979-991 draws
// rand() % k for v = 0..V-1 on one thread).  With P(x) = x^31 - x^28 - 1,
// s_{m0+t} = sum_i [x^t mod P]_i * s_{m0+i}, so every block rebuilds its own
// start window from the jump polynomial x^{m0} and every thread then needs one
// 31-term dot product.  All arithmetic is exact modulo 2^32.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kColorBlock) k_color(ColorArgs a)
{
    __shared__ uint32_t W[31];
    const int b = blockIdx.x;
    const int col = blockIdx.y;
    const uint32_t *w0 = a.window + 31 * col;
    if (threadIdx.x < 31) {
        uint32_t q[31];
#pragma unroll
        for (int j = 0; j < 31; ++j) q[j] = a.jump[b * 31 + j];
        for (int s = 0; s < (int)threadIdx.x; ++s) {   // q <- x*q mod P
            uint32_t t = q[30];
#pragma unroll
            for (int j = 30; j > 0; --j) q[j] = q[j - 1];
            q[0] = t;
            q[28] += t;
        }
        uint32_t acc = 0;
#pragma unroll
        for (int j = 0; j < 31; ++j) acc += q[j] * w0[j];
        W[threadIdx.x] = acc;
    }
    __syncthreads();
    const int64_t v = (int64_t)b * kColorBlock + threadIdx.x;
    if (v < a.V) {
        uint32_t s = 0;
#pragma unroll
        for (int i = 0; i < 31; ++i) s += __ldg(a.coef + i * kColorBlock + threadIdx.x) * W[i];
        const int r = (int)(s >> 1);
        a.color[col * a.color_stride + (int64_t)a.perm[v] * a.vertex_stride] = (uint8_t)(r % a.k);
    }
}

void launch_color(const ColorArgs &a, int ncolorings, cudaStream_t st)
{
    if (a.V == 0 || ncolorings == 0) return;
    dim3 grid(a.nblocks, ncolorings);
    k_color<<<grid, kColorBlock, 0, st>>>(a);
}

// ---------------------------------------------------------------------------
// Relabelling: internal vertex v = original iperm[v]; its neighbour list keeps
// the original order (which fixes the summation order) with ids mapped
// through perm.  One warp per vertex.
// ---------------------------------------------------------------------------
__global__ void k_remap(int32_t V, const int32_t *__restrict__ old_off, const int32_t *__restrict__ old_adj,
                        const int32_t *__restrict__ new_off, const int32_t *__restrict__ iperm,
                        const int32_t *__restrict__ perm, int32_t *__restrict__ new_adj, int32_t *bad)
{
    const int lane = threadIdx.x & 31;
    const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t v = w; v < V; v += nw) {
        const int32_t o = iperm[v];
        const int32_t b = old_off[o], e = old_off[o + 1], d = new_off[v];
        for (int32_t i = b + lane; i < e; i += 32) {
            const int32_t u = old_adj[i];
            if ((uint32_t)u < (uint32_t)V) {
                new_adj[d + (i - b)] = perm[u];
            } else {
                new_adj[d + (i - b)] = 0;
                atomicMin(bad, i);
            }
        }
    }
}

void launch_remap(int32_t V, const int32_t *old_off, const int32_t *old_adj, const int32_t *new_off,
                  const int32_t *iperm, const int32_t *perm, int32_t *new_adj, int32_t *bad, cudaStream_t st)
{
    if (V == 0) return;
    int blocks = std::min<int64_t>(((int64_t)V * 32 + 255) / 256, 148 * 16);
    k_remap<<<blocks, 256, 0, st>>>(V, old_off, old_adj, new_off, iperm, perm, new_adj, bad);
}

// ---------------------------------------------------------------------------
// K2: one sub-template step over all tiles (plain form); the tile body is
// fused_tile (tile.cuh), shared with the persistent batched kernel.
// ---------------------------------------------------------------------------
template <typename T, int NT, int Q, bool PK>
__global__ void __launch_bounds__(NT) k_fused(StageDesc d)
{
    extern __shared__ __align__(32) unsigned char smem_raw[];
    if (d.ticket) {
        // tiles in vertex order (degree-descending: the heaviest first), each
        // CTA taking the next one when it is done (fused_tile ends with a
        // barrier, so the shared word is read before it is written again)
        __shared__ int s_tile;
        for (;;) {
            if (threadIdx.x == 0) s_tile = d.tile_begin + atomicAdd(d.ticket, 1);
            __syncthreads();
            const int tile = s_tile;
            if (tile >= d.ntiles) break;
            fused_tile<T, NT, Q, PK>(d, tile, smem_raw);
        }
        return;
    }
    for (int tile = d.tile_begin + blockIdx.x; tile < d.ntiles; tile += gridDim.x) fused_tile<T, NT, Q, PK>(d, tile, smem_raw);
}

template <typename T, int NT>
__global__ void __launch_bounds__(NT) k_hub(HubArgs h)
{
    __shared__ __align__(32) unsigned char smem_raw[NT * 32];
    for (int item = blockIdx.x; item < h.total_chunks; item += gridDim.x) hub_item<T, NT>(h, item, smem_raw);
}

// Exact-order hub aggregation (hub_item_exact): one warp per (hub, 32-column
// group) item, items in hub order (degree-descending: the longest lists
// first), W warps a CTA, each with a ring of NSLOT staging tiles.  The
// variants trade warps per SM against batches in flight per warp; the
// autotuner picks one per row width.
int hub_variants() { return 6; }

// Items are taken from a ticket counter: every warp takes the next item when
// it is done with its last, so the long lists (the first items) do not end up
// behind a fixed share of the others on the same warp.
template <typename T, int W, int NSLOT, int BR>
__global__ void __launch_bounds__(32 * W) k_hub_exact(HubArgs h)
{
    extern __shared__ __align__(32) unsigned char smem_raw[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char *wsmem = smem_raw + (size_t)warp * hub_warp_bytes<T, NSLOT, BR>();
    const int items = h.hub_count * ((h.L_a + 31) / 32);
    for (;;) {
        int item = 0;
        if (lane == 0) item = atomicAdd(h.ticket, 1);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= items) break;
        hub_item_exact<T, NSLOT, BR>(h, item, wsmem);
    }
}

template <typename T, int W, int NSLOT, int BR = 32>
static void launch_hub_exact_v(const HubArgs &h, int sm_count, cudaStream_t st)
{
    const int items = h.hub_count * ((h.L_a + 31) / 32);
    constexpr size_t smem = (size_t)W * hub_warp_bytes<T, NSLOT, BR>();
    static_assert(smem <= 227 * 1024, "a CTA's rings must fit shared memory");
    auto kern = k_hub_exact<T, W, NSLOT, BR>;
    if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * W, smem) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    const int grid = std::max(1, std::min((items + W - 1) / W, sm_count * per_sm));
    cudaMemsetAsync(h.ticket, 0, sizeof(int32_t), st);
    kern<<<grid, 32 * W, smem, st>>>(h);
}

template <typename T>
static void launch_hub_exact(const HubArgs &h, int sm_count, cudaStream_t st, int variant)
{
    // (warps, ring depth, batch rows): 32-row tiles are 4.6 KB (FP32) / 8.7 KB
    // (FP64), and every variant stays under 227 KB a CTA; the deep rings serve
    // stages whose few long hub lists are latency-bound, the many-warp ones
    // wide stages; 64-row batches (FP32 only: FP64 would need 256 registers
    // for the two batches in flight) halve the work around the adds
    constexpr bool D = sizeof(T) == 8;
    switch (variant) {
    case 1: launch_hub_exact_v<T, 4, 6>(h, sm_count, st); break;
    case 2: launch_hub_exact_v<T, D ? 2 : 4, 12>(h, sm_count, st); break;
    case 3: launch_hub_exact_v<T, D ? 1 : 2, 24>(h, sm_count, st); break;
    case 4:
        if constexpr (D) launch_hub_exact_v<T, 2, 6>(h, sm_count, st);
        else launch_hub_exact_v<T, 2, 12, 64>(h, sm_count, st);
        break;
    case 5:
        if constexpr (D) launch_hub_exact_v<T, 1, 12>(h, sm_count, st);
        else launch_hub_exact_v<T, 4, 6, 64>(h, sm_count, st);
        break;
    default: launch_hub_exact_v<T, D ? 4 : 8, D ? 3 : 6>(h, sm_count, st); break;
    }
}

// Threads per vertex (gather_group) and chunks per thread (gather_q) of the
// aggregation: Q = `want`, or the smallest Q that keeps nine in ten threads
// busy.  False when Q = `want` needs more threads than the CTA has.
bool choose_gather(StageDesc &d, bool fp64, int want = 0)
{
    if (d.aux_leaf) {
        d.gather_q = 1;
        d.gather_group = 1;
        return want <= 1;
    }
    const int CH = fp64 ? 4 : 8;   // elements of a 32-byte chunk
    const int nchunk = (d.aux_cols + CH - 1) / CH;
    const int NT = d.nthreads;
    if (want > 0) {
        const int G = (nchunk + want - 1) / want;
        if (G > NT) return false;
        d.gather_q = want;
        d.gather_group = std::max(1, G);
        return true;
    }
    int bestQ = 4, bestG = (nchunk + 3) / 4, bestActive = -1;
    for (int Q : {1, 2, 4}) {
        const int G = (nchunk + Q - 1) / Q;
        if (G > NT) continue;
        const int active = (NT / G) * G;
        if (active >= (NT * 9) / 10) { bestQ = Q; bestG = G; bestActive = active; break; }
        if (active > bestActive) { bestQ = Q; bestG = G; bestActive = active; }
    }
    d.gather_q = bestQ;
    d.gather_group = std::max(1, bestG);
    return true;
}

bool packed_ok(const StageDesc &d, bool fp64, int tv)
{
    return !fp64 && tv == 32 && d.nb == 1 && !d.main_leaf && !d.is_root && !d.scaled && d.aoff && d.moff;
}

bool blocked_ok(const StageDesc &d, bool fp64, int tv, int nt)
{
    return !fp64 && (tv == 32 || tv == 16) && (nt == 256 || nt == 512) && d.nb == 1 && d.blk && d.blk_shape > 0 &&
           d.blk_nblocks > 0 && !d.main_leaf && !d.is_root && !d.scaled;
}

// The stage's block tables in the rooted (rooted = 1) or the plain form.
static void pick_blocks(StageDesc &d, int rooted)
{
    d.rooted = rooted;
    d.blk = rooted ? d.rblk : d.ublk;
    d.blk_shape = rooted ? d.rblk_shape : d.ublk_shape;
    d.blk_nblocks = rooted ? d.rblk_nblocks : d.ublk_nblocks;
}

bool shape_fits(const StageDesc &d0, bool fp64, int tv, int nt, int packed, size_t limit, size_t &bytes, int &oc,
                int rooted = 0)
{
    if (rooted && (packed != 2 || !d0.rblk || d0.nb != 1 || d0.aux_leaf)) return false;
    StageDesc d = d0;
    pick_blocks(d, rooted);
    if (packed == 1 && !packed_ok(d, fp64, tv)) return false;
    if (packed == 2 && !blocked_ok(d, fp64, tv, nt)) return false;
    const int La_rows = d.aux_leaf ? d.nb * d.k : (rooted ? d.r_La : d.aux_cols);
    const int Lm_rows = d.main_leaf ? 0 : (rooted ? d.r_Lm : d.main_cols);
    // staged output columns: one coloring's L_s, or the launch's wide columns
    // (nb row pitches) in chunks of a multiple of 4
    const int wide = d.nb == 1 ? d.L_s : d.nb * d.s_cstride;
    oc = (d.is_root || d.main_leaf) ? 0 : (packed == 2 ? (rooted ? d.r_Ls : d.L_s) : std::min(wide, nt >= 1024 ? 256 : 128));
    bytes = fp64 ? tile_smem_bytes<double>(La_rows, Lm_rows, oc, tv, false, d.nb)
                 : tile_smem_bytes<float>(La_rows, Lm_rows, oc, tv, packed == 1, d.nb);
    if (bytes > limit) return false;
    if (!d.aux_leaf) {
        const int CH = fp64 ? 4 : 8;   // elements of a 32-byte chunk
        const int nchunk = (d.aux_cols + CH - 1) / CH;
        if (nchunk > 4 * nt) return false;
    }
    return true;
}

bool flat_ok(const StageDesc &d, const TileShape &sh)
{
    return d.cmask && d.ucact && !d.aux_leaf && d.nb == 1 && sh.tile_v <= 32 && !sh.nomask &&
           (d.main_leaf || (sh.packed == 2 && sh.rooted));
}

bool set_shape(StageDesc &d, bool fp64, const TileShape &sh)
{
    size_t bytes;
    int oc;
    if (!shape_fits(d, fp64, sh.tile_v, sh.threads, sh.packed, 227 * 1024, bytes, oc, sh.rooted)) return false;
    pick_blocks(d, sh.rooted);
    d.tile_v = sh.tile_v;
    d.nthreads = sh.threads;
    d.packed = sh.packed;
    d.out_chunk = oc;
    d.smem = bytes;
    d.ntiles = (d.V + sh.tile_v - 1) / sh.tile_v;
    if (sh.nomask) d.cmask = nullptr;
    d.cact = nullptr;
    if (sh.flat) {
        // only where every aggregate column read lacks the vertex's color (the
        // rooted eMA, a one-hot main): the inactive chunks are then never read
        if (!flat_ok(d, sh)) return false;
        d.cact = d.ucact;
    }
    return choose_gather(d, fp64, sh.q);
}

std::vector<TileShape> candidate_shapes(const StageDesc &d, bool fp64)
{
    std::vector<TileShape> all, out;
    const bool heavy = !d.main_leaf && !d.is_root && (int64_t)d.S * d.L_s >= 512;
    if (d.aux_leaf) all = {{256, 256, 0}, {64, 256, 0}, {32, 256, 0}, {128, 512, 0}};
    else if (heavy)
        all = {{32, 1024, 1}, {32, 512, 1}, {32, 256, 1}, {32, 1024, 0}, {32, 512, 0}, {32, 256, 0},
               {16, 256, 0}, {16, 512, 0}, {16, 1024, 0}};
    else if (!d.aux_leaf && d.L_a >= 128)   // wide gathers: more threads per CTA for loads in flight
        all = {{8, 256, 0}, {16, 256, 0}, {32, 256, 0}, {32, 512, 0}, {8, 512, 0}, {16, 512, 0}, {16, 1024, 0}};
    else all = {{8, 256, 0}, {16, 256, 0}, {32, 256, 0}, {32, 512, 0}};
    if (d.ublk_shape > 0)   // register-blocked eMA
        for (TileShape t : {TileShape{32, 256, 2}, TileShape{32, 512, 2}, TileShape{16, 256, 2}, TileShape{16, 512, 2}})
            all.push_back(t);
    if (d.rblk_shape > 0) {   // register-blocked eMA in the rooted form
        for (TileShape t : {TileShape{32, 256, 2}, TileShape{32, 512, 2}, TileShape{16, 256, 2}, TileShape{16, 512, 2}}) {
            t.rooted = 1;
            all.push_back(t);
        }
    }
    for (auto &c : all) {
        size_t bytes;
        int oc;
        if (!shape_fits(d, fp64, c.tile_v, c.threads, c.packed, 227 * 1024, bytes, oc, c.rooted)) continue;
        out.push_back(c);
        // with chunk masks: also without them (the masks save loads but not the
        // instructions around them)
        if (d.cmask && !c.nomask) {
            TileShape t = c;
            t.nomask = 1;
            StageDesc f = d;
            if (set_shape(f, fp64, t)) out.push_back(t);
        }
        // wide aggregations: also the other chunk counts per thread (more chunks
        // per thread share one neighbour id and row address among them)
        if (!d.aux_leaf && d.aux_cols >= 64) {
            StageDesc e = d;
            if (!set_shape(e, fp64, c)) continue;
            for (int q : {1, 2, 4}) {
                if (q == e.gather_q) continue;
                TileShape t = c;
                t.q = q;
                StageDesc f = d;
                if (set_shape(f, fp64, t)) out.push_back(t);
            }
        }
        // the flat aggregation over the active chunks, at each chunk count
        if (flat_ok(d, c) && d.aux_cols >= 64) {
            for (int q : {1, 2, 4}) {
                TileShape t = c;
                t.q = q;
                t.flat = 1;
                StageDesc f = d;
                if (set_shape(f, fp64, t)) out.push_back(t);
            }
        }
    }
    return out;
}

bool plan_fused(StageDesc &d, bool fp64, int sm_count, FusedConfig &cfg)
{
    const bool heavy = !d.main_leaf && !d.is_root && (int64_t)d.S * d.L_s >= 512;
    std::vector<int> tvs;
    if (d.aux_leaf) tvs = {256, 128, 64, 32, 16, 8};
    else tvs = {32, 16, 8};
    const size_t limits[3] = {56 * 1024, 113 * 1024, 227 * 1024};
    bool ok = false;
    d.packed = 0;
    // the register-blocked eMA when the stage has one (its sums are those of the
    // per-output loop), the rooted form first
    for (int rooted : {1, 0})
        for (TileShape t : {TileShape{32, 256, 2}, TileShape{16, 256, 2}, TileShape{32, 512, 2}, TileShape{16, 512, 2}}) {
            t.rooted = rooted;
            if (!ok && (rooted ? d.rblk_shape : d.ublk_shape) > 0) ok = set_shape(d, fp64, t);
        }
    if (heavy && !ok) {
        // 32-vertex tiles keep the eMA free of bank conflicts; a wide tile gets 512 threads
        const int pk = packed_ok(d, fp64, 32) ? 1 : 0;
        size_t bytes;
        int oc;
        if (shape_fits(d, fp64, 32, 512, pk, 227 * 1024, bytes, oc))
            ok = set_shape(d, fp64, TileShape{32, bytes > 113 * 1024 ? 512 : 256, pk});
    }
    for (int li = 0; !ok && li < 3; ++li)
        for (int tv : tvs) {
            size_t bytes;
            int oc;
            if (shape_fits(d, fp64, tv, 256, 0, limits[li], bytes, oc)) { ok = set_shape(d, fp64, TileShape{tv, 256, 0}); break; }
            if (shape_fits(d, fp64, tv, 512, 0, limits[li], bytes, oc)) { ok = set_shape(d, fp64, TileShape{tv, 512, 0}); break; }
        }
    if (!ok) return false;
    // the flat aggregation where the chosen shape allows it (the autotuner
    // times both)
    if (d.ucact) {
        TileShape t{d.tile_v, d.nthreads, d.packed};
        t.rooted = d.rooted;
        t.flat = 1;
        StageDesc f = d;
        if (flat_ok(f, t) && set_shape(f, fp64, t)) d = f;
    }
    cfg.tile_v = d.tile_v;
    cfg.q = d.gather_q;
    cfg.smem = d.smem;
    cfg.grid = sm_count;
    return true;
}

template <typename T, int NT>
static void launch_fused_q(const StageDesc &d, const FusedConfig &cfg, cudaStream_t st)
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
    if (d.packed == 1) {
        switch (d.gather_q) {
        case 1: go(k_fused<float, NT, 1, true>); break;
        case 2: go(k_fused<float, NT, 2, true>); break;
        default: go(k_fused<float, NT, 4, true>); break;
        }
        return;
    }
    switch (d.gather_q) {
    case 1: go(k_fused<T, NT, 1, false>); break;
    case 2: go(k_fused<T, NT, 2, false>); break;
    default: go(k_fused<T, NT, 4, false>); break;
    }
}

void launch_fused(const StageDesc &d, bool fp64, const FusedConfig &cfg, cudaStream_t st)
{
    if (d.V == 0) return;
    if (!fp64 && d.packed == 2) {
        launch_fused_blk(d, cfg, st);
        return;
    }
    if (fp64) {
        if (d.nthreads == 1024) launch_fused_q<double, 1024>(d, cfg, st);
        else if (d.nthreads == 512) launch_fused_q<double, 512>(d, cfg, st);
        else launch_fused_q<double, 256>(d, cfg, st);
    } else {
        if (d.nthreads == 1024) launch_fused_q<float, 1024>(d, cfg, st);
        else if (d.nthreads == 512) launch_fused_q<float, 512>(d, cfg, st);
        else launch_fused_q<float, 256>(d, cfg, st);
    }
}

void launch_hub(const HubArgs &h, bool fp64, int sm_count, cudaStream_t st, int variant)
{
    if (h.hub_count == 0 || h.total_chunks == 0) return;
    if (h.exact_order && !h.k_leaf) {   // colour counts are exact integers in any order
        if (fp64) launch_hub_exact<double>(h, sm_count, st, variant);
        else launch_hub_exact<float>(h, sm_count, st, variant);
        return;
    }
    const int grid = std::max(1, std::min(h.total_chunks, sm_count * 8));
    if (fp64) k_hub<double, 256><<<grid, 256, 0, st>>>(h);
    else k_hub<float, 256><<<grid, 256, 0, st>>>(h);
}

// ---------------------------------------------------------------------------
// Colored adjacency of one coloring: neighbour id | its color << 28.
__global__ void k_color_adj(const int32_t *__restrict__ adj, int64_t nnz, const uint8_t *__restrict__ color,
                            int64_t cstride, int32_t *__restrict__ adjc)
{
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nnz; e += (int64_t)gridDim.x * blockDim.x) {
        const int32_t u = adj[e];
        adjc[e] = u | ((int32_t)color[(size_t)u * cstride] << 28);
    }
}

void launch_color_adj(const int32_t *adj, int64_t nnz, const uint8_t *color, int64_t cstride, int32_t *adjc,
                      cudaStream_t st)
{
    if (nnz <= 0) return;
    const int grid = (int)std::min<int64_t>((nnz + 255) / 256, 148 * 32);
    k_color_adj<<<grid, 256, 0, st>>>(adj, nnz, color, cstride, adjc);
}

// ---------------------------------------------------------------------------
// K3: the per-coloring sum of the root partials, FP64 with Kahan
// compensation, in a fixed order (one CTA, strided per thread, then a
// fixed-shape tree), times the scale (1e12 for the pruned modes).
// ---------------------------------------------------------------------------
__global__ void k_root_reduce(const double *__restrict__ partial, int32_t n, double scale, double *out)
{
    __shared__ double ss[256], cc[256], pp[256];
    const double r = block_sum_partials(partial, n, scale, ss, cc, pp);
    if (threadIdx.x == 0) *out = r;
}

void launch_root_reduce(const double *partial, int32_t n, double scale, double *out, cudaStream_t st)
{
    k_root_reduce<<<1, 256, 0, st>>>(partial, n, scale, out);
}

// ---------------------------------------------------------------------------
// isPruned=0 on a CSC graph (CountMat::countNonBottomeOriginal,
// CountMat.cpp:851-977): for every output color set i in lexicographic order
// and every split j in order, one SpMV adds the aux column auxSplit[i][j] of
// every neighbour onto CountMat::_bufVec -- a buffer that is zeroed once, at
// CountMat::initialization (CountMat.cpp:52-59), and never again, so it keeps
// accumulating over splits, sub-templates and colorings (spmvNaiveSplit adds,
// CSCGraph.hpp:219-239) -- and arrayWiseFMANaive adds bufVec * main to the
// output column (DataTableColMajor.cpp:502-510); the root is an FP32 buffer.
// Every vertex's bufVec entry is its own sequential chain of FP32 adds in
// neighbour order, so one thread per vertex reproduces it exactly; the work
// per vertex is degree x (sum over sub-templates of outputs x splits), as in
// the reference.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kOriginalThreads) k_original(OriginalArgs a)
{
    __shared__ double red[kOriginalThreads / 32];
    const int v = blockIdx.x * kOriginalThreads + threadIdx.x;
    double rootv = 0.0;
    if (v < a.V) {
        float buf = a.buf[v];
        const int cv = a.color[v];
        const int beg = a.off[v], end = a.off[v + 1];
        for (int i = 0; i < a.L_s; ++i) {
            const int o = a.c2c[i];
            float acc = 0.f;
            for (int j = 0; j < a.S; ++j) {
                const uint32_t pk = a.split[(size_t)j * a.split_stride + o];
                const int mc = (int)(pk & 0xffffu), ac = (int)(pk >> 16);
                for (int e = beg; e < end; ++e) {
                    const int u = a.adj[e];
                    const float x = a.aux_leaf ? (a.color[u] == ac ? 1.f : 0.f) : a.aux[(size_t)u * a.aux_pitch + ac];
                    buf = __fadd_rn(buf, x);
                }
                const float m = a.main_leaf ? (cv == mc ? 1.f : 0.f) : a.main[(size_t)v * a.main_pitch + mc];
                acc = __fadd_rn(acc, __fmul_rn(buf, m));
            }
            if (a.is_root) rootv = (double)acc;
            else a.out[(size_t)v * a.out_pitch + o] = acc;
        }
        if (!a.is_root)
            for (int o = a.L_s; o < a.out_pitch; ++o) a.out[(size_t)v * a.out_pitch + o] = 0.f;   // row padding
        a.buf[v] = buf;
        if (a.is_root && a.root_vertex) a.root_vertex[v] = rootv;
    }
    if (!a.is_root) return;
    // the block's root values summed in a fixed order
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) rootv = __dadd_rn(rootv, __shfl_down_sync(0xffffffffu, rootv, o));
    if (lane == 0) red[warp] = rootv;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < kOriginalThreads / 32; ++w) s = __dadd_rn(s, red[w]);
        a.partial[blockIdx.x] = s;
    }
}

int launch_original(const OriginalArgs &a, cudaStream_t st)
{
    const int blocks = (a.V + kOriginalThreads - 1) / kOriginalThreads;
    if (blocks > 0) k_original<<<blocks, kOriginalThreads, 0, st>>>(a);
    return blocks;
}

}  // namespace sg
