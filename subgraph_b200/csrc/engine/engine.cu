// Host side of the device engine.
#include "engine.hpp"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>

#include <queue>

#include "blk_sched.hpp"
#include "kernels.cuh"
#include "tile.cuh"

namespace sg {

#define SG_CK(call)                                                                               \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess)                                                                    \
            return Status{3, std::string(#call) + ": " + cudaGetErrorString(e_)};                 \
    } while (0)

#define SG_CKS(st)                 \
    do {                           \
        Status s_ = (st);          \
        if (s_.code) return s_;    \
    } while (0)

// ---------------------------------------------------------------------------
// glibc TYPE_3 stream: window s_0..s_30 of the lag-31 recurrence after
// srandom(seed) (its r_0..r_30 by Schrage's 16807 multiply, s = r_3..r_30,
// r_0, r_1, r_2) and polynomial arithmetic modulo P(x) = x^31 - x^28 - 1.
// ---------------------------------------------------------------------------
void glibc_window(uint32_t seed, uint32_t w[31])
{
    if (seed == 0) seed = 1;
    int32_t r[31];
    int32_t word = (int32_t)seed;
    r[0] = word;
    for (int i = 1; i < 31; ++i) {
        int32_t hi = word / 127773, lo = word % 127773;
        word = 16807 * lo - 2836 * hi;
        if (word < 0) word += 2147483647;
        r[i] = word;
    }
    for (int i = 0; i < 28; ++i) w[i] = (uint32_t)r[i + 3];
    for (int i = 0; i < 3; ++i) w[28 + i] = (uint32_t)r[i];
}

namespace {

using Poly = std::vector<uint32_t>;   // 31 coefficients

Poly poly_mulmod(const Poly &a, const Poly &b)
{
    uint32_t c[61] = {0};
    for (int i = 0; i < 31; ++i) {
        if (!a[i]) continue;
        for (int j = 0; j < 31; ++j) c[i + j] += a[i] * b[j];
    }
    for (int d = 60; d >= 31; --d) {   // x^d = x^(d-3) + x^(d-31)
        c[d - 3] += c[d];
        c[d - 31] += c[d];
        c[d] = 0;
    }
    return Poly(c, c + 31);
}

Poly poly_xpow(uint64_t n)
{
    Poly r(31, 0), base(31, 0);
    r[0] = 1;
    base[1] = 1;
    while (n) {
        if (n & 1) r = poly_mulmod(r, base);
        base = poly_mulmod(base, base);
        n >>= 1;
    }
    return r;
}

int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

// Device buffers reused across count() calls on one graph.
struct Workspace {
    void *arena = nullptr;
    size_t arena_bytes = 0;
    uint8_t *colors = nullptr;
    size_t colors_bytes = 0;
    double *partial = nullptr;
    size_t partial_bytes = 0;
    double *raw = nullptr;
    size_t raw_bytes = 0;
    uint32_t *windows = nullptr;
    size_t windows_bytes = 0;
    void *hub_partial = nullptr;
    size_t hub_partial_bytes = 0;
    int32_t *chunk_start = nullptr;
    size_t chunk_start_bytes = 0;
    double *root_vertex = nullptr;
    size_t root_vertex_bytes = 0;
    int32_t *adjc = nullptr;           // [nnz] neighbour id | color << 28 of the coloring in slot 0
    size_t adjc_bytes = 0;
    float *orig_buf = nullptr;         // [V] isPruned=0 (CSC) aggregation buffer, internal order
    size_t orig_buf_bytes = 0;
    int32_t *hub_ticket = nullptr;     // exact-order hub kernel's item counters, one per concurrent stream
    size_t hub_ticket_bytes = 0;
    int32_t *tile_ticket = nullptr;    // fused kernels' tile counters, one per concurrent stream
    size_t tile_ticket_bytes = 0;
    uint64_t generation = 0;   // bumped whenever a buffer above is re-allocated
};

struct DevicePlanTables {
    std::vector<uint32_t *> split;   // per sub
    std::vector<int32_t *> c2c;      // per sub: output column of each color set in lexicographic order
    std::vector<int16_t *> rem;      // per sub
    std::vector<uint32_t *> aoff, moff;  // per sub: packed-layout byte offsets (FP32)
    std::vector<int32_t *> blk;      // per sub: register-blocked eMA column tables, or null
    std::vector<int32_t> blk_shape, blk_nblocks;
    // per sub: the rooted form (StageDesc::rooted), or null
    std::vector<int32_t *> rblk;
    std::vector<int32_t> rblk_shape, rblk_nblocks, r_Ls, r_La, r_Lm;
    std::vector<uint32_t *> agg_chunk;
    std::vector<int16_t *> main_full, out_rank;
    // per sub with a non-leaf aux child: [k][chunks] masks for 32-byte chunks (8 FP32 / 4 FP64 columns)
    std::vector<uint16_t *> cmask_f32, cmask_f64;
    std::vector<int32_t> cmf32_stride, cmf64_stride;
    // per sub with chunk masks: [k][chunks + 1] count and list of the chunks
    // holding a set that lacks c (StageDesc::cact)
    std::vector<uint16_t *> cact_f32, cact_f64;
    // per sub with chunk masks: [k][32-column groups] masks of the exact-order
    // hub items (HubArgs::gmask)
    std::vector<uint16_t *> hub_gmask;
    std::vector<int32_t> hgm_stride;
};

// The work queue of one batch shape (plan, slots, mode, hubs), built once per
// graph and replayed as a CUDA graph.
struct BatchPlan {
    int slots = 0;
    int nstages = 0, total_items = 0;
    int root_tiles = 0;
    size_t smem = 0;
    BatchStage *d_stages = nullptr;
    int *d_done = nullptr;         // [nstages] completed items
    BatchCtl *d_ctl = nullptr;
    double *d_raw = nullptr;       // [slots] raw counts of the batch
    void *d_hub = nullptr;         // hub partial rows, one region per (slot, sub)
    cudaGraphExec_t exec = nullptr;
    uint64_t generation = 0;       // workspace generation the pointers belong to
    std::vector<BatchStage> host_stages;
};

void free_batch(BatchPlan &b, cudaStream_t stream)
{
    if (b.exec) cudaGraphExecDestroy(b.exec);
    for (void *p : {(void *)b.d_stages, (void *)b.d_done, (void *)b.d_ctl, (void *)b.d_raw, b.d_hub})
        if (p) cudaFreeAsync(p, stream);
    b = BatchPlan();
}

struct GraphState {
    Workspace ws;
    std::map<std::string, BatchPlan> batches; // batch shape -> work queue
    std::vector<cudaStream_t> streams;        // job streams (created on first use)
};

std::string shape_key(const StageDesc &d, bool fp64, int hubs)
{
    char b[160];
    std::snprintf(b, sizeof b, "%d/%d/%d/%d/%d/%d/%d/%d/%d/%d", d.L_s, d.S, d.L_m, d.L_a, d.main_leaf, d.aux_leaf,
                  d.is_root, (int)fp64, d.k, hubs);
    return b;
}

std::map<const DeviceGraph *, GraphState> g_state;
std::mutex g_state_mu;

// Device copies of a plan's index tables.  They depend on the plan alone, so
// one copy per (device, plan) serves every graph (a graph uploaded per call
// finds them ready); release_plan_tables frees them with the plan.
std::map<std::pair<int, uint64_t>, DevicePlanTables> g_plan_tables;   // guarded by g_state_mu

void free_plan_tables(DevicePlanTables &t)
{
    auto drop = [](auto &v) {
        for (auto *p : v)
            if (p) cudaFree(p);
    };
    drop(t.split), drop(t.c2c), drop(t.rem), drop(t.aoff), drop(t.moff), drop(t.blk), drop(t.rblk);
    drop(t.agg_chunk), drop(t.main_full), drop(t.out_rank), drop(t.cmask_f32), drop(t.cmask_f64);
    drop(t.cact_f32), drop(t.cact_f64), drop(t.hub_gmask);
    t = DevicePlanTables();
}

// Autotuner results, process-wide: a graph with the same signature (another
// handle of the same CSC arrays, as the end-to-end path creates per call)
// reuses them.  Key: graph signature | stage shape.
std::map<std::string, TileShape> g_tuned;
std::map<std::string, int> g_hub_tuned;   // exact-order hub kernel variant per graph | row width

std::string graph_sig(const DeviceGraph &g)
{
    char b[96];
    std::snprintf(b, sizeof b, "%d/%d/%lld/%d|", g.device, g.V, (long long)g.nnz, g.max_degree);
    return b;
}

GraphState &state_of(const DeviceGraph &g)
{
    std::lock_guard<std::mutex> lk(g_state_mu);
    return g_state[&g];
}

// Device memory comes from the stream-ordered allocator of the device's
// default pool, which keeps freed memory (release threshold = max): the
// buffers of a destroyed graph are reused by the next one without new
// driver allocations.
void keep_pool_memory(int device)
{
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t thr = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
}

uint64_t g_grow_count = 0;   // re-allocations so far (the workspace generation)

Status grow(void **p, size_t *have, size_t need, cudaStream_t st)
{
    if (need <= *have) return Status::ok();
    ++g_grow_count;
    if (*p) cudaFreeAsync(*p, st);
    *p = nullptr;
    *have = 0;
    cudaError_t e = cudaMallocAsync(p, need, st);
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return Status{2, "device allocation of " + std::to_string(need) + " bytes failed: " + cudaGetErrorString(e)};
    }
    *have = need;
    return Status::ok();
}
template <typename T> Status growT(T **p, size_t *have, size_t need, cudaStream_t st) { return grow((void **)p, have, need, st); }

// Register-blocked eMA tables of sub s: the output color sets (|s| colors out
// of k) partitioned greedily into blocks U of |s|+1 colors, each block the
// column ids of its held sets, streamed sets and outputs (-1: computed by
// another block), laid out as blk::Shape::ROW words.  Every assigned
// output's product sequence under the block schedule is checked against the
// split tables (main_split/aux_split in split order); any difference, or a
// shape without a blocked kernel, leaves the sub on the per-output loop.
// The tables of an index structure: k colors, outputs of n colors, mains of
// pm colors (a sub's own, or the rooted one over k - 1 colors).
struct IndexView {
    int k, n, pm, L, S;
    const int32_t *comb_to_count, *main_split, *aux_split;
};

bool build_blocks(const IndexView &st, std::vector<int32_t> &rows, int &nblocks, int &shape);

bool build_blocks(const Plan &p, int s, std::vector<int32_t> &rows, int &nblocks, int &shape)
{
    const SubTemplate &st = p.subs[s];
    const int pm = p.subs[st.main].size;
    nblocks = 0;
    shape = 0;
    if (s == 0 || pm < 2) return false;
    const IndexView iv{p.k, st.size, pm, st.L, st.S, st.comb_to_count.data(), st.main_split.data(),
                       st.aux_split.data()};
    return build_blocks(iv, rows, nblocks, shape);
}

bool build_blocks(const IndexView &st, std::vector<int32_t> &rows, int &nblocks, int &shape)
{
    const int k = st.k, n = st.n, pm = st.pm;
    nblocks = 0;
    shape = (pm < 1 || n + 1 > k) ? 0 : blk::shape_id(n, pm);
    blk::View v;
    if (!shape || !blk::view_by_id(shape, v)) return false;
    auto colex = [&](unsigned mask) {
        int c[32], m = 0;
        for (int b = 0; b < k; ++b)
            if (mask >> b & 1) c[m++] = b;
        return (int)colex_rank(c, m);
    };
    std::vector<int> lex_of_col(st.L, -1);
    for (int i = 0; i < st.L; ++i) lex_of_col[st.comb_to_count[i]] = i;
    std::vector<char> done(st.L, 0);
    int left = st.L;
    auto gain = [&](unsigned U) {
        int g = 0;
        for (int b = 0; b < k; ++b)
            if ((U >> b & 1) && !done[colex(U & ~(1u << b))]) ++g;
        return g;
    };
    // lazy greedy: the superset covering the most unassigned outputs first
    std::priority_queue<std::pair<int, unsigned>> pq;
    for (unsigned U = 0; U < (1u << k); ++U)
        if (__builtin_popcount(U) == n + 1) pq.push({gain(U), U});
    rows.clear();
    while (left > 0 && !pq.empty()) {
        const auto top = pq.top();
        pq.pop();
        const int g = gain(top.second);
        if (g != top.first) {
            if (g > 0) pq.push({g, top.second});
            continue;
        }
        const unsigned U = top.second;
        int pos[32], m = 0;
        for (int b = 0; b < k; ++b)
            if (U >> b & 1) pos[m++] = b;
        auto global = [&](unsigned local) {
            unsigned gm = 0;
            for (int i = 0; i < m; ++i)
                if (local >> i & 1) gm |= 1u << pos[i];
            return gm;
        };
        std::vector<int32_t> row(v.ROW, 0);
        for (int i = 0; i < v.NH; ++i) row[i] = colex(global(v.held[i]));
        for (int i = 0; i < v.NS; ++i) row[v.NH4 + i] = colex(global(v.str[i]));
        for (int i = 0; i < v.NO4; ++i) row[v.NH4 + v.NS4 + i] = -1;
        for (int o = 0; o < v.NO; ++o) {
            const int col = colex(global(v.out[o]));
            if (!done[col]) {
                done[col] = 1;
                --left;
                row[v.NH4 + v.NS4 + o] = col;
            }
        }
        rows.insert(rows.end(), row.begin(), row.end());
        ++nblocks;
    }
    if (left != 0) return false;
    // the schedule's product order of every output against the split tables
    for (int b = 0; b < nblocks; ++b) {
        const int32_t *row = rows.data() + (size_t)b * v.ROW;
        for (int o = 0; o < v.NO; ++o) {
            const int col = row[v.NH4 + v.NS4 + o];
            if (col < 0) continue;
            const int i = lex_of_col[col];
            int j = 0;
            for (int t = 0; t < v.NS; ++t)
                for (int c = 0; c < v.PER; ++c) {
                    if (v.po[t * v.PER + c] != o) continue;
                    const int hcol = row[v.ph[t * v.PER + c]], tcol = row[v.NH4 + t];
                    const int mc = v.hold_main ? hcol : tcol, ac = v.hold_main ? tcol : hcol;
                    if (i < 0 || j >= st.S || st.main_split[(size_t)i * st.S + j] != mc ||
                        st.aux_split[(size_t)i * st.S + j] != ac)
                        return false;
                    ++j;
                }
            if (j != st.S) return false;
        }
    }
    return true;
}

// the `size` colors (ascending) of the color set with colex rank r
void colex_unrank(int size, int64_t r, int *out)
{
    for (int t = size; t >= 1; --t) {
        int x = t - 1;
        while (binom(x + 1, t) <= r) ++x;
        out[t - 1] = x;
        r -= binom(x, t);
    }
}

// Chunk masks of sub s's aggregation (aux child of >= 2 colors): bit c_u of
// mask[c][j] is set when column chunk j (w columns) holds a color set that
// contains c_u and lacks c.  A vertex of color c reads chunk j of a
// neighbour of color c_u only then: the neighbour's other entries are exact
// zeros (its own color is in every non-zero set), and the columns containing
// c are read by no output or meet a main entry that is an exact zero.
Status upload_chunk_masks(DeviceGraph &g, const Plan &p, int s, DevicePlanTables &out)
{
    const SubTemplate &a = p.subs[p.subs[s].aux];
    const int k = p.k, na = a.size;
    if (na < 2 || k > 16) return Status::ok();
    std::vector<unsigned> am(a.L);
    int el[32];
    for (int t = 0; t < a.L; ++t) {
        colex_unrank(na, t, el);
        unsigned m = 0;
        for (int i = 0; i < na; ++i) m |= 1u << el[i];
        am[t] = m;
    }
    {
        // the exact-order hub items' 32-column groups (FP32 and FP64 alike)
        const int ng = (a.L + 31) / 32;
        std::vector<uint16_t> gm((size_t)k * ng, 0);
        for (int c = 0; c < k; ++c)
            for (int j = 0; j < ng; ++j)
                for (int t = j * 32; t < std::min(a.L, j * 32 + 32); ++t)
                    if (!(am[t] >> c & 1)) gm[(size_t)c * ng + j] |= (uint16_t)(am[t] & 0xffffu);
        SG_CK(cudaMallocAsync(&out.hub_gmask[s], gm.size() * 2, g.stream));
        SG_CK(cudaMemcpyAsync(out.hub_gmask[s], gm.data(), gm.size() * 2, cudaMemcpyHostToDevice, g.stream));
        SG_CK(cudaStreamSynchronize(g.stream));   // `gm` is pageable and goes out of scope
        out.hgm_stride[s] = ng;
    }
    for (int w : {8, 4}) {   // chunk columns: FP32, FP64
        const int nch = (a.L + w - 1) / w;
        std::vector<uint16_t> cm((size_t)k * nch, 0);
        for (int c = 0; c < k; ++c)
            for (int j = 0; j < nch; ++j)
                for (int t = j * w; t < std::min(a.L, j * w + w); ++t)
                    if (!(am[t] >> c & 1)) cm[(size_t)c * nch + j] |= (uint16_t)(am[t] & 0xffffu);
        // a chunk is active for c when some set in it lacks c: its mask is then
        // non-zero (every set holds a color)
        std::vector<uint16_t> ca((size_t)k * (nch + 1), 0);
        for (int c = 0; c < k; ++c) {
            uint16_t *row = &ca[(size_t)c * (nch + 1)];
            for (int j = 0; j < nch; ++j)
                if (cm[(size_t)c * nch + j]) row[1 + row[0]++] = (uint16_t)j;
        }
        uint16_t *&dst = w == 8 ? out.cmask_f32[s] : out.cmask_f64[s];
        uint16_t *&dca = w == 8 ? out.cact_f32[s] : out.cact_f64[s];
        SG_CK(cudaMallocAsync(&dst, cm.size() * 2, g.stream));
        SG_CK(cudaMallocAsync(&dca, ca.size() * 2, g.stream));
        SG_CK(cudaMemcpyAsync(dst, cm.data(), cm.size() * 2, cudaMemcpyHostToDevice, g.stream));
        SG_CK(cudaMemcpyAsync(dca, ca.data(), ca.size() * 2, cudaMemcpyHostToDevice, g.stream));
        SG_CK(cudaStreamSynchronize(g.stream));   // `cm` and `ca` are pageable and go out of scope
        (w == 8 ? out.cmf32_stride : out.cmf64_stride)[s] = nch;
    }
    return Status::ok();
}

// The rooted form of sub s (main and aux of two colors or more): the index
// structure of a stage of |s|-1 colors with mains of |main|-1 over k-1 colors,
// its register-blocked tables, and per vertex color c the compaction tables:
// the rank of every aggregate column lacking c (per 8-column chunk: the first
// rank and the mask of such columns), the table column of every rooted main
// set (the sets holding c, in colex order), and the rooted rank of every
// output column holding c.  Colex order restricted to the sets lacking (or
// holding) c is the colex order of those sets with c removed and the colors
// above c renumbered, so each rank is the count of such columns before it.
Status upload_rooted(DeviceGraph &g, const Plan &p, int s, DevicePlanTables &out)
{
    const SubTemplate &st = p.subs[s];
    const SubTemplate &m = p.subs[st.main], &a = p.subs[st.aux];
    const int k = p.k, n = st.size, pm = m.size, na = a.size;
    if (s == 0 || pm < 2 || na < 2 || k < 3) return Status::ok();
    int L = 0, S = 0;
    std::vector<int32_t> c2c, ms, as;
    index_tables(k - 1, n - 1, pm - 1, L, S, c2c, ms, as);
    const IndexView iv{k - 1, n - 1, pm - 1, L, S, c2c.data(), ms.data(), as.data()};
    std::vector<int32_t> rows;
    int nb = 0, shape = 0;
    if (!build_blocks(iv, rows, nb, shape)) return Status::ok();
    auto mask_of = [&](int size, int col) {
        int el[32];
        colex_unrank(size, col, el);
        unsigned msk = 0;
        for (int i = 0; i < size; ++i) msk |= 1u << el[i];
        return msk;
    };
    const int La = a.L, Lm = m.L, Ls = st.L, nch = (La + 7) / 8;
    const int rLa = (int)binom(k - 1, na), rLm = (int)binom(k - 1, pm - 1);
    std::vector<uint32_t> ach((size_t)k * nch, 0u);
    std::vector<int16_t> mf((size_t)k * rLm, 0), orank((size_t)k * Ls, -1);
    std::vector<unsigned> amask(La), mmask(Lm), omask(Ls);
    for (int t = 0; t < La; ++t) amask[t] = mask_of(na, t);
    for (int t = 0; t < Lm; ++t) mmask[t] = mask_of(pm, t);
    for (int t = 0; t < Ls; ++t) omask[t] = mask_of(n, t);
    for (int c = 0; c < k; ++c) {
        int rank = 0;
        for (int q = 0; q < nch; ++q) {
            uint32_t lack = 0;
            const int base = rank;
            for (int i = 0; i < 8; ++i) {
                const int t = q * 8 + i;
                if (t < La && !(amask[t] >> c & 1u)) { lack |= 1u << i; ++rank; }
            }
            ach[(size_t)c * nch + q] = (uint32_t)base | lack << 16;
        }
        int r = 0;
        for (int t = 0; t < Lm; ++t)
            if (mmask[t] >> c & 1u) mf[(size_t)c * rLm + r++] = (int16_t)t;
        int o = 0;
        for (int t = 0; t < Ls; ++t)
            if (omask[t] >> c & 1u) orank[(size_t)c * Ls + t] = (int16_t)o++;
        if (rank != rLa || r != rLm || o != L) return Status{1, "rooted tables: column counts do not match"};
    }
    SG_CK(cudaMallocAsync(&out.rblk[s], rows.size() * 4, g.stream));
    SG_CK(cudaMallocAsync(&out.agg_chunk[s], ach.size() * 4, g.stream));
    SG_CK(cudaMallocAsync(&out.main_full[s], mf.size() * 2, g.stream));
    SG_CK(cudaMallocAsync(&out.out_rank[s], orank.size() * 2, g.stream));
    SG_CK(cudaMemcpyAsync(out.rblk[s], rows.data(), rows.size() * 4, cudaMemcpyHostToDevice, g.stream));
    SG_CK(cudaMemcpyAsync(out.agg_chunk[s], ach.data(), ach.size() * 4, cudaMemcpyHostToDevice, g.stream));
    SG_CK(cudaMemcpyAsync(out.main_full[s], mf.data(), mf.size() * 2, cudaMemcpyHostToDevice, g.stream));
    SG_CK(cudaMemcpyAsync(out.out_rank[s], orank.data(), orank.size() * 2, cudaMemcpyHostToDevice, g.stream));
    SG_CK(cudaStreamSynchronize(g.stream));   // the host vectors go out of scope
    out.rblk_shape[s] = shape;
    out.rblk_nblocks[s] = nb;
    out.r_Ls[s] = L;
    out.r_La[s] = rLa;
    out.r_Lm[s] = rLm;
    return Status::ok();
}

Status upload_plan(DeviceGraph &g, const Plan &p, DevicePlanTables &out)
{
    out.rblk.assign(p.nsub(), nullptr);
    out.rblk_shape.assign(p.nsub(), 0);
    out.rblk_nblocks.assign(p.nsub(), 0);
    out.r_Ls.assign(p.nsub(), 0);
    out.r_La.assign(p.nsub(), 0);
    out.r_Lm.assign(p.nsub(), 0);
    out.agg_chunk.assign(p.nsub(), nullptr);
    out.main_full.assign(p.nsub(), nullptr);
    out.out_rank.assign(p.nsub(), nullptr);
    out.cmask_f32.assign(p.nsub(), nullptr);
    out.cmask_f64.assign(p.nsub(), nullptr);
    out.cact_f32.assign(p.nsub(), nullptr);
    out.cact_f64.assign(p.nsub(), nullptr);
    out.hub_gmask.assign(p.nsub(), nullptr);
    out.hgm_stride.assign(p.nsub(), 0);
    out.cmf32_stride.assign(p.nsub(), 0);
    out.cmf64_stride.assign(p.nsub(), 0);
    out.blk.assign(p.nsub(), nullptr);
    out.blk_shape.assign(p.nsub(), 0);
    out.blk_nblocks.assign(p.nsub(), 0);
    out.split.assign(p.nsub(), nullptr);
    out.c2c.assign(p.nsub(), nullptr);
    out.rem.assign(p.nsub(), nullptr);
    out.aoff.assign(p.nsub(), nullptr);
    out.moff.assign(p.nsub(), nullptr);
    for (int s = 0; s < p.nsub(); ++s) {
        const SubTemplate &st = p.subs[s];
        if (st.size <= 1) continue;
        // [split j][output column], columns padded to a multiple of 4 (zero pairs)
        const size_t Lsp = (size_t)(st.L + 3) / 4 * 4;
        std::vector<uint32_t> sp(Lsp * st.S, 0u);
        for (int i = 0; i < st.L; ++i) {
            int o = st.comb_to_count[i];
            for (int j = 0; j < st.S; ++j)
                sp[(size_t)j * Lsp + o] = (uint32_t)st.main_split[(size_t)i * st.S + j] |
                                          ((uint32_t)st.aux_split[(size_t)i * st.S + j] << 16);
        }
        SG_CK(cudaMallocAsync(&out.split[s], sp.size() * 4, g.stream));
        SG_CK(cudaMemcpyAsync(out.split[s], sp.data(), sp.size() * 4, cudaMemcpyHostToDevice, g.stream));
        SG_CK(cudaMallocAsync(&out.c2c[s], (size_t)st.L * 4, g.stream));
        SG_CK(cudaMemcpyAsync(out.c2c[s], st.comb_to_count.data(), (size_t)st.L * 4, cudaMemcpyHostToDevice, g.stream));
        SG_CK(cudaStreamSynchronize(g.stream));   // `sp` is pageable and goes out of scope
        if (p.subs[st.main].size > 1 && s != 0) {
            // packed eMA: byte offsets of the aggregate row and of the main row
            // (main rows follow the La_rows aggregate rows) in the shared tile
            const uint32_t rowb = (uint32_t)(kPackedRow * sizeof(float));
            const uint32_t La_rows = p.subs[st.aux].size == 1 ? (uint32_t)p.k : (uint32_t)p.subs[st.aux].L;
            std::vector<uint32_t> ao(sp.size(), 0u), mo(sp.size(), La_rows * rowb);
            for (size_t i = 0; i < sp.size(); ++i) {
                ao[i] = (sp[i] >> 16) * rowb;
                mo[i] = (La_rows + (sp[i] & 0xffffu)) * rowb;
            }
            SG_CK(cudaMallocAsync(&out.aoff[s], ao.size() * 4, g.stream));
            SG_CK(cudaMallocAsync(&out.moff[s], mo.size() * 4, g.stream));
            SG_CK(cudaMemcpyAsync(out.aoff[s], ao.data(), ao.size() * 4, cudaMemcpyHostToDevice, g.stream));
            SG_CK(cudaMemcpyAsync(out.moff[s], mo.data(), mo.size() * 4, cudaMemcpyHostToDevice, g.stream));
            SG_CK(cudaStreamSynchronize(g.stream));
        }
        {
            std::vector<int32_t> rows;
            int nb = 0, shape = 0;
            if (build_blocks(p, s, rows, nb, shape)) {
                SG_CK(cudaMallocAsync(&out.blk[s], rows.size() * 4, g.stream));
                SG_CK(cudaMemcpyAsync(out.blk[s], rows.data(), rows.size() * 4, cudaMemcpyHostToDevice, g.stream));
                SG_CK(cudaStreamSynchronize(g.stream));
                out.blk_shape[s] = shape;
                out.blk_nblocks[s] = nb;
            }
        }
        if (p.subs[st.main].size == 1) {
            std::vector<int16_t> rem((size_t)st.L * p.k, -1);
            for (int i = 0; i < st.L; ++i) {
                int o = st.comb_to_count[i];
                for (int j = 0; j < st.S; ++j)
                    rem[(size_t)o * p.k + st.main_split[(size_t)i * st.S + j]] = (int16_t)st.aux_split[(size_t)i * st.S + j];
            }
            SG_CK(cudaMallocAsync(&out.rem[s], rem.size() * 2, g.stream));
            SG_CK(cudaMemcpyAsync(out.rem[s], rem.data(), rem.size() * 2, cudaMemcpyHostToDevice, g.stream));
        }
        SG_CKS(upload_chunk_masks(g, p, s, out));
        SG_CKS(upload_rooted(g, p, s, out));
    }
    SG_CK(cudaStreamSynchronize(g.stream));
    return Status::ok();
}

struct Hubs {
    int32_t count = 0, chunk = 0, total_chunks = 0;
    bool exact_order = false;
};

// Vertices of degree above `thr` (the first `count` of the degree-descending
// order) are aggregated by the hub kernel.  In exact order each hub is one
// chunk, summed in neighbour-list order with its columns split among lanes
// (the same sums as the per-tile aggregation); otherwise in neighbour chunks
// of `thr` neighbours, one hub item each, whose partial rows are added in
// chunk order (another summation order).
Hubs plan_hubs(const DeviceGraph &g, int thr, bool exact_order)
{
    Hubs h;
    if (thr <= 0) return h;
    h.exact_order = exact_order;
    h.chunk = exact_order ? std::max(thr, g.max_degree) : thr;
    while (h.count < g.V && g.h_degree[h.count] > thr) {
        h.total_chunks += (g.h_degree[h.count] + h.chunk - 1) / h.chunk;
        ++h.count;
    }
    return h;
}

}  // namespace

DeviceGraph::~DeviceGraph()
{
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    {
        std::lock_guard<std::mutex> lk(g_state_mu);
        auto it = g_state.find(this);
        if (it != g_state.end()) {
            Workspace &w = it->second.ws;
            for (void *p : {w.arena, (void *)w.colors, (void *)w.partial, (void *)w.raw, (void *)w.windows, w.hub_partial,
                            (void *)w.chunk_start, (void *)w.root_vertex, (void *)w.adjc, (void *)w.orig_buf,
                            (void *)w.hub_ticket, (void *)w.tile_ticket})
                if (p) cudaFreeAsync(p, stream);
            for (auto &kv : it->second.batches) free_batch(kv.second, stream);
            for (cudaStream_t js : it->second.streams) {
                cudaStreamSynchronize(js);
                cudaStreamDestroy(js);
            }

            g_state.erase(it);
        }
    }
    for (void *p : {(void *)d_off, (void *)d_adj, (void *)d_perm, (void *)d_iperm, (void *)d_jump, (void *)d_coef})
        if (p) cudaFreeAsync(p, stream);
    if (stream) {
        cudaStreamSynchronize(stream);
        cudaStreamDestroy(stream);
    }
    cudaSetDevice(prev);
}

Status new_device_graph(int device, int32_t V, int64_t nnz, std::unique_ptr<DeviceGraph> &out)
{
    int ndev = 0;
    SG_CK(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) return Status{1, "no CUDA device " + std::to_string(device)};
    SG_CK(cudaSetDevice(device));
    auto g = std::make_unique<DeviceGraph>();
    g->device = device;
    g->V = V;
    g->nnz = nnz;
    SG_CK(cudaDeviceGetAttribute(&g->sm_count, cudaDevAttrMultiProcessorCount, device));
    SG_CK(cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking));
    keep_pool_memory(device);
    out = std::move(g);
    return Status::ok();
}

// Jump-ahead polynomials of the coloring blocks: block b starts x^(341 + b *
// kColorBlock) into the glibc stream.  They depend on nothing but b, so one
// process-wide prefix serves every graph (extended when a larger graph needs
// more blocks); the coefficients of x^t (t < kColorBlock) likewise.
static std::mutex g_jump_mu;
static std::vector<uint32_t> g_jump;   // [blocks][31]
static Poly g_jump_next;               // the polynomial of the next block
static std::vector<uint32_t> g_coef;   // [31][kColorBlock]

static void color_tables(int blocks, std::vector<uint32_t> &jump, std::vector<uint32_t> &coef)
{
    std::lock_guard<std::mutex> lk(g_jump_mu);
    if (g_coef.empty()) {
        g_coef.assign((size_t)31 * kColorBlock, 0u);
        Poly q(31, 0);
        q[0] = 1;
        for (int t = 0; t < kColorBlock; ++t) {
            for (int i = 0; i < 31; ++i) g_coef[(size_t)i * kColorBlock + t] = q[i];
            uint32_t top = q[30];
            for (int j = 30; j > 0; --j) q[j] = q[j - 1];
            q[0] = top;
            q[28] += top;
        }
        g_jump_next = poly_xpow(341);
    }
    if ((int64_t)g_jump.size() < (int64_t)blocks * 31) {
        const Poly step = poly_xpow(kColorBlock);
        while ((int64_t)g_jump.size() < (int64_t)blocks * 31) {
            g_jump.insert(g_jump.end(), g_jump_next.begin(), g_jump_next.end());
            g_jump_next = poly_mulmod(g_jump_next, step);
        }
    }
    jump.assign(g_jump.begin(), g_jump.begin() + (size_t)blocks * 31);
    coef = g_coef;
}

// The common tail of every graph upload: the degree order (on the device),
// the relabelled adjacency (k_remap from the original-order device arrays,
// which this frees) and the coloring jump-ahead tables.
Status graph_finish(DeviceGraph &gr, int32_t *d_old_off, int32_t *d_old_adj)
{
    DeviceGraph *g = &gr;
    const int32_t V = g->V;
    const int64_t nnz = g->nnz;
    cudaStream_t st = g->stream;
    SG_CK(cudaMallocAsync(&g->d_off, sizeof(int32_t) * ((size_t)V + 1), st));
    SG_CK(cudaMallocAsync(&g->d_adj, sizeof(int32_t) * std::max<int64_t>(nnz, 1), st));
    SG_CK(cudaMallocAsync(&g->d_perm, sizeof(int32_t) * std::max<int32_t>(V, 1), st));
    SG_CK(cudaMallocAsync(&g->d_iperm, sizeof(int32_t) * std::max<int32_t>(V, 1), st));
    SG_CKS(degree_order(V, d_old_off, g->d_iperm, g->d_perm, g->d_off, g->h_degree, st));
    g->max_degree = V ? g->h_degree[0] : 0;
    int32_t *d_bad = nullptr;
    const int32_t none = INT32_MAX;
    int32_t bad = none;
    SG_CK(cudaMallocAsync(&d_bad, sizeof(int32_t), st));
    SG_CK(cudaMemcpyAsync(d_bad, &none, sizeof(int32_t), cudaMemcpyHostToDevice, st));
    launch_remap(V, d_old_off, d_old_adj, g->d_off, g->d_iperm, g->d_perm, g->d_adj, d_bad, st);
    SG_CK(cudaGetLastError());
    SG_CK(cudaMemcpyAsync(&bad, d_bad, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    cudaFreeAsync(d_bad, st);
    // coloring jump-ahead tables
    g->color_blocks = (V + kColorBlock - 1) / kColorBlock;
    std::vector<uint32_t> jump, coef;
    color_tables(std::max(g->color_blocks, 1), jump, coef);
    SG_CK(cudaMallocAsync(&g->d_jump, jump.size() * 4, st));
    SG_CK(cudaMallocAsync(&g->d_coef, coef.size() * 4, st));
    SG_CK(cudaMemcpyAsync(g->d_jump, jump.data(), jump.size() * 4, cudaMemcpyHostToDevice, st));
    SG_CK(cudaMemcpyAsync(g->d_coef, coef.data(), coef.size() * 4, cudaMemcpyHostToDevice, st));
    cudaFreeAsync(d_old_off, st);
    cudaFreeAsync(d_old_adj, st);
    SG_CK(cudaStreamSynchronize(st));
    if (bad != none) return Status{1, "neighbour id out of range at entry " + std::to_string(bad)};
    return Status::ok();
}

void release_plan_tables(uint64_t uid)
{
    std::lock_guard<std::mutex> lk(g_state_mu);
    int prev = -1;
    for (auto it = g_plan_tables.begin(); it != g_plan_tables.end();) {
        if (it->first.second != uid) {
            ++it;
            continue;
        }
        if (prev < 0) cudaGetDevice(&prev);
        cudaSetDevice(it->first.first);
        free_plan_tables(it->second);   // cudaFree waits for the device's work
        it = g_plan_tables.erase(it);
    }
    if (prev >= 0) cudaSetDevice(prev);
}

Status graph_create(const int32_t *offsets, const int32_t *neighbors, int32_t V, int64_t nnz, int device,
                    std::unique_ptr<DeviceGraph> &out)
{
    if (V < 0 || nnz < 0 || nnz > 0x7fffffffLL) return Status{1, "vertex or entry count out of range"};
    if (!offsets || (nnz > 0 && !neighbors)) return Status{1, "null graph array"};
    if (offsets[0] != 0 || offsets[V] != nnz) return Status{1, "offsets[0] must be 0 and offsets[V] must equal nnz"};
    for (int32_t v = 0; v < V; ++v)
        if (offsets[v + 1] < offsets[v]) return Status{1, "offsets are not monotone"};
    // neighbour ids are range-checked by the remap kernel (graph_finish)
    std::unique_ptr<DeviceGraph> g;
    SG_CKS(new_device_graph(device, V, nnz, g));
    int32_t *d_old_off = nullptr, *d_old_adj = nullptr;
    cudaStream_t st = g->stream;
    SG_CK(cudaMallocAsync(&d_old_off, sizeof(int32_t) * ((size_t)V + 1), st));
    SG_CK(cudaMallocAsync(&d_old_adj, sizeof(int32_t) * std::max<int64_t>(nnz, 1), st));
    SG_CK(cudaMemcpyAsync(d_old_off, offsets, sizeof(int32_t) * ((size_t)V + 1), cudaMemcpyHostToDevice, st));
    if (nnz) SG_CK(cudaMemcpyAsync(d_old_adj, neighbors, sizeof(int32_t) * nnz, cudaMemcpyHostToDevice, st));
    SG_CKS(graph_finish(*g, d_old_off, d_old_adj));
    out = std::move(g);
    return Status::ok();
}

namespace {

struct RunCtx {
    DeviceGraph &g;
    const Plan &p;
    GraphState &gs;
    DevicePlanTables *tab;
    bool fp64;
    size_t es;
    size_t arena_per_coloring;
    Hubs hubs;
    int32_t hub_pitch;
    int64_t launches = 0;
    int mode;
    int root_tiles = 0;
    // profiling: event pairs around every hub and fused launch
    bool profile = false;
    bool autotune = false;
    bool blocked = true;     // register-blocked eMA allowed
    bool rooted = true;      // its rooted form allowed
    bool flat = true;        // the flat aggregation allowed
    int lay = 1;             // colorings interleaved per table row (grouped batched form)
    size_t arena_base = 0;   // byte offset of this context's tables in the arena (job queues)
    bool exact = false;      // no fused products (packed eMA), no hub chunks
    bool use_adjc = false;   // one coloring at a time per slot: neighbour ids carry their colors
    void *hub_region = nullptr;  // this context's hub partial rows (job streams), else the workspace's
    int ticket = 0;              // its hub item and tile counters (job streams: the stream's)
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> fused_ev, hub_ev;
    std::vector<std::pair<int, double>> fused_sub;   // per fused launch: sub, compulsory bytes
    double fused_alg_bytes = 0, fused_gather_bytes = 0;
};

Status ev_pair(std::vector<std::pair<cudaEvent_t, cudaEvent_t>> &v)
{
    cudaEvent_t a, b;
    SG_CK(cudaEventCreate(&a));
    SG_CK(cudaEventCreate(&b));
    v.push_back({a, b});
    return Status::ok();
}

double ev_sum(std::vector<std::pair<cudaEvent_t, cudaEvent_t>> &v)
{
    double t = 0;
    for (auto &e : v) {
        float ms = 0;
        cudaEventElapsedTime(&ms, e.first, e.second);
        t += ms;
        cudaEventDestroy(e.first);
        cudaEventDestroy(e.second);
    }
    v.clear();
    return t;
}

// The sub whose fused launches took the most summed time (profile mode):
// its launches, time and compulsory bytes.  Reads the events before ev_sum
// releases them.
void top_stage(RunCtx &c, CountStats *stats)
{
    std::map<int, std::pair<double, double>> per;   // sub -> (ms, bytes)
    std::map<int, int64_t> n;
    for (size_t i = 0; i < c.fused_ev.size() && i < c.fused_sub.size(); ++i) {
        float ms = 0;
        cudaEventElapsedTime(&ms, c.fused_ev[i].first, c.fused_ev[i].second);
        auto &e = per[c.fused_sub[i].first];
        e.first += ms;
        e.second += c.fused_sub[i].second;
        ++n[c.fused_sub[i].first];
    }
    stats->top_sub = -1;
    for (auto &kv : per)
        if (kv.second.first > stats->top_ms) {
            stats->top_sub = kv.first;
            stats->top_ms = kv.second.first;
            stats->top_alg_bytes = kv.second.second;
            stats->top_launches = n[kv.first];
        }
}

Status prepare(RunCtx &c, int ncolor_slots, int ncolorings_total)
{
    DeviceGraph &g = c.g;
    GraphState &gs = c.gs;
    Workspace &w = gs.ws;
    const size_t V = (size_t)g.V;
    c.arena_per_coloring = (size_t)(c.mode == kModeOriginal ? c.p.arena_units_all : c.p.arena_units) * V * c.es;
    SG_CKS(grow(&w.arena, &w.arena_bytes, std::max<size_t>(16, c.arena_per_coloring * ncolor_slots), g.stream));
    SG_CKS(growT(&w.colors, &w.colors_bytes, std::max<size_t>(16, V * ncolor_slots), g.stream));
    SG_CKS(growT(&w.tile_ticket, &w.tile_ticket_bytes, 4 * 64, g.stream));
    SG_CKS(growT(&w.partial, &w.partial_bytes, 8 * ((V / 8 + 2) * ncolor_slots), g.stream));
    SG_CKS(growT(&w.raw, &w.raw_bytes, 8 * (size_t)std::max(ncolorings_total, 1), g.stream));
    SG_CKS(growT(&w.windows, &w.windows_bytes, 4 * 31 * (size_t)std::max(ncolorings_total, 1), g.stream));
    if (c.use_adjc)   // one colour-tagged adjacency per coloring of a slot (the interleaved group's)
        SG_CKS(growT(&w.adjc, &w.adjc_bytes, std::max<size_t>(16, 4 * (size_t)g.nnz * c.lay), g.stream));
    if (c.mode == kModeOriginal) SG_CKS(growT(&w.orig_buf, &w.orig_buf_bytes, std::max<size_t>(16, 4 * V), g.stream));
    if (c.hubs.count > 0) {
        // a partial row holds the aux columns (or colour counts) of up to c.lay colorings
        int32_t maxp = round_up(c.lay * c.p.k, 8);
        for (int s : c.p.process_order) {
            const SubTemplate &st = c.p.subs[s];
            const SubTemplate &a = c.p.subs[st.aux];
            if (a.size > 1) maxp = std::max<int32_t>(maxp, c.lay * c.p.table_pitch[st.aux]);
        }
        c.hub_pitch = maxp;
        SG_CKS(grow(&w.hub_partial, &w.hub_partial_bytes, (size_t)c.hubs.total_chunks * maxp * c.es, g.stream));
        std::vector<int32_t> cs((size_t)c.hubs.count + 1, 0);
        for (int h = 0; h < c.hubs.count; ++h) cs[h + 1] = cs[h] + (g.h_degree[h] + c.hubs.chunk - 1) / c.hubs.chunk;
        SG_CKS(growT(&w.chunk_start, &w.chunk_start_bytes, 4 * cs.size(), g.stream));
        SG_CK(cudaMemcpyAsync(w.chunk_start, cs.data(), 4 * cs.size(), cudaMemcpyHostToDevice, g.stream));
        SG_CKS(growT(&w.hub_ticket, &w.hub_ticket_bytes, 4 * 64, g.stream));
    }
    return Status::ok();
}

// Table of sub `sub` in color slot `slot`; with c.lay colorings interleaved
// the table is [V][lay][pitch] at lay times the per-coloring offset.
void *table_ptr(RunCtx &c, int slot, int sub)
{
    const int64_t off = c.mode == kModeOriginal ? c.p.table_offset_all[sub] : c.p.table_offset[sub];
    return (char *)c.gs.ws.arena + c.arena_base + c.arena_per_coloring * slot + (size_t)c.lay * off * c.g.V * c.es;
}

// A sub whose table an earlier sub of the same structure already computed
// (Plan::same_as) is not run again; the isPruned=0 CSC mode runs every sub.
bool shared_table(const RunCtx &c, int s) { return c.mode != kModeOriginal && c.p.same_as[s] >= 0; }

// neighbour ids with their color in the top 4 bits: ids below 2^28, colors below 16
bool adjc_ok(const DeviceGraph &g, const Plan &p) { return g.V < (1 << 28) && p.k <= 16 && g.nnz > 0; }

// The descriptor of one sub-template step of the coloring in color slot `slot`,
// or of colorings [b0, b0 + nb) of an interleaved group (c.lay > 1, slot 0);
// shape fields are left for plan_fused / set_shape.
StageDesc make_stage(RunCtx &c, int slot, int s, double *root_vertex, int b0 = 0, int nb = 1)
{
    const Plan &p = c.p;
    const SubTemplate &sub = p.subs[s];
    const SubTemplate &m = p.subs[sub.main], &a = p.subs[sub.aux];
    DeviceGraph &g = c.g;
    Workspace &w = c.gs.ws;
    StageDesc d{};
    d.V = g.V;
    d.L_s = sub.L;
    d.S = sub.S;
    d.k = p.k;
    d.ticket = w.tile_ticket ? w.tile_ticket + c.ticket : nullptr;
    d.main_leaf = m.size == 1;
    d.aux_leaf = a.size == 1;
    d.L_m = m.L;
    d.L_a = a.L;
    d.is_root = s == 0;
    d.scaled = (c.mode == kModeReference && s == p.scaled_sub && s != 0) ? 1 : 0;
    d.root_float = c.mode == kModeOriginal || c.mode == kModeOriginalCSR;
    const int L = c.lay;
    const int ps = s == 0 ? 0 : p.table_pitch[s];
    const int pm = d.main_leaf ? 0 : p.table_pitch[sub.main];
    const int pa = d.aux_leaf ? 0 : p.table_pitch[sub.aux];
    d.nb = nb;
    d.cstride = L;
    d.out_pitch = L * ps;
    d.main_pitch = L * pm;
    d.aux_pitch = L * pa;
    d.aux_cols = d.aux_leaf ? nb * p.k : (nb == 1 ? a.L : nb * pa);   // one-hot: the histogram's columns
    d.a_cstride = d.aux_leaf ? p.k : pa;
    d.main_cols = nb == 1 ? m.L : nb * pm;
    d.m_cstride = pm;
    d.out_w = nb * ps;
    d.s_cstride = ps;
    d.rp_stride = g.V / 8 + 2;
    d.main = d.main_leaf ? nullptr : (char *)table_ptr(c, slot, sub.main) + (size_t)b0 * pm * c.es;
    d.aux = d.aux_leaf ? nullptr : (char *)table_ptr(c, slot, sub.aux) + (size_t)b0 * pa * c.es;
    d.out = s == 0 ? nullptr : (char *)table_ptr(c, slot, s) + (size_t)b0 * ps * c.es;
    d.split = c.tab->split[s];
    d.split_stride = (sub.L + 3) / 4 * 4;
    d.rem = c.tab->rem[s];
    // the packed eMA fuses multiply and add: only outside exact mode
    d.aoff = c.exact ? nullptr : c.tab->aoff[s];
    d.moff = c.exact ? nullptr : c.tab->moff[s];
    // the blocked eMA keeps the split order of every output: exact mode may use it
    d.blk = (c.fp64 || !c.blocked) ? nullptr : c.tab->blk[s];
    d.blk_shape = d.blk ? c.tab->blk_shape[s] : 0;
    d.blk_nblocks = d.blk ? c.tab->blk_nblocks[s] : 0;
    d.ublk = d.blk;
    d.ublk_shape = d.blk_shape;
    d.ublk_nblocks = d.blk_nblocks;
    // the rooted form skips exact-zero products: FP32 reference arithmetic only
    // (isPruned=0 tables may hold inf, where a skipped 0 * inf would be NaN);
    // one coloring a launch (of an interleaved group: a strided view of it)
    if (!c.fp64 && c.blocked && c.rooted && c.mode == kModeReference && nb == 1 && c.tab->rblk[s]) {
        d.rblk = c.tab->rblk[s];
        d.rblk_shape = c.tab->rblk_shape[s];
        d.rblk_nblocks = c.tab->rblk_nblocks[s];
        d.r_Ls = c.tab->r_Ls[s];
        d.r_La = c.tab->r_La[s];
        d.r_Lm = c.tab->r_Lm[s];
        d.agg_chunk = c.tab->agg_chunk[s];
        d.main_full = c.tab->main_full[s];
        d.out_rank = c.tab->out_rank[s];
    }
    d.color = w.colors + (size_t)slot * g.V + b0;
    if (c.use_adjc && nb == 1) {
        d.adjc = w.adjc + ((size_t)slot * L + b0) * g.nnz;
        d.cmask = c.fp64 ? c.tab->cmask_f64[s] : c.tab->cmask_f32[s];
        d.cmask_stride = c.fp64 ? c.tab->cmf64_stride[s] : c.tab->cmf32_stride[s];
        d.ucact = !c.flat ? nullptr : c.fp64 ? c.tab->cact_f64[s] : c.tab->cact_f32[s];
        d.cact_stride = d.cmask_stride + 1;
    }
    d.off = g.d_off;
    d.adj = g.d_adj;
    d.root_partial = w.partial + (size_t)(slot + b0) * (g.V / 8 + 2);
    d.root_vertex = nb == 1 ? root_vertex : nullptr;
    return d;
}

// The hub aggregation feeding stage d, writing its partial rows to `partial`;
// also points d at those rows.
HubArgs make_hub(RunCtx &c, StageDesc &d, void *partial, int s)
{
    DeviceGraph &g = c.g;
    HubArgs h{};
    h.hub_count = c.hubs.count;
    h.chunk = c.hubs.chunk;
    h.L_a = d.aux_cols;
    h.aux_pitch = d.aux_pitch;
    h.row_pitch = c.hub_pitch;
    h.k_leaf = d.aux_leaf ? c.p.k : 0;
    h.nb = d.nb;
    h.cstride = d.cstride;
    h.color = d.color;
    h.adjc = d.adjc;
    h.total_chunks = c.hubs.total_chunks;
    h.chunk_start = c.gs.ws.chunk_start;
    h.exact_order = c.hubs.exact_order ? 1 : 0;
    h.off = g.d_off;
    h.adj = g.d_adj;
    h.aux = d.aux;
    h.partial = partial;
    h.ticket = c.gs.ws.hub_ticket ? c.gs.ws.hub_ticket + c.ticket : nullptr;
    // skipped slices need the exact-zero structure of the reference and FP64
    // tables (isPruned=0 runs no hub kernel) and the colour-tagged ids
    if (h.exact_order && !h.k_leaf && d.adjc && d.nb == 1 && c.tab->hub_gmask[s] &&
        (c.mode == kModeReference || c.mode == kModeFP64)) {
        h.gmask = c.tab->hub_gmask[s];
        h.gmask_stride = c.tab->hgm_stride[s];
    }
    d.hub_count = c.hubs.count;
    d.hub_pitch = c.hub_pitch;
    d.hub_chunk_start = c.gs.ws.chunk_start;
    d.hub_partial = partial;
    return h;
}

// One isPruned=0 step on a CSC graph (k_original): the running aggregation
// buffer is the workspace's orig_buf.
Status run_stage_original(RunCtx &c, int slot, int s, double *root_vertex, cudaStream_t st)
{
    const Plan &p = c.p;
    const SubTemplate &sub = p.subs[s];
    const SubTemplate &m = p.subs[sub.main], &a = p.subs[sub.aux];
    OriginalArgs o{};
    o.V = c.g.V;
    o.L_s = sub.L;
    o.S = sub.S;
    o.split_stride = (sub.L + 3) / 4 * 4;
    o.split = c.tab->split[s];
    o.c2c = c.tab->c2c[s];
    o.main_leaf = m.size == 1;
    o.aux_leaf = a.size == 1;
    o.is_root = s == 0;
    o.main = o.main_leaf ? nullptr : (const float *)table_ptr(c, slot, sub.main);
    o.main_pitch = o.main_leaf ? 0 : p.table_pitch[sub.main];
    o.aux = o.aux_leaf ? nullptr : (const float *)table_ptr(c, slot, sub.aux);
    o.aux_pitch = o.aux_leaf ? 0 : p.table_pitch[sub.aux];
    o.out = s == 0 ? nullptr : (float *)table_ptr(c, slot, s);
    o.out_pitch = s == 0 ? 0 : p.table_pitch[s];
    o.color = c.gs.ws.colors + (size_t)slot * c.g.V;
    o.off = c.g.d_off;
    o.adj = c.g.d_adj;
    o.buf = c.gs.ws.orig_buf;
    o.partial = c.gs.ws.partial + (size_t)slot * (c.g.V / 8 + 2);
    o.root_vertex = root_vertex;
    const int blocks = launch_original(o, st);
    c.launches += 1;
    if (s == 0) c.root_tiles = blocks;
    SG_CK(cudaGetLastError());
    return Status::ok();
}

// One sub-template step of the coloring in color slot `slot`.
Status run_stage(RunCtx &c, int slot, int s, double *root_vertex, cudaStream_t st, int b0 = 0, int nb = 1)
{
    if (c.mode == kModeOriginal) return run_stage_original(c, slot, s, root_vertex, st);
    if (shared_table(c, s)) return Status::ok();
    DeviceGraph &g = c.g;
    StageDesc d = make_stage(c, slot, s, root_vertex, b0, nb);
    if (c.hubs.count > 0) {
        HubArgs h = make_hub(c, d, c.hub_region ? c.hub_region : c.gs.ws.hub_partial, s);
        int variant = 0;
        if (h.exact_order && !h.k_leaf) {
            // the exact-order hub kernel's (threads, ring depth) pair: timed once per
            // graph and row width (all variants compute the same rows)
            const std::string key = graph_sig(g) + "hub/" + std::to_string(h.L_a) + "/" + std::to_string(h.hub_count) +
                                    "/" + std::to_string((int)c.fp64);
            bool have = false;
            {
                std::lock_guard<std::mutex> lk(g_state_mu);
                auto it = g_hub_tuned.find(key);
                if (it != g_hub_tuned.end()) { variant = it->second; have = true; }
            }
            if (!have && c.autotune) {
                cudaEvent_t e0, e1;
                SG_CK(cudaEventCreate(&e0));
                SG_CK(cudaEventCreate(&e1));
                float best = 1e30f;
                for (int vv = 0; vv < hub_variants(); ++vv) {
                    launch_hub(h, c.fp64, g.sm_count, st, vv);   // untimed: module load
                    SG_CK(cudaEventRecord(e0, st));
                    launch_hub(h, c.fp64, g.sm_count, st, vv);
                    SG_CK(cudaEventRecord(e1, st));
                    SG_CK(cudaEventSynchronize(e1));
                    SG_CK(cudaGetLastError());
                    float t = 0;
                    cudaEventElapsedTime(&t, e0, e1);
                    c.launches += 2;
                    if (t < best) { best = t; variant = vv; }
                    if (std::getenv("SG_TUNE_LOG"))
                        std::fprintf(stderr, "[sg tune] hub %s variant %d: %.3f ms\n", key.c_str(), vv, t);
                }
                cudaEventDestroy(e0);
                cudaEventDestroy(e1);
                std::lock_guard<std::mutex> lk(g_state_mu);
                g_hub_tuned[key] = variant;
            }
        }
        if (c.profile) {
            SG_CKS(ev_pair(c.hub_ev));
            SG_CK(cudaEventRecord(c.hub_ev.back().first, st));
        }
        launch_hub(h, c.fp64, g.sm_count, st, variant);
        if (c.profile) SG_CK(cudaEventRecord(c.hub_ev.back().second, st));
        c.launches += 1;
    }
    FusedConfig cfg;
    if (!plan_fused(d, c.fp64, g.sm_count, cfg))
        return Status{6, "sub-template " + std::to_string(s) + " needs more shared memory than a CTA has"};
    {
        // autotuner: the first time a stage shape runs on this graph, time every
        // (tile vertices, CTA threads) candidate on the real inputs; all of them
        // compute the same values, so the trial launches only cost time
        const std::string key = graph_sig(g) + shape_key(d, c.fp64, c.hubs.count) + (d.aoff ? "/pk" : "/ex") +
                                (d.blk ? "/bk" : "") + (d.rblk ? "/rt" : "") + "/n" + std::to_string(d.nb) + "/l" +
                                std::to_string(c.lay);
        TileShape pick{d.tile_v, d.nthreads, d.packed};
        bool have = false;
        {
            std::lock_guard<std::mutex> lk(g_state_mu);
            auto it = g_tuned.find(key);
            if (it != g_tuned.end()) { pick = it->second; have = true; }
        }
        if (!have && c.autotune) {
            cudaEvent_t e0, e1;
            SG_CK(cudaEventCreate(&e0));
            SG_CK(cudaEventCreate(&e1));
            float best = 1e30f;
            for (auto cand : candidate_shapes(d, c.fp64)) {
                StageDesc dc = d;
                if (!set_shape(dc, c.fp64, cand)) continue;
                FusedConfig cc = cfg;
                cc.smem = dc.smem;
                // one untimed launch (the first launch of a kernel also loads its
                // module), then the faster of two timed ones
                launch_fused(dc, c.fp64, cc, st);
                float ms = 1e30f;
                for (int rep = 0; rep < 2; ++rep) {
                    SG_CK(cudaEventRecord(e0, st));
                    launch_fused(dc, c.fp64, cc, st);
                    SG_CK(cudaEventRecord(e1, st));
                    SG_CK(cudaEventSynchronize(e1));
                    SG_CK(cudaGetLastError());
                    float t = 0;
                    cudaEventElapsedTime(&t, e0, e1);
                    ms = std::min(ms, t);
                }
                c.launches += 3;
                if (ms < best) { best = ms; pick = cand; }
                if (std::getenv("SG_TUNE_LOG"))
                    std::fprintf(stderr, "[sg tune] sub %d shape %s tile %d threads %d packed %d q %d group %d mask %d: %.3f ms\n",
                                 s, key.c_str(), cand.tile_v, cand.threads, cand.packed, dc.gather_q, dc.gather_group,
                                 dc.cact ? 2 : dc.cmask ? 1 : 0, ms);
            }
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            std::lock_guard<std::mutex> lk(g_state_mu);
            g_tuned[key] = pick;
            have = true;
        }
        if (have && set_shape(d, c.fp64, pick)) cfg.smem = d.smem;
    }
    if (c.profile) {
        SG_CKS(ev_pair(c.fused_ev));
        SG_CK(cudaEventRecord(c.fused_ev.back().first, st));
    }
    launch_fused(d, c.fp64, cfg, st);
    if (c.profile) {
        SG_CK(cudaEventRecord(c.fused_ev.back().second, st));
        // compulsory traffic: main and aux tables read once (a one-hot child is read
        // as the colors array: one element per vertex), the output written once and
        // the adjacency read once (offsets + neighbour ids)
        const double V = (double)g.V, nb = (double)d.nb;
        const double lm = d.main_leaf ? 1.0 : (double)d.L_m, la = d.aux_leaf ? 1.0 : (double)d.L_a;
        const double alg = nb * (double)c.es * V * (lm + la + (s ? (double)d.L_s : 0.0)) + 4.0 * (V + 1 + (double)g.nnz);
        c.fused_alg_bytes += alg;
        c.fused_sub.push_back({s, alg});
        c.fused_gather_bytes += nb * (double)c.es * (double)g.nnz * (d.aux_leaf ? 0.25 : (double)d.L_a);
    }
    c.launches += 1;
    if (s == 0) c.root_tiles = d.ntiles;
    SG_CK(cudaGetLastError());
    return Status::ok();
}

// Colors of colorings [first_coloring, +n) into slots [slot0, +n); on the
// one-coloring-at-a-time path also the colored adjacency of slot 0.
Status launch_colors(RunCtx &c, int slot0, int first_coloring, int n, cudaStream_t st)
{
    ColorArgs a{};
    a.V = c.g.V;
    a.k = c.p.k;
    a.nblocks = c.g.color_blocks;
    a.jump = c.g.d_jump;
    a.coef = c.g.d_coef;
    a.window = c.gs.ws.windows + 31 * (size_t)first_coloring;
    a.perm = c.g.d_perm;
    a.color = c.gs.ws.colors + (size_t)slot0 * c.g.V;
    a.color_stride = c.lay == 1 ? c.g.V : 1;   // [n][V], or interleaved [V][lay]
    a.vertex_stride = c.lay;
    launch_color(a, n, st);
    c.launches += 1;
    if (c.use_adjc && (c.lay == 1 ? n == 1 : n <= c.lay)) {
        // one colour-tagged adjacency per coloring: slot slot0's, or each of the
        // interleaved group's (colours [V][lay])
        for (int b = 0; b < (c.lay == 1 ? 1 : n); ++b) {
            launch_color_adj(c.g.d_adj, c.g.nnz, c.gs.ws.colors + (size_t)slot0 * c.g.V + b, c.lay,
                             c.gs.ws.adjc + ((size_t)slot0 * c.lay + b) * c.g.nnz, st);
            c.launches += 1;
        }
    }
    SG_CK(cudaGetLastError());
    return Status::ok();
}

Status make_ctx_tables(DeviceGraph &g, const Plan &p, GraphState &, DevicePlanTables *&tab)
{
    const std::pair<int, uint64_t> key{g.device, p.uid};
    {
        std::lock_guard<std::mutex> lk(g_state_mu);
        auto it = g_plan_tables.find(key);
        if (it != g_plan_tables.end()) {
            tab = &it->second;
            return Status::ok();
        }
    }
    // uploaded on this graph's stream and synchronised (upload_plan), so any
    // stream may read them afterwards
    DevicePlanTables t;
    Status st = upload_plan(g, p, t);
    if (st.code) {
        free_plan_tables(t);
        return st;
    }
    std::lock_guard<std::mutex> lk(g_state_mu);
    auto ins = g_plan_tables.try_emplace(key, std::move(t));
    if (!ins.second) free_plan_tables(t);   // another thread uploaded them first
    tab = &ins.first->second;
    return Status::ok();
}

Status upload_windows(RunCtx &c, uint32_t seed_base, int n)
{
    std::vector<uint32_t> win((size_t)n * 31);
    for (int i = 0; i < n; ++i) glibc_window(seed_base + (uint32_t)i, &win[(size_t)i * 31]);
    SG_CK(cudaMemcpyAsync(c.gs.ws.windows, win.data(), win.size() * 4, cudaMemcpyHostToDevice, c.g.stream));
    SG_CK(cudaStreamSynchronize(c.g.stream));   // `win` is pageable and goes out of scope
    return Status::ok();
}

// Tile shape of a stage in the persistent kernel (1024 threads, one CTA per SM).
// Tile shape of a stage in the persistent kernel (kBatchThreads threads, up
// to two CTAs per SM): the candidates that leave room for two CTAs first.
std::vector<TileShape> batch_candidates(const StageDesc &d)
{
    const bool heavy = !d.main_leaf && !d.is_root && (int64_t)d.S * d.L_s >= 512;
    if (d.aux_leaf) return {{256, kBatchThreads, 0}, {128, kBatchThreads, 0}, {64, kBatchThreads, 0}, {32, kBatchThreads, 0}};
    if (heavy) return {{32, kBatchThreads, 1}, {32, kBatchThreads, 0}, {16, kBatchThreads, 0}, {8, kBatchThreads, 0}};
    return {{32, kBatchThreads, 0}, {16, kBatchThreads, 0}, {8, kBatchThreads, 0}};
}

bool batch_shape(StageDesc &d, bool fp64)
{
    const std::vector<TileShape> cands = batch_candidates(d);
    for (auto &t : cands) {
        StageDesc e = d;
        if (set_shape(e, fp64, t) && e.smem <= 113 * 1024) {
            d = e;
            return true;
        }
    }
    for (auto &t : cands)
        if (set_shape(d, fp64, t)) return true;
    return false;
}

// The persistent kernel runs the tile body of the plain kernel of the same
// thread count, so a stage's queue shape is chosen by timing the candidates
// (those under 113 KB of shared memory when any fit) through that kernel on
// the stage's own buffers: trial launches read whatever the inputs hold and
// write the stage's output, which the queue rewrites.  Cached process-wide by
// graph signature and stage shape.
std::map<std::string, TileShape> g_batch_tuned;

Status queue_shape(RunCtx &c, StageDesc &d)
{
    const std::string key = graph_sig(c.g) + shape_key(d, c.fp64, c.hubs.count) + (d.aoff ? "/pk" : "/ex") + "/queue";
    {
        std::lock_guard<std::mutex> lk(g_state_mu);
        auto it = g_batch_tuned.find(key);
        if (it != g_batch_tuned.end() && set_shape(d, c.fp64, it->second)) return Status::ok();
    }
    if (!c.autotune) {
        if (!batch_shape(d, c.fp64)) return Status{6, "a sub-template needs more shared memory than a CTA has"};
        return Status::ok();
    }
    std::vector<TileShape> fit, all;
    for (const TileShape &t : batch_candidates(d)) {
        StageDesc e = d;
        if (!set_shape(e, c.fp64, t)) continue;
        all.push_back(t);
        if (e.smem <= 113 * 1024) fit.push_back(t);
    }
    const std::vector<TileShape> &cands = fit.empty() ? all : fit;
    if (cands.empty()) return Status{6, "a sub-template needs more shared memory than a CTA has"};
    cudaStream_t st = c.g.stream;
    // the queue is built before its colorings' colors exist, and colors are
    // indices (histogram rows, rem lookups): give the trial launches valid
    // ones (0 < k); the queue's own color launch overwrites them
    SG_CK(cudaMemsetAsync(const_cast<uint8_t *>(d.color), 0, (size_t)c.g.V * (size_t)d.cstride, st));
    cudaEvent_t e0, e1;
    SG_CK(cudaEventCreate(&e0));
    SG_CK(cudaEventCreate(&e1));
    float best = 1e30f;
    TileShape pick = cands.front();
    for (const TileShape &t : cands) {
        StageDesc e = d;
        set_shape(e, c.fp64, t);
        FusedConfig cfg;
        cfg.tile_v = e.tile_v;
        cfg.q = e.gather_q;
        cfg.smem = e.smem;
        cfg.grid = c.g.sm_count;
        launch_fused(e, c.fp64, cfg, st);
        float ms = 1e30f;
        for (int rep = 0; rep < 2; ++rep) {
            SG_CK(cudaEventRecord(e0, st));
            launch_fused(e, c.fp64, cfg, st);
            SG_CK(cudaEventRecord(e1, st));
            SG_CK(cudaEventSynchronize(e1));
            SG_CK(cudaGetLastError());
            float tt = 0;
            cudaEventElapsedTime(&tt, e0, e1);
            ms = std::min(ms, tt);
        }
        if (ms < best) { best = ms; pick = t; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    {
        std::lock_guard<std::mutex> lk(g_state_mu);
        g_batch_tuned[key] = pick;
    }
    set_shape(d, c.fp64, pick);
    return Status::ok();
}

// The queue stages of one coloring slot of context c: per sub (in processing
// order, one call per sub) the hub chunks (when the graph has hubs) and the
// fused tile groups.  `fused` / `hub` map the slot's subs to stage indices;
// `hub_region` is this (slot, sub)'s partial-row buffer.
struct QueueSlot {
    std::vector<int> proc_index, fused, hub;
    int root_tiles = 0;
    explicit QueueSlot(const Plan &p) : proc_index(p.nsub(), -1), fused(p.nsub(), -1), hub(p.nsub(), -1)
    {
        for (size_t i = 0; i < p.process_order.size(); ++i) proc_index[p.process_order[i]] = (int)i;
    }
};

Status add_queue_stage(RunCtx &c, int slot, int s, void *hub_region, QueueSlot &q, std::vector<BatchStage> &S,
                       int &item, size_t &smem)
{
    const Plan &p = c.p;
    const SubTemplate &sub = p.subs[s];
    if (shared_table(c, s)) {   // its readers wait for the sub that computes the table
        q.fused[s] = q.fused[p.same_as[s]];
        return Status::ok();
    }
    StageDesc d = make_stage(c, slot, s, nullptr);
    if (c.hubs.count > 0) {
        BatchStage hs{};
        hs.kind = kStageHub;
        hs.h = make_hub(c, d, hub_region, s);
        hs.first_item = item;
        hs.nitems = (c.hubs.total_chunks + kHubItemChunks - 1) / kHubItemChunks;
        if (p.subs[sub.aux].size > 1) hs.deps[hs.ndeps++] = q.fused[sub.aux];
        item += hs.nitems;
        q.hub[s] = (int)S.size();
        S.push_back(hs);
    }
    SG_CKS(queue_shape(c, d));
    BatchStage fs{};
    fs.kind = kStageFused;
    fs.d = d;
    fs.tiles_per_item = std::max(1, 1024 / d.tile_v);
    fs.first_item = item;
    fs.nitems = (d.ntiles + fs.tiles_per_item - 1) / fs.tiles_per_item;
    std::vector<int> deps;
    if (p.subs[sub.main].size > 1) deps.push_back(q.fused[sub.main]);
    if (p.subs[sub.aux].size > 1) deps.push_back(q.fused[sub.aux]);
    if (c.hubs.count > 0) deps.push_back(q.hub[s]);
    // write after read: the arena gives this table the range of tables
    // already consumed; their consumers may still be reading it
    if (s != 0) {
        const int64_t lo = p.table_offset[s], hi = lo + p.table_pitch[s];
        for (int x : p.process_order) {
            if (x == s) break;
            const int par = p.subs[x].parent;
            if (x == 0 || par < 0 || par >= p.nsub() || q.proc_index[par] >= q.proc_index[s]) continue;
            const int64_t xlo = p.table_offset[x], xhi = xlo + p.table_pitch[x];
            if (xlo < hi && lo < xhi) {
                const int dep = q.fused[par];
                if (std::find(deps.begin(), deps.end(), dep) == deps.end()) deps.push_back(dep);
            }
        }
    }
    if ((int)deps.size() > kBatchMaxDeps)
        return Status{6, "sub-template " + std::to_string(s) + " needs more queue dependencies than a stage holds"};
    for (int dep : deps) fs.deps[fs.ndeps++] = dep;
    item += fs.nitems;
    smem = std::max(smem, d.smem);
    if (s == 0) q.root_tiles = d.ntiles;
    q.fused[s] = (int)S.size();
    S.push_back(fs);
    return Status::ok();
}

// Builds the work queue of a batch of `slots` colorings: for every sub in
// processing order and every slot, the hub chunks (when the graph has hubs)
// and the fused tile groups of that (slot, sub) stage.
Status build_batch(RunCtx &c, int slots, bool poison, BatchPlan &bp)
{
    const Plan &p = c.p;
    DeviceGraph &g = c.g;
    const int nproc = (int)p.process_order.size();
    const size_t hub_region = (size_t)c.hubs.total_chunks * (size_t)std::max(c.hub_pitch, 4) * c.es;
    if (c.hubs.count > 0) {
        const size_t bytes = std::max<size_t>(16, hub_region * (size_t)slots * nproc);
        SG_CK(cudaMallocAsync(&bp.d_hub, bytes, g.stream));
    }
    std::vector<QueueSlot> qs(slots, QueueSlot(p));
    std::vector<BatchStage> &S = bp.host_stages;
    S.clear();
    int item = 0;
    size_t smem = (size_t)kBatchThreads * 32;   // hub items' lane partials
    for (int s : p.process_order)
        for (int b = 0; b < slots; ++b) {
            void *region = c.hubs.count > 0
                               ? (char *)bp.d_hub + hub_region * ((size_t)b * nproc + qs[b].proc_index[s])
                               : nullptr;
            SG_CKS(add_queue_stage(c, b, s, region, qs[b], S, item, smem));
        }
    bp.root_tiles = qs[0].root_tiles;
    if (poison) {
        // test hook: a stage no item belongs to; the first fused stage waits on it
        BatchStage ds{};
        ds.kind = kStageFused;
        ds.first_item = item;
        ds.nitems = 1;
        for (auto &st : S)
            if (st.kind == kStageFused && st.ndeps < kBatchMaxDeps) { st.deps[st.ndeps++] = (int)S.size(); break; }
        S.push_back(ds);
    }
    bp.slots = slots;
    bp.nstages = (int)S.size();
    bp.total_items = item;
    bp.smem = smem;
    SG_CK(cudaMallocAsync(&bp.d_stages, sizeof(BatchStage) * S.size(), g.stream));
    SG_CK(cudaMemcpyAsync(bp.d_stages, S.data(), sizeof(BatchStage) * S.size(), cudaMemcpyHostToDevice, g.stream));
    SG_CK(cudaMallocAsync(&bp.d_done, sizeof(int) * S.size(), g.stream));
    SG_CK(cudaMallocAsync(&bp.d_ctl, sizeof(BatchCtl), g.stream));
    SG_CK(cudaMallocAsync(&bp.d_raw, sizeof(double) * slots, g.stream));
    SG_CK(cudaStreamSynchronize(g.stream));
    return Status::ok();
}

// The launches of one batch: colors of every slot, the queue reset, the
// persistent kernel and the per-slot root sums.
Status enqueue_batch(RunCtx &c, BatchPlan &bp, long long wait_cycles, cudaStream_t st)
{
    SG_CKS(launch_colors(c, 0, 0, bp.slots, st));
    SG_CK(cudaMemsetAsync(bp.d_done, 0, sizeof(int) * bp.nstages, st));
    SG_CK(cudaMemsetAsync(bp.d_ctl, 0, sizeof(BatchCtl), st));
    SG_CK(launch_persistent(bp.d_stages, bp.nstages, bp.total_items, bp.d_done, bp.d_ctl, wait_cycles, bp.smem,
                            c.fp64, c.g.sm_count, st));
    const double scale = c.mode == kModeReference ? 1.0e12 : 1.0;
    launch_root_reduce_slots(c.gs.ws.partial, (int64_t)(c.g.V / 8 + 2), bp.root_tiles, scale, bp.d_raw, bp.slots, st);
    SG_CK(cudaGetLastError());
    c.launches += 3;
    return Status::ok();
}

// Batched form: `batch` colorings per persistent launch, each batch replayed
// from a CUDA graph.  Slots are admitted by free device memory.
Status count_batched(RunCtx &c, const CountOptions &o, double *raw, CountStats *stats)
{
    DeviceGraph &g = c.g;
    const Plan &p = c.p;
    cudaStream_t st = g.stream;
    const size_t V = (size_t)g.V;
    int slots = std::min(o.batch, o.n_colorings);
    {
        // admission: a slot needs its table arena, colors, root partials and hub rows
        size_t free_b = 0, total_b = 0;
        SG_CK(cudaMemGetInfo(&free_b, &total_b));
        const size_t held = c.gs.ws.arena_bytes;   // reused by the batch
        const size_t per_slot = (size_t)p.arena_units * V * c.es + V + 8 * (V / 8 + 2) +
                                (size_t)c.hubs.total_chunks * (size_t)std::max(c.hub_pitch, 4) * c.es *
                                    p.process_order.size();
        const size_t budget = (size_t)((double)(free_b + held) * 0.9);
        const int fit = per_slot ? (int)std::min<size_t>(budget / per_slot, (size_t)slots) : slots;
        if (fit < 1) return Status{2, "not enough device memory for one coloring's tables"};
        slots = std::min(slots, fit);
    }
    SG_CKS(prepare(c, slots, o.n_colorings));
    // any re-allocation since a queue was built (by any call) may have moved its buffers
    c.gs.ws.generation = g_grow_count;
    // queues built on buffers that have since moved are stale
    for (auto it = c.gs.batches.begin(); it != c.gs.batches.end();) {
        if (it->second.generation != c.gs.ws.generation) {
            free_batch(it->second, st);
            it = c.gs.batches.erase(it);
        } else {
            ++it;
        }
    }
    const long long wait_cycles = (long long)(o.wait_limit_ms > 0 ? o.wait_limit_ms : 2000) * 2000000LL;
    cudaEvent_t e0, e1;
    SG_CK(cudaEventCreate(&e0));
    SG_CK(cudaEventCreate(&e1));
    double total_ms = 0;
    for (int c0 = 0; c0 < o.n_colorings; c0 += slots) {
        const int nb = std::min(slots, o.n_colorings - c0);
        char key[200];
        std::snprintf(key, sizeof key, "%llu/%d/%d/%d/%d/%d", (unsigned long long)p.uid, nb, c.mode, c.hubs.count,
                      (int)c.exact, o.test_unsatisfiable_wait);
        auto it = c.gs.batches.find(key);
        if (it == c.gs.batches.end()) {
            BatchPlan bp;
            bp.generation = c.gs.ws.generation;
            SG_CKS(build_batch(c, nb, o.test_unsatisfiable_wait != 0, bp));
            it = c.gs.batches.emplace(key, std::move(bp)).first;
        }
        BatchPlan &bp = it->second;
        SG_CKS(upload_windows(c, o.seed_base + (uint32_t)c0, nb));
        SG_CK(cudaEventRecord(e0, st));
        if (!bp.exec) {
            // first use: run the launches directly (sets kernel attributes), then capture them
            SG_CKS(enqueue_batch(c, bp, wait_cycles, st));
            SG_CK(cudaStreamSynchronize(st));
            cudaGraph_t graph;
            SG_CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            Status cs = enqueue_batch(c, bp, wait_cycles, st);
            cudaError_t ce = cudaStreamEndCapture(st, &graph);
            if (cs.code) return cs;
            SG_CK(ce);
            SG_CK(cudaGraphInstantiate(&bp.exec, graph, 0));
            cudaGraphDestroy(graph);
            c.launches -= 3;   // the captured launches are counted when replayed
        } else {
            SG_CK(cudaGraphLaunch(bp.exec, st));
            c.launches += 3;
        }
        SG_CK(cudaEventRecord(e1, st));
        SG_CK(cudaMemcpyAsync(c.gs.ws.raw + c0, bp.d_raw, sizeof(double) * nb, cudaMemcpyDeviceToDevice, st));
        BatchCtl ctl{};
        SG_CK(cudaMemcpyAsync(&ctl, bp.d_ctl, sizeof ctl, cudaMemcpyDeviceToHost, st));
        SG_CK(cudaStreamSynchronize(st));
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        total_ms += ms;
        if (ctl.error)
            return Status{4, "batched queue: a work item waited longer than the limit for its inputs (stage " +
                                 std::to_string(ctl.error_stage) + ")"};
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    SG_CK(cudaMemcpyAsync(raw, c.gs.ws.raw, sizeof(double) * o.n_colorings, cudaMemcpyDeviceToHost, st));
    SG_CK(cudaStreamSynchronize(st));
    if (stats) {
        stats->device_ms = total_ms;
        stats->kernel_launches = c.launches;
        stats->table_bytes = (int64_t)(c.arena_per_coloring * slots);
    }
    return Status::ok();
}

}  // namespace

// Interleaved groups: colorings per launch of each stage.  Every candidate
// nb in (lay, lay/2, ..., 1) whose tile fits shared memory is timed over a
// whole stage pass (all its launches, each with tuned tile shapes) once per
// graph, stage shape and group size; the fastest is kept.  Passes recompute
// the same table from the same inputs (an output never overlaps its inputs
// in the arena), so trial passes are harmless.
std::map<std::string, int> g_group_nb;

Status run_stage_group(RunCtx &c, int s, cudaStream_t st)
{
    if (shared_table(c, s)) return Status::ok();
    const int L = c.lay;
    auto pass = [&](int nb) -> Status {
        for (int b0 = 0; b0 < L; b0 += nb) SG_CKS(run_stage(c, 0, s, nullptr, st, b0, std::min(nb, L - b0)));
        return Status::ok();
    };
    if (L == 1) return pass(1);
    StageDesc d1 = make_stage(c, 0, s, nullptr, 0, 1);
    const std::string key = graph_sig(c.g) + shape_key(d1, c.fp64, c.hubs.count) + "/lay" + std::to_string(L) +
                            (c.exact ? "/ex" : "") + (c.blocked ? "/bk" : "");
    int nb = 0;
    {
        std::lock_guard<std::mutex> lk(g_state_mu);
        auto it = g_group_nb.find(key);
        if (it != g_group_nb.end()) nb = it->second;
    }
    if (nb == 0) {
        std::vector<int> cands;
        for (int n = L;; n = (n + 1) / 2) {
            StageDesc dn = make_stage(c, 0, s, nullptr, 0, n);
            FusedConfig cfg;
            if (plan_fused(dn, c.fp64, c.g.sm_count, cfg)) cands.push_back(n);
            if (n == 1) break;
        }
        if (cands.empty()) return Status{6, "sub-template " + std::to_string(s) + " needs more shared memory than a CTA has"};
        nb = cands.front();
        if (c.autotune && cands.size() > 1) {
            cudaEvent_t e0, e1;
            SG_CK(cudaEventCreate(&e0));
            SG_CK(cudaEventCreate(&e1));
            float best = 1e30f;
            for (int n : cands) {
                SG_CKS(pass(n));   // tunes the tile shapes of this nb
                SG_CK(cudaEventRecord(e0, st));
                SG_CKS(pass(n));
                SG_CK(cudaEventRecord(e1, st));
                SG_CK(cudaEventSynchronize(e1));
                float ms = 0;
                cudaEventElapsedTime(&ms, e0, e1);
                if (std::getenv("SG_TUNE_LOG"))
                    std::fprintf(stderr, "[sg tune] sub %d group %d colorings per launch %d: %.3f ms\n", s, L, n, ms);
                if (ms < best) { best = ms; nb = n; }
            }
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
        }
        std::lock_guard<std::mutex> lk(g_state_mu);
        g_group_nb[key] = nb;
    }
    return pass(nb);
}

// Grouped batched form: `batch` colorings interleaved per table row ([V][B]
// colors, [V][B][pitch] tables), every stage launched for several colorings
// at once so one pass over a vertex's neighbour list serves all of them.
// The group size is admitted by free device memory.
Status count_grouped(RunCtx &c, const CountOptions &o, double *raw, CountStats *stats)
{
    DeviceGraph &g = c.g;
    const Plan &p = c.p;
    cudaStream_t st = g.stream;
    int B = std::max(1, std::min(o.batch, o.n_colorings));
    {
        size_t free_b = 0, total_b = 0;
        SG_CK(cudaMemGetInfo(&free_b, &total_b));
        const size_t V = (size_t)g.V;
        const size_t per = (size_t)p.arena_units * V * c.es + V + 8 * (V / 8 + 2);
        const size_t have = c.gs.ws.arena_bytes + c.gs.ws.colors_bytes + c.gs.ws.partial_bytes;
        while (B > 1 && per * (size_t)B > (size_t)((double)(free_b + have) * 0.85)) B = (B + 1) / 2;
    }
    c.lay = B;
    c.use_adjc = adjc_ok(g, p);
    SG_CKS(prepare(c, B, o.n_colorings));
    SG_CKS(upload_windows(c, o.seed_base, o.n_colorings));
    cudaEvent_t e0, e1;
    SG_CK(cudaEventCreate(&e0));
    SG_CK(cudaEventCreate(&e1));
    SG_CK(cudaEventRecord(e0, st));
    const double scale = o.mode == kModeReference ? 1.0e12 : 1.0;
    for (int g0 = 0; g0 < o.n_colorings; g0 += B) {
        c.lay = std::min(B, o.n_colorings - g0);
        SG_CKS(launch_colors(c, 0, g0, c.lay, st));
        for (int s : p.process_order) SG_CKS(run_stage_group(c, s, st));
        launch_root_reduce_slots(c.gs.ws.partial, (int64_t)(g.V / 8 + 2), c.root_tiles, scale, c.gs.ws.raw + g0, c.lay,
                                 st);
        c.launches += 1;
        SG_CK(cudaGetLastError());
    }
    SG_CK(cudaEventRecord(e1, st));
    SG_CK(cudaMemcpyAsync(raw, c.gs.ws.raw, sizeof(double) * o.n_colorings, cudaMemcpyDeviceToHost, st));
    SG_CK(cudaStreamSynchronize(st));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (stats) {
        stats->device_ms = ms;
        stats->kernel_launches = c.launches;
        stats->table_bytes = (int64_t)(c.arena_per_coloring * B);
        stats->fused_launches = (int64_t)c.fused_ev.size();
        top_stage(c, stats);
        stats->fused_ms = ev_sum(c.fused_ev);
        stats->hub_ms = ev_sum(c.hub_ev);
        stats->fused_alg_bytes = c.fused_alg_bytes;
        stats->fused_gather_bytes = c.fused_gather_bytes;
    }
    ev_sum(c.fused_ev);
    ev_sum(c.hub_ev);
    return Status::ok();
}

Status count(DeviceGraph &g, const Plan &p, const CountOptions &o, double *raw, CountStats *stats)
{
    if (o.n_colorings < 1) return Status{1, "n_colorings must be >= 1"};
    if (o.mode < 0 || o.mode > 3) return Status{1, "unknown count mode"};
    if (p.k > 255) return Status{1, "too many colors"};
    if (g.V >= (1 << 28)) return Status{1, "counting supports graphs of fewer than 2^28 vertices"};
    SG_CK(cudaSetDevice(g.device));
    GraphState &gs = state_of(g);
    RunCtx c{g, p, gs, nullptr, o.mode == kModeFP64, (size_t)(o.mode == kModeFP64 ? 8 : 4), 0, {}, 0, 0, o.mode, 0};
    SG_CKS(make_ctx_tables(g, p, gs, c.tab));
    c.exact = o.exact != 0;
    // hubs in exact order (the per-tile sums) on the plain and grouped forms;
    // the persistent queue chunks them (another summation order), or in exact
    // mode aggregates every vertex in its tile
    const bool queue = o.batch > 0 && o.persistent && o.mode != kModeOriginal;
    c.hubs = queue ? plan_hubs(g, c.exact ? 0 : o.hub_threshold, false) : plan_hubs(g, o.hub_threshold, true);
    c.profile = o.profile != 0;
    c.autotune = o.autotune != 0;
    c.blocked = o.blocked != 0;
    c.rooted = o.rooted != 0;
    c.flat = o.flat != 0;
    // mode 2 carries its aggregation buffer from one coloring to the next, so
    // its colorings always run one after another (the plain form)
    if (o.batch > 0 && o.mode != kModeOriginal)
        return o.persistent ? count_batched(c, o, raw, stats) : count_grouped(c, o, raw, stats);
    const int slots = 1;
    c.use_adjc = adjc_ok(g, p);
    SG_CKS(prepare(c, slots, o.n_colorings));
    SG_CKS(upload_windows(c, o.seed_base, o.n_colorings));
    cudaStream_t st = g.stream;
    if (o.mode == kModeOriginal) {
        if (o.orig_state)
            SG_CK(cudaMemcpyAsync(gs.ws.orig_buf, o.orig_state, 4 * (size_t)g.V, cudaMemcpyHostToDevice, st));
        else
            SG_CK(cudaMemsetAsync(gs.ws.orig_buf, 0, 4 * (size_t)g.V, st));
    }
    cudaEvent_t e0, e1;
    SG_CK(cudaEventCreate(&e0));
    SG_CK(cudaEventCreate(&e1));
    SG_CK(cudaEventRecord(e0, st));
    const double scale = o.mode == kModeReference ? 1.0e12 : 1.0;
    for (int col = 0; col < o.n_colorings; ++col) {
        SG_CKS(launch_colors(c, 0, col, 1, st));
        for (int s : p.process_order) SG_CKS(run_stage(c, 0, s, nullptr, st));
        launch_root_reduce(gs.ws.partial, c.root_tiles, scale, gs.ws.raw + col, st);
        c.launches += 1;
        SG_CK(cudaGetLastError());
    }
    SG_CK(cudaEventRecord(e1, st));
    SG_CK(cudaMemcpyAsync(raw, gs.ws.raw, sizeof(double) * o.n_colorings, cudaMemcpyDeviceToHost, st));
    if (o.mode == kModeOriginal && o.orig_state)
        SG_CK(cudaMemcpyAsync(o.orig_state, gs.ws.orig_buf, 4 * (size_t)g.V, cudaMemcpyDeviceToHost, st));
    SG_CK(cudaStreamSynchronize(st));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (stats) {
        stats->device_ms = ms;
        stats->kernel_launches = c.launches;
        stats->table_bytes = (int64_t)(c.arena_per_coloring * slots);
        stats->fused_launches = (int64_t)c.fused_ev.size();
        top_stage(c, stats);
        stats->fused_ms = ev_sum(c.fused_ev);
        stats->hub_ms = ev_sum(c.hub_ev);
        stats->fused_alg_bytes = c.fused_alg_bytes;
        stats->fused_gather_bytes = c.fused_gather_bytes;
    }
    ev_sum(c.fused_ev);
    ev_sum(c.hub_ev);
    return Status::ok();
}

Status debug_colors(DeviceGraph &g, int k, uint32_t seed, int32_t *colors)
{
    if (k < 1 || k > 255) return Status{1, "k out of range"};
    SG_CK(cudaSetDevice(g.device));
    GraphState &gs = state_of(g);
    Plan dummy;
    dummy.k = k;
    RunCtx c{g, dummy, gs, nullptr, false, 4, 0, {}, 0, 0, 0, 0};
    SG_CKS(growT(&gs.ws.colors, &gs.ws.colors_bytes, std::max<size_t>(16, (size_t)g.V), g.stream));
    SG_CKS(growT(&gs.ws.windows, &gs.ws.windows_bytes, 4 * 31, g.stream));
    SG_CKS(upload_windows(c, seed, 1));
    SG_CKS(launch_colors(c, 0, 0, 1, g.stream));
    std::vector<uint8_t> ci(g.V);
    std::vector<int32_t> perm(g.V);
    if (g.V) {
        SG_CK(cudaMemcpyAsync(ci.data(), gs.ws.colors, g.V, cudaMemcpyDeviceToHost, g.stream));
        SG_CK(cudaMemcpyAsync(perm.data(), g.d_perm, 4 * (size_t)g.V, cudaMemcpyDeviceToHost, g.stream));
    }
    SG_CK(cudaStreamSynchronize(g.stream));
    for (int32_t v = 0; v < g.V; ++v) colors[v] = ci[perm[v]];
    return Status::ok();
}

static Status run_partial(DeviceGraph &g, const Plan &p, uint32_t seed, int mode, int hub_threshold, int upto,
                          RunCtx &c, GraphState &gs)
{
    if (g.V >= (1 << 28)) return Status{1, "counting supports graphs of fewer than 2^28 vertices"};
    SG_CKS(make_ctx_tables(g, p, gs, c.tab));
    // the parity helpers run the reference's operation order; vertices above
    // hub_threshold go through the exact-order hub kernel
    c.exact = true;
    c.hubs = plan_hubs(g, hub_threshold, true);
    c.use_adjc = adjc_ok(g, p);
    SG_CKS(prepare(c, 1, 1));
    SG_CKS(upload_windows(c, seed, 1));
    SG_CKS(launch_colors(c, 0, 0, 1, g.stream));
    if (mode == kModeOriginal) SG_CK(cudaMemsetAsync(gs.ws.orig_buf, 0, 4 * (size_t)g.V, g.stream));
    for (int s : p.process_order) {
        if (s < upto) break;
        SG_CKS(run_stage(c, 0, s, upto == 0 ? gs.ws.root_vertex : nullptr, g.stream));
    }
    SG_CK(cudaStreamSynchronize(g.stream));
    return Status::ok();
}

Status debug_sub_table(DeviceGraph &g, const Plan &p, uint32_t seed, int mode, int hub_threshold, int s, void *out)
{
    if (s <= 0 || s >= p.nsub()) return Status{1, "sub index must be in [1, nsub)"};
    SG_CK(cudaSetDevice(g.device));
    GraphState &gs = state_of(g);
    RunCtx c{g, p, gs, nullptr, mode == kModeFP64, (size_t)(mode == kModeFP64 ? 8 : 4), 0, {}, 0, 0, mode, 0};
    const SubTemplate &sub = p.subs[s];
    std::vector<int32_t> perm(g.V);
    if (g.V) SG_CK(cudaMemcpy(perm.data(), g.d_perm, 4 * (size_t)g.V, cudaMemcpyDeviceToHost));
    const size_t V = (size_t)g.V;
    if (sub.size == 1) {
        std::vector<int32_t> col(V);
        SG_CKS(debug_colors(g, p.k, seed, col.data()));
        for (int cc = 0; cc < sub.L; ++cc)
            for (size_t v = 0; v < V; ++v) {
                double val = col[v] == cc ? 1.0 : 0.0;
                if (c.fp64) ((double *)out)[cc * V + v] = val;
                else ((float *)out)[cc * V + v] = (float)val;
            }
        return Status::ok();
    }
    SG_CKS(run_partial(g, p, seed, mode, hub_threshold, s, c, gs));
    const int P = p.table_pitch[s];
    std::vector<char> rows(V * P * c.es);
    if (V) SG_CK(cudaMemcpy(rows.data(), table_ptr(c, 0, s), rows.size(), cudaMemcpyDeviceToHost));
    for (size_t v = 0; v < V; ++v)
        for (int cc = 0; cc < sub.L; ++cc) {
            size_t src = ((size_t)perm[v] * P + cc) * c.es, dst = ((size_t)cc * V + v) * c.es;
            std::memcpy((char *)out + dst, rows.data() + src, c.es);
        }
    return Status::ok();
}

Status debug_root(DeviceGraph &g, const Plan &p, uint32_t seed, int mode, int hub_threshold, double *root, double *raw)
{
    SG_CK(cudaSetDevice(g.device));
    GraphState &gs = state_of(g);
    RunCtx c{g, p, gs, nullptr, mode == kModeFP64, (size_t)(mode == kModeFP64 ? 8 : 4), 0, {}, 0, 0, mode, 0};
    SG_CKS(growT(&gs.ws.root_vertex, &gs.ws.root_vertex_bytes, 8 * std::max<size_t>(1, (size_t)g.V), g.stream));
    SG_CKS(run_partial(g, p, seed, mode, hub_threshold, 0, c, gs));
    std::vector<double> rv(g.V);
    std::vector<int32_t> perm(g.V);
    if (g.V) {
        SG_CK(cudaMemcpy(rv.data(), gs.ws.root_vertex, 8 * (size_t)g.V, cudaMemcpyDeviceToHost));
        SG_CK(cudaMemcpy(perm.data(), g.d_perm, 4 * (size_t)g.V, cudaMemcpyDeviceToHost));
    }
    for (int32_t v = 0; v < g.V; ++v) root[v] = rv[perm[v]];
    if (raw) {
        double s = 0;
        for (int32_t v = 0; v < g.V; ++v) s += root[v];
        *raw = mode == kModeReference ? s * 1.0e12 : s;
    }
    return Status::ok();
}

}  // namespace sg

namespace sg {

// ---------------------------------------------------------------------------
// Job queues: one coloring each of jobs with different templates on one
// graph, run as persistent work-queue launches.  Jobs are admitted in waves
// by free device memory (each job's table arena, colors, root partials and
// hub rows); a wave's stages go into one queue level by level (every job's
// first sub, then every job's second, ...), each stage depending only on
// earlier stages of its own job.  The CTA that completes a job's root stage
// stamps %globaltimer, which gives each job's latency from the launch start.
// ---------------------------------------------------------------------------
Status count_jobs_streams(DeviceGraph &g, const std::vector<const Plan *> &plans, const uint32_t *seeds,
                          const CountOptions &o, double *raw, double *job_ms, CountStats *stats);

Status count_jobs(DeviceGraph &g, const std::vector<const Plan *> &plans, const uint32_t *seeds,
                  const CountOptions &o, double *raw, double *job_ms, CountStats *stats)
{
    if (o.mode == kModeOriginal)
        return Status{6, "mode 2 (isPruned=0 on a CSC graph) carries its aggregation buffer from one coloring to the "
                         "next: count such jobs with sg_count one after another"};
    if (o.mode < 0 || o.mode > 3) return Status{1, "unknown count mode"};
    if (!o.persistent) return count_jobs_streams(g, plans, seeds, o, raw, job_ms, stats);
    const int n = (int)plans.size();
    if (n < 1) return Status{1, "no jobs"};
    if (!seeds || !raw) return Status{1, "null argument"};
    if (o.mode < 0 || o.mode > 3) return Status{1, "unknown count mode"};
    for (const Plan *p : plans)
        if (!p) return Status{1, "null template plan"};
    if (g.V >= (1 << 28)) return Status{1, "counting supports graphs of fewer than 2^28 vertices"};
    SG_CK(cudaSetDevice(g.device));
    GraphState &gs = state_of(g);
    Workspace &w = gs.ws;
    const bool fp64 = o.mode == kModeFP64;
    const size_t es = fp64 ? 8 : 4;
    const size_t V = (size_t)g.V;
    cudaStream_t st = g.stream;
    const Hubs hubs = plan_hubs(g, o.exact ? 0 : o.hub_threshold, false);

    // one context per job: its plan's device tables, its tables at arena_base
    std::vector<RunCtx> ctx;
    ctx.reserve(n);
    int32_t hub_pitch = 8;
    for (int j = 0; j < n; ++j) {
        const Plan &p = *plans[j];
        ctx.push_back(RunCtx{g, p, gs, nullptr, fp64, es, 0, hubs, 0, 0, o.mode, 0});
        RunCtx &c = ctx.back();
        SG_CKS(make_ctx_tables(g, p, gs, c.tab));
        c.exact = o.exact != 0;
        c.autotune = o.autotune != 0;
        hub_pitch = std::max<int32_t>(hub_pitch, (int32_t)round_up(p.k, 8));
        for (int s : p.process_order) {
            const SubTemplate &a = p.subs[p.subs[s].aux];
            if (a.size > 1) hub_pitch = std::max<int32_t>(hub_pitch, p.table_pitch[p.subs[s].aux]);
        }
    }
    for (RunCtx &c : ctx) c.hub_pitch = hub_pitch;
    if (hubs.count > 0) {
        std::vector<int32_t> cs((size_t)hubs.count + 1, 0);
        for (int h = 0; h < hubs.count; ++h) cs[h + 1] = cs[h] + (g.h_degree[h] + hubs.chunk - 1) / hubs.chunk;
        SG_CKS(growT(&w.chunk_start, &w.chunk_start_bytes, 4 * cs.size(), st));
        SG_CK(cudaMemcpyAsync(w.chunk_start, cs.data(), 4 * cs.size(), cudaMemcpyHostToDevice, st));
        SG_CK(cudaStreamSynchronize(st));
    }
    const size_t hub_region = (size_t)hubs.total_chunks * (size_t)hub_pitch * es;
    const long long wait_cycles = (long long)(o.wait_limit_ms > 0 ? o.wait_limit_ms : 2000) * 2000000LL;
    const double scale = o.mode == kModeReference ? 1.0e12 : 1.0;
    cudaEvent_t e0, e1;
    SG_CK(cudaEventCreate(&e0));
    SG_CK(cudaEventCreate(&e1));
    double total_ms = 0;
    int64_t launches = 0;
    for (int j0 = 0; j0 < n;) {
        // admission: jobs while their tables fit the free memory (at least one)
        size_t free_b = 0, total_b = 0;
        SG_CK(cudaMemGetInfo(&free_b, &total_b));
        const size_t budget = (size_t)((double)(free_b + w.arena_bytes) * 0.85);
        size_t arena_sum = 0, hub_sum = 0;
        int j1 = j0;
        while (j1 < n && j1 - j0 < 4096) {
            const size_t a = (size_t)plans[j1]->arena_units * V * es;
            const size_t h = hubs.count > 0 ? hub_region * plans[j1]->process_order.size() : 0;
            const size_t per = a + h + V + 8 * (V / 8 + 2);
            if (j1 > j0 && arena_sum + hub_sum + per > budget) break;
            arena_sum += a;
            hub_sum += h;
            ++j1;
        }
        const int nj = j1 - j0;
        SG_CKS(grow(&w.arena, &w.arena_bytes, std::max<size_t>(16, arena_sum), st));
        SG_CKS(growT(&w.colors, &w.colors_bytes, std::max<size_t>(16, V * nj), st));
        SG_CKS(growT(&w.partial, &w.partial_bytes, 8 * ((V / 8 + 2) * nj), st));
        SG_CKS(growT(&w.windows, &w.windows_bytes, 4 * 31 * (size_t)nj, st));
        {
            std::vector<uint32_t> win((size_t)nj * 31);
            for (int j = 0; j < nj; ++j) glibc_window(seeds[j0 + j], &win[(size_t)j * 31]);
            SG_CK(cudaMemcpyAsync(w.windows, win.data(), win.size() * 4, cudaMemcpyHostToDevice, st));
            SG_CK(cudaStreamSynchronize(st));
        }
        // the wave's queue
        void *d_hub = nullptr;
        if (hubs.count > 0) SG_CK(cudaMallocAsync(&d_hub, std::max<size_t>(16, hub_sum), st));
        std::vector<QueueSlot> qs;
        qs.reserve(nj);
        std::vector<size_t> hub_off(nj, 0);
        size_t base = 0, hoff = 0;
        int maxlev = 0;
        for (int j = 0; j < nj; ++j) {
            RunCtx &c = ctx[j0 + j];
            c.arena_base = base;
            c.arena_per_coloring = 0;
            base += (size_t)c.p.arena_units * V * es;
            hub_off[j] = hoff;
            hoff += hubs.count > 0 ? hub_region * c.p.process_order.size() : 0;
            qs.emplace_back(c.p);
            maxlev = std::max(maxlev, (int)c.p.process_order.size());
        }
        std::vector<BatchStage> S;
        int item = 0;
        size_t smem = (size_t)kBatchThreads * 32;
        for (int lev = 0; lev < maxlev; ++lev)
            for (int j = 0; j < nj; ++j) {
                RunCtx &c = ctx[j0 + j];
                if (lev >= (int)c.p.process_order.size()) continue;
                const int s = c.p.process_order[lev];
                void *region = hubs.count > 0 ? (char *)d_hub + hub_off[j] + hub_region * (size_t)qs[j].proc_index[s]
                                              : nullptr;
                SG_CKS(add_queue_stage(c, j, s, region, qs[j], S, item, smem));
            }
        std::vector<int32_t> tiles(nj);
        for (int j = 0; j < nj; ++j) tiles[j] = qs[j].root_tiles;
        BatchStage *d_stages = nullptr;
        int *d_done = nullptr;
        BatchCtl *d_ctl = nullptr;
        unsigned long long *d_end = nullptr;
        double *d_raw = nullptr;
        int32_t *d_tiles = nullptr;
        SG_CK(cudaMallocAsync(&d_stages, sizeof(BatchStage) * S.size(), st));
        SG_CK(cudaMallocAsync(&d_done, sizeof(int) * S.size(), st));
        SG_CK(cudaMallocAsync(&d_ctl, sizeof(BatchCtl), st));
        SG_CK(cudaMallocAsync(&d_end, sizeof(unsigned long long) * S.size(), st));
        SG_CK(cudaMallocAsync(&d_raw, sizeof(double) * nj, st));
        SG_CK(cudaMallocAsync(&d_tiles, sizeof(int32_t) * nj, st));
        SG_CK(cudaMemcpyAsync(d_stages, S.data(), sizeof(BatchStage) * S.size(), cudaMemcpyHostToDevice, st));
        SG_CK(cudaMemcpyAsync(d_tiles, tiles.data(), sizeof(int32_t) * nj, cudaMemcpyHostToDevice, st));
        SG_CK(cudaMemsetAsync(d_done, 0, sizeof(int) * S.size(), st));
        SG_CK(cudaMemsetAsync(d_ctl, 0, sizeof(BatchCtl), st));
        SG_CK(cudaMemsetAsync(d_end, 0, sizeof(unsigned long long) * S.size(), st));
        SG_CK(cudaStreamSynchronize(st));   // `S` and `tiles` are pageable host memory
        SG_CK(cudaEventRecord(e0, st));
        for (int j = 0; j < nj; ++j) SG_CKS(launch_colors(ctx[j0 + j], j, j, 1, st));
        SG_CK(launch_persistent(d_stages, (int)S.size(), item, d_done, d_ctl, wait_cycles, smem, fp64, g.sm_count, st,
                                d_end));
        launch_root_reduce_slots(w.partial, (int64_t)(V / 8 + 2), 0, scale, d_raw, nj, st, d_tiles);
        SG_CK(cudaGetLastError());
        SG_CK(cudaEventRecord(e1, st));
        launches += nj + 2;
        BatchCtl ctl{};
        std::vector<unsigned long long> ends(S.size());
        SG_CK(cudaMemcpyAsync(raw + j0, d_raw, sizeof(double) * nj, cudaMemcpyDeviceToHost, st));
        SG_CK(cudaMemcpyAsync(&ctl, d_ctl, sizeof ctl, cudaMemcpyDeviceToHost, st));
        SG_CK(cudaMemcpyAsync(ends.data(), d_end, sizeof(unsigned long long) * S.size(), cudaMemcpyDeviceToHost, st));
        SG_CK(cudaStreamSynchronize(st));
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        total_ms += ms;
        for (void *q : {(void *)d_stages, (void *)d_done, (void *)d_ctl, (void *)d_end, (void *)d_raw, (void *)d_tiles,
                        d_hub})
            if (q) cudaFreeAsync(q, st);
        if (ctl.error) {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            return Status{4, "job queue: a work item waited longer than the limit for its inputs (stage " +
                                 std::to_string(ctl.error_stage) + ")"};
        }
        if (job_ms)
            for (int j = 0; j < nj; ++j) {
                const unsigned long long e = ends[qs[j].fused[0]];
                job_ms[j0 + j] = e > ctl.t0 ? (double)(e - ctl.t0) * 1e-6 : 0.0;
            }
        j0 = j1;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (stats) {
        stats->device_ms = total_ms;
        stats->kernel_launches = launches;
        stats->table_bytes = (int64_t)w.arena_bytes;
    }
    return Status::ok();
}

// ---------------------------------------------------------------------------
// Job streams, stream form: every job runs the plain form's tuned stage
// launches (register-blocked eMA, colour-tagged neighbours, chunk masks) on
// one of S CUDA streams; stream s owns table slot s (the largest job's arena),
// its colors, colour-tagged adjacency, root partials and hub rows, and takes
// jobs s, s+S, ... in order, so slots are reused only by later jobs of the
// same stream.  The launches of different streams overlap on the GPU, which
// fills it when one job's launches are short.  Each job's latency is the
// time from the common start event to the end of its root sum.
// ---------------------------------------------------------------------------
Status count_jobs_streams(DeviceGraph &g, const std::vector<const Plan *> &plans, const uint32_t *seeds,
                          const CountOptions &o, double *raw, double *job_ms, CountStats *stats)
{
    const int n = (int)plans.size();
    if (n < 1) return Status{1, "no jobs"};
    if (!seeds || !raw) return Status{1, "null argument"};
    if (o.mode < 0 || o.mode > 3) return Status{1, "unknown count mode"};
    for (const Plan *p : plans)
        if (!p) return Status{1, "null template plan"};
    if (g.V >= (1 << 28)) return Status{1, "counting supports graphs of fewer than 2^28 vertices"};
    SG_CK(cudaSetDevice(g.device));
    GraphState &gs = state_of(g);
    Workspace &w = gs.ws;
    const bool fp64 = o.mode == kModeFP64;
    const size_t es = fp64 ? 8 : 4;
    const size_t V = (size_t)g.V;
    cudaStream_t st = g.stream;
    const Hubs hubs = plan_hubs(g, o.hub_threshold, true);
    std::vector<RunCtx> ctx;
    ctx.reserve(n);
    size_t max_arena = 16;
    int32_t hub_pitch = 8;
    for (int j = 0; j < n; ++j) {
        const Plan &p = *plans[j];
        ctx.push_back(RunCtx{g, p, gs, nullptr, fp64, es, 0, hubs, 0, 0, o.mode, 0});
        RunCtx &c = ctx.back();
        SG_CKS(make_ctx_tables(g, p, gs, c.tab));
        c.exact = o.exact != 0;
        c.autotune = o.autotune != 0;
        c.blocked = o.blocked != 0;
        c.rooted = o.rooted != 0;
        c.flat = o.flat != 0;
        c.use_adjc = adjc_ok(g, p);
        max_arena = std::max(max_arena, (size_t)p.arena_units * V * es);
        hub_pitch = std::max<int32_t>(hub_pitch, (int32_t)round_up(p.k, 8));
        for (int s : p.process_order)
            if (p.subs[p.subs[s].aux].size > 1) hub_pitch = std::max<int32_t>(hub_pitch, p.table_pitch[p.subs[s].aux]);
    }
    const bool adjc = ctx[0].use_adjc;
    const size_t hub_region = (size_t)hubs.total_chunks * (size_t)hub_pitch * es;
    // streams admitted by free memory: a slot holds one job's tables, colors,
    // colour-tagged adjacency, root partials and hub rows
    int S = std::max(1, std::min(o.batch > 0 ? o.batch : 8, n));
    {
        size_t free_b = 0, total_b = 0;
        SG_CK(cudaMemGetInfo(&free_b, &total_b));
        const size_t per = max_arena + V + 8 * (V / 8 + 2) + hub_region + (adjc ? 4 * (size_t)g.nnz : 0);
        const size_t have = w.arena_bytes + w.hub_partial_bytes + w.adjc_bytes;
        while (S > 1 && per * (size_t)S > (size_t)((double)(free_b + have) * 0.85)) --S;
    }
    SG_CKS(grow(&w.arena, &w.arena_bytes, max_arena * S, st));
    SG_CKS(growT(&w.colors, &w.colors_bytes, std::max<size_t>(16, V * S), st));
    SG_CKS(growT(&w.partial, &w.partial_bytes, 8 * (V / 8 + 2) * S, st));
    SG_CKS(growT(&w.raw, &w.raw_bytes, 8 * (size_t)n, st));
    SG_CKS(growT(&w.windows, &w.windows_bytes, 4 * 31 * (size_t)n, st));
    if (adjc) SG_CKS(growT(&w.adjc, &w.adjc_bytes, std::max<size_t>(16, 4 * (size_t)g.nnz * S), st));
    if (hubs.count > 0) {
        SG_CKS(grow(&w.hub_partial, &w.hub_partial_bytes, std::max<size_t>(16, hub_region * S), st));
        std::vector<int32_t> cs((size_t)hubs.count + 1, 0);
        for (int h = 0; h < hubs.count; ++h) cs[h + 1] = cs[h] + (g.h_degree[h] + hubs.chunk - 1) / hubs.chunk;
        SG_CKS(growT(&w.chunk_start, &w.chunk_start_bytes, 4 * cs.size(), st));
        SG_CK(cudaMemcpyAsync(w.chunk_start, cs.data(), 4 * cs.size(), cudaMemcpyHostToDevice, st));
        SG_CKS(growT(&w.hub_ticket, &w.hub_ticket_bytes, 4 * (size_t)std::max(64, S), st));
        SG_CK(cudaStreamSynchronize(st));   // `cs` is pageable and goes out of scope
    }
    SG_CKS(growT(&w.tile_ticket, &w.tile_ticket_bytes, 4 * (size_t)std::max(64, S), st));
    {
        std::vector<uint32_t> win((size_t)n * 31);
        for (int j = 0; j < n; ++j) glibc_window(seeds[j], &win[(size_t)j * 31]);
        SG_CK(cudaMemcpyAsync(w.windows, win.data(), win.size() * 4, cudaMemcpyHostToDevice, st));
        SG_CK(cudaStreamSynchronize(st));
    }
    while ((int)gs.streams.size() < S) {
        cudaStream_t js;
        SG_CK(cudaStreamCreateWithFlags(&js, cudaStreamNonBlocking));
        gs.streams.push_back(js);
    }
    for (RunCtx &c : ctx) {
        c.arena_per_coloring = max_arena;
        c.hub_pitch = hub_pitch;
    }
    std::vector<cudaEvent_t> ev_end(n, nullptr);
    cudaEvent_t ev0;
    SG_CK(cudaEventCreate(&ev0));
    for (int j = 0; j < n; ++j) SG_CK(cudaEventCreate(&ev_end[j]));
    SG_CK(cudaEventRecord(ev0, st));
    for (int s = 0; s < S; ++s) SG_CK(cudaStreamWaitEvent(gs.streams[s], ev0, 0));
    const double scale = o.mode == kModeReference ? 1.0e12 : 1.0;
    int64_t launches = 0;
    Status status = Status::ok();
    for (int j = 0; j < n && !status.code; ++j) {
        const int s = j % S;
        cudaStream_t js = gs.streams[s];
        RunCtx &c = ctx[j];
        c.hub_region = hubs.count > 0 ? (char *)w.hub_partial + hub_region * s : nullptr;
        c.ticket = s;
        status = launch_colors(c, s, j, 1, js);
        for (int sub : c.p.process_order)
            if (!status.code) status = run_stage(c, s, sub, nullptr, js);
        if (status.code) break;
        launch_root_reduce(w.partial + (size_t)s * (V / 8 + 2), c.root_tiles, scale, w.raw + j, js);
        cudaEventRecord(ev_end[j], js);
        launches += c.launches + 1;
    }
    // join: the default stream waits for every job stream
    for (int s = 0; s < S; ++s) {
        cudaEvent_t e;
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) == cudaSuccess) {
            cudaEventRecord(e, gs.streams[s]);
            cudaStreamWaitEvent(st, e, 0);
            cudaEventDestroy(e);
        }
    }
    if (!status.code) SG_CK(cudaMemcpyAsync(raw, w.raw, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    SG_CK(cudaStreamSynchronize(st));
    double total = 0;
    for (int j = 0; j < n; ++j) {
        float ms = 0;
        if (!status.code && cudaEventElapsedTime(&ms, ev0, ev_end[j]) == cudaSuccess) {
            if (job_ms) job_ms[j] = ms;
            total = std::max(total, (double)ms);
        }
        cudaEventDestroy(ev_end[j]);
    }
    cudaEventDestroy(ev0);
    if (status.code) return status;
    if (stats) {
        stats->device_ms = total;
        stats->kernel_launches = launches;
        stats->table_bytes = (int64_t)(max_arena * S);
    }
    return Status::ok();
}

}  // namespace sg
