// C ABI (include/sg_api.h) over the host planner and the device engine.
#include "../../include/sg_api.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <memory>
#include <string>
#include <vector>

#include "engine/engine.hpp"
#include "host/graph_io.hpp"
#include "host/plan.hpp"

struct sg_graph_s {
    std::unique_ptr<sg::DeviceGraph> g;
};
struct sg_plan_s {
    sg::Template t;
    sg::Plan p;
};
struct sg_countmat_s {
    sg_graph graph = nullptr;
    int32_t thd_num = 1, itr_num = 1, isPruned = 1, useSPMM = 1, vtuneStart = -1, calc_aut = 0;
    uint32_t seed = 0;
    bool seeded = false;
    bool initialized = false;
    bool csr = false;                 // the graph was given as the CSRGraph
    std::vector<double> raw;
    std::vector<float> orig_state;    // isPruned=0 on a CSC graph: CountMat::_bufVec, zeroed at
                                      // initialization and carried from one compute() to the next
};

namespace {

thread_local std::string t_err;

sg_status fail(sg_status code, const std::string &msg)
{
    t_err = msg;
    return code;
}
sg_status from(const sg::Status &s) { return s.code ? fail(s.code, s.msg) : SG_OK; }

template <typename T> T *dup_array(const std::vector<T> &v)
{
    T *p = (T *)std::malloc(sizeof(T) * (v.empty() ? 1 : v.size()));
    if (p && !v.empty()) std::memcpy(p, v.data(), sizeof(T) * v.size());
    return p;
}

#define SG_GUARD_BEGIN try {
#define SG_GUARD_END                                                              \
    }                                                                             \
    catch (const std::bad_alloc &) { return fail(SG_ERR_OOM, "host allocation failed"); } \
    catch (const std::exception &e) { return fail(SG_ERR_INVALID, e.what()); }

}  // namespace

namespace sg {
void set_last_error(const std::string &msg) { t_err = msg; }
}

extern "C" {

const char *sg_last_error(void) { return t_err.c_str(); }
const char *sg_version(void) { return "subgraph_b200 0.1 (sm_100a)"; }
void sg_free(void *p) { std::free(p); }

sg_status sg_edgelist_read(const char *path, int32_t *V, int64_t *E, int32_t **src, int32_t **dst)
{
    SG_GUARD_BEGIN
    if (!path || !V || !E || !src || !dst) return fail(SG_ERR_INVALID, "null argument");
    sg::EdgeListData el;
    std::string err;
    if (!sg::read_edge_list(path, el, err)) return fail(err.rfind("cannot", 0) == 0 ? SG_ERR_IO : SG_ERR_INVALID, err);
    *V = el.V;
    *E = (int64_t)el.src.size();
    *src = dup_array(el.src);
    *dst = dup_array(el.dst);
    return SG_OK;
    SG_GUARD_END
}

sg_status sg_edgelist_write(const char *path, int32_t V, int64_t E, const int32_t *src, const int32_t *dst)
{
    SG_GUARD_BEGIN
    if (!path || E < 0 || (E > 0 && (!src || !dst))) return fail(SG_ERR_INVALID, "null argument");
    sg::EdgeListData el;
    el.V = V;
    el.src.assign(src, src + E);
    el.dst.assign(dst, dst + E);
    std::string err;
    if (!sg::write_edge_list(path, el, err)) return fail(SG_ERR_IO, err);
    return SG_OK;
    SG_GUARD_END
}

sg_status sg_csc_build(int32_t V, int64_t E, const int32_t *src, const int32_t *dst, int32_t **indexCol,
                       int32_t **indexRow, int32_t **degList)
{
    SG_GUARD_BEGIN
    if (E < 0 || (E > 0 && (!src || !dst)) || !indexCol || !indexRow || !degList) return fail(SG_ERR_INVALID, "null argument");
    sg::CSC g;
    std::string err;
    if (!sg::build_csc(V, src, dst, E, g, err)) return fail(SG_ERR_INVALID, err);
    *indexCol = dup_array(g.indexCol);
    *indexRow = dup_array(g.indexRow);
    *degList = dup_array(g.degList);
    return SG_OK;
    SG_GUARD_END
}

sg_status sg_csr_build(int32_t V, int64_t E, const int32_t *src, const int32_t *dst, int32_t **indexRow,
                       int32_t **indexCol, int32_t **degList)
{
    SG_GUARD_BEGIN
    if (E < 0 || (E > 0 && (!src || !dst)) || !indexCol || !indexRow || !degList) return fail(SG_ERR_INVALID, "null argument");
    sg::CSR g;
    std::string err;
    if (!sg::build_csr(V, src, dst, E, g, err)) return fail(SG_ERR_INVALID, err);
    *indexRow = dup_array(g.indexRow);
    *indexCol = dup_array(g.indexCol);
    *degList = dup_array(g.degList);
    return SG_OK;
    SG_GUARD_END
}

sg_status sg_graph_data_write(const char *path, int32_t V, int32_t numEdges, const int32_t *indexCol,
                              const int32_t *indexRow, const int32_t *degList)
{
    SG_GUARD_BEGIN
    if (!path || V < 0 || !indexCol || !degList) return fail(SG_ERR_INVALID, "null argument");
    sg::CSC g;
    g.V = V;
    g.numEdges = numEdges;
    g.indexCol.assign(indexCol, indexCol + V + 1);
    int32_t nnz = indexCol[V];
    if (nnz < 0 || (nnz > 0 && !indexRow)) return fail(SG_ERR_INVALID, "bad indexCol");
    g.indexRow.assign(indexRow, indexRow + nnz);
    g.degList.assign(degList, degList + V);
    std::string err;
    if (!sg::write_graph_data(path, g, err)) return fail(SG_ERR_IO, err);
    return SG_OK;
    SG_GUARD_END
}

sg_status sg_graph_data_read(const char *path, int32_t *V, int32_t *numEdges, int32_t **indexCol,
                             int32_t **indexRow, int32_t **degList)
{
    SG_GUARD_BEGIN
    if (!path || !V || !numEdges || !indexCol || !indexRow || !degList) return fail(SG_ERR_INVALID, "null argument");
    sg::CSC g;
    std::string err;
    if (!sg::read_graph_data(path, g, err)) return fail(err.rfind("cannot", 0) == 0 ? SG_ERR_IO : SG_ERR_INVALID, err);
    *V = g.V;
    *numEdges = g.numEdges;
    *indexCol = dup_array(g.indexCol);
    *indexRow = dup_array(g.indexRow);
    *degList = dup_array(g.degList);
    return SG_OK;
    SG_GUARD_END
}

sg_status sg_graph_data_encode(int32_t V, int32_t numEdges, const int32_t *offsets, const int32_t *neighbors,
                               const int32_t *degList, void **buf, int64_t *bytes)
{
    SG_GUARD_BEGIN
    if (V < 0 || !offsets || !degList || !buf || !bytes) return fail(SG_ERR_INVALID, "null argument");
    sg::CSC g;
    g.V = V;
    g.numEdges = numEdges;
    g.indexCol.assign(offsets, offsets + V + 1);
    int32_t nnz = offsets[V];
    if (nnz < 0 || (nnz > 0 && !neighbors)) return fail(SG_ERR_INVALID, "bad offsets");
    g.indexRow.assign(neighbors, neighbors + nnz);
    g.degList.assign(degList, degList + V);
    std::string b;
    sg::encode_graph_data(g, b);
    void *p = std::malloc(std::max<size_t>(b.size(), 1));
    if (!p) return fail(SG_ERR_OOM, "host allocation failed");
    std::memcpy(p, b.data(), b.size());
    *buf = p;
    *bytes = (int64_t)b.size();
    return SG_OK;
    SG_GUARD_END
}

sg_status sg_graph_data_decode(const void *buf, int64_t bytes, int32_t *V, int32_t *numEdges, int32_t **offsets,
                               int32_t **neighbors, int32_t **degList)
{
    SG_GUARD_BEGIN
    if ((!buf && bytes > 0) || bytes < 0 || !V || !numEdges || !offsets || !neighbors || !degList)
        return fail(SG_ERR_INVALID, "null argument");
    sg::CSC g;
    std::string err;
    if (!sg::decode_graph_data((const char *)buf, (size_t)bytes, "graph.data buffer", g, err))
        return fail(SG_ERR_INVALID, err);
    *V = g.V;
    *numEdges = g.numEdges;
    *offsets = dup_array(g.indexCol);
    *neighbors = dup_array(g.indexRow);
    *degList = dup_array(g.degList);
    return SG_OK;
    SG_GUARD_END
}

sg_status sg_rmat_generate(int32_t scale, int32_t edge_factor, double a, double b, double c, uint64_t seed,
                           int32_t *V, int64_t *E, int32_t **src, int32_t **dst)
{
    SG_GUARD_BEGIN
    if (!V || !E || !src || !dst) return fail(SG_ERR_INVALID, "null argument");
    sg::EdgeListData el;
    std::string err;
    if (!sg::rmat_generate(scale, edge_factor, a, b, c, seed, el, err)) return fail(SG_ERR_INVALID, err);
    *V = el.V;
    *E = (int64_t)el.src.size();
    *src = dup_array(el.src);
    *dst = dup_array(el.dst);
    return SG_OK;
    SG_GUARD_END
}

static sg_status finish_plan(sg::Template &t, sg_plan *out)
{
    auto h = std::make_unique<sg_plan_s>();
    h->t = t;
    std::string err;
    if (!sg::make_plan(h->t, h->p, err)) return fail(SG_ERR_INVALID, err);
    *out = h.release();
    return SG_OK;
}

sg_status sg_plan_create(int32_t n, int32_t m, const int32_t *src, const int32_t *dst, sg_plan *out)
{
    SG_GUARD_BEGIN
    if (!out || m < 0 || (m > 0 && (!src || !dst))) return fail(SG_ERR_INVALID, "null argument");
    std::vector<std::pair<int, int>> edges;
    for (int i = 0; i < m; ++i) edges.push_back({src[i], dst[i]});
    sg::Template t;
    std::string err;
    if (!sg::Template::from_edges(n, edges, t, err)) return fail(SG_ERR_INVALID, err);
    return finish_plan(t, out);
    SG_GUARD_END
}

sg_status sg_plan_read(const char *path, sg_plan *out)
{
    SG_GUARD_BEGIN
    if (!path || !out) return fail(SG_ERR_INVALID, "null argument");
    sg::Template t;
    std::string err;
    if (!sg::read_template(path, t, err)) return fail(err.rfind("cannot", 0) == 0 ? SG_ERR_IO : SG_ERR_INVALID, err);
    return finish_plan(t, out);
    SG_GUARD_END
}

void sg_plan_destroy(sg_plan p)
{
    if (!p) return;
    sg::release_plan_tables(p->p.uid);
    delete p;
}

sg_status sg_plan_info(sg_plan p, int32_t *k, int32_t *nsub, int32_t *scaled_sub, int64_t *arena_units)
{
    if (!p) return fail(SG_ERR_INVALID, "null plan");
    if (k) *k = p->p.k;
    if (nsub) *nsub = p->p.nsub();
    if (scaled_sub) *scaled_sub = p->p.scaled_sub;
    if (arena_units) *arena_units = p->p.arena_units;
    return SG_OK;
}

sg_status sg_plan_sub(sg_plan p, int32_t s, int32_t info[7])
{
    if (!p || !info) return fail(SG_ERR_INVALID, "null argument");
    if (s < 0 || s >= p->p.nsub()) return fail(SG_ERR_INVALID, "sub index out of range");
    const sg::SubTemplate &st = p->p.subs[s];
    info[0] = st.size;
    info[1] = st.main;
    info[2] = st.aux;
    info[3] = st.parent;
    info[4] = st.L;
    info[5] = st.S;
    info[6] = p->p.table_pitch[s];
    return SG_OK;
}

sg_status sg_plan_tables(sg_plan p, int32_t s, int32_t *c2c, int32_t *msplit, int32_t *asplit)
{
    if (!p) return fail(SG_ERR_INVALID, "null plan");
    if (s < 0 || s >= p->p.nsub()) return fail(SG_ERR_INVALID, "sub index out of range");
    const sg::SubTemplate &st = p->p.subs[s];
    if (c2c) std::memcpy(c2c, st.comb_to_count.data(), 4 * st.comb_to_count.size());
    if (msplit && !st.main_split.empty()) std::memcpy(msplit, st.main_split.data(), 4 * st.main_split.size());
    if (asplit && !st.aux_split.empty()) std::memcpy(asplit, st.aux_split.data(), 4 * st.aux_split.size());
    return SG_OK;
}

sg_status sg_plan_automorphisms(sg_plan p, int32_t *count)
{
    if (!p || !count) return fail(SG_ERR_INVALID, "null argument");
    *count = sg::count_automorphisms(p->t);
    return SG_OK;
}

sg_status sg_plan_shared_tables(sg_plan p, int32_t *same_as)
{
    if (!p || !same_as) return fail(SG_ERR_INVALID, "null argument");
    for (int s = 0; s < p->p.nsub(); ++s) same_as[s] = p->p.same_as[s];
    return SG_OK;
}

sg_status sg_plan_sub_edges(sg_plan p, int32_t s, int32_t *n, int32_t *src, int32_t *dst)
{
    if (!p || !n) return fail(SG_ERR_INVALID, "null argument");
    if (s < 0 || s >= p->p.nsub()) return fail(SG_ERR_INVALID, "sub index out of range");
    const sg::Template &t = p->p.subs[s].tree;
    *n = t.n;
    for (size_t i = 0; i < t.edges.size(); ++i) {
        if (src) src[i] = t.edges[i].first;
        if (dst) dst[i] = t.edges[i].second;
    }
    return SG_OK;
}

sg_status sg_graph_create(const int32_t *offsets, const int32_t *neighbors, int32_t V, int64_t nnz, int32_t device,
                          sg_graph *out)
{
    SG_GUARD_BEGIN
    if (!out) return fail(SG_ERR_INVALID, "null argument");
    auto h = std::make_unique<sg_graph_s>();
    sg_status st = from(sg::graph_create(offsets, neighbors, V, nnz, device, h->g));
    if (st) return st;
    *out = h.release();
    return SG_OK;
    SG_GUARD_END
}

sg_status sg_graph_create_edges(int32_t V, const int32_t *src, const int32_t *dst, int64_t E, int32_t device,
                                sg_graph *out)
{
    SG_GUARD_BEGIN
    if (!out) return fail(SG_ERR_INVALID, "null argument");
    auto h = std::make_unique<sg_graph_s>();
    sg_status st = from(sg::graph_from_edges(V, src, dst, E, device, h->g));
    if (st) return st;
    *out = h.release();
    return SG_OK;
    SG_GUARD_END
}

sg_status sg_graph_create_text(const char *path, int32_t device, sg_graph *out)
{
    SG_GUARD_BEGIN
    if (!out || !path) return fail(SG_ERR_INVALID, "null argument");
    auto h = std::make_unique<sg_graph_s>();
    sg_status st = from(sg::graph_from_text(path, device, h->g));
    if (st) return st;
    *out = h.release();
    return SG_OK;
    SG_GUARD_END
}

sg_status sg_graph_create_rmat(int32_t scale, int32_t edge_factor, double a, double b, double c, uint64_t seed,
                               int32_t device, sg_graph *out)
{
    SG_GUARD_BEGIN
    if (!out) return fail(SG_ERR_INVALID, "null argument");
    auto h = std::make_unique<sg_graph_s>();
    sg_status st = from(sg::graph_from_rmat(scale, edge_factor, a, b, c, seed, device, h->g));
    if (st) return st;
    *out = h.release();
    return SG_OK;
    SG_GUARD_END
}

sg_status sg_graph_download_csc(sg_graph g, int32_t *offsets, int32_t *neighbors)
{
    SG_GUARD_BEGIN
    if (!g) return fail(SG_ERR_INVALID, "null graph");
    return from(sg::graph_download_csc(*g->g, offsets, neighbors));
    SG_GUARD_END
}

void sg_graph_destroy(sg_graph g) { delete g; }

sg_status sg_graph_info(sg_graph g, int32_t *V, int64_t *nnz, int32_t *max_degree)
{
    if (!g) return fail(SG_ERR_INVALID, "null graph");
    if (V) *V = g->g->V;
    if (nnz) *nnz = g->g->nnz;
    if (max_degree) *max_degree = g->g->max_degree;
    return SG_OK;
}

void sg_count_opts_default(sg_count_opts *o)
{
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->n_colorings = 1;
    o->mode = SG_MODE_REFERENCE;
    o->hub_threshold = 1024;
}

namespace {
sg::CountOptions count_options(const sg_count_opts *o)
{
    sg::CountOptions co;
    co.n_colorings = o->n_colorings;
    co.seed_base = o->seed_base;
    co.mode = o->mode;
    co.batch = o->batch;
    co.hub_threshold = o->hub_threshold;
    co.profile = o->profile;
    co.autotune = o->no_autotune ? 0 : 1;
    co.exact = o->exact ? 1 : 0;
    co.wait_limit_ms = o->wait_limit_ms;
    co.blocked = o->no_blocked ? 0 : 1;
    co.rooted = o->no_rooted ? 0 : 1;
    co.flat = o->no_flat ? 0 : 1;
    co.persistent = o->persistent;
    return co;
}
}  // namespace

sg_status sg_count(sg_graph g, sg_plan p, const sg_count_opts *o, double *raw, sg_count_stats *stats)
{
    SG_GUARD_BEGIN
    if (!g || !p || !o || !raw) return fail(SG_ERR_INVALID, "null argument");
    sg::CountOptions co = count_options(o);
    sg::CountStats cs;
    sg_status st = from(sg::count(*g->g, p->p, co, raw, &cs));
    if (st) return st;
    if (stats) {
        stats->device_ms = cs.device_ms;
        stats->kernel_launches = cs.kernel_launches;
        stats->table_bytes = cs.table_bytes;
        stats->fused_ms = cs.fused_ms;
        stats->fused_launches = cs.fused_launches;
        stats->fused_alg_bytes = cs.fused_alg_bytes;
        stats->fused_gather_bytes = cs.fused_gather_bytes;
        stats->hub_ms = cs.hub_ms;
        stats->top_sub = cs.top_sub;
        stats->top_launches = cs.top_launches;
        stats->top_ms = cs.top_ms;
        stats->top_alg_bytes = cs.top_alg_bytes;
    }
    return SG_OK;
    SG_GUARD_END
}

sg_status sg_debug_count_unsatisfiable_wait(sg_graph g, sg_plan p, const sg_count_opts *o, double *raw)
{
    SG_GUARD_BEGIN
    if (!g || !p || !o || !raw) return fail(SG_ERR_INVALID, "null argument");
    if (o->batch < 1) return fail(SG_ERR_INVALID, "the wait test runs the batched form: batch must be >= 1");
    sg::CountOptions co = count_options(o);
    co.persistent = 1;
    co.test_unsatisfiable_wait = 1;
    return from(sg::count(*g->g, p->p, co, raw, nullptr));
    SG_GUARD_END
}

sg_status sg_count_jobs(sg_graph g, int32_t n_jobs, const sg_plan *plans, const uint32_t *seeds,
                        const sg_count_opts *o, double *raw, double *job_ms, sg_count_stats *stats)
{
    SG_GUARD_BEGIN
    if (!g || !plans || !seeds || !o || !raw) return fail(SG_ERR_INVALID, "null argument");
    if (n_jobs < 1) return fail(SG_ERR_INVALID, "n_jobs must be >= 1");
    std::vector<const sg::Plan *> ps((size_t)n_jobs);
    for (int32_t j = 0; j < n_jobs; ++j) {
        if (!plans[j]) return fail(SG_ERR_INVALID, "null plan in the job list");
        ps[j] = &plans[j]->p;
    }
    sg::CountOptions co;
    co.mode = o->mode;
    co.hub_threshold = o->hub_threshold;
    co.exact = o->exact ? 1 : 0;
    co.wait_limit_ms = o->wait_limit_ms;
    co.autotune = o->no_autotune ? 0 : 1;
    co.persistent = o->persistent ? 1 : 0;
    co.batch = o->batch;
    co.blocked = o->no_blocked ? 0 : 1;
    co.rooted = o->no_rooted ? 0 : 1;
    co.flat = o->no_flat ? 0 : 1;
    sg::CountStats cs;
    sg_status st = from(sg::count_jobs(*g->g, ps, seeds, co, raw, job_ms, &cs));
    if (st) return st;
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        stats->device_ms = cs.device_ms;
        stats->kernel_launches = cs.kernel_launches;
        stats->table_bytes = cs.table_bytes;
    }
    return SG_OK;
    SG_GUARD_END
}

static int factorial_int(int n) { return n <= 1 ? 1 : n * factorial_int(n - 1); }

sg_status sg_estimate(const double *raw, int32_t n, int32_t k, int32_t automorphisms, double *out)
{
    if (!raw || !out || n < 1 || k < 1 || automorphisms < 1) return fail(SG_ERR_INVALID, "bad argument");
    double sum = 0.0;
    for (int i = 0; i < n; ++i) sum += raw[i];
    double mean = sum / (double)n;
    // factorial in int as CountMat::factorial (CountMat.cpp:993-999)
    double prob = factorial_int(k) / ((double)factorial_int(0) * std::pow((double)k, (double)k));
    *out = std::floor(mean / (prob * (double)automorphisms) + 0.5);
    return SG_OK;
}

sg_status sg_colors(sg_graph g, int32_t k, uint32_t seed, int32_t *colors)
{
    SG_GUARD_BEGIN
    if (!g || !colors) return fail(SG_ERR_INVALID, "null argument");
    return from(sg::debug_colors(*g->g, k, seed, colors));
    SG_GUARD_END
}

sg_status sg_debug_sub_table(sg_graph g, sg_plan p, uint32_t seed, int32_t mode, int32_t hub_threshold, int32_t s,
                             void *out)
{
    SG_GUARD_BEGIN
    if (!g || !p || !out) return fail(SG_ERR_INVALID, "null argument");
    return from(sg::debug_sub_table(*g->g, p->p, seed, mode, hub_threshold, s, out));
    SG_GUARD_END
}

sg_status sg_debug_root(sg_graph g, sg_plan p, uint32_t seed, int32_t mode, int32_t hub_threshold, double *root,
                        double *raw)
{
    SG_GUARD_BEGIN
    if (!g || !p || !root) return fail(SG_ERR_INVALID, "null argument");
    return from(sg::debug_root(*g->g, p->p, seed, mode, hub_threshold, root, raw));
    SG_GUARD_END
}

sg_status sg_countmat_create(sg_countmat *out)
{
    if (!out) return fail(SG_ERR_INVALID, "null argument");
    *out = new sg_countmat_s();
    return SG_OK;
}

void sg_countmat_destroy(sg_countmat cm) { delete cm; }

sg_status sg_countmat_initialization(sg_countmat cm, sg_graph csr_graph, sg_graph csc_graph, int32_t thd_num,
                                     int32_t itr_num, int32_t isPruned, int32_t useSPMM, int32_t vtuneStart,
                                     int32_t calculate_automorphisms)
{
    if (!cm) return fail(SG_ERR_INVALID, "null countmat");
    if ((csr_graph == nullptr) == (csc_graph == nullptr))
        return fail(SG_ERR_INVALID, "exactly one of the CSR and CSC graphs must be given");
    if (itr_num < 1) return fail(SG_ERR_INVALID, "itr_num must be >= 1");
    cm->graph = csr_graph ? csr_graph : csc_graph;
    cm->csr = csr_graph != nullptr;
    cm->orig_state.assign((size_t)cm->graph->g->V, 0.0f);
    cm->thd_num = thd_num;
    cm->itr_num = itr_num;
    cm->isPruned = isPruned;
    cm->useSPMM = useSPMM;
    cm->vtuneStart = vtuneStart;
    cm->calc_aut = calculate_automorphisms;
    cm->initialized = true;
    return SG_OK;
}

sg_status sg_countmat_set_seed(sg_countmat cm, uint32_t seed_base)
{
    if (!cm) return fail(SG_ERR_INVALID, "null countmat");
    cm->seed = seed_base;
    cm->seeded = true;
    return SG_OK;
}

sg_status sg_countmat_compute(sg_countmat cm, sg_plan templates, int32_t isEstimate, int32_t verbose, double *result)
{
    SG_GUARD_BEGIN
    if (!cm || !templates || !result) return fail(SG_ERR_INVALID, "null argument");
    if (!cm->initialized) return fail(SG_ERR_INVALID, "CountMat not initialized");
    if (isEstimate) { *result = 0.0; return SG_OK; }
    sg_count_opts o;
    sg_count_opts_default(&o);
    o.n_colorings = cm->itr_num;
    o.seed_base = cm->seeded ? cm->seed : (uint32_t)std::time(nullptr);
    // isPruned=0 differs by graph type: the CSC path accumulates its SpMV buffer
    // (CountMat.cpp:931, CSCGraph.hpp:219-239), the CSR path overwrites it
    // (CSRGraph::SpMVNaiveFull, CSRGraph.cpp:190-208); useSPMM selects between
    // aggregations with identical results (CountMat.cpp:325-554 vs 556-849)
    o.mode = cm->isPruned ? SG_MODE_REFERENCE : (cm->csr ? SG_MODE_ORIGINAL_CSR : SG_MODE_ORIGINAL);
    cm->raw.assign((size_t)cm->itr_num, 0.0);
    sg::CountOptions co = count_options(&o);
    if (o.mode == SG_MODE_ORIGINAL) co.orig_state = cm->orig_state.data();
    sg::CountStats stats;
    sg_status st = from(sg::count(*cm->graph->g, templates->p, co, cm->raw.data(), &stats));
    if (st) return st;
    const int k = templates->p.k;
    if (verbose) {
        std::printf("\nTime for count per iter: %9.6lf seconds\n", stats.device_ms / 1000.0 / cm->itr_num);
        std::fflush(stdout);
    }
    double sum = 0.0;
    for (double r : cm->raw) sum += r;
    double finalCount = sum / (double)cm->itr_num;
    double prob = factorial_int(k) / ((double)factorial_int(0) * std::pow((double)k, (double)k));
    int aut = cm->calc_aut ? sg::count_automorphisms(templates->t) : 1;
    if (verbose) {
        std::printf("Final raw count is %e\n", finalCount);
        std::printf("Prob is %f\n", prob);
    }
    finalCount = std::floor(finalCount / (prob * (double)aut) + 0.5);
    if (verbose) {
        std::printf("Final count is %e\n", finalCount);
        std::fflush(stdout);
    }
    *result = finalCount;
    return SG_OK;
    SG_GUARD_END
}

sg_status sg_countmat_raw(sg_countmat cm, double *raw)
{
    if (!cm || !raw) return fail(SG_ERR_INVALID, "null argument");
    std::memcpy(raw, cm->raw.data(), sizeof(double) * cm->raw.size());
    return SG_OK;
}

}  // extern "C"
