// Input preparation on the GPU: edge-list text parsing, the CSC of the
// symmetrised adjacency, and an R-MAT generator with deduplication, each
// ending in a DeviceGraph (engine.cu, graph_finish) without a host copy of the
// adjacency.  Problems in the input (ids out of range, malformed or missing
// lines) are recorded in an error word on the device and reported as a
// status; no kernel reads outside its buffers.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "engine.hpp"

namespace sg {

#define IG_CK(call)                                                                               \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess)                                                                    \
            return Status{3, std::string(#call) + ": " + cudaGetErrorString(e_)};                 \
    } while (0)
#define IG_CKS(st)                 \
    do {                           \
        Status s_ = (st);          \
        if (s_.code) return s_;    \
    } while (0)

namespace {

enum : int32_t { kErrRange = 1, kErrNoSpace = 2, kErrNegative = 4 };

// ---------------------------------------------------------------------------
// CSC: entries (column, row) of both directions of every edge as 64-bit keys
// (column << 32 | row), sorted: the rows of every column come out ascending,
// duplicates and self loops kept (CSCGraph.hpp:95-178).
// ---------------------------------------------------------------------------
__global__ void k_edge_keys(int64_t E, int32_t V, const int32_t *__restrict__ src, const int32_t *__restrict__ dst,
                            uint64_t *__restrict__ keys, int32_t *__restrict__ deg, int32_t *err)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < E; i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t u = src[i], v = dst[i];
        if ((uint32_t)u >= (uint32_t)V || (uint32_t)v >= (uint32_t)V) {
            atomicOr(err, kErrRange);
            keys[2 * i] = keys[2 * i + 1] = 0;   // vertex 0, never read: the call fails
            continue;
        }
        keys[2 * i] = ((uint64_t)(uint32_t)v << 32) | (uint32_t)u;       // column v gets row u
        keys[2 * i + 1] = ((uint64_t)(uint32_t)u << 32) | (uint32_t)v;   // column u gets row v
        atomicAdd(deg + v, 1);
        atomicAdd(deg + u, 1);
    }
}

__global__ void k_key_rows(int64_t n, const uint64_t *__restrict__ keys, int32_t *__restrict__ rows)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        rows[i] = (int32_t)(uint32_t)(keys[i] & 0xffffffffull);
}

int grid_for(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 16)); }

__global__ void k_degree_keys(int32_t V, const int32_t *__restrict__ off, uint32_t *__restrict__ key,
                              int32_t *__restrict__ ids)
{
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < V; v += (int64_t)gridDim.x * blockDim.x) {
        key[v] = (uint32_t)(INT32_MAX - (off[v + 1] - off[v]));
        ids[v] = (int32_t)v;
    }
}

__global__ void k_degree_order(int32_t V, const uint32_t *__restrict__ key, const int32_t *__restrict__ iperm,
                               int32_t *__restrict__ perm, int32_t *__restrict__ deg)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= V; i += (int64_t)gridDim.x * blockDim.x) {
        if (i == V) {
            deg[V] = 0;
            continue;
        }
        perm[iperm[i]] = (int32_t)i;
        deg[i] = INT32_MAX - (int32_t)key[i];
    }
}

}  // namespace

Status degree_order(int32_t V, const int32_t *d_old_off, int32_t *d_iperm, int32_t *d_perm, int32_t *d_new_off,
                    std::vector<int32_t> &h_degree, cudaStream_t st)
{
    h_degree.assign(V, 0);
    if (V == 0) {
        IG_CK(cudaMemsetAsync(d_new_off, 0, sizeof(int32_t), st));
        return Status::ok();
    }
    uint32_t *key = nullptr, *key_sorted = nullptr;
    int32_t *ids = nullptr, *deg = nullptr;
    IG_CK(cudaMallocAsync(&key, 4 * (size_t)V, st));
    IG_CK(cudaMallocAsync(&key_sorted, 4 * (size_t)V, st));
    IG_CK(cudaMallocAsync(&ids, 4 * (size_t)V, st));
    IG_CK(cudaMallocAsync(&deg, 4 * ((size_t)V + 1), st));
    k_degree_keys<<<grid_for(V), 256, 0, st>>>(V, d_old_off, key, ids);
    IG_CK(cudaGetLastError());
    size_t sort_bytes = 0, scan_bytes = 0;
    IG_CK(cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, key, key_sorted, ids, d_iperm, (int)V, 0, 32, st));
    IG_CK(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, deg, d_new_off, V + 1, st));
    void *tmp = nullptr;
    IG_CK(cudaMallocAsync(&tmp, std::max<size_t>(std::max(sort_bytes, scan_bytes), 16), st));
    IG_CK(cub::DeviceRadixSort::SortPairs(tmp, sort_bytes, key, key_sorted, ids, d_iperm, (int)V, 0, 32, st));
    k_degree_order<<<grid_for((int64_t)V + 1), 256, 0, st>>>(V, key_sorted, d_iperm, d_perm, deg);
    IG_CK(cudaGetLastError());
    IG_CK(cub::DeviceScan::ExclusiveSum(tmp, scan_bytes, deg, d_new_off, V + 1, st));
    IG_CK(cudaMemcpyAsync(h_degree.data(), deg, 4 * (size_t)V, cudaMemcpyDeviceToHost, st));
    for (void *p : {(void *)key, (void *)key_sorted, (void *)ids, (void *)deg, tmp}) cudaFreeAsync(p, st);
    IG_CK(cudaStreamSynchronize(st));   // h_degree is pageable
    return Status::ok();
}

namespace {

// CSC of E host-or-device edges (device arrays here) into device offsets and
// rows.
Status build_csc_device(int32_t V, const int32_t *d_src, const int32_t *d_dst, int64_t E, cudaStream_t st,
                        int32_t *&d_off, int32_t *&d_rows)
{
    const int64_t nnz = 2 * E;
    if (nnz > 0x7fffffffLL) return Status{1, "too many edges"};
    uint64_t *keys = nullptr, *sorted = nullptr;
    int32_t *d_deg = nullptr, *d_err = nullptr;
    IG_CK(cudaMallocAsync(&keys, 8 * (size_t)std::max<int64_t>(nnz, 1), st));
    IG_CK(cudaMallocAsync(&sorted, 8 * (size_t)std::max<int64_t>(nnz, 1), st));
    IG_CK(cudaMallocAsync(&d_deg, 4 * ((size_t)V + 1), st));
    IG_CK(cudaMallocAsync(&d_err, 4, st));
    IG_CK(cudaMemsetAsync(d_deg, 0, 4 * ((size_t)V + 1), st));
    IG_CK(cudaMemsetAsync(d_err, 0, 4, st));
    if (E > 0) k_edge_keys<<<grid_for(E), 256, 0, st>>>(E, V, d_src, d_dst, keys, d_deg, d_err);
    IG_CK(cudaGetLastError());
    int32_t err = 0;
    IG_CK(cudaMemcpyAsync(&err, d_err, 4, cudaMemcpyDeviceToHost, st));
    IG_CK(cudaStreamSynchronize(st));
    if (err) {
        cudaFreeAsync(keys, st), cudaFreeAsync(sorted, st), cudaFreeAsync(d_deg, st), cudaFreeAsync(d_err, st);
        return Status{1, "edge endpoint out of range [0, V)"};
    }
    // sort the keys (only the bits the ids use)
    int end_bit = 32;
    while (end_bit < 64 && (((uint64_t)1 << (end_bit - 32)) <= (uint64_t)std::max(V - 1, 0))) ++end_bit;
    size_t tmp_bytes = 0;
    void *tmp = nullptr;
    IG_CK(cub::DeviceRadixSort::SortKeys(nullptr, tmp_bytes, keys, sorted, (int)nnz, 0, end_bit, st));
    IG_CK(cudaMallocAsync(&tmp, std::max<size_t>(tmp_bytes, 16), st));
    if (nnz) IG_CK(cub::DeviceRadixSort::SortKeys(tmp, tmp_bytes, keys, sorted, (int)nnz, 0, end_bit, st));
    IG_CK(cudaMallocAsync(&d_rows, 4 * (size_t)std::max<int64_t>(nnz, 1), st));
    if (nnz) k_key_rows<<<grid_for(nnz), 256, 0, st>>>(nnz, sorted, d_rows);
    IG_CK(cudaGetLastError());
    // offsets: exclusive scan of the degrees
    IG_CK(cudaMallocAsync(&d_off, 4 * ((size_t)V + 1), st));
    size_t scan_bytes = 0;
    IG_CK(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, d_deg, d_off, V + 1, st));
    void *scan_tmp = nullptr;
    IG_CK(cudaMallocAsync(&scan_tmp, std::max<size_t>(scan_bytes, 16), st));
    IG_CK(cub::DeviceScan::ExclusiveSum(scan_tmp, scan_bytes, d_deg, d_off, V + 1, st));
    for (void *p : {(void *)keys, (void *)sorted, (void *)d_deg, (void *)d_err, tmp, scan_tmp}) cudaFreeAsync(p, st);
    return Status::ok();
}

Status finish_from_device_edges(int32_t V, int32_t *d_src, int32_t *d_dst, int64_t E, std::unique_ptr<DeviceGraph> &g)
{
    cudaStream_t st = g->stream;
    int32_t *d_off = nullptr, *d_rows = nullptr;
    Status s = build_csc_device(V, d_src, d_dst, E, st, d_off, d_rows);
    cudaFreeAsync(d_src, st);
    cudaFreeAsync(d_dst, st);
    if (s.code) return s;
    g->V = V;
    g->nnz = 2 * E;
    return graph_finish(*g, d_off, d_rows);
}

// ---------------------------------------------------------------------------
// Edge-list text.  The body (after the two header lines) is split into lines;
// line j (j < E) must hold a space: the field before the first space is u,
// the rest of the line v, each converted like atoi (leading blanks, sign,
// digits).  For lines of that form this is exactly the getline(' ') /
// getline('\n') reading of EdgeList.cpp:46-60.
// ---------------------------------------------------------------------------
__device__ int32_t d_atoi(const char *b, const char *e)
{
    while (b < e && (*b == ' ' || *b == '\t' || *b == '\n' || *b == '\r' || *b == '\v' || *b == '\f')) ++b;
    bool neg = false;
    if (b < e && (*b == '+' || *b == '-')) { neg = (*b == '-'); ++b; }
    int64_t v = 0;
    while (b < e && *b >= '0' && *b <= '9') { v = v * 10 + (*b - '0'); if (v > 0x7fffffffLL) v = 0x7fffffffLL + 1; ++b; }
    return (int32_t)(neg ? -v : v);
}

struct LineStart {
    const char *text;
    __host__ __device__ bool operator()(int64_t i) const { return i == 0 || text[i - 1] == '\n'; }
};

__global__ void k_count_lines(const char *__restrict__ text, int64_t n, unsigned long long *count)
{
    unsigned long long c = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        c += (i == 0 || text[i - 1] == '\n') ? 1 : 0;
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, c);
}

__global__ void k_parse_lines(const char *__restrict__ text, int64_t n, const int64_t *__restrict__ starts,
                              int64_t nlines, int64_t E, int32_t *__restrict__ src, int32_t *__restrict__ dst,
                              int32_t *err, int32_t *max_id)
{
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < E; j += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = starts[j];
        const int64_t e = j + 1 < nlines ? starts[j + 1] - 1 : n;   // the newline, or the end of the text
        int64_t sp = s;
        while (sp < e && text[sp] != ' ') ++sp;
        if (sp >= e) {
            atomicOr(err, kErrNoSpace);
            src[j] = dst[j] = 0;
            continue;
        }
        const int32_t a = d_atoi(text + s, text + sp), b = d_atoi(text + sp + 1, text + e);
        if (a < 0 || b < 0) {
            atomicOr(err, kErrNegative);
            src[j] = dst[j] = 0;
            continue;
        }
        src[j] = a;
        dst[j] = b;
        atomicMax(max_id, max(a, b));
    }
}

__global__ void k_mark_used(int64_t E, const int32_t *__restrict__ src, const int32_t *__restrict__ dst, int32_t *used)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < E; i += (int64_t)gridDim.x * blockDim.x) {
        used[src[i]] = 1;
        used[dst[i]] = 1;
    }
}

__global__ void k_renumber(int64_t E, int32_t *src, int32_t *dst, const int32_t *__restrict__ vid)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < E; i += (int64_t)gridDim.x * blockDim.x) {
        src[i] = vid[src[i]];
        dst[i] = vid[dst[i]];
    }
}

// header fields the way the host reader takes them: getline('\n') + atoi
bool header_field(const char *&p, const char *end, int32_t &v)
{
    if (p >= end) return false;
    const char *q = (const char *)std::memchr(p, '\n', (size_t)(end - p));
    const char *fe = q ? q : end;
    const char *b = p;
    while (b < fe && (*b == ' ' || *b == '\t' || *b == '\r' || *b == '\v' || *b == '\f')) ++b;
    bool neg = false;
    if (b < fe && (*b == '+' || *b == '-')) { neg = (*b == '-'); ++b; }
    int64_t x = 0;
    while (b < fe && *b >= '0' && *b <= '9') { x = x * 10 + (*b - '0'); if (x > 0x7fffffffLL) x = 0x7fffffffLL + 1; ++b; }
    v = (int32_t)(neg ? -x : x);
    p = q ? q + 1 : end;
    return true;
}

// ---------------------------------------------------------------------------
// R-MAT on the GPU: counter-based SplitMix64 draws (a vertex's permutation
// key from (seed, vertex), the quadrant of edge e at level l from (seed, e,
// l)), so every draw is independent of the thread that makes it: the same
// seed gives the same graph.  Vertex ids are scrambled by sorting random
// keys, self loops dropped, edges canonicalised (min, max), sorted and
// deduplicated, and vertex 2^scale - 1 kept non-isolated (the largest id in
// use becomes it), as the host generator does with its sequential stream.
// ---------------------------------------------------------------------------
__host__ __device__ inline uint64_t splitmix(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

__global__ void k_perm_keys(int64_t n, uint64_t seed, uint64_t *keys, int32_t *ids)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        keys[i] = splitmix(seed ^ splitmix((uint64_t)i * 2 + 1));
        ids[i] = (int32_t)i;
    }
}

__global__ void k_rmat_edges(int64_t m, int scale, double a, double ab, double abc, uint64_t seed,
                             const int32_t *__restrict__ perm, uint64_t *__restrict__ keys)
{
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += (int64_t)gridDim.x * blockDim.x) {
        int64_t u = 0, v = 0;
        const uint64_t base = splitmix(seed ^ splitmix((uint64_t)e * 2));
        for (int l = 0; l < scale; ++l) {
            const double r = (double)(splitmix(base + (uint64_t)l) >> 11) * (1.0 / 9007199254740992.0);
            const int64_t bu = r >= ab ? 1 : 0;
            const int64_t bv = ((r >= a && r < ab) || r >= abc) ? 1 : 0;
            u |= bu << l;
            v |= bv << l;
        }
        const uint32_t pu = (uint32_t)perm[u], pv = (uint32_t)perm[v];
        keys[e] = pu == pv ? ~0ull : ((uint64_t)min(pu, pv) << 32) | (uint64_t)max(pu, pv);
    }
}

__global__ void k_split_keys(int64_t n, const uint64_t *__restrict__ keys, uint32_t top, uint32_t max_used,
                             int32_t *__restrict__ src, int32_t *__restrict__ dst)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t lo = (uint32_t)(keys[i] >> 32), hi = (uint32_t)(keys[i] & 0xffffffffull);
        src[i] = (int32_t)lo;
        dst[i] = (int32_t)(hi == max_used ? top : hi);   // the largest id in use becomes 2^scale - 1
    }
}

__global__ void k_max_hi(int64_t n, const uint64_t *__restrict__ keys, uint32_t *out)
{
    uint32_t m = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        m = max(m, (uint32_t)(keys[i] & 0xffffffffull));
    atomicMax(out, m);
}

// ---------------------------------------------------------------------------
// CSC in original vertex order: internal vertex iv (original iperm[iv]) owns
// off[iv] .. off[iv+1]; its neighbours map back through iperm.
// ---------------------------------------------------------------------------
__global__ void k_unmap(int32_t V, const int32_t *__restrict__ off, const int32_t *__restrict__ adj,
                        const int32_t *__restrict__ iperm, const int32_t *__restrict__ orig_off, int32_t *__restrict__ out)
{
    const int lane = threadIdx.x & 31;
    const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t iv = w; iv < V; iv += nw) {
        const int32_t o = orig_off[iperm[iv]], b = off[iv], e = off[iv + 1];
        for (int32_t i = b + lane; i < e; i += 32) out[o + (i - b)] = iperm[adj[i]];
    }
}

}  // namespace

Status graph_from_edges(int32_t V, const int32_t *src, const int32_t *dst, int64_t E, int device,
                        std::unique_ptr<DeviceGraph> &out)
{
    if (V < 0 || E < 0 || 2 * E > 0x7fffffffLL) return Status{1, "vertex or edge count out of range"};
    if (E > 0 && (!src || !dst)) return Status{1, "null edge array"};
    std::unique_ptr<DeviceGraph> g;
    IG_CKS(new_device_graph(device, V, 2 * E, g));
    cudaStream_t st = g->stream;
    int32_t *d_src = nullptr, *d_dst = nullptr;
    IG_CK(cudaMallocAsync(&d_src, 4 * (size_t)std::max<int64_t>(E, 1), st));
    IG_CK(cudaMallocAsync(&d_dst, 4 * (size_t)std::max<int64_t>(E, 1), st));
    if (E) {
        IG_CK(cudaMemcpyAsync(d_src, src, 4 * (size_t)E, cudaMemcpyHostToDevice, st));
        IG_CK(cudaMemcpyAsync(d_dst, dst, 4 * (size_t)E, cudaMemcpyHostToDevice, st));
    }
    IG_CKS(finish_from_device_edges(V, d_src, d_dst, E, g));
    out = std::move(g);
    return Status::ok();
}

Status graph_from_text(const std::string &path, int device, std::unique_ptr<DeviceGraph> &out)
{
    FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) return Status{5, "cannot open " + path};
    std::fseek(f, 0, SEEK_END);
    const long len = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    std::string buf(len > 0 ? (size_t)len : 0, '\0');
    const size_t got = len > 0 ? std::fread(&buf[0], 1, (size_t)len, f) : 0;
    std::fclose(f);
    if (len < 0 || got != (size_t)len) return Status{5, "short read on " + path};
    const char *p = buf.data(), *end = p + buf.size();
    int32_t V = 0, E = 0;
    if (!header_field(p, end, V) || !header_field(p, end, E)) return Status{1, path + ": missing header"};
    if (V < 0 || E < 0) return Status{1, path + ": negative vertex or edge count"};
    const int64_t n = end - p;
    std::unique_ptr<DeviceGraph> g;
    IG_CKS(new_device_graph(device, V, 2 * (int64_t)E, g));
    cudaStream_t st = g->stream;
    char *d_text = nullptr;
    int64_t *d_starts = nullptr, *d_nlines = nullptr;
    int32_t *d_src = nullptr, *d_dst = nullptr, *d_err = nullptr, *d_max = nullptr;
    IG_CK(cudaMallocAsync(&d_text, (size_t)std::max<int64_t>(n, 1), st));
    IG_CK(cudaMallocAsync(&d_nlines, 8, st));
    IG_CK(cudaMemsetAsync(d_nlines, 0, 8, st));
    if (n) IG_CK(cudaMemcpyAsync(d_text, p, (size_t)n, cudaMemcpyHostToDevice, st));
    // count the line starts first: the selection output holds exactly them
    unsigned long long nstart = 0;
    if (n) k_count_lines<<<grid_for(n), 256, 0, st>>>(d_text, n, reinterpret_cast<unsigned long long *>(d_nlines));
    IG_CK(cudaMemcpyAsync(&nstart, d_nlines, 8, cudaMemcpyDeviceToHost, st));
    IG_CK(cudaStreamSynchronize(st));
    IG_CK(cudaMallocAsync(&d_starts, 8 * (size_t)std::max<unsigned long long>(nstart, 1), st));
    IG_CK(cudaMallocAsync(&d_src, 4 * (size_t)std::max(E, 1), st));
    IG_CK(cudaMallocAsync(&d_dst, 4 * (size_t)std::max(E, 1), st));
    IG_CK(cudaMallocAsync(&d_err, 8, st));
    d_max = d_err + 1;
    IG_CK(cudaMemsetAsync(d_err, 0, 8, st));
    IG_CK(cudaMemsetAsync(d_nlines, 0, 8, st));
    // line starts: positions i with i == 0 or text[i-1] == '\n'
    size_t tmp_bytes = 0;
    void *tmp = nullptr;
    cub::CountingInputIterator<int64_t> idx(0);
    if (n) {
        IG_CK(cub::DeviceSelect::If(nullptr, tmp_bytes, idx, d_starts, d_nlines, n, LineStart{d_text}, st));
        IG_CK(cudaMallocAsync(&tmp, std::max<size_t>(tmp_bytes, 16), st));
        IG_CK(cub::DeviceSelect::If(tmp, tmp_bytes, idx, d_starts, d_nlines, n, LineStart{d_text}, st));
    }
    int64_t nlines = 0;
    IG_CK(cudaMemcpyAsync(&nlines, d_nlines, 8, cudaMemcpyDeviceToHost, st));
    IG_CK(cudaStreamSynchronize(st));
    auto cleanup = [&]() {
        for (void *q : {(void *)d_text, (void *)d_starts, (void *)d_nlines, (void *)d_err, tmp}) if (q) cudaFreeAsync(q, st);
    };
    if (nlines < E) {
        cleanup();
        cudaFreeAsync(d_src, st), cudaFreeAsync(d_dst, st);
        cudaStreamSynchronize(st);
        return Status{1, path + ": truncated edge list (" + std::to_string(nlines) + " of " + std::to_string(E) + " edges)"};
    }
    if (E) k_parse_lines<<<grid_for(E), 256, 0, st>>>(d_text, n, d_starts, nlines, E, d_src, d_dst, d_err, d_max);
    IG_CK(cudaGetLastError());
    int32_t hs[2] = {0, 0};
    IG_CK(cudaMemcpyAsync(hs, d_err, 8, cudaMemcpyDeviceToHost, st));
    IG_CK(cudaStreamSynchronize(st));
    cleanup();
    if (hs[0]) {
        cudaFreeAsync(d_src, st), cudaFreeAsync(d_dst, st);
        cudaStreamSynchronize(st);
        return Status{1, path + ((hs[0] & kErrNegative) ? ": negative vertex id" : ": an edge line without a space")};
    }
    // hole removal (EdgeList.cpp:70-113): only when the largest id is not V-1
    const int32_t max_id = hs[1];
    if (E == 0 && max_id != V - 1) V = 0;   // no id in use: the host reader's hole removal leaves none
    if (E > 0 && max_id != V - 1) {
        int32_t *used = nullptr, *vid = nullptr;
        IG_CK(cudaMallocAsync(&used, 4 * ((size_t)max_id + 2), st));
        IG_CK(cudaMallocAsync(&vid, 4 * ((size_t)max_id + 2), st));
        IG_CK(cudaMemsetAsync(used, 0, 4 * ((size_t)max_id + 2), st));
        k_mark_used<<<grid_for(E), 256, 0, st>>>(E, d_src, d_dst, used);
        size_t sb = 0;
        void *stmp = nullptr;
        IG_CK(cub::DeviceScan::ExclusiveSum(nullptr, sb, used, vid, max_id + 2, st));
        IG_CK(cudaMallocAsync(&stmp, std::max<size_t>(sb, 16), st));
        IG_CK(cub::DeviceScan::ExclusiveSum(stmp, sb, used, vid, max_id + 2, st));
        k_renumber<<<grid_for(E), 256, 0, st>>>(E, d_src, d_dst, vid);
        IG_CK(cudaGetLastError());
        IG_CK(cudaMemcpyAsync(&V, vid + max_id + 1, 4, cudaMemcpyDeviceToHost, st));
        IG_CK(cudaStreamSynchronize(st));
        for (void *q : {(void *)used, (void *)vid, stmp}) cudaFreeAsync(q, st);
    }
    IG_CKS(finish_from_device_edges(V, d_src, d_dst, E, g));
    out = std::move(g);
    return Status::ok();
}

Status graph_from_rmat(int scale, int edge_factor, double a, double b, double c, uint64_t seed, int device,
                       std::unique_ptr<DeviceGraph> &out)
{
    if (scale < 1 || scale > 30 || edge_factor < 1) return Status{1, "scale must be in [1,30], edge_factor >= 1"};
    if (a < 0 || b < 0 || c < 0 || a + b + c > 1.0) return Status{1, "invalid R-MAT initiator"};
    const int64_t n = int64_t(1) << scale;
    const int64_t m = (int64_t)edge_factor * n;
    if (m > 0x3fffffffLL) return Status{1, "too many edges"};
    std::unique_ptr<DeviceGraph> g;
    IG_CKS(new_device_graph(device, (int32_t)n, 0, g));
    cudaStream_t st = g->stream;
    // vertex scramble: ids sorted by random keys
    uint64_t *pk = nullptr, *pk2 = nullptr;
    int32_t *ids = nullptr, *perm = nullptr;
    IG_CK(cudaMallocAsync(&pk, 8 * (size_t)n, st));
    IG_CK(cudaMallocAsync(&pk2, 8 * (size_t)n, st));
    IG_CK(cudaMallocAsync(&ids, 4 * (size_t)n, st));
    IG_CK(cudaMallocAsync(&perm, 4 * (size_t)n, st));
    k_perm_keys<<<grid_for(n), 256, 0, st>>>(n, seed, pk, ids);
    size_t tb = 0;
    void *tmp = nullptr;
    IG_CK(cub::DeviceRadixSort::SortPairs(nullptr, tb, pk, pk2, ids, perm, (int)n, 0, 64, st));
    IG_CK(cudaMallocAsync(&tmp, std::max<size_t>(tb, 16), st));
    IG_CK(cub::DeviceRadixSort::SortPairs(tmp, tb, pk, pk2, ids, perm, (int)n, 0, 64, st));
    cudaFreeAsync(tmp, st);
    // edges as canonical keys, self loops as the all-ones key (sorted last)
    uint64_t *keys = nullptr, *sorted = nullptr, *uniq = nullptr;
    int64_t *d_count = nullptr;
    IG_CK(cudaMallocAsync(&keys, 8 * (size_t)m, st));
    IG_CK(cudaMallocAsync(&sorted, 8 * (size_t)m, st));
    IG_CK(cudaMallocAsync(&uniq, 8 * (size_t)m, st));
    IG_CK(cudaMallocAsync(&d_count, 8, st));
    k_rmat_edges<<<grid_for(m), 256, 0, st>>>(m, scale, a, a + b, a + b + c, seed, perm, keys);
    IG_CK(cub::DeviceRadixSort::SortKeys(nullptr, tb, keys, sorted, (int)m, 0, 64, st));
    IG_CK(cudaMallocAsync(&tmp, std::max<size_t>(tb, 16), st));
    IG_CK(cub::DeviceRadixSort::SortKeys(tmp, tb, keys, sorted, (int)m, 0, 64, st));
    cudaFreeAsync(tmp, st);
    IG_CK(cub::DeviceSelect::Unique(nullptr, tb, sorted, uniq, d_count, (int)m, st));
    IG_CK(cudaMallocAsync(&tmp, std::max<size_t>(tb, 16), st));
    IG_CK(cub::DeviceSelect::Unique(tmp, tb, sorted, uniq, d_count, (int)m, st));
    cudaFreeAsync(tmp, st);
    int64_t cnt = 0;
    uint64_t last = 0;
    IG_CK(cudaMemcpyAsync(&cnt, d_count, 8, cudaMemcpyDeviceToHost, st));
    IG_CK(cudaStreamSynchronize(st));
    if (cnt > 0) {
        IG_CK(cudaMemcpyAsync(&last, uniq + cnt - 1, 8, cudaMemcpyDeviceToHost, st));
        IG_CK(cudaStreamSynchronize(st));
        if (last == ~0ull) --cnt;   // the self-loop key
    }
    // the largest id in use (every key has lo < hi, so it is the largest hi)
    uint32_t *d_mx = reinterpret_cast<uint32_t *>(d_count);
    IG_CK(cudaMemsetAsync(d_mx, 0, 4, st));
    if (cnt) k_max_hi<<<grid_for(cnt), 256, 0, st>>>(cnt, uniq, d_mx);
    uint32_t mx = 0;
    IG_CK(cudaMemcpyAsync(&mx, d_mx, 4, cudaMemcpyDeviceToHost, st));
    IG_CK(cudaStreamSynchronize(st));
    int32_t *d_src = nullptr, *d_dst = nullptr;
    IG_CK(cudaMallocAsync(&d_src, 4 * (size_t)std::max<int64_t>(cnt, 1), st));
    IG_CK(cudaMallocAsync(&d_dst, 4 * (size_t)std::max<int64_t>(cnt, 1), st));
    // renaming the largest id in use to 2^scale - 1 keeps the key order: it is
    // the largest hi of its lo in every key it appears in
    if (cnt) k_split_keys<<<grid_for(cnt), 256, 0, st>>>(cnt, uniq, (uint32_t)(n - 1), mx, d_src, d_dst);
    IG_CK(cudaGetLastError());
    for (void *q : {(void *)pk, (void *)pk2, (void *)ids, (void *)perm, (void *)keys, (void *)sorted, (void *)uniq,
                    (void *)d_count})
        cudaFreeAsync(q, st);
    IG_CKS(finish_from_device_edges((int32_t)n, d_src, d_dst, cnt, g));
    out = std::move(g);
    return Status::ok();
}

Status graph_download_csc(DeviceGraph &g, int32_t *offsets, int32_t *neighbors)
{
    if (!offsets || (g.nnz > 0 && !neighbors)) return Status{1, "null output array"};
    IG_CK(cudaSetDevice(g.device));
    const int32_t V = g.V;
    std::vector<int32_t> iperm(V);
    cudaStream_t st = g.stream;
    if (V) IG_CK(cudaMemcpyAsync(iperm.data(), g.d_iperm, 4 * (size_t)V, cudaMemcpyDeviceToHost, st));
    IG_CK(cudaStreamSynchronize(st));
    // original-order offsets from the internal-order degrees
    std::vector<int32_t> deg(V);
    for (int32_t i = 0; i < V; ++i) deg[iperm[i]] = g.h_degree[i];
    offsets[0] = 0;
    for (int32_t v = 0; v < V; ++v) offsets[v + 1] = offsets[v] + deg[v];
    if (g.nnz == 0) return Status::ok();
    int32_t *d_oo = nullptr, *d_out = nullptr;
    IG_CK(cudaMallocAsync(&d_oo, 4 * ((size_t)V + 1), st));
    IG_CK(cudaMallocAsync(&d_out, 4 * (size_t)g.nnz, st));
    IG_CK(cudaMemcpyAsync(d_oo, offsets, 4 * ((size_t)V + 1), cudaMemcpyHostToDevice, st));
    k_unmap<<<(int)std::min<int64_t>(((int64_t)V * 32 + 255) / 256, 148 * 16), 256, 0, st>>>(V, g.d_off, g.d_adj,
                                                                                            g.d_iperm, d_oo, d_out);
    IG_CK(cudaGetLastError());
    IG_CK(cudaMemcpyAsync(neighbors, d_out, 4 * (size_t)g.nnz, cudaMemcpyDeviceToHost, st));
    IG_CK(cudaStreamSynchronize(st));
    cudaFreeAsync(d_oo, st);
    cudaFreeAsync(d_out, st);
    IG_CK(cudaStreamSynchronize(st));
    return Status::ok();
}

}  // namespace sg
