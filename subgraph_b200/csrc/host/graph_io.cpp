// Host-side graph inputs.  Behaviour follows the reference loaders cited per
// function; the implementation is linear-time (counting passes instead of the
// per-column std::sort) and checks its inputs.
#include "graph_io.hpp"

#include <algorithm>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>

namespace sg {

namespace {

bool slurp(const std::string &path, std::string &buf, std::string &err)
{
    FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) { err = "cannot open " + path + ": " + std::strerror(errno); return false; }
    std::fseek(f, 0, SEEK_END);
    long n = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    if (n < 0) { std::fclose(f); err = "cannot size " + path; return false; }
    buf.resize((size_t)n);
    size_t got = n ? std::fread(&buf[0], 1, (size_t)n, f) : 0;
    std::fclose(f);
    if (got != (size_t)n) { err = "short read on " + path; return false; }
    return true;
}

// atoi() of the bytes [b, e): leading blanks, optional sign, digits.
int32_t atoi_range(const char *b, const char *e)
{
    while (b < e && (*b == ' ' || *b == '\t' || *b == '\n' || *b == '\r' || *b == '\v' || *b == '\f')) ++b;
    bool neg = false;
    if (b < e && (*b == '+' || *b == '-')) { neg = (*b == '-'); ++b; }
    int64_t v = 0;
    while (b < e && *b >= '0' && *b <= '9') { v = v * 10 + (*b - '0'); if (v > 0x7fffffffLL) v = 0x7fffffffLL + 1; ++b; }
    return (int32_t)(neg ? -v : v);
}

// Reads the next field the way std::getline(stream, line, delim) does and
// converts it with atoi.  Returns false at end of input.
bool next_field(const char *&p, const char *end, char delim, int32_t &v)
{
    if (p >= end) return false;
    const char *q = (const char *)std::memchr(p, delim, (size_t)(end - p));
    const char *fe = q ? q : end;
    v = atoi_range(p, fe);
    p = q ? q + 1 : end;
    return true;
}

}  // namespace

bool read_edge_list(const std::string &path, EdgeListData &out, std::string &err)
{
    std::string buf;
    if (!slurp(path, buf, err)) return false;
    const char *p = buf.data(), *end = p + buf.size();
    int32_t V, E;
    if (!next_field(p, end, '\n', V) || !next_field(p, end, '\n', E)) { err = path + ": missing header"; return false; }
    if (V < 0 || E < 0) { err = path + ": negative vertex or edge count"; return false; }
    out.src.resize((size_t)E);
    out.dst.resize((size_t)E);
    int32_t max_id = 0;
    for (int32_t j = 0; j < E; ++j) {
        int32_t a, b;
        if (!next_field(p, end, ' ', a) || !next_field(p, end, '\n', b)) {
            err = path + ": truncated edge list (" + std::to_string(j) + " of " + std::to_string(E) + " edges)";
            return false;
        }
        if (a < 0 || b < 0) { err = path + ": negative vertex id"; return false; }
        out.src[j] = a;
        out.dst[j] = b;
        max_id = std::max(max_id, std::max(a, b));
    }
    // hole removal (EdgeList.cpp:70-113): only when the largest id is not V-1
    if (max_id != V - 1) {
        std::vector<int32_t> vid((size_t)max_id + 1, 0);
        for (int32_t i = 0; i < E; ++i) { vid[out.src[i]] = 1; vid[out.dst[i]] = 1; }
        int32_t itr = 0;
        for (int32_t i = 0; i <= max_id; ++i)
            if (vid[i] == 1) vid[i] = itr++;
        V = itr;
        for (int32_t i = 0; i < E; ++i) { out.src[i] = vid[out.src[i]]; out.dst[i] = vid[out.dst[i]]; }
    }
    out.V = V;
    return true;
}

bool write_edge_list(const std::string &path, const EdgeListData &el, std::string &err)
{
    FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) { err = "cannot create " + path + ": " + std::strerror(errno); return false; }
    std::vector<char> out;
    out.reserve(el.src.size() * 16 + 64);
    char tmp[64];
    int n = std::snprintf(tmp, sizeof tmp, "%d\n%zu\n", el.V, el.src.size());
    out.insert(out.end(), tmp, tmp + n);
    for (size_t i = 0; i < el.src.size(); ++i) {
        n = std::snprintf(tmp, sizeof tmp, "%d %d\n", el.src[i], el.dst[i]);
        out.insert(out.end(), tmp, tmp + n);
    }
    bool ok = std::fwrite(out.data(), 1, out.size(), f) == out.size();
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) err = "write failed on " + path;
    return ok;
}

namespace {

bool check_edges(int32_t V, const int32_t *src, const int32_t *dst, int64_t E, std::string &err)
{
    if (V < 0) { err = "negative vertex count"; return false; }
    if (2 * E > 0x7fffffffLL) { err = "2*E exceeds the int32 nnz range of the reference format"; return false; }
    for (int64_t i = 0; i < E; ++i)
        if (src[i] < 0 || src[i] >= V || dst[i] < 0 || dst[i] >= V) {
            err = "edge " + std::to_string(i) + " has an endpoint outside [0, V)";
            return false;
        }
    return true;
}

}  // namespace

bool build_csr(int32_t V, const int32_t *src, const int32_t *dst, int64_t E, CSR &out, std::string &err)
{
    if (!check_edges(V, src, dst, E, err)) return false;
    out.V = V;
    out.numEdges = (int32_t)E;
    out.degList.assign((size_t)V, 0);
    for (int64_t i = 0; i < E; ++i) { out.degList[src[i]]++; out.degList[dst[i]]++; }
    out.indexRow.assign((size_t)V + 1, 0);
    for (int32_t i = 0; i < V; ++i) out.indexRow[i + 1] = out.indexRow[i] + out.degList[i];
    out.indexCol.assign((size_t)out.indexRow[V], 0);
    std::vector<int32_t> pos(out.indexRow.begin(), out.indexRow.end() - 1);
    // CSRGraph.cpp:82-96: the source row gets dst, then the destination row gets src
    for (int64_t i = 0; i < E; ++i) {
        out.indexCol[pos[src[i]]++] = dst[i];
        out.indexCol[pos[dst[i]]++] = src[i];
    }
    return true;
}

bool build_csc(int32_t V, const int32_t *src, const int32_t *dst, int64_t E, CSC &out, std::string &err)
{
    // The symmetrised matrix has entry (r, c) exactly as often as (c, r), so
    // walking the rows in ascending order and appending each row id r to the
    // columns of its entries yields every column's rows in ascending order:
    // the same arrays as the per-column std::sort of CSCGraph.hpp:172-175.
    CSR rows;
    if (!build_csr(V, src, dst, E, rows, err)) return false;
    out.V = V;
    out.numEdges = (int32_t)E;
    out.degList = rows.degList;
    out.indexCol = rows.indexRow;
    out.indexRow.assign(rows.indexCol.size(), 0);
    std::vector<int32_t> pos(out.indexCol.begin(), out.indexCol.end() - 1);
    for (int32_t r = 0; r < V; ++r)
        for (int32_t e = rows.indexRow[r]; e < rows.indexRow[r + 1]; ++e)
            out.indexRow[pos[rows.indexCol[e]]++] = r;
    return true;
}

void encode_graph_data(const CSC &g, std::string &buf)
{
    const size_t V = (size_t)g.V, nnz = g.indexRow.size();
    buf.assign(8 + 4 * (V + V + 1 + 2 * nnz), '\0');
    char *p = &buf[0];
    const int32_t hdr[2] = {g.numEdges, g.V};
    const float one = 1.0f;
    std::memcpy(p, hdr, 8);
    p += 8;
    if (V) std::memcpy(p, g.degList.data(), 4 * V);
    p += 4 * V;
    std::memcpy(p, g.indexCol.data(), 4 * (V + 1));
    p += 4 * (V + 1);
    if (nnz) std::memcpy(p, g.indexRow.data(), 4 * nnz);
    p += 4 * nnz;
    for (size_t e = 0; e < nnz; ++e) std::memcpy(p + 4 * e, &one, 4);
}

bool decode_graph_data(const char *data, size_t n, const std::string &what, CSC &g, std::string &err)
{
    auto rd = [&](size_t off) { int32_t v; std::memcpy(&v, data + off, 4); return v; };
    if (n < 8) { err = what + ": truncated header"; return false; }
    int32_t ne = rd(0), V = rd(4);
    if (V < 0) { err = what + ": negative vertex count"; return false; }
    size_t off_deg = 8, off_col = off_deg + 4 * (size_t)V, off_row = off_col + 4 * ((size_t)V + 1);
    if (n < off_row) { err = what + ": truncated offsets"; return false; }
    int32_t nnz = rd(off_row - 4);
    if (nnz < 0 || n != off_row + 8 * (size_t)nnz) {
        err = what + ": size does not match numVertices/indexCol (expected " +
              std::to_string(off_row + 8 * (size_t)(nnz < 0 ? 0 : nnz)) + " bytes, have " + std::to_string(n) + ")";
        return false;
    }
    g.numEdges = ne;
    g.V = V;
    g.degList.resize((size_t)V);
    g.indexCol.resize((size_t)V + 1);
    g.indexRow.resize((size_t)nnz);
    if (V) std::memcpy(g.degList.data(), data + off_deg, 4 * (size_t)V);
    std::memcpy(g.indexCol.data(), data + off_col, 4 * ((size_t)V + 1));
    if (nnz) std::memcpy(g.indexRow.data(), data + off_row, 4 * (size_t)nnz);
    if (g.indexCol[0] != 0) { err = what + ": indexCol[0] != 0"; return false; }
    for (int32_t i = 0; i < V; ++i)
        if (g.indexCol[i + 1] < g.indexCol[i]) { err = what + ": indexCol not monotone"; return false; }
    for (int32_t e = 0; e < nnz; ++e)
        if (g.indexRow[e] < 0 || g.indexRow[e] >= V) { err = what + ": row id out of range"; return false; }
    return true;
}

bool write_graph_data(const std::string &path, const CSC &g, std::string &err)
{
    std::string buf;
    encode_graph_data(g, buf);
    FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) { err = "cannot create " + path + ": " + std::strerror(errno); return false; }
    bool ok = std::fwrite(buf.data(), 1, buf.size(), f) == buf.size();
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) err = "write failed on " + path;
    return ok;
}

bool read_graph_data(const std::string &path, CSC &g, std::string &err)
{
    std::string buf;
    if (!slurp(path, buf, err)) return false;
    return decode_graph_data(buf.data(), buf.size(), path, g, err);
}

namespace {

struct Xoshiro256 {
    uint64_t s[4];
    explicit Xoshiro256(uint64_t seed)
    {
        for (int i = 0; i < 4; ++i) {  // splitmix64 expansion of the seed
            seed += 0x9e3779b97f4a7c15ULL;
            uint64_t z = seed;
            z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
            z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
            s[i] = z ^ (z >> 31);
        }
    }
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t next()
    {
        uint64_t r = rotl(s[1] * 5, 7) * 9, t = s[1] << 17;
        s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3];
        s[2] ^= t; s[3] = rotl(s[3], 45);
        return r;
    }
    double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
};

}  // namespace

bool rmat_generate(int scale, int edge_factor, double a, double b, double c, uint64_t seed,
                   EdgeListData &out, std::string &err)
{
    if (scale < 1 || scale > 30 || edge_factor < 1) { err = "scale must be in [1,30], edge_factor >= 1"; return false; }
    if (a < 0 || b < 0 || c < 0 || a + b + c > 1.0) { err = "invalid R-MAT initiator"; return false; }
    const int64_t n = int64_t(1) << scale;
    const int64_t m = (int64_t)edge_factor * n;
    Xoshiro256 rng(seed);
    std::vector<uint64_t> keys;
    keys.reserve((size_t)m);
    std::vector<int64_t> perm((size_t)n);
    for (int64_t i = 0; i < n; ++i) perm[i] = i;
    for (int64_t i = n - 1; i > 0; --i) {
        int64_t j = (int64_t)(rng.next() % (uint64_t)(i + 1));
        std::swap(perm[i], perm[j]);
    }
    const double ab = a + b, abc = a + b + c;
    for (int64_t e = 0; e < m; ++e) {
        int64_t u = 0, v = 0;
        for (int l = 0; l < scale; ++l) {
            double r = rng.uniform();
            int64_t bu = r >= ab ? 1 : 0;
            int64_t bv = ((r >= a && r < ab) || r >= abc) ? 1 : 0;
            u |= bu << l;
            v |= bv << l;
        }
        u = perm[u];
        v = perm[v];
        if (u == v) continue;
        int64_t lo = std::min(u, v), hi = std::max(u, v);
        keys.push_back(((uint64_t)lo << 32) | (uint64_t)hi);
    }
    std::sort(keys.begin(), keys.end());
    keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
    // keep the last id in use so that max_id == V-1 (no hole removal on load)
    int64_t top = n - 1;
    bool top_used = false;
    int64_t max_used = -1;
    for (uint64_t k : keys) {
        int64_t lo = (int64_t)(k >> 32), hi = (int64_t)(k & 0xffffffffULL);
        if (lo == top || hi == top) top_used = true;
        max_used = std::max(max_used, hi);
    }
    if (!top_used && max_used >= 0) {
        for (uint64_t &k : keys) {
            int64_t lo = (int64_t)(k >> 32), hi = (int64_t)(k & 0xffffffffULL);
            if (lo == max_used) lo = top;
            if (hi == max_used) hi = top;
            k = ((uint64_t)std::min(lo, hi) << 32) | (uint64_t)std::max(lo, hi);
        }
        std::sort(keys.begin(), keys.end());
    }
    out.V = (int32_t)n;
    out.src.resize(keys.size());
    out.dst.resize(keys.size());
    for (size_t i = 0; i < keys.size(); ++i) {
        out.src[i] = (int32_t)(keys[i] >> 32);
        out.dst[i] = (int32_t)(keys[i] & 0xffffffffULL);
    }
    return true;
}

}  // namespace sg
