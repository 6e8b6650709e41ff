// Template planning.  The sub-template list, its order and the index tables
// must equal the reference's exactly (they decide which sub is scaled and how
// every count-table column is addressed), so the steps follow the reference's
// algorithm; the code is organised differently:
//  * a split is a breadth-first walk from the root that skips the cut edge,
//    with vertices relabelled in discovery order (DivideTemplates.cpp:153-246);
//  * the final order is breadth-first over the binary split tree, main child
//    before aux child, which is the fixed point of the reference's bubble sort
//    on parent indices (DivideTemplates.cpp:264-327);
//  * split tables come from the complement rule (the aux colors of a split are
//    the color set minus the main colors), which is what the reference's
//    reversed lexicographic pairing produces (IndexSys.cpp:395-414).
#include "plan.hpp"

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <deque>
#include <functional>
#include <map>
#include <string>

namespace sg {

int64_t binom(int n, int k)
{
    if (k < 0 || k > n) return 0;
    if (k * 2 > n) k = n - k;
    int64_t r = 1;
    for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
    return r;
}

int32_t colex_rank(const int *c, int size)
{
    // IndexSys::get_color_hash (IndexSys.cpp:303-313) with 0-based colors
    int64_t r = 0;
    for (int i = 0; i < size; ++i) r += binom(c[i], i + 1);
    return (int32_t)r;
}

void index_tables(int k, int size, int msz, int &L, int &S, std::vector<int32_t> &comb_to_count,
                  std::vector<int32_t> &main_split, std::vector<int32_t> &aux_split)
{
    L = (int)binom(k, size);
    comb_to_count.assign(L, 0);
    S = size > 1 ? (int)binom(size, msz) : 0;
    main_split.assign((size_t)L * S, 0);
    aux_split.assign((size_t)L * S, 0);
    std::vector<int> set(size), sel(msz > 0 ? msz : 1);
    for (int i = 0; i < size; ++i) set[i] = i;
    for (int li = 0; li < L; ++li) {
        comb_to_count[li] = colex_rank(set.data(), size);
        if (size > 1) {
            for (int i = 0; i < msz; ++i) sel[i] = i;
            for (int j = 0; j < S; ++j) {
                int mc[kMaxColors], ac[kMaxColors], nm = 0, na = 0;
                for (int q = 0, w = 0; q < size; ++q) {
                    if (w < msz && sel[w] == q) { mc[nm++] = set[q]; ++w; }
                    else ac[na++] = set[q];
                }
                main_split[(size_t)li * S + j] = colex_rank(mc, nm);
                aux_split[(size_t)li * S + j] = colex_rank(ac, na);
                // next lexicographic msz-subset of positions
                for (int q = msz - 1; q >= 0; --q)
                    if (sel[q] < size - msz + q) { ++sel[q]; for (int r = q + 1; r < msz; ++r) sel[r] = sel[r - 1] + 1; break; }
            }
        }
        // next lexicographic size-subset of colors
        for (int q = size - 1; q >= 0; --q)
            if (set[q] < k - size + q) { ++set[q]; for (int r = q + 1; r < size; ++r) set[r] = set[r - 1] + 1; break; }
    }
}

bool Template::from_edges(int n, const std::vector<std::pair<int, int>> &edges, Template &t, std::string &err)
{
    if (n < 2) { err = "template needs at least 2 vertices"; return false; }
    if (n > kMaxColors) { err = "template has " + std::to_string(n) + " vertices; at most " + std::to_string(kMaxColors) + " are supported"; return false; }
    if ((int)edges.size() != n - 1) { err = "template is not a tree (needs n-1 edges)"; return false; }
    t.n = n;
    t.edges = edges;
    t.adj.assign(n, {});
    for (auto &e : edges) {
        if (e.first < 0 || e.first >= n || e.second < 0 || e.second >= n || e.first == e.second) {
            err = "template edge endpoint out of range or self loop";
            return false;
        }
        t.adj[e.first].push_back(e.second);
        t.adj[e.second].push_back(e.first);
    }
    // connected?
    std::vector<char> seen(n, 0);
    std::vector<int> st{0};
    seen[0] = 1;
    int cnt = 1;
    while (!st.empty()) {
        int a = st.back();
        st.pop_back();
        for (int b : t.adj[a])
            if (!seen[b]) { seen[b] = 1; ++cnt; st.push_back(b); }
    }
    if (cnt != n) { err = "template is not connected"; return false; }
    return true;
}

bool read_template(const std::string &path, Template &t, std::string &err)
{
    FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) { err = "cannot open template " + path; return false; }
    std::string buf;
    char tmp[4096];
    size_t got;
    while ((got = std::fread(tmp, 1, sizeof tmp, f)) > 0) buf.append(tmp, got);
    std::fclose(f);
    // same field rules as the graph reader: getline('\n') twice, then ' ' / '\n'
    const char *p = buf.data(), *end = p + buf.size();
    auto field = [&](char delim, int &v) {
        if (p >= end) return false;
        const char *q = (const char *)std::memchr(p, delim, (size_t)(end - p));
        std::string s(p, q ? q : end);
        v = std::atoi(s.c_str());
        p = q ? q + 1 : end;
        return true;
    };
    int n, m;
    if (!field('\n', n) || !field('\n', m)) { err = path + ": missing template header"; return false; }
    if (m < 0 || m > 4 * kMaxColors) { err = path + ": bad template edge count"; return false; }
    std::vector<std::pair<int, int>> edges;
    int max_id = 0;
    for (int j = 0; j < m; ++j) {
        int a, b;
        if (!field(' ', a) || !field('\n', b)) { err = path + ": truncated template"; return false; }
        if (a < 0 || b < 0) { err = path + ": negative template vertex id"; return false; }
        edges.push_back({a, b});
        max_id = std::max(max_id, std::max(a, b));
    }
    if (max_id != n - 1 && max_id < 4 * kMaxColors) {
        // hole removal of Graph.cpp:40-69 (the vertex count is kept, as there)
        std::vector<int> vid(max_id + 1, 0);
        for (auto &e : edges) { vid[e.first] = 1; vid[e.second] = 1; }
        int itr = 0;
        for (int i = 0; i <= max_id; ++i) if (vid[i]) vid[i] = itr++;
        for (auto &e : edges) { e.first = vid[e.first]; e.second = vid[e.second]; }
    }
    return Template::from_edges(n, edges, t, err);
}

namespace {

// The subtree on `root`'s side of the edge (root, cut), vertices relabelled in
// breadth-first discovery order (root -> 0), edges in discovery order.
Template extract_side(const Template &t, int root, int cut)
{
    std::vector<int> label(t.n, -1), order{root};
    std::vector<std::pair<int, int>> edges;
    label[root] = 0;
    for (size_t i = 0; i < order.size(); ++i) {
        int a = order[i];
        for (int b : t.adj[a]) {
            if (b == cut || label[b] >= 0) continue;   // the cut side, or a's parent
            label[b] = (int)order.size();
            order.push_back(b);
            edges.push_back({label[a], label[b]});
        }
    }
    Template s;
    s.n = (int)order.size();
    s.edges = edges;
    s.adj.assign(s.n, {});
    for (auto &e : edges) { s.adj[e.first].push_back(e.second); s.adj[e.second].push_back(e.first); }
    return s;
}

struct SplitNode {
    Template tree;
    int main = -1, aux = -1;
};

}  // namespace

int count_automorphisms(const Template &t)
{
    // |Aut| of a tree from canonical forms rooted at its center (the reference
    // enumerates all n! permutations; the predicate it tests is equivalent to
    // the automorphism condition, so the counts agree).
    int n = t.n;
    if (n <= 1) return 1;
    std::vector<int> deg(n), layer;
    for (int i = 0; i < n; ++i) { deg[i] = (int)t.adj[i].size(); if (deg[i] <= 1) layer.push_back(i); }
    int remaining = n;
    while (remaining > 2) {
        std::vector<int> next;
        remaining -= (int)layer.size();
        for (int v : layer) {
            deg[v] = 0;
            for (int w : t.adj[v]) if (deg[w] > 0 && --deg[w] == 1) next.push_back(w);
        }
        layer.swap(next);
    }
    std::map<std::vector<int>, int> ids;
    std::function<std::pair<int, int64_t>(int, int)> canon = [&](int v, int par) -> std::pair<int, int64_t> {
        std::vector<std::pair<int, int64_t>> ch;
        for (int w : t.adj[v]) if (w != par) ch.push_back(canon(w, v));
        std::sort(ch.begin(), ch.end());
        int64_t a = 1;
        std::vector<int> key;
        for (size_t i = 0; i < ch.size();) {
            size_t j = i;
            while (j < ch.size() && ch[j].first == ch[i].first) { a *= ch[j].second; ++j; }
            for (size_t f = 2; f <= j - i; ++f) a *= (int64_t)f;
            i = j;
        }
        for (auto &c : ch) key.push_back(c.first);
        auto it = ids.find(key);
        int id = it == ids.end() ? (ids[key] = (int)ids.size()) : it->second;
        return {id, a};
    };
    if (layer.size() == 1) return (int)canon(layer[0], -1).second;
    auto a = canon(layer[0], layer[1]);
    auto b = canon(layer[1], layer[0]);
    int64_t r = a.second * b.second * (a.first == b.first ? 2 : 1);
    return (int)r;
}

bool make_plan(const Template &t, Plan &p, std::string &err)
{
    if (t.n < 2 || t.n > kMaxColors) { err = "template size out of range"; return false; }
    // ---- division: depth-first numbering as DivideTemplates::divide assigns it
    std::vector<SplitNode> nodes(1);
    nodes[0].tree = t;
    std::function<void(int)> divide = [&](int x) {
        const Template &cur = nodes[x].tree;
        int cut = cur.adj[0][0];                          // first neighbour of the root
        SplitNode m, a;
        m.tree = extract_side(cur, 0, cut);
        a.tree = extract_side(cur, cut, 0);
        int mi = (int)nodes.size();
        nodes.push_back(m);
        nodes.push_back(a);
        nodes[x].main = mi;
        nodes[x].aux = mi + 1;
        if (nodes[mi].tree.n > 1) divide(mi);
        if (nodes[mi + 1].tree.n > 1) divide(mi + 1);
    };
    divide(0);
    // ---- order: breadth-first over the split tree, main before aux
    std::vector<int> order{0}, pos(nodes.size(), -1);
    for (size_t i = 0; i < order.size(); ++i) {
        int x = order[i];
        if (nodes[x].main >= 0) { order.push_back(nodes[x].main); order.push_back(nodes[x].aux); }
    }
    for (size_t i = 0; i < order.size(); ++i) pos[order[i]] = (int)i;
    const int ns = (int)order.size();
    p = Plan();
    p.k = t.n;
    p.subs.resize(ns);
    for (int i = 0; i < ns; ++i) {
        const SplitNode &nd = nodes[order[i]];
        SubTemplate &s = p.subs[i];
        s.tree = nd.tree;
        s.size = nd.tree.n;
        if (nd.main >= 0) { s.main = pos[nd.main]; s.aux = pos[nd.aux]; }
    }
    for (int i = 0; i < ns; ++i)
        if (p.subs[i].main != kDummy) { p.subs[p.subs[i].main].parent = i; p.subs[p.subs[i].aux].parent = i; }
    // ---- index tables
    for (int si = 0; si < ns; ++si) {
        SubTemplate &s = p.subs[si];
        const int msz = s.size > 1 ? p.subs[s.main].size : 0;
        index_tables(p.k, s.size, msz, s.L, s.S, s.comb_to_count, s.main_split, s.aux_split);
    }
    // ---- processing order (CountMat.cpp:277: s = n-1 .. 0) and the scaled sub
    for (int si = ns - 1; si >= 0; --si)
        if (p.subs[si].size > 1) {
            p.process_order.push_back(si);
            if (p.scaled_sub < 0) p.scaled_sub = si;
        }
    // ---- tables computed once.  A sub's table is a function of its rooted
    // shape and split structure (its main and aux children's, recursively: the
    // splits, the index tables and every operand follow from them) and of
    // whether the scaled sub lies below it (its 1e-12 reaches every table
    // above it), so two subs with the same signature have equal tables.
    // Children have higher indices and are processed first.
    {
        std::vector<std::string> sig(ns);
        for (int si = ns - 1; si >= 0; --si) {
            const SubTemplate &s = p.subs[si];
            sig[si] = s.size == 1 ? std::string("1")
                                  : "(" + sig[s.main] + "," + sig[s.aux] + ")" + (si == p.scaled_sub ? "s" : "");
        }
        p.same_as.assign(ns, -1);
        std::map<std::string, int> first;
        for (int si : p.process_order) {
            if (si == 0) continue;   // the root has no table
            auto it = first.find(sig[si]);
            if (it == first.end()) first.emplace(sig[si], si);
            else p.same_as[si] = it->second;
        }
    }
    // ---- count-table arena: a table lives from its sub's step to its last
    // reader's (its parent's; for a shared table, the last of its subs'
    // parents).  Rows an aggregation gathers (a parent's aux child) are
    // 32-byte aligned for its 256-bit loads; main-child rows, read element by
    // element, keep 16-byte rows; a shared table takes the wider of its subs'.
    p.table_pitch.assign(ns, 0);
    {
        std::vector<int> need8(ns, 0);
        for (int si : p.process_order) {
            if (si == 0) continue;
            const SubTemplate &s = p.subs[si];
            const int r = p.same_as[si] >= 0 ? p.same_as[si] : si;
            if (s.parent >= 0 && s.parent < ns && p.subs[s.parent].aux == si) need8[r] = 1;
        }
        for (int si : p.process_order) {
            if (si == 0) continue;
            const int r = p.same_as[si] >= 0 ? p.same_as[si] : si;
            const int L = p.subs[si].L;
            p.table_pitch[si] = need8[r] ? (L + 7) / 8 * 8 : (L + 3) / 4 * 4;
        }
    }
    auto plan_arena = [&](bool share, std::vector<int64_t> &offset, int64_t &units) {
        offset.assign(ns, -1);
        std::vector<std::pair<int64_t, int64_t>> freel;   // (offset, length), sorted
        int64_t top = 0;
        auto alloc = [&](int64_t len) {
            for (size_t i = 0; i < freel.size(); ++i)
                if (freel[i].second >= len) {
                    int64_t off = freel[i].first;
                    freel[i].first += len;
                    freel[i].second -= len;
                    if (freel[i].second == 0) freel.erase(freel.begin() + i);
                    return off;
                }
            int64_t off = top;
            top += len;
            return off;
        };
        auto release = [&](int64_t off, int64_t len) {
            freel.push_back({off, len});
            std::sort(freel.begin(), freel.end());
            std::vector<std::pair<int64_t, int64_t>> merged;
            for (auto &f : freel) {
                if (!merged.empty() && merged.back().first + merged.back().second == f.first)
                    merged.back().second += f.second;
                else merged.push_back(f);
            }
            if (!merged.empty() && merged.back().first + merged.back().second == top) {
                top = merged.back().first;
                merged.pop_back();
            }
            freel.swap(merged);
        };
        auto owner = [&](int si) { return share && p.same_as[si] >= 0 ? p.same_as[si] : si; };
        std::vector<int> readers(ns, 0);   // per owning sub: parents still to run
        for (int si : p.process_order)
            if (si != 0) ++readers[owner(si)];
        int64_t peak = 0;
        for (int si : p.process_order) {
            const SubTemplate &s = p.subs[si];
            if (si > 0) {
                // arena slots are whole multiples of 8 units, so every table
                // starts 32-byte aligned for any V
                if (owner(si) != si) offset[si] = offset[owner(si)];
                else offset[si] = alloc((p.table_pitch[si] + 7) / 8 * 8);
                peak = std::max(peak, top);
            }
            for (int c : {s.main, s.aux})
                if (p.subs[c].size > 1 && --readers[owner(c)] == 0)
                    release(offset[owner(c)], (p.table_pitch[c] + 7) / 8 * 8);
        }
        units = peak;
    };
    plan_arena(true, p.table_offset, p.arena_units);
    plan_arena(false, p.table_offset_all, p.arena_units_all);
    p.automorphisms = 1;
    static std::atomic<uint64_t> next_uid{1};
    p.uid = next_uid++;
    return true;
}

}  // namespace sg
