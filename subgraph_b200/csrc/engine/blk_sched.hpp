// Register-blocked eMA: compile-time schedules (plain C++17, shared by the
// host planner and the device code).
//
// A sub s with |s| = N colors, main child of P colors and aux child of
// Qa = N - P colors computes, for every N-set O of colors,
//     out[O] = sum over splits j of main[M_j] * agg[O \ M_j],
// the M_j being the P-subsets of O in lex order (IndexSys.cpp:383-414; the
// complements O \ M_j then come in reverse lex order).  All N-subsets O of
// one (N+1)-set U share their operands: the P-subsets and the Qa-subsets of
// U.  A block keeps one of the two families (the smaller, "held") in
// registers and streams the other once from shared memory, in lex order for
// mains and reverse lex order for aux sets: every output of U then receives
// its terms in exactly its split order, so the sums are bit-identical to the
// per-output loop.  Sets are bit masks over the positions 0..N of U.
#pragma once
#include <cstdint>

namespace sg {
namespace blk {

constexpr int binom(int n, int k)
{
    if (k < 0 || k > n) return 0;
    long long r = 1;
    for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
    return (int)r;
}

// the k-subsets of {0..m-1}, lex order of their sorted position tuples
constexpr void lex_subsets(int m, int k, unsigned *out)
{
    int idx[32] = {};
    for (int i = 0; i < k; ++i) idx[i] = i;
    const int n = binom(m, k);
    for (int c = 0; c < n; ++c) {
        unsigned mask = 0;
        for (int i = 0; i < k; ++i) mask |= 1u << idx[i];
        out[c] = mask;
        int i = k - 1;
        while (i >= 0 && idx[i] == m - k + i) --i;
        if (i < 0) break;
        ++idx[i];
        for (int j = i + 1; j < k; ++j) idx[j] = idx[j - 1] + 1;
    }
}

template <int N, int P> struct Shape {
    static constexpr int M = N + 1;                 // |U|
    static constexpr int Qa = N - P;
    static constexpr bool kHoldMain = binom(M, P) <= binom(M, Qa);
    static constexpr int HS = kHoldMain ? P : Qa;   // held subset size
    static constexpr int TS = N - HS;               // streamed subset size
    static constexpr int NH = binom(M, HS), NS = binom(M, TS), NO = M;
    static constexpr int PER = HS + 1;              // outputs containing one streamed set
    static constexpr int NH4 = (NH + 3) / 4 * 4, NS4 = (NS + 3) / 4 * 4, NO4 = (NO + 3) / 4 * 4;
    static constexpr int ROW = NH4 + NS4 + NO4;     // int32 words of a block's column table
};

template <int N, int P> struct Table {
    using S = Shape<N, P>;
    unsigned held[S::NH] = {};
    unsigned str[S::NS] = {};
    unsigned out[S::NO] = {};
    int po[S::NS][S::PER] = {};   // output slot of the (streamed set, k-th containing output) pair
    int ph[S::NS][S::PER] = {};   // held slot of its other factor
};

template <int N, int P> constexpr Table<N, P> make_table()
{
    using S = Shape<N, P>;
    Table<N, P> t{};
    lex_subsets(S::M, S::HS, t.held);
    unsigned lex[S::NS] = {};
    lex_subsets(S::M, S::TS, lex);
    for (int i = 0; i < S::NS; ++i) t.str[i] = S::kHoldMain ? lex[S::NS - 1 - i] : lex[i];
    lex_subsets(S::M, N, t.out);
    for (int i = 0; i < S::NS; ++i) {
        int c = 0;
        for (int o = 0; o < S::NO; ++o) {
            if ((t.out[o] & t.str[i]) != t.str[i]) continue;
            const unsigned h = t.out[o] & ~t.str[i];
            int hi = -1;
            for (int j = 0; j < S::NH; ++j)
                if (t.held[j] == h) hi = j;
            t.po[i][c] = o;
            t.ph[i][c] = hi;
            ++c;
        }
    }
    return t;
}

template <int N, int P> struct Sched {
    static constexpr Table<N, P> tab = make_table<N, P>();
};

// The shapes with a blocked kernel: (N, P) with N <= 11 and at most 64 held
// values.  P >= 2 for a sub's own split structure (a one-hot main has its own
// path); the P = 1 shapes serve the rooted form, where a stage of shape
// (N + 1, P + 1) is computed per vertex over the other k - 1 colors and its
// main operands (the sets holding the vertex's color) are not one-hot.
// Index 0 means "no blocked path"; shape ids are 1 + the position in this list.
#define SG_BLK_SHAPES_A(X) X(3, 2) X(4, 2) X(4, 3) X(5, 2) X(5, 3) X(5, 4) X(6, 2) X(6, 3)
#define SG_BLK_SHAPES_B(X) X(6, 4) X(6, 5) X(7, 2) X(7, 3) X(7, 4) X(7, 5)
#define SG_BLK_SHAPES_C(X) X(7, 6) X(8, 2) X(8, 6) X(8, 7) X(9, 2) X(9, 7)
#define SG_BLK_SHAPES_D(X) X(9, 8) X(10, 2) X(10, 8) X(10, 9) X(11, 10)
#define SG_BLK_SHAPES_E(X) X(2, 1) X(3, 1) X(4, 1) X(5, 1) X(6, 1) X(7, 1) X(8, 1) X(9, 1) X(10, 1)
#define SG_BLK_SHAPES(X) \
    SG_BLK_SHAPES_A(X) SG_BLK_SHAPES_B(X) SG_BLK_SHAPES_C(X) SG_BLK_SHAPES_D(X) SG_BLK_SHAPES_E(X)

// Runtime view of one shape's schedule (host planner).
struct View {
    int N = 0, P = 0, M = 0, HS = 0, TS = 0, NH = 0, NS = 0, NO = 0, PER = 0, NH4 = 0, NS4 = 0, NO4 = 0, ROW = 0;
    bool hold_main = false;
    const unsigned *held = nullptr, *str = nullptr, *out = nullptr;
    const int *po = nullptr, *ph = nullptr;   // [NS][PER]
};

template <int N, int P> View view_of()
{
    using S = Shape<N, P>;
    const Table<N, P> &t = Sched<N, P>::tab;
    View v;
    v.N = N; v.P = P; v.M = S::M; v.HS = S::HS; v.TS = S::TS; v.NH = S::NH; v.NS = S::NS; v.NO = S::NO;
    v.PER = S::PER; v.NH4 = S::NH4; v.NS4 = S::NS4; v.NO4 = S::NO4; v.ROW = S::ROW; v.hold_main = S::kHoldMain;
    v.held = t.held; v.str = t.str; v.out = t.out;
    v.po = &t.po[0][0]; v.ph = &t.ph[0][0];
    return v;
}

// shape id of (n, p), 0 when there is no blocked kernel for it
inline int shape_id(int n, int p)
{
    int id = 0, k = 0;
#define SG_BLK_ID(NN, PP) ++k; if (n == NN && p == PP) id = k;
    SG_BLK_SHAPES(SG_BLK_ID)
#undef SG_BLK_ID
    return id;
}

inline bool view_by_id(int id, View &v)
{
    int k = 0;
#define SG_BLK_VIEW(NN, PP) if (++k == id) { v = view_of<NN, PP>(); return true; }
    SG_BLK_SHAPES(SG_BLK_VIEW)
#undef SG_BLK_VIEW
    return false;
}

}  // namespace blk
}  // namespace sg
