// Template planning: the tree template, its division into sub-templates
// (DivideTemplates), the color-set index tables (IndexSys) and the memory plan
// of the count tables.  Pure host code, no CUDA.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace sg {

constexpr int kMaxColors = 16;     // C(16,8) = 12870 columns: split ids fit in uint16
constexpr int kDummy = 93620;      // the reference's DUMMY_VAL (Helper.hpp:7)

// A tree template with adjacency lists in edge-file order (Graph.cpp:82-129).
struct Template {
    int n = 0;
    std::vector<std::pair<int, int>> edges;
    std::vector<std::vector<int>> adj;
    static bool from_edges(int n, const std::vector<std::pair<int, int>> &edges, Template &t, std::string &err);
};

// Graph::read_enlist (Graph.cpp:9-80): "n\nm\nu v\n...".
bool read_template(const std::string &path, Template &t, std::string &err);

struct SubTemplate {
    int size = 0;
    int main = kDummy, aux = kDummy, parent = kDummy;   // indices into Plan::subs
    Template tree;                                      // relabelled subtree, root 0
    // index tables (meaningful when size > 1); lex order i of the color sets
    int L = 0;                          // C(k, size): columns of this sub's table
    int S = 0;                          // C(size, |main|): splits per color set
    std::vector<int32_t> comb_to_count; // [L] lex index -> colex column
    std::vector<int32_t> main_split;    // [L][S] main column per (lex set, split)
    std::vector<int32_t> aux_split;     // [L][S] aux column per (lex set, split)
};

struct Plan {
    uint64_t uid = 0;                    // unique per make_plan call (device-table cache key)
    int k = 0;
    std::vector<SubTemplate> subs;       // DivideTemplates order (after sort_tps)
    std::vector<int> process_order;      // subs of size > 1, in the order the DP runs them
    int scaled_sub = -1;                 // the first non-bottom sub processed (1e-12 scale)
    int automorphisms = 1;

    // Tables computed once: same_as[s] = a sub processed before s whose table
    // equals s's (the same rooted split structure all the way down and the same
    // position relative to the scaled sub), else -1.  Such subs share one table.
    std::vector<int> same_as;

    // count-table arena, in units of "V elements" (a table of pitch P uses P units)
    std::vector<int64_t> table_offset;   // per sub (shared tables at one offset), -1 when the sub has no table
    std::vector<int32_t> table_pitch;    // row pitch (elements): multiple of 8 for aux children, else of 4
    int64_t arena_units = 0;
    // the arena with every sub's table computed and held on its own (the
    // isPruned=0 CSC mode, whose running buffer makes each step's table differ)
    std::vector<int64_t> table_offset_all;
    int64_t arena_units_all = 0;

    int nsub() const { return (int)subs.size(); }
};

// IndexSys tables of a color-set size `size` on k colors with main subsets of
// msz colors (IndexSys.cpp:169-436): comb_to_count[L] (lex index -> colex
// column), main_split / aux_split [L][S] (main column and the complement's aux
// column of the j-th lex msz-subset).
void index_tables(int k, int size, int msz, int &L, int &S, std::vector<int32_t> &comb_to_count,
                  std::vector<int32_t> &main_split, std::vector<int32_t> &aux_split);

// DivideTemplates::DivideTp + sort_tps (DivideTemplates.cpp:6-327) and
// IndexSys::initialization (IndexSys.cpp:9-57, 169-436), then the table plan.
bool make_plan(const Template &t, Plan &p, std::string &err);

// The automorphism count of CountMat::automorphismNum (CountMat.cpp:1498-1572).
int count_automorphisms(const Template &t);

int64_t binom(int n, int k);
int32_t colex_rank(const int *sorted_colors0, int size);   // 0-based colors

}  // namespace sg
