/*
 * Graph.hpp -- drop-in for the reference's template Graph (Graph.hpp:11-66):
 * read_enlist reads "n\nm\nu v\n..." (Graph.cpp:9-80) and build_graph takes
 * the edges directly (Graph.cpp:82-129); either also plans the template
 * (DivideTemplates + IndexSys, sg_plan_read / sg_plan_create), which
 * CountMat::compute then uses.
 */
#ifndef SUBGRAPH_B200_GRAPH_HPP
#define SUBGRAPH_B200_GRAPH_HPP

#include <string>

#include "Helper.hpp"

class Graph {
public:
    Graph() = default;
    Graph(const Graph &) = delete;
    Graph &operator=(const Graph &) = delete;
    ~Graph() { release(); }

    void read_enlist(string file_name)
    {
        release();
        sg_shim::check(sg_plan_read(file_name.c_str(), &plan_), "Graph::read_enlist");
        load_counts();
    }
    void build_graph(int vert, int edge, int *src_edge, int *dst_edge)
    {
        release();
        sg_shim::check(sg_plan_create(vert, edge, src_edge, dst_edge, &plan_), "Graph::build_graph");
        load_counts();
    }

    int get_vert_num() const { return vert_num_; }
    int get_edge_num() const { return vert_num_ > 0 ? vert_num_ - 1 : 0; }   // templates are trees
    void release()
    {
        if (plan_) sg_plan_destroy(plan_);
        plan_ = nullptr;
        vert_num_ = 0;
    }

    // the planned template (library handle; owned by this object)
    sg_plan plan() const { return plan_; }

private:
    void load_counts()
    {
        int32_t k = 0, nsub = 0, scaled = 0;
        int64_t units = 0;
        sg_shim::check(sg_plan_info(plan_, &k, &nsub, &scaled, &units), "Graph");
        vert_num_ = k;
    }
    sg_plan plan_ = nullptr;
    int vert_num_ = 0;
};

#endif
