/*
 * CountMat.hpp -- drop-in for the reference's CountMat (CountMat.hpp:19-191):
 *   initialization(CSRGraph*, CSCGraph<int32_t,float>*, thd_num, itr_num,
 *                  isPruned, useSPMM, vtuneStart, calculate_automorphisms)
 *                  exactly one graph non-null (CountMat.cpp:21-77)
 *   compute(Graph&, isEstimate)  runs itr_num colorings on the GPU, prints the
 *                  reference's report lines ("Time for count per iter",
 *                  "Final raw count is", "Prob is", "Final count is",
 *                  CountMat.cpp:213,251,254,261) and returns the rounded
 *                  estimate (CountMat.cpp:79-266)
 * thd_num and vtuneStart are accepted for interface parity.  Colorings are
 * seeded from time(0) as in the reference unless setSeed() gives a base
 * (coloring c then uses srand(base + c)).  With isPruned=0 on a CSC graph the
 * SpMV buffer carries from one compute() to the next, as the reference's
 * _bufVec does.
 */
#ifndef SUBGRAPH_B200_COUNTMAT_HPP
#define SUBGRAPH_B200_COUNTMAT_HPP

#include <vector>

#include "CSCGraph.hpp"
#include "CSRGraph.hpp"
#include "Graph.hpp"
#include "Helper.hpp"

class CountMat {
public:
    typedef int32_t idxType;
    typedef float valType;

    CountMat() { sg_shim::check(sg_countmat_create(&cm_), "CountMat"); }
    CountMat(const CountMat &) = delete;
    CountMat &operator=(const CountMat &) = delete;
    ~CountMat() { sg_countmat_destroy(cm_); }

    void initialization(CSRGraph *graph, CSCGraph<int32_t, float> *graphCSC, int thd_num, int itr_num,
                        int isPruned, int useSPMM, int vtuneStart = -1, bool calculate_automorphisms = false)
    {
        if ((graph == nullptr) == (graphCSC == nullptr))
            throw sg_error(SG_ERR_INVALID, "CountMat::initialization: exactly one of the CSR and CSC graphs");
        sg_graph csr = graph ? graph->deviceGraph() : nullptr;
        sg_graph csc = graphCSC ? graphCSC->deviceGraph() : nullptr;
        sg_shim::check(sg_countmat_initialization(cm_, csr, csc, thd_num, itr_num, isPruned, useSPMM, vtuneStart,
                                                  calculate_automorphisms ? 1 : 0),
                       "CountMat::initialization");
        itr_num_ = itr_num;
    }

    double compute(Graph &templates, bool isEstimate = false)
    {
        double r = 0.0;
        sg_shim::check(sg_countmat_compute(cm_, templates.plan(), isEstimate ? 1 : 0, 1, &r), "CountMat::compute");
        return r;
    }

    // not in the reference: a fixed seed base, and the per-coloring raw counts
    // of the last compute()
    void setSeed(uint32_t seed_base) { sg_shim::check(sg_countmat_set_seed(cm_, seed_base), "CountMat::setSeed"); }
    std::vector<double> rawCounts()
    {
        std::vector<double> r((size_t)(itr_num_ > 0 ? itr_num_ : 0));
        if (!r.empty()) sg_shim::check(sg_countmat_raw(cm_, r.data()), "CountMat::rawCounts");
        return r;
    }

private:
    sg_countmat cm_ = nullptr;
    int itr_num_ = 0;
};

#endif
