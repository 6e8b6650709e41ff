// ref_harness.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Drives the compiled reference (CountMat, CSCGraph, EdgeList, DivideTemplates,
// IndexSys from the reference's own sources, see build_ref.sh) and writes its
// full-precision intermediate results to a directory, so the oracle
// restatement and the CUDA path can be pinned against them.
//
// Determinism: CountMat::colorInit seeds with srand(time(0) + thread)
// (CountMat.cpp:984).  This file defines time() so that coloring c of a run
// with base seed S sees time() == S + c, and the coloring region runs on one
// OpenMP thread, which makes the reference's coloring the glibc stream of
// srand(S + c).  Every other parallel region runs on `threads` threads.
//
// Usage: ref_oracle <graph.txt> <template> <ncolorings> <seed_base> <threads>
//                   <outdir> [dump_tables] [automorphisms] [isPruned] [useSPMM]
//                   [csr] [light]
//   isPruned, useSPMM: CountMat::initialization's flags (default 1, 1), which
//     select countNonBottomePrunedSPMM / countNonBottomePruned /
//     countNonBottomeOriginal (CountMat.cpp:291-302);
//   csr=1: the graph is a CSRGraph (CSRGraph::createFromEdgeListFile) instead
//     of a CSCGraph;
//   light=1: only raw.txt, times.txt and aut.txt are written (large graphs).
// Writes: outdir/csc_col.i32, csc_row.i32 (or csr_row.i32, csr_col.i32 for
//         csr=1), plan.txt, colors.i32 (ncol x V), raw.txt (one %.17g per
//         coloring), times.txt (seconds of each coloring), tables/s<k>.f32
//         (coloring 0, column-major [L][V], only when dump_tables=1), aut.txt.
// Colorings run in order 0..ncol-1 on one CountMat, as compute() runs them
// (isPruned=0 on a CSC graph carries CountMat::_bufVec from one SpMV to the
// next, across colorings, CountMat.cpp:931); with dump_tables=1 coloring 0 is
// the dumped one.
#include <vector>
#include <algorithm>
#include <string>
#include <fstream>
#include <iostream>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <sys/stat.h>
#include <omp.h>

#define private public
#include "CountMat.hpp"
#include "EdgeList.hpp"
#include "CSRGraph.hpp"
#undef private

static long g_time_base = 0;
extern "C" time_t time(time_t *t)
{
    time_t v = (time_t)g_time_base;
    if (t) *t = v;
    return v;
}

static void write_bin(const std::string &path, const void *p, size_t bytes)
{
    FILE *f = fopen(path.c_str(), "wb");
    if (!f) { perror(path.c_str()); exit(3); }
    if (bytes) fwrite(p, 1, bytes, f);
    fclose(f);
}

// One coloring: colorCounting (CountMat.cpp:268-322) step by step, with the
// reference's own per-step functions, so that (i) the coloring runs on one
// OpenMP thread (deterministic glibc stream) while every other parallel region
// -- several use omp_get_max_threads(), e.g. the SpMM transposes at
// CountMat.cpp:699-730 -- runs on `thds` threads, and (ii) with `dump` every
// sub-template table can be copied out right after it is computed (its parent
// later overwrites it in place with the aggregation).  The per-sub
// "Mem utilization" report line and its /proc read are left out.
static double counting(CountMat &cm, const std::string &dir, bool dump, int thds)
{
    omp_set_num_threads(1);
    cm.colorInit();
    omp_set_num_threads(thds);
    double countTotal = 0.0;
    cm._isScaled = 0;
    int V = cm._vert_num;
    for (int s = cm._total_sub_num - 1; s >= 0; --s) {
        int subSize = cm._subtmp_array[s].get_vert_num();
        int mainIdx = cm.div_tp.get_main_node_idx(s);
        int auxIdx = cm.div_tp.get_aux_node_idx(s);
        cm._dTable.initSubTempTable(s, mainIdx, auxIdx);
        int *idxCombToCount = (cm.indexer.getSubCToCount())[s];
        if (subSize == 1)
            cm._dTable.countCurBottom(idxCombToCount, cm._colors_local);
        else if (cm._isPruned == 1)
            countTotal = cm._useSPMM == 1 ? cm.countNonBottomePrunedSPMM(s) : cm.countNonBottomePruned(s);
        else
            countTotal = cm.countNonBottomeOriginal(s);
        if (dump && s > 0 && (subSize > 1 || s == cm._total_sub_num - 1)) {
            int L = cm._dTable.getTableLen(s);
            std::vector<float> buf((size_t)L * V);
            for (int c = 0; c < L; ++c)
                std::memcpy(&buf[(size_t)c * V], cm._dTable.getCurTableArray(c), sizeof(float) * V);
            write_bin(dir + "/tables/s" + std::to_string(s) + ".f32", buf.data(), buf.size() * sizeof(float));
        }
        if (mainIdx != DUMMY_VAL) cm._dTable.cleanSubTempTable(mainIdx, false);
        if (auxIdx != DUMMY_VAL) cm._dTable.cleanSubTempTable(auxIdx, false);
    }
    return countTotal;
}

int main(int argc, char **argv)
{
    if (argc < 7) {
        fprintf(stderr, "usage: %s graph template ncol seed_base threads outdir [dump_tables] [aut]\n", argv[0]);
        return 2;
    }
    std::string graph = argv[1], tmpl = argv[2], dir = argv[6];
    int ncol = atoi(argv[3]);
    long seed = atol(argv[4]);
    int thds = atoi(argv[5]);
    int dump_tables = argc > 7 ? atoi(argv[7]) : 0;
    int want_aut = argc > 8 ? atoi(argv[8]) : 0;
    int is_pruned = argc > 9 ? atoi(argv[9]) : 1;
    int use_spmm = argc > 10 ? atoi(argv[10]) : 1;
    int use_csr = argc > 11 ? atoi(argv[11]) : 0;
    int light = argc > 12 ? atoi(argv[12]) : 0;
    mkdir(dir.c_str(), 0755);
    mkdir((dir + "/tables").c_str(), 0755);

    EdgeList elist(graph);
    CSCGraph<int32_t, float> csc;
    CSRGraph csr;
    int V = 0, nnz = 0;
    if (use_csr) {
        csr.createFromEdgeListFile(elist.getNumVertices(), elist.getNumEdges(), elist.getSrcList(), elist.getDstList(),
                                   false, false, false);
        V = csr.getNumVertices();
        nnz = csr.getNNZ();
        if (!light) {
            write_bin(dir + "/csr_row.i32", csr.getIndexRow(), sizeof(int32_t) * (V + 1));
            write_bin(dir + "/csr_col.i32", csr.getIndexCol(), sizeof(int32_t) * (size_t)nnz);
        }
    } else {
        csc.createFromEdgeListFile(elist.getNumVertices(), elist.getNumEdges(), elist.getSrcList(), elist.getDstList(),
                                   false);
        csc.splitCSC(4 * thds);
        V = csc.getNumVertices();
        nnz = csc.getNNZ();
        if (!light) {
            write_bin(dir + "/csc_col.i32", csc.getIndexCol(), sizeof(int32_t) * (V + 1));
            write_bin(dir + "/csc_row.i32", csc.getIndexRow(), sizeof(int32_t) * (size_t)nnz);
        }
    }

    Graph input_template;
    input_template.read_enlist(tmpl);

    omp_set_num_threads(thds);
    CountMat cm;
    cm.initialization(use_csr ? &csr : nullptr, use_csr ? nullptr : &csc, thds, ncol, is_pruned, use_spmm, -1, false);

    // CountMat::compute setup (CountMat.cpp:82-125, 174-197)
    cm._templates = &input_template;
    cm._color_num = input_template.get_vert_num();
    cm.div_tp.DivideTp(input_template);
    cm.div_tp.sort_tps();
    cm._subtmp_array = cm.div_tp.get_subtps();
    cm._total_sub_num = cm.div_tp.get_subtps_num();
    cm.indexer.initialization(cm._color_num, cm._total_sub_num, &cm._subtmp_array, &cm.div_tp);
    cm._dTable.initDataTable(cm._subtmp_array, &cm.indexer, cm._total_sub_num, cm._color_num, V, thds, 1, cm._bufMatCols);
    int k = cm._color_num;
    // as CountMat::compute allocates it (CountMat.cpp:174-197), so that the
    // destructor's frees match
    cm._bufVecLeaf = (float **)malloc(k * sizeof(float *));
    if (use_spmm == 0) {
        for (int i = 0; i < k; ++i) cm._bufVecLeaf[i] = (float *)aligned_alloc(64, ((size_t)V * sizeof(float) + 63) / 64 * 64);
    } else {
        cm._bufVecLeaf[0] = (float *)aligned_alloc(64, ((size_t)V * k * sizeof(float) + 63) / 64 * 64);
        for (int i = 1; i < k; ++i) cm._bufVecLeaf[i] = cm._bufVecLeaf[0] + (size_t)i * V;
    }

    // plan: one line per sub, then its tables
    if (!light) {
        FILE *f = fopen((dir + "/plan.txt").c_str(), "w");
        int n = cm._total_sub_num;
        fprintf(f, "k %d nsub %d V %d nnz %d\n", k, n, V, nnz);
        int **comb = cm.indexer.getCombTable();
        for (int s = 0; s < n; ++s) {
            int sz = cm._subtmp_array[s].get_vert_num();
            int m = cm.div_tp.get_main_node_idx(s), a = cm.div_tp.get_aux_node_idx(s);
            int par = cm.div_tp.parents[s];
            int L = comb[k][sz];
            int S = sz > 1 ? comb[sz][cm.indexer.getSubsSize()[m]] : 0;
            fprintf(f, "sub %d size %d main %d aux %d parent %d L %d S %d\n", s, sz, m, a, par, L, S);
            int *c2c = cm.indexer.getCombToCountTable()[s];
            fprintf(f, "c2c");
            for (int i = 0; i < L; ++i) fprintf(f, " %d", c2c[i]);
            fprintf(f, "\n");
            if (sz > 1) {
                int **ms = cm.indexer.getSplitToCountTable()[0][s];
                int **as = cm.indexer.getSplitToCountTable()[1][s];
                fprintf(f, "msplit");
                for (int i = 0; i < L; ++i) for (int j = 0; j < S; ++j) fprintf(f, " %d", ms[i][j]);
                fprintf(f, "\nasplit");
                for (int i = 0; i < L; ++i) for (int j = 0; j < S; ++j) fprintf(f, " %d", as[i][j]);
                fprintf(f, "\n");
            }
        }
        fclose(f);
    }

    std::vector<int32_t> colors(light ? 0 : (size_t)ncol * V);
    FILE *fr = fopen((dir + "/raw.txt").c_str(), "w");
    FILE *ft = fopen((dir + "/times.txt").c_str(), "w");
    for (int c = 0; c < ncol; ++c) {
        g_time_base = seed + c;
        const double t0 = omp_get_wtime();
        const bool dump = c == 0 && dump_tables;
        const double raw = counting(cm, dir, dump, thds);
        if (dump) {
            FILE *f = fopen((dir + "/raw_dump.txt").c_str(), "w");
            fprintf(f, "%.17g\n", raw);
            fclose(f);
        }
        const double t1 = omp_get_wtime();
        if (!light) std::memcpy(&colors[(size_t)c * V], cm._colors_local, sizeof(int32_t) * V);
        fprintf(fr, "%.17g\n", raw);
        fprintf(ft, "%.9f\n", t1 - t0);
        fflush(fr);
        fflush(ft);
    }
    fclose(fr);
    fclose(ft);
    if (!light) write_bin(dir + "/colors.i32", colors.data(), colors.size() * sizeof(int32_t));
    {
        FILE *f = fopen((dir + "/aut.txt").c_str(), "w");
        fprintf(f, "%d\n", want_aut ? cm.automorphismNum() : 1);
        fclose(f);
    }
    // estimate as CountMat::compute prints it (CountMat.cpp:246-264)
    return 0;
}
