// sc-main: the reference's command line (sc-main.cpp:1556-1805) over the C ABI.
//
//   sc-main graph template iterations threads load_binary write_binary
//           [isPruned useSPMM vtuneStart benchItr]
//
// graph is a text edge list ("V\nE\nu v\n...") or, with load_binary=1, a
// graph.data file; write_binary=1 writes ./graph.data.  The report lines are
// the reference's: "Time for count per iter", "Final raw count is", "Prob is",
// "Final count is".  Counting runs on CUDA device SG_DEVICE (default 0);
// colorings are seeded srand(SG_SEED_BASE + c) when SG_SEED_BASE is set, else
// from time(0) like the reference.  The reference's unrelated eMA triad
// benchmark that precedes loading (sc-main.cpp:1606) is not run.
#include <sys/time.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "sg_api.h"

static double now()
{
    struct timeval tp;
    gettimeofday(&tp, nullptr);
    return (double)tp.tv_sec + 1e-6 * (double)tp.tv_usec;
}

static int die(const char *what)
{
    std::fprintf(stderr, "sc-main: %s: %s\n", what, sg_last_error());
    return 1;
}

int main(int argc, char **argv)
{
    if (argc < 7) {
        std::fprintf(stderr,
                     "usage: %s graph template iterations threads load_binary write_binary "
                     "[isPruned useSPMM vtuneStart benchItr]\n",
                     argv[0]);
        return 2;
    }
    const std::string graph_name = argv[1], template_name = argv[2];
    const int iterations = std::atoi(argv[3]);
    const int comp_thds = std::atoi(argv[4]);
    const int load_binary = std::atoi(argv[5]);
    const int write_binary = std::atoi(argv[6]);
    const int isPruned = argc > 7 ? std::atoi(argv[7]) : 1;
    const int useSPMM = argc > 8 ? std::atoi(argv[8]) : 1;
    const int vtuneStart = argc > 9 ? std::atoi(argv[9]) : -1;
    const bool calculate_automorphism = false;   // sc-main.cpp:1568
    const int device = std::getenv("SG_DEVICE") ? std::atoi(std::getenv("SG_DEVICE")) : 0;
    if (iterations < 1) {
        std::fprintf(stderr, "sc-main: iterations must be >= 1\n");
        return 2;
    }

    std::printf("Start loading datasets\n");
    std::fflush(stdout);
    double start = now();
    int32_t V = 0, numEdges = 0;
    int32_t *indexCol = nullptr, *indexRow = nullptr, *degList = nullptr;
    if (load_binary) {
        if (sg_graph_data_read(graph_name.c_str(), &V, &numEdges, &indexCol, &indexRow, &degList) != SG_OK)
            return die("loading graph.data");
        std::printf("CSC Format Total vertices is : %d\n", V);
        std::printf("CSC Format Total Edges is : %d\n", numEdges);
    } else {
        int64_t E = 0;
        int32_t *src = nullptr, *dst = nullptr;
        std::printf("File name: %s\n", graph_name.c_str());
        if (sg_edgelist_read(graph_name.c_str(), &V, &E, &src, &dst) != SG_OK) return die("reading the edge list");
        std::printf("Vert: %d, Edge: %lld\n", V, (long long)E);
        if (sg_csc_build(V, E, src, dst, &indexCol, &indexRow, &degList) != SG_OK) return die("building the CSC");
        numEdges = (int32_t)E;
        sg_free(src);
        sg_free(dst);
    }
    if (write_binary && sg_graph_data_write("graph.data", V, numEdges, indexCol, indexRow, degList) != SG_OK)
        return die("writing graph.data");
    std::printf("Prepare Datasets using %f secs\n", now() - start);
    std::fflush(stdout);

    sg_plan tmpl = nullptr;
    if (sg_plan_read(template_name.c_str(), &tmpl) != SG_OK) return die("reading the template");
    sg_graph g = nullptr;
    if (sg_graph_create(indexCol, indexRow, V, (int64_t)indexCol[V], device, &g) != SG_OK)
        return die("uploading the graph");
    sg_countmat cm = nullptr;
    sg_countmat_create(&cm);
    if (sg_countmat_initialization(cm, nullptr, g, comp_thds, iterations, isPruned, useSPMM, vtuneStart,
                                   calculate_automorphism ? 1 : 0) != SG_OK)
        return die("initialising the counter");
    if (const char *s = std::getenv("SG_SEED_BASE")) sg_countmat_set_seed(cm, (uint32_t)std::strtoul(s, nullptr, 10));
    double result = 0.0;
    if (sg_countmat_compute(cm, tmpl, 0, 1, &result) != SG_OK) return die("counting");
    sg_countmat_destroy(cm);
    sg_graph_destroy(g);
    sg_plan_destroy(tmpl);
    sg_free(indexCol);
    sg_free(indexRow);
    sg_free(degList);
    return 0;
}
