// sc-main: the reference's command line (sc-main.cpp:1556-1805), written
// against the C++ drop-in headers (include/subgraph_b200/*.hpp), which carry
// the reference's class names and signatures over the C ABI.  The engine calls
// below are the reference main's own sequence: EdgeList -> CSCGraph (or
// CSRGraph)::createFromEdgeListFile -> splitCSC, or deserialize for
// load_binary; serialize for write_binary; Graph::read_enlist;
// CountMat::initialization; CountMat::compute.
//
//   sc-main graph template iterations threads load_binary write_binary
//           [isPruned useSPMM vtuneStart benchItr]
//
// graph is a text edge list ("V\nE\nu v\n...") or, with load_binary=1, a
// graph.data file; write_binary=1 writes ./graph.data.  The report lines are
// the reference's: "Time for count per iter", "Final raw count is", "Prob is",
// "Final count is".  Counting runs on CUDA device SG_DEVICE (default 0);
// colorings are seeded srand(SG_SEED_BASE + c) when SG_SEED_BASE is set, else
// from time(0) like the reference.  The reference hard-codes the CSC graph
// (useCSC, sc-main.cpp:1576); SG_USE_CSR=1 selects its CSRGraph branch.  The
// reference's unrelated eMA triad benchmark that precedes loading
// (sc-main.cpp:1606) is not run.
#include <fcntl.h>
#include <unistd.h>

#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <string>

#include "subgraph_b200/CountMat.hpp"
#include "subgraph_b200/EdgeList.hpp"

static int run(int argc, char **argv)
{
    const string graph_name = argv[1], template_name = argv[2];
    const int iterations = std::atoi(argv[3]);
    const int comp_thds = std::atoi(argv[4]);
    const int load_binary = std::atoi(argv[5]);
    const int write_binary = std::atoi(argv[6]);
    const int isPruned = argc > 7 ? std::atoi(argv[7]) : 1;
    const int useSPMM = argc > 8 ? std::atoi(argv[8]) : 1;
    const int vtuneStart = argc > 9 ? std::atoi(argv[9]) : -1;
    const bool calculate_automorphism = false;   // sc-main.cpp:1568
    const bool useCSC = !(std::getenv("SG_USE_CSR") && std::atoi(std::getenv("SG_USE_CSR")));
    const bool useMKL = false, useRcm = false;
    if (iterations < 1) {
        std::fprintf(stderr, "sc-main: iterations must be >= 1\n");
        return 2;
    }

    CSRGraph *csrInputG = nullptr;
    CSCGraph<int32_t, float> *cscInputG = nullptr;
    if (!useCSC)
        csrInputG = new CSRGraph();
    else
        cscInputG = new CSCGraph<int32_t, float>();
    Graph input_template;

    std::printf("Start loading datasets\n");
    std::fflush(stdout);
    double startTime = utility::timer();
    if (load_binary) {
        int input_file = open(graph_name.c_str(), O_RDONLY);
        if (input_file < 0) throw sg_error(SG_ERR_IO, "cannot open " + graph_name);
        if (csrInputG != nullptr) {
            csrInputG->deserialize(input_file, useMKL, useRcm);
        } else {
            cscInputG->deserialize(input_file);
            cscInputG->splitCSC(4 * comp_thds);
        }
        close(input_file);
        std::printf("%s Format Total vertices is : %d\n", useCSC ? "CSC" : "CSR",
                    useCSC ? cscInputG->getNumVertices() : csrInputG->getNumVertices());
    } else {
        double iotStart = utility::timer();
        EdgeList elist(graph_name);
        std::cout << "Disk Load Text Data using " << (utility::timer() - iotStart) << " s" << std::endl;
        if (csrInputG != nullptr) {
            csrInputG->createFromEdgeListFile(elist.getNumVertices(), elist.getNumEdges(), elist.getSrcList(),
                                              elist.getDstList(), useMKL, useRcm, false);
        } else {
            cscInputG->createFromEdgeListFile(elist.getNumVertices(), elist.getNumEdges(), elist.getSrcList(),
                                              elist.getDstList(), false);
            cscInputG->splitCSC(4 * comp_thds);
        }
    }
    if (write_binary) {
        ofstream output_file("graph.data", ios::binary);
        if (csrInputG != nullptr)
            csrInputG->serialize(output_file);
        else
            cscInputG->serialize(output_file);
        output_file.close();
        if (!output_file) throw sg_error(SG_ERR_IO, "writing graph.data");
    }
    std::printf("Prepare Datasets using %f secs\n", utility::timer() - startTime);
    std::fflush(stdout);

    input_template.read_enlist(template_name);
    CountMat executor;
    executor.initialization(csrInputG, cscInputG, comp_thds, iterations, isPruned, useSPMM, vtuneStart,
                            calculate_automorphism);
    if (const char *s = std::getenv("SG_SEED_BASE")) executor.setSeed((uint32_t)std::strtoul(s, nullptr, 10));
    executor.compute(input_template, false);

    delete csrInputG;
    delete cscInputG;
    return 0;
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
    try {
        return run(argc, argv);
    } catch (const std::exception &e) {
        std::fprintf(stderr, "sc-main: %s\n", e.what());
        return 1;
    }
}
