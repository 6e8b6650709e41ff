/*
 * CSRGraph.hpp -- drop-in for the reference's CSRGraph (CSRGraph.hpp:20-146):
 *   createFromEdgeListFile  row offsets and neighbours in edge-file insertion
 *                           order, both directions (CSRGraph.cpp:16-108;
 *                           sg_csr_build).  useMKL / useRcm are accepted and
 *                           ignored: MKL and the SpMP reordering are not part
 *                           of this library, and the reference's -DNEC build
 *                           compiles both out.
 *   serialize/deserialize   CSRGraph.cpp:236-295 (the graph.data layout with
 *                           row offsets and column ids)
 * CountMat counts on it with the CSR semantics of the reference
 * (SpMVNaiveFull neighbour order, CSRGraph.cpp:190-208).
 */
#ifndef SUBGRAPH_B200_CSRGRAPH_HPP
#define SUBGRAPH_B200_CSRGRAPH_HPP

#include <fstream>

#include "Helper.hpp"

class CSRGraph {
public:
    typedef int32_t idxType;
    typedef float valType;

    CSRGraph() = default;

    idxType getNumVertices() { return _a.V; }
    idxType getNNZ() { return _a.nnz(); }
    idxType *getIndexRow() { return _a.off.p; }
    idxType *getIndexCol() { return _a.nbr.p; }
    idxType *getDegList() { return _a.deg.p; }
    idxType *getColIdx(idxType rowId) { return _a.nbr.p + _a.off.p[rowId]; }
    idxType getRowLen(idxType rowId) { return _a.off.p[rowId + 1] - _a.off.p[rowId]; }
    bool useMKL() { return false; }

    void createFromEdgeListFile(idxType numVerts, idxType numEdges, idxType *srcList, idxType *dstList,
                                bool useMKL = false, bool useRcm = false, bool isBenchmark = false)
    {
        (void)useMKL;
        (void)useRcm;
        (void)isBenchmark;
        int32_t *row = nullptr, *col = nullptr, *deg = nullptr;
        sg_shim::check(sg_csr_build(numVerts, numEdges, srcList, dstList, &row, &col, &deg),
                       "CSRGraph::createFromEdgeListFile");
        _a.set(numVerts, numEdges, row, col, deg);
    }

    void serialize(ofstream &outputFile)
    {
        const std::string b = _a.encode();
        outputFile.write(b.data(), (std::streamsize)b.size());
    }
    void deserialize(int inputFile, bool useMKL = false, bool useRcm = false)
    {
        (void)useMKL;
        (void)useRcm;
        _a.decode(sg_shim::read_fd(inputFile));
    }

    sg_graph deviceGraph() { return _a.device_graph(); }

private:
    sg_shim::Adjacency _a;
};

#endif
