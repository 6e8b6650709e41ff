/*
 * CSCGraph.hpp -- drop-in for the reference's CSCGraph<idxType, valType>
 * (CSCGraph.hpp:22-90), the graph type CountMat counts on:
 *   createFromEdgeListFile  CSC of the symmetrised adjacency, both directions
 *                           inserted, duplicates kept, rows ascending per
 *                           column (CSCGraph.hpp:95-178; sg_csc_build)
 *   splitCSC                accepted for interface parity (the GPU kernels
 *                           need no row-owner split, CSCGraph.hpp:180-217)
 *   serialize/deserialize   the graph.data layout (CSCGraph.hpp:427-463)
 * Only CSCGraph<int32_t, float> exists, as in the reference's use.  The
 * arrays live in host memory; the first CountMat that counts on the graph
 * uploads them to the GPU.
 */
#ifndef SUBGRAPH_B200_CSCGRAPH_HPP
#define SUBGRAPH_B200_CSCGRAPH_HPP

#include <fstream>
#include <type_traits>
#include <vector>

#include "Helper.hpp"

template <class idxType, class valType> class CSCGraph {
    static_assert(std::is_same<idxType, int32_t>::value && std::is_same<valType, float>::value,
                  "the library provides CSCGraph<int32_t, float>");

public:
    CSCGraph() = default;

    idxType getNumVertices() { return _a.V; }
    idxType getNNZ() { return _a.nnz(); }
    idxType *getIndexRow() { return _a.nbr.p; }
    idxType *getIndexCol() { return _a.off.p; }
    idxType *getDegList() { return _a.deg.p; }
    idxType *getRowIdx(idxType colId) { return _a.nbr.p + _a.off.p[colId]; }
    idxType getColLen(idxType colId) { return _a.off.p[colId + 1] - _a.off.p[colId]; }

    void createFromEdgeListFile(idxType numVerts, idxType numEdges, idxType *srcList, idxType *dstList,
                                bool isBenchmark = false)
    {
        (void)isBenchmark;
        int32_t *col = nullptr, *row = nullptr, *deg = nullptr;
        sg_shim::check(sg_csc_build(numVerts, numEdges, srcList, dstList, &col, &row, &deg),
                       "CSCGraph::createFromEdgeListFile");
        _a.set(numVerts, numEdges, col, row, deg);
    }

    void splitCSC(idxType numsplits) { (void)numsplits; }

    void serialize(ofstream &outputFile)
    {
        const std::string b = _a.encode();
        outputFile.write(b.data(), (std::streamsize)b.size());
    }
    void deserialize(int inputFile) { _a.decode(sg_shim::read_fd(inputFile)); }

    // the device copy of this graph (library handle; owned by the graph)
    sg_graph deviceGraph() { return _a.device_graph(); }

private:
    sg_shim::Adjacency _a;
};

#endif
