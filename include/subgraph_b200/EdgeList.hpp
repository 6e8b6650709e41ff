/*
 * EdgeList.hpp -- drop-in for the reference's EdgeList (EdgeList.hpp:19-66):
 * the text edge list "V\nE\nu v\n..." with its hole removal
 * (EdgeList::readfromEdgeList, EdgeList.cpp:34-116), read by sg_edgelist_read.
 */
#ifndef SUBGRAPH_B200_EDGELIST_HPP
#define SUBGRAPH_B200_EDGELIST_HPP

#include "Helper.hpp"

class EdgeList {
public:
    typedef int32_t idxType;

    EdgeList() : _numEdges(-1), _numVertices(-1) {}
    // noVerticesNum != 0 selects the reference's tab-separated reader that
    // writes rmat.txt (EdgeList.cpp:208-282), a conversion tool that is not
    // part of the counting path: it is rejected here.
    explicit EdgeList(string fileName, int noVerticesNum = 0) : _numEdges(-1), _numVertices(-1)
    {
        if (noVerticesNum) throw sg_error(SG_ERR_UNSUPPORTED, "EdgeList: the no-vertex-count reader is not provided");
        int32_t V = 0;
        int64_t E = 0;
        int32_t *s = nullptr, *d = nullptr;
        sg_shim::check(sg_edgelist_read(fileName.c_str(), &V, &E, &s, &d), "EdgeList");
        _src.reset(s);
        _dst.reset(d);
        if (E > INT32_MAX) throw sg_error(SG_ERR_INVALID, "EdgeList: more than 2^31-1 edges");
        _numVertices = V;
        _numEdges = (idxType)E;
    }

    idxType getNumEdges() { return _numEdges; }
    idxType getNumVertices() { return _numVertices; }
    idxType *getSrcList() { return _src.p; }
    idxType *getDstList() { return _dst.p; }

private:
    idxType _numEdges;
    idxType _numVertices;
    sg_shim::LibArray<int32_t> _src, _dst;
};

#endif
