// Host-side graph inputs: text edge lists, CSC / CSR construction, the binary
// graph.data format and a seeded R-MAT generator.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace sg {

// An edge list as EdgeList produces it (EdgeList.cpp:34-116): V, then E pairs.
struct EdgeListData {
    int32_t V = 0;
    std::vector<int32_t> src, dst;
};

// Text format "V\nE\nu v\n..." (EdgeList::readfromEdgeList, EdgeList.cpp:34-116),
// including its hole removal when the largest id is not V-1. Returns false
// with a message on I/O or format errors.
bool read_edge_list(const std::string &path, EdgeListData &out, std::string &err);
bool write_edge_list(const std::string &path, const EdgeListData &el, std::string &err);

// CSC of the symmetrised adjacency (CSCGraph::createFromEdgeListFile,
// CSCGraph.hpp:95-178): each edge inserted in both directions, duplicates and
// self loops kept, the rows of every column ascending.
struct CSC {
    int32_t V = 0;
    int32_t numEdges = 0;
    std::vector<int32_t> indexCol;  // V+1
    std::vector<int32_t> indexRow;  // nnz
    std::vector<int32_t> degList;   // V
};
bool build_csc(int32_t V, const int32_t *src, const int32_t *dst, int64_t E, CSC &out, std::string &err);

// CSR (CSRGraph::createFromEdgeListFile, CSRGraph.cpp:16-108): the same
// insertion, but neighbours stay in insertion order (no sort).
struct CSR {
    int32_t V = 0;
    int32_t numEdges = 0;
    std::vector<int32_t> indexRow;  // V+1 (row offsets)
    std::vector<int32_t> indexCol;  // nnz (column ids)
    std::vector<int32_t> degList;
};
bool build_csr(int32_t V, const int32_t *src, const int32_t *dst, int64_t E, CSR &out, std::string &err);

// graph.data (CSCGraph::serialize/deserialize, CSCGraph.hpp:427-463): int32
// numEdges, numVertices, degList[V], indexCol[V+1], indexRow[nnz], float
// edgeVal[nnz] (all 1.0).
// The CSR form (CSRGraph::serialize/deserialize, CSRGraph.cpp:236-295) is the
// same layout with row offsets and column ids in place of indexCol/indexRow.
bool write_graph_data(const std::string &path, const CSC &g, std::string &err);
bool read_graph_data(const std::string &path, CSC &g, std::string &err);
// the same bytes in memory (`what` names the source in error messages)
void encode_graph_data(const CSC &g, std::string &buf);
bool decode_graph_data(const char *data, size_t n, const std::string &what, CSC &g, std::string &err);

// Seeded R-MAT / Kronecker generator: E = edge_factor * 2^scale draws with
// initiator (a, b, c, 1-a-b-c), vertex ids scrambled by a seeded permutation,
// self loops dropped, edges canonicalised (min,max), sorted and deduplicated.
// Vertex 2^scale-1 is kept non-isolated so the text file round-trips without
// hole removal.
bool rmat_generate(int scale, int edge_factor, double a, double b, double c, uint64_t seed,
                   EdgeListData &out, std::string &err);

}  // namespace sg
