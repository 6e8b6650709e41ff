// Host side of the device engine: device-resident graphs, plans and the
// counting pipelines (plain: launches per coloring and sub; batched: one
// persistent work-queue launch for many colorings).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../host/plan.hpp"
#include "stage.cuh"

namespace sg {

struct Status {
    int code = 0;       // 0 ok; see include/sg_api.h for the codes
    std::string msg;
    static Status ok() { return {}; }
};

// A graph resident on one GPU.  Vertices are relabelled by descending degree
// (ties by id) so that tiles of consecutive vertices have similar work and the
// highest-degree rows share cache lines; each neighbour list keeps the order
// of the input adjacency, which fixes the floating-point summation order.
struct DeviceGraph {
    int device = 0;
    int32_t V = 0;
    int64_t nnz = 0;
    int32_t max_degree = 0;
    int32_t *d_off = nullptr;     // [V+1] internal order
    int32_t *d_adj = nullptr;     // [nnz]
    int32_t *d_perm = nullptr;    // original -> internal
    int32_t *d_iperm = nullptr;   // internal -> original
    std::vector<int32_t> h_degree;   // internal order (descending)
    // coloring jump-ahead tables
    int32_t color_blocks = 0;
    uint32_t *d_jump = nullptr;   // [color_blocks][31]
    uint32_t *d_coef = nullptr;   // [31][1024]
    cudaStream_t stream = nullptr;
    int sm_count = 148;
    ~DeviceGraph();
};

struct CountOptions {
    int32_t n_colorings = 1;
    uint32_t seed_base = 0;
    int32_t mode = kModeReference;
    int32_t batch = 0;              // > 0: colorings per batch (interleaved group); 0: plain
    int32_t persistent = 0;         // batched: one persistent work-queue launch per batch instead
    int32_t hub_threshold = 1024;   // degree above which a vertex is aggregated in chunks; 0 = never
    int32_t profile = 0;            // time every fused launch with CUDA events
    int32_t autotune = 1;           // time the tile-shape candidates of new stage shapes once per graph
    int32_t exact = 0;              // reference operation order everywhere: no hub chunks, no fused products
    int32_t wait_limit_ms = 0;      // batched queue: time a dependency wait may take (0 = 2000 ms)
    int32_t test_unsatisfiable_wait = 0;   // test hook: the first fused stage waits on a counter nothing sets
    int32_t blocked = 1;            // register-blocked eMA where a stage has one (same values)
    int32_t rooted = 1;             // its rooted form where a stage has one (same values)
    int32_t flat = 1;               // flat aggregation over the active chunks where it applies (same values)
    float *orig_state = nullptr;    // mode 2: host [V] aggregation buffer (original vertex order is not
                                    // needed: internal order, opaque to the caller) carried in and out;
                                    // null: start from zeros
};

struct CountStats {
    double device_ms = 0;       // CUDA-event time of the counting launches
    int64_t kernel_launches = 0;
    int64_t table_bytes = 0;    // device bytes of count tables
    double fused_ms = 0;        // profile: summed time of the fused launches
    int64_t fused_launches = 0;
    double fused_alg_bytes = 0; // compulsory bytes of the fused launches
    double fused_gather_bytes = 0;
    double hub_ms = 0;
    int32_t top_sub = -1;       // profile: the sub whose fused launches took the most time
    int64_t top_launches = 0;
    double top_ms = 0, top_alg_bytes = 0;
};

Status graph_create(const int32_t *offsets, const int32_t *neighbors, int32_t V, int64_t nnz, int device,
                    std::unique_ptr<DeviceGraph> &out);
// Frees the device copies of a plan's index tables (kept per device and plan
// for every graph that counts with it); called when the plan is destroyed.
void release_plan_tables(uint64_t uid);

// Pieces of a graph upload shared by the host-array and device-array paths:
// a DeviceGraph with its stream, and the tail that orders the vertices by
// degree (on the device, from the original-order offsets), relabels the
// original-order device adjacency (both freed here) and builds the coloring
// tables.
Status new_device_graph(int device, int32_t V, int64_t nnz, std::unique_ptr<DeviceGraph> &out);
Status graph_finish(DeviceGraph &g, int32_t *d_old_off, int32_t *d_old_adj);
// The degree order of V vertices on the device (engine/input_gpu.cu): iperm =
// the vertices by descending degree, ties by ascending id (a stable radix sort
// on INT32_MAX - degree: the order of a stable counting sort by descending
// degree), perm its inverse, new_off the exclusive sum of the ordered degrees;
// the ordered degrees are copied to the host.
Status degree_order(int32_t V, const int32_t *d_old_off, int32_t *d_iperm, int32_t *d_perm, int32_t *d_new_off,
                    std::vector<int32_t> &h_degree, cudaStream_t st);

// Input preparation on the GPU (engine/input_gpu.cu), each ending in a
// DeviceGraph without a host copy of the adjacency:
//   graph_from_edges   host edge arrays -> CSC of the symmetrised adjacency
//                      (CSCGraph::createFromEdgeListFile semantics) on the GPU
//   graph_from_text    an edge-list text file ("V\nE\nu v\n...", EdgeList.cpp:34-116)
//                      parsed on the GPU, hole removal included
//   graph_from_rmat    an R-MAT graph generated, deduplicated and built on the GPU
// and graph_download_csc: the CSC in original vertex order back to the host.
Status graph_from_edges(int32_t V, const int32_t *src, const int32_t *dst, int64_t E, int device,
                        std::unique_ptr<DeviceGraph> &out);
Status graph_from_text(const std::string &path, int device, std::unique_ptr<DeviceGraph> &out);
Status graph_from_rmat(int scale, int edge_factor, double a, double b, double c, uint64_t seed, int device,
                       std::unique_ptr<DeviceGraph> &out);
Status graph_download_csc(DeviceGraph &g, int32_t *offsets, int32_t *neighbors);

// Runs n_colorings colorings, writes the raw colorful counts (host).
Status count(DeviceGraph &g, const Plan &p, const CountOptions &o, double *raw, CountStats *stats);

// One coloring each of jobs of different templates on one graph (job j:
// plans[j], seeded srand(seeds[j])), run as persistent work-queue launches
// (waves admitted by free memory).  job_ms (optional): per-job latency from
// the start of its wave's launch to the completion of its root stage.
Status count_jobs(DeviceGraph &g, const std::vector<const Plan *> &plans, const uint32_t *seeds,
                  const CountOptions &o, double *raw, double *job_ms, CountStats *stats);

// Parity helpers: colors of one seed (original order), the table of sub s
// after one coloring (column-major [L][V], original order), per-vertex root.
Status debug_colors(DeviceGraph &g, int k, uint32_t seed, int32_t *colors);
Status debug_sub_table(DeviceGraph &g, const Plan &p, uint32_t seed, int mode, int hub_threshold, int s, void *out);
Status debug_root(DeviceGraph &g, const Plan &p, uint32_t seed, int mode, int hub_threshold, double *root, double *raw);

// host-side coloring tables (also used by tests through the C ABI)
void glibc_window(uint32_t seed, uint32_t w[31]);

}  // namespace sg
