/*
 * sg_api.h -- C ABI of subgraph_b200, a B200 (sm_100a) implementation of
 * dsc-nec/subgraph's color-coding tree-template counting engine.
 *
 * Conventions
 *   - Every call returns sg_status (SG_OK = 0); sg_last_error() gives the
 *     message of the last failure on the calling thread.  No exception crosses
 *     the ABI.
 *   - Pointers in the signatures are HOST pointers.  Arrays returned by the
 *     library (sg_edgelist_read, ...) are malloc'd and released with sg_free.
 *   - Device memory is owned by the library (per sg_graph).  A graph handle is
 *     used by one host thread at a time.
 *   - Vertex ids, offsets and neighbour counts are int32 like the reference's
 *     idxType (CountMat.hpp:24); nnz <= 2^31-1.
 *
 * Each declaration names the reference interface it replaces (file:line in
 * the dsc-nec/subgraph tree).
 */
#ifndef SG_API_H
#define SG_API_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t sg_status;
#define SG_OK 0
#define SG_ERR_INVALID 1      /* bad argument, malformed input file */
#define SG_ERR_OOM 2          /* device or host allocation failed / over budget */
#define SG_ERR_CUDA 3         /* CUDA runtime error */
#define SG_ERR_TIMEOUT 4      /* a bounded device wait gave up */
#define SG_ERR_IO 5           /* file could not be read or written */
#define SG_ERR_UNSUPPORTED 6  /* shape or option not supported */

typedef struct sg_graph_s *sg_graph;   /* device-resident adjacency */
typedef struct sg_plan_s *sg_plan;     /* template + sub-templates + index tables */
typedef struct sg_countmat_s *sg_countmat;

/* count modes */
#define SG_MODE_REFERENCE 0   /* FP32 tables, the reference's arithmetic (isPruned=1) */
#define SG_MODE_FP64 1        /* FP64 tables, no scaling: high-precision oracle mode */
/* isPruned=0 (CountMat::countNonBottomeOriginal, CountMat.cpp:851-977): FP32,
 * no 1e-12 scaling, FP32 root buffer, one SpMV per (output, split) pair.  On
 * the reference's CSC graph the SpMV adds onto CountMat::_bufVec, which is
 * zeroed only at initialization, so the aggregate accumulates over every
 * split, sub-template and coloring of the run (CountMat.cpp:52-59, 931;
 * CSCGraph.hpp:219-239): SG_MODE_ORIGINAL reproduces that, each sg_count
 * call starting from a zero buffer (a fresh CountMat) and running its
 * colorings one after another whatever `batch` says.  On a CSRGraph the SpMV
 * overwrites its output (CSRGraph::SpMVNaiveFull, CSRGraph.cpp:190-208):
 * SG_MODE_ORIGINAL_CSR, a fresh aggregation for every split. */
#define SG_MODE_ORIGINAL 2
#define SG_MODE_ORIGINAL_CSR 3

const char *sg_last_error(void);
const char *sg_version(void);
void sg_free(void *p);

/* ---- host-side inputs (no GPU needed) --------------------------------- */

/* EdgeList::EdgeList(fileName) / readfromEdgeList (EdgeList.hpp:28-36,
 * EdgeList.cpp:34-116): "V\nE\nu v\n..." with hole removal. */
sg_status sg_edgelist_read(const char *path, int32_t *V, int64_t *E, int32_t **src, int32_t **dst);
sg_status sg_edgelist_write(const char *path, int32_t V, int64_t E, const int32_t *src, const int32_t *dst);

/* CSCGraph::createFromEdgeListFile (CSCGraph.hpp:64-65, 95-178).
 * indexCol[V+1], indexRow[2E], degList[V] are malloc'd by the library. */
sg_status sg_csc_build(int32_t V, int64_t E, const int32_t *src, const int32_t *dst,
                       int32_t **indexCol, int32_t **indexRow, int32_t **degList);

/* CSRGraph::createFromEdgeListFile (CSRGraph.hpp:112-113, CSRGraph.cpp:16-108):
 * row offsets indexRow[V+1], neighbours indexCol[2E] in insertion order. */
sg_status sg_csr_build(int32_t V, int64_t E, const int32_t *src, const int32_t *dst,
                       int32_t **indexRow, int32_t **indexCol, int32_t **degList);

/* CSCGraph::serialize / deserialize (CSCGraph.hpp:71-72, 427-463): graph.data */
sg_status sg_graph_data_write(const char *path, int32_t V, int32_t numEdges, const int32_t *indexCol,
                              const int32_t *indexRow, const int32_t *degList);
sg_status sg_graph_data_read(const char *path, int32_t *V, int32_t *numEdges, int32_t **indexCol,
                             int32_t **indexRow, int32_t **degList);
/* The same bytes in memory, for callers that hold the stream or descriptor
 * themselves (CSCGraph::serialize(ofstream&), deserialize(int fd),
 * CSCGraph.hpp:71-72; CSRGraph::serialize/deserialize, CSRGraph.cpp:236-295,
 * whose layout is the same with row offsets and column ids): *buf is
 * malloc'd (release with sg_free). */
sg_status sg_graph_data_encode(int32_t V, int32_t numEdges, const int32_t *offsets, const int32_t *neighbors,
                               const int32_t *degList, void **buf, int64_t *bytes);
sg_status sg_graph_data_decode(const void *buf, int64_t bytes, int32_t *V, int32_t *numEdges, int32_t **offsets,
                               int32_t **neighbors, int32_t **degList);

/* Synthetic input: seeded R-MAT (no reference counterpart in the product; the
 * reference's inputs come from graph500's make_graph, make_graph.h:21-35). */
sg_status sg_rmat_generate(int32_t scale, int32_t edge_factor, double a, double b, double c, uint64_t seed,
                           int32_t *V, int64_t *E, int32_t **src, int32_t **dst);

/* ---- template planning (no GPU needed) ---------------------------------- */

/* Graph::read_enlist (Graph.hpp:29) + DivideTemplates::DivideTp/sort_tps
 * (DivideTemplates.hpp:21-23) + IndexSys::initialization (IndexSys.hpp:31). */
sg_status sg_plan_create(int32_t n, int32_t m, const int32_t *src, const int32_t *dst, sg_plan *out);
sg_status sg_plan_read(const char *template_path, sg_plan *out);
void sg_plan_destroy(sg_plan p);
/* k, number of subs, the scaled sub, arena size in units of V elements */
sg_status sg_plan_info(sg_plan p, int32_t *k, int32_t *nsub, int32_t *scaled_sub, int64_t *arena_units);
/* per sub: size, main, aux, parent (93620 = none, DivideTemplates.hpp:26-29),
 * L = C(k,size), S = C(size,|main|), table pitch (DataTableColMajor.hpp:27-35) */
sg_status sg_plan_sub(sg_plan p, int32_t s, int32_t info[7]);
/* IndexSys tables of sub s (IndexSys.hpp:35-39): c2c[L], msplit[L*S], asplit[L*S] */
sg_status sg_plan_tables(sg_plan p, int32_t s, int32_t *c2c, int32_t *msplit, int32_t *asplit);
/* CountMat::automorphismNum (CountMat.hpp:110) */
sg_status sg_plan_automorphisms(sg_plan p, int32_t *count);
/* the edges of sub s's relabelled subtree (DivideTemplates::get_subtps) */
sg_status sg_plan_sub_edges(sg_plan p, int32_t s, int32_t *n, int32_t *src, int32_t *dst);
/* Tables computed once (no counterpart in the reference, which computes every
 * sub): same_as[s] (nsub entries) = the sub processed before s whose table
 * equals s's -- the same rooted split structure below it and the same
 * position relative to the 1e-12-scaled sub -- so s reuses that table and is
 * not computed again; -1 when s computes its own (every sub in the isPruned=0
 * CSC mode, whose running buffer makes each step's table its own). */
sg_status sg_plan_shared_tables(sg_plan p, int32_t *same_as);

/* ---- device graph -------------------------------------------------------- */

/* Uploads an adjacency given per vertex in summation order: a CSC
 * (indexCol, indexRow) as CountMat uses it (CountMat.hpp:32, CountMat.cpp:
 * 686-735) or a CSR (indexRow, indexCol) for the CSRGraph path. */
sg_status sg_graph_create(const int32_t *offsets, const int32_t *neighbors, int32_t V, int64_t nnz,
                          int32_t device, sg_graph *out);

/* Input preparation on the GPU, each ending in a graph handle without a host
 * copy of the adjacency:
 *  - sg_graph_create_edges: CSC of the symmetrised adjacency of host edge
 *    arrays built on the GPU (CSCGraph::createFromEdgeListFile,
 *    CSCGraph.hpp:95-178: both directions, duplicates and self loops kept,
 *    rows of every column ascending);
 *  - sg_graph_create_text: an edge-list text file ("V\nE\nu v\n...",
 *    EdgeList::readfromEdgeList, EdgeList.cpp:34-116) parsed on the GPU, hole
 *    removal included; every edge line must contain a space (the field before
 *    it is u, the rest of the line v), other lines are an error;
 *  - sg_graph_create_rmat: an R-MAT graph (initiator a, b, c, 1-a-b-c,
 *    edge_factor * 2^scale draws) generated, deduplicated and built on the
 *    GPU from counter-based SplitMix64 draws (the same seed gives the same
 *    graph; a different stream from sg_rmat_generate's);
 *  - sg_graph_download_csc: the CSC of a graph in original vertex order
 *    (offsets[V+1], neighbors[nnz]), e.g. to write graph.data. */
sg_status sg_graph_create_edges(int32_t V, const int32_t *src, const int32_t *dst, int64_t E, int32_t device,
                                sg_graph *out);
sg_status sg_graph_create_text(const char *path, int32_t device, sg_graph *out);
sg_status sg_graph_create_rmat(int32_t scale, int32_t edge_factor, double a, double b, double c, uint64_t seed,
                               int32_t device, sg_graph *out);
sg_status sg_graph_download_csc(sg_graph g, int32_t *offsets, int32_t *neighbors);
void sg_graph_destroy(sg_graph g);
sg_status sg_graph_info(sg_graph g, int32_t *V, int64_t *nnz, int32_t *max_degree);

/* ---- counting ------------------------------------------------------------- */

typedef struct {
    int32_t n_colorings;    /* iterations (CountMat::initialization itr_num) */
    uint32_t seed_base;     /* coloring c uses srand(seed_base + c) */
    int32_t mode;           /* SG_MODE_* */
    int32_t batch;          /* > 0: colorings per batch (batched form); 0: plain */
    int32_t hub_threshold;  /* degree above which aggregation is chunked; 0 = never
                               (exact reference arithmetic for every vertex) */
    int32_t profile;        /* != 0: time every fused launch with CUDA events */
    int32_t no_autotune;    /* != 0: use the default tile shapes instead of timing the
                               candidates of each new stage shape once per graph */
    int32_t exact;          /* != 0: the reference's FP32 operations in the reference's
                               order for every vertex and product (no fused multiply-add,
                               no hub chunking): per-vertex values bit-identical to the
                               reference; otherwise products may be fused (one rounding).
                               Hub neighbour lists are summed in the reference's order in
                               the plain and grouped forms either way; the persistent form
                               sums them in chunks unless exact is set */
    int32_t wait_limit_ms;  /* batched form: how long a work item may wait for its inputs
                               before the call fails with SG_ERR_TIMEOUT (0 = 2000 ms) */
    int32_t no_blocked;     /* 1: no register-blocked eMA (every output computed by its
                               own split loop); the two forms give identical values */
    int32_t persistent;     /* batched form: 1 = one persistent work-queue launch per batch
                               (colorings in separate table slots); 0 = interleaved groups
                               (the batch's colorings share table rows and neighbour passes) */
    int32_t no_rooted;      /* 1: no rooted form of the register-blocked eMA (a vertex of color c
                               computes only the outputs and products whose sets hold c, over
                               the other k-1 colors); the two give identical values */
    int32_t no_flat;        /* 1: no flat aggregation (the tile's vertices each take a fixed group
                               of threads, which also walk the column chunks no output of the
                               vertex reads); the two give identical values */
} sg_count_opts;

typedef struct {
    double device_ms;        /* CUDA-event time of the counting launches */
    int64_t kernel_launches; /* kernels launched by the call */
    int64_t table_bytes;     /* device bytes of count tables */
    /* with profile != 0: the fused aggregation+eMA launches */
    double fused_ms;         /* summed CUDA-event time of the fused launches */
    int64_t fused_launches;
    double fused_alg_bytes;  /* compulsory bytes of those launches: every input table
                                read once, the output written once, the adjacency once */
    double fused_gather_bytes; /* neighbour-row bytes the aggregation reads (4*nnz*L_a) */
    double hub_ms;           /* summed time of the hub aggregation launches */
    /* with profile != 0: the sub-template whose fused launches took the most
       time (the dominant kernel), its launches, summed time and compulsory bytes */
    int32_t top_sub;
    int64_t top_launches;
    double top_ms;
    double top_alg_bytes;
} sg_count_stats;

void sg_count_opts_default(sg_count_opts *o);

/* CountMat::colorCounting per coloring (CountMat.cpp:268-322): raw colorful
 * counts, one per coloring, into raw[n_colorings] (host).  Graphs of 2^28 or
 * more vertices are rejected (SG_ERR_INVALID): neighbour ids carry their
 * color in the top 4 bits of a 32-bit word. */
sg_status sg_count(sg_graph g, sg_plan p, const sg_count_opts *o, double *raw, sg_count_stats *stats);

/* A stream of jobs with different templates on one graph: job j counts one
 * coloring of plans[j] seeded srand(seeds[j]) into raw[j].  Default form: the
 * jobs' stage launches (those of sg_count) are spread over opts.batch CUDA
 * streams (0: 8; fewer when device memory is short), each stream with its own
 * table slot, so the launches of different jobs overlap.  opts.persistent = 1:
 * the jobs run as persistent work-queue launches instead (all their
 * sub-template stages in one queue, waves admitted by free device memory).
 * From opts also: mode, hub_threshold, exact, wait_limit_ms, no_autotune,
 * no_blocked.  job_ms (optional, n_jobs): each job's latency from the start of
 * the call's launches (stream form) or of its wave's launch (persistent form)
 * to the end of its last stage.  The reference
 * runs one template per CountMat::compute (CountMat.cpp:79-266); this is the
 * batched mixed-template form with no single counterpart there. */
sg_status sg_count_jobs(sg_graph g, int32_t n_jobs, const sg_plan *plans, const uint32_t *seeds,
                        const sg_count_opts *opts, double *raw, double *job_ms, sg_count_stats *stats);

/* CountMat::compute's final estimate (CountMat.cpp:246-264):
 * floor(mean(raw) / (k!/k^k * automorphisms) + 0.5). */
sg_status sg_estimate(const double *raw, int32_t n, int32_t k, int32_t automorphisms, double *out);

/* ---- parity helpers ------------------------------------------------------- */

/* CountMat::colorInit on one thread (CountMat.cpp:979-991): colors[V] in
 * original vertex order. */
sg_status sg_colors(sg_graph g, int32_t k, uint32_t seed, int32_t *colors);
/* the count table of sub s after one coloring (DataTableColMajor columns,
 * column-major [L][V], original order; float or double by mode) */
sg_status sg_debug_sub_table(sg_graph g, sg_plan p, uint32_t seed, int32_t mode, int32_t hub_threshold,
                             int32_t s, void *out);
/* per-vertex root values (bufLastSub, CountMat.cpp:815-831) and their sum */
sg_status sg_debug_root(sg_graph g, sg_plan p, uint32_t seed, int32_t mode, int32_t hub_threshold,
                        double *root, double *raw);
/* Test of the bounded waits (no counterpart in the reference): sg_count in the
 * persistent batched form (opts->batch colorings per batch) with one extra
 * dependency of the first fused stage on a counter that nothing increments,
 * so the call must end with SG_ERR_TIMEOUT after opts->wait_limit_ms and
 * leave the device usable.  Only for tests; sg_count has no such option. */
sg_status sg_debug_count_unsatisfiable_wait(sg_graph g, sg_plan p, const sg_count_opts *o, double *raw);

/* The coloring of sg_colors for callers that cannot allocate device memory
 * (no counterpart in the reference).  Frameworks that reserve all GPU memory
 * in their own pool at start-up, and pipelines that cannot take the device
 * synchronisation an allocation implies, pass the output buffer themselves:
 * d_colors is a DEVICE array of V int32 written with rand() % k after
 * srand(seed), in vertex order, on `stream` (a cudaStream_t; NULL = legacy
 * stream).  The call allocates nothing: its scratch (the glibc stream's
 * jump-ahead tables, 8.3 MB) is a fixed array in the library that every GPU
 * that loads the library keeps until the process exits; V is limited to 2^26
 * and larger V is rejected with SG_ERR_INVALID.  The first call on a device
 * is its set-up: it looks up the array's device address and fills the whole
 * array with one synchronous copy from host memory, so that first call must
 * not be made while a stream is being captured.  Every later call only
 * launches one kernel on `stream` (no copy, no synchronisation).  All calls
 * share the array; after the set-up they only read it, so calls that overlap
 * on the GPU do not disturb one another, and concurrent first calls from
 * several host threads are serialised by a lock. */
sg_status sg_colors_noalloc(int32_t V, int32_t k, uint32_t seed, int32_t *d_colors, void *stream);

/* ---- CountMat mirror ---------------------------------------------------- */

/* CountMat::initialization (CountMat.hpp:32-33).  Exactly one of the graphs is
 * given, as in the reference (CountMat.cpp:27-30); thd_num is accepted for
 * interface parity (the GPU ignores it). */
sg_status sg_countmat_create(sg_countmat *out);
void sg_countmat_destroy(sg_countmat cm);
sg_status sg_countmat_initialization(sg_countmat cm, sg_graph csr_graph, sg_graph csc_graph, int32_t thd_num,
                                     int32_t itr_num, int32_t isPruned, int32_t useSPMM, int32_t vtuneStart,
                                     int32_t calculate_automorphisms);
/* seed base for the colorings (the reference seeds with time(0)) */
sg_status sg_countmat_set_seed(sg_countmat cm, uint32_t seed_base);
/* CountMat::compute (CountMat.hpp:35): prints the reference's report lines to
 * stdout when verbose != 0 and returns the rounded estimate in *result. */
sg_status sg_countmat_compute(sg_countmat cm, sg_plan templates, int32_t isEstimate, int32_t verbose, double *result);
/* per-coloring raw counts of the last compute (n = itr_num) */
sg_status sg_countmat_raw(sg_countmat cm, double *raw);

#ifdef __cplusplus
}
#endif

#endif /* SG_API_H */
