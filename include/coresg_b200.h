/* coresg_b200.h -- C ABI of the B200 (sm_100a) engine for the CORE-SG hot path.
 *
 * The engine keeps a CORE-SG resident in HBM (padded points, the k_max-NN arrays,
 * the bridge edges and the derived undirected edge list) and runs, on one GPU:
 * Dynamic NN-Descent, core distances, mutual-reachability reweighting, the per-mpts
 * MST extraction (plain and as one batched persistent sweep), and the anti-hub
 * bridge selection.  Citations are path:line in the reference project
 * (voidosama/Incremental-CORE-SG).
 *
 * Conventions
 *   - Every function returns a cs_status; on failure cs_last_error(ctx) holds the
 *     message (per context; cs_last_error(NULL) is the calling thread's last error,
 *     for failures before a context exists).  Mirrors the bool + thread-local
 *     last_error() of include/coresg/cuda_api.hpp:22-23 / cuda/cuda_runtime_api.cu:17-23.
 *   - Plain pointers and sizes only.  "host" pointers are caller-owned host memory;
 *     the engine copies through its own pinned staging.  Distances cross the
 *     boundary in metric units (L2 distance, not squared), like nndescent_gpu.
 *   - One CUDA stream per context; calls on one context are serialised by a
 *     per-context mutex.  There is no CPU fallback: a device failure is an error.
 *   - Out of device memory is CS_ERR_OOM, never a crash (src/cuda_backend.cpp:88-103
 *     records OOM as a result; the caller decides what to do).
 */
#ifndef CORESG_B200_H
#define CORESG_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t cs_status;
enum {
    CS_OK = 0,
    CS_ERR_INVALID = 1,     /* bad argument (null pointer, size, mpts > k_max, ...) */
    CS_ERR_CUDA = 2,        /* a CUDA runtime call failed */
    CS_ERR_OOM = 3,         /* device allocation failed */
    CS_ERR_TIMEOUT = 4,     /* a bounded device-side wait ran out; the context stays usable */
    CS_ERR_UNSUPPORTED = 5, /* metric / size the device path does not cover */
    CS_ERR_STATE = 6        /* call out of order (e.g. extract before a graph is loaded) */
};

/* Metric codes, as coresg::cuda::MetricCode (include/coresg/cuda_api.hpp:30-33). */
enum { CS_METRIC_L2 = 0, CS_METRIC_COSINE = 1 };

/* Same layout as coresg::Edge (include/coresg/types.hpp:20-33): u < v, weight w. */
typedef struct {
    uint32_t u;
    uint32_t v;
    float w;
} cs_edge;

/* Same fields as coresg::cuda::NndConfig (include/coresg/cuda_api.hpp:35-46). */
typedef struct {
    uint32_t n;
    uint32_t dim;
    uint32_t stride; /* padded row length in floats (multiple of 8, dataset.hpp:21) */
    uint32_t k;
    uint32_t sample; /* smpN; sampled old neighbours capped at 3 * sample */
    uint32_t iters;
    uint64_t seed;
    int32_t metric;
    float delta;         /* stop when a round's updates <= delta * k * n */
    int32_t random_fill; /* top up unfilled slots with random candidates first */
} cs_nnd_config;

typedef struct cs_ctx cs_ctx;
typedef struct cs_graph cs_graph;

/* ---- device and context (cuda/cuda_runtime_api.cu:25-79) ------------------- */

/* Replaces coresg::cuda::device_count (include/coresg/cuda_api.hpp:48). */
cs_status cs_device_count(int32_t* out_count);
/* Replaces get_device_props + device_memory (include/coresg/cuda_api.hpp:49, :80). */
cs_status cs_device_props(int32_t device, char* name, size_t name_len, size_t* total_mem,
                          size_t* free_mem, int32_t* sm_count, int32_t* cc_major,
                          int32_t* cc_minor);
/* Replaces coresg::cuda::last_error (include/coresg/cuda_api.hpp:52). */
const char* cs_last_error(const cs_ctx* ctx);

/* A context binds one device and owns one stream plus cached device scratch.  The
 * reference binds a device per call (cudaSetDevice in nndescent_gpu); a context is
 * the per-slot state that src/cuda_backend.cpp keeps per JobScheduler thread. */
cs_status cs_ctx_create(int32_t device, cs_ctx** out_ctx);
void cs_ctx_destroy(cs_ctx* ctx);
/* Release cached scratch (coresg::cuda::release_thread_cache, cuda_api.hpp:84;
 * Backend::trim, backend.hpp:91). */
cs_status cs_ctx_trim(cs_ctx* ctx);
/* The context's CUDA stream (a cudaStream_t), on which every call of this context
 * runs its device work: a caller orders its own work after the engine's on it (the
 * multi-GPU gather of a partitioned sweep runs its collective there).  Valid until
 * cs_ctx_destroy. */
void* cs_ctx_stream(const cs_ctx* ctx);
/* Number of engine kernel launches issued on this context so far. */
uint64_t cs_ctx_launches(const cs_ctx* ctx);
/* Device allocations (cudaMalloc) the library has made in this process so far,
 * and their bytes (freed buffers included).  After cs_graph_reserve(g, rows), an
 * insert of any batch that keeps the graph within `rows` makes none, except when
 * the k-NN graph then has more than 4x (+ 64) the components it had at the last
 * bridge selection before the reserve, when the bridges leave components apart (the
 * repair pass), or when the rows come with a stride above dim. */
void cs_device_allocs(uint64_t* out_count, uint64_t* out_bytes);

/* ---- the two device entry points the reference's CUDA backend binds -------- */

/* Dynamic NN-Descent on host buffers, start to finish: upload, optional random
 * fill, <= iters rounds with the delta stop rule, download.  Replaces
 * coresg::cuda::nndescent_gpu (include/coresg/cuda_api.hpp:57-59,
 * cuda/nndescent_kernels.cu:295-437).  ids/dists/flags are n*k, counts n; dists in
 * metric units; out_updates may be NULL. */
cs_status cs_nndescent(cs_ctx* ctx, const cs_nnd_config* cfg, const float* host_vectors,
                       uint32_t* ids, float* dists, uint8_t* flags, uint32_t* counts,
                       uint64_t* out_updates);

/* Rows [r0, r1) of the m x m mutual-reachability matrix max(d(i,j), core_i, core_j),
 * 0 on the diagonal.  Replaces coresg::cuda::mrd_block_gpu
 * (include/coresg/cuda_api.hpp:62-65, cuda/mrd_kernels.cu:218-243). */
cs_status cs_mrd_block(cs_ctx* ctx, const float* host_pts, size_t m, uint32_t dim,
                       uint32_t stride, int32_t metric, const float* host_core, size_t r0,
                       size_t r1, float* host_out);

/* ---- resident CORE-SG -------------------------------------------------------- */

/* An empty device-resident CORE-SG with the given dimensionality and k_max
 * (CoreSG state of include/coresg/coresg.hpp:198-204). k_max <= 64. */
cs_status cs_graph_create(cs_ctx* ctx, uint32_t dim, uint32_t k_max, int32_t metric,
                          cs_graph** out_graph);
void cs_graph_destroy(cs_graph* g);

/* n rows of `dim` floats (row_stride floats apart) -> padded device rows
 * (Dataset::append, include/coresg/dataset.hpp:55-68; cosine rows are normalised). */
cs_status cs_graph_set_points(cs_graph* g, const float* rows, uint64_t n, uint32_t row_stride);
/* Append further rows (CoreSG::insert's Dataset::append + KnnGraph::grow). */
cs_status cs_graph_append_points(cs_graph* g, const float* rows, uint64_t count,
                                 uint32_t row_stride);
/* k-NN arrays in the KnnGraph layout (include/coresg/knn_graph.hpp:191-197): n*k ids
 * (0xFFFFFFFF unfilled), n*k dists (+inf unfilled, ascending), n*k flags, n counts.
 * flags may be NULL (all zero). */
cs_status cs_graph_set_knn(cs_graph* g, const uint32_t* ids, const float* dists,
                           const uint8_t* flags, const uint32_t* counts, uint64_t n);
cs_status cs_graph_get_knn(cs_graph* g, uint32_t* ids, float* dists, uint8_t* flags,
                           uint32_t* counts);
/* Bridge ("missing") edges with base distances (CoreSG::missing_edges,
 * include/coresg/coresg.hpp:155). */
cs_status cs_graph_set_bridges(cs_graph* g, const cs_edge* edges, uint64_t m);
cs_status cs_graph_get_bridges(cs_graph* g, cs_edge* out, uint64_t cap, uint64_t* out_count);
/* Capacity for `rows` nodes (Dataset::reserve, include/coresg/dataset.hpp:50): the
 * resident arrays, the edge list, and the scratch of NN-Descent, inserts and the
 * bridge selection are allocated for that many nodes now, and the sweep buffers are
 * sized for it when next built, so inserts that stay within it allocate no device
 * memory (cs_device_allocs states the exceptions; a fresh allocation of a few
 * hundred MB took from a few ms to over a second here).  Never shrinks. */
cs_status cs_graph_reserve(cs_graph* g, uint64_t rows);
/* n, k_max, dim, stride, undirected k-NN edge count (KnnGraph::undirected_edge_count,
 * src/knn_graph.cpp:202-217), bridge count.  Any pointer may be NULL. */
cs_status cs_graph_info(cs_graph* g, uint64_t* n, uint32_t* k_max, uint32_t* dim,
                        uint32_t* stride, uint64_t* knn_edges, uint64_t* bridges);

/* CORESG01 files, byte-compatible with CoreSG::save / CoreSG::load
 * (src/io.cpp:195-330): padded rows, k-NN arrays, bridges, repair count.
 * Connectivity and hubness are derived state and are not stored (as in the
 * reference); cs_select_bridges recomputes them. */
cs_status cs_graph_save(cs_graph* g, const char* path);
/* The extraction's text outputs, byte for byte as coresg::write_edges_tsv /
 * write_labels_tsv (src/io.cpp:131-145, apps/coresg_cli.cpp:563-570): "u\tv\tweight"
 * with the weight in scientific notation, 9 digits; "id\tlabel". */
cs_status cs_write_edges_tsv(const char* path, const cs_edge* edges, uint64_t m);
cs_status cs_write_labels_tsv(const char* path, const uint32_t* labels, uint64_t n);
/* Result `index` of the last sweep (its tree, and its labels when the sweep computed
 * them) straight from the device to those files; either path may be NULL. */
cs_status cs_sweep_write_tsv(cs_graph* g, uint32_t index, const char* edges_path,
                             const char* labels_path);
cs_status cs_graph_load(cs_ctx* ctx, const char* path, cs_graph** out_graph);

/* ---- build: NN-Descent on the resident points + bridges --------------------- */

/* k-NN graph of the resident points by Dynamic NN-Descent (IncrementalKnn::build
 * with one instance, src/incremental_knn.cpp:1003-1050 -> nndescent_gpu): random
 * fill, <= iters rounds, delta stop.  sample/iters/seed/delta as NNDescentParams
 * (include/coresg/nndescent.hpp:45-71).  out_updates, out_rounds may be NULL. */
cs_status cs_knn_build(cs_graph* g, uint32_t sample, uint32_t iters, double delta, uint64_t seed,
                       uint64_t* out_updates, uint32_t* out_rounds);
/* Of the last cs_knn_build: distance evaluations of the local joins (the statistic
 * NNDescentStats::distance_evals, include/coresg/nndescent.hpp:73-78; 3 x dim FLOP
 * each) and device milliseconds of the random fill + rounds. */
cs_status cs_knn_build_stats(cs_graph* g, uint64_t* out_evals, double* out_device_ms);

/* Parameters of cs_insert; cs_insert_defaults fills the reference's defaults
 * (coresg_cli: sample 16, iters 10, refine-iters 5, context-per-new 2.0,
 * owned-warm-fraction 0.25, refine-per-new 2.0; IncrementalKnnParams:
 * refine_max_fraction 0.25; seeding search with 8k expansions). */
typedef struct {
    uint32_t sample;            /* smpN of both descents */
    uint32_t instance_iters;    /* rounds over the new points and their context */
    uint32_t refine_iters;      /* rounds of the restricted refinement */
    double context_per_new;     /* context nodes per new point in the first descent */
    double owned_warm_fraction; /* fraction of a new point's seeds it keeps (rest: random batch points) */
    double refine_per_new;      /* refinement-set cap per new point (0: no per-point cap) */
    double refine_max_fraction; /* active-set cap as a fraction of n (>= 1: none) */
    double delta;               /* stop when a round's updates <= delta * k * |active| */
    uint32_t max_expand;        /* seeding search expansions per point (0: 8k) */
    uint32_t reverse_cap;       /* reverse neighbours the search expands per node (search_reverse_cap) */
    uint64_t seed;
    int32_t reselect_bridges;   /* 1: re-select the anti-hub bridges afterwards */
} cs_insert_params;
void cs_insert_defaults(cs_insert_params* p);

/* Incremental insertion of `count` rows (CoreSG::insert, src/coresg.cpp:325-389 ->
 * IncrementalKnn::insert, src/incremental_knn.cpp:1155-1252), all on device and over
 * the one resident graph: the rows are appended; each new point is seeded by a beam
 * search over the base graph (the anchored seeding search, :118-216); the seeds are
 * inserted both ways (:1195-1200); a restricted Dynamic NN-Descent runs over the new
 * points and two rings of their neighbourhoods in discovery order, capped as
 * refinement_set (:927-987); then, optionally, the bridges are re-selected.  The
 * reference splits an insert into instances to bound per-device memory; here the
 * whole graph is resident, so one active set plays every instance: a descent over the
 * new points and their context (new points keep owned_warm_fraction of their seeds
 * and are topped up with random points of the batch, src/incremental_knn.cpp:808-840),
 * then the restricted refinement.
 * out_active, out_updates may be NULL. */
/* Stages of the last cs_insert on a graph (IncrementalKnnStats,
 * include/coresg/incremental_knn.hpp:270-300): device milliseconds of the reverse
 * index, the seeding search + seed application, the instance descent, the
 * restricted refinement and the finalisation, and host milliseconds of the bridge
 * re-selection and of the whole call. */
typedef struct {
    uint64_t new_points;
    uint64_t instance_nodes;  /* new points + context */
    uint64_t refine_nodes;
    uint64_t updates;
    uint32_t rounds;          /* descent rounds run (instance + refinement) */
    uint32_t reserved0;
    double reverse_ms, search_ms, instance_ms, refine_ms, finish_ms, bridges_ms, total_ms;
} cs_insert_stats;
cs_status cs_insert_stats_get(cs_graph* g, cs_insert_stats* out);

cs_status cs_insert(cs_graph* g, const float* rows, uint64_t count, uint32_t row_stride,
                    const cs_insert_params* params, uint64_t* out_active, uint64_t* out_updates);

/* Anti-hub bridges for the current k-NN graph, all on device: connectivity
 * (src/connectivity.cpp:99-139), reverse degrees and scores (src/hubness.cpp:44-158,
 * :302-352), selection with the per-component quota (:424-521), the MRD MST over the
 * selected set stored with base distances (src/coresg.cpp:97-141) and the
 * connectivity repair (src/coresg.cpp:171-258).  Replaces the bridges half of
 * CoreSG::build/insert (src/coresg.cpp:487-516, :565-583) with the defaults of
 * CoreSGParams/HubnessParams.  Results: the graph's bridge set; counts optional. */
cs_status cs_select_bridges(cs_graph* g, uint64_t* out_selected, uint64_t* out_bridges,
                            uint64_t* out_repair, uint32_t* out_knn_components);
/* Stages of the last cs_select_bridges (or of the re-selection inside cs_insert),
 * device milliseconds between stage boundaries on the context stream (host steps
 * between them included), as CoreSGStats::hubness_seconds / missing_seconds /
 * repair_seconds (include/coresg/coresg.hpp:108-138) and HubnessStats
 * (include/coresg/hubness.hpp:121-142) split the reference's build. */
typedef struct {
    double connectivity_ms;  /* union-find over the k-NN lists, dense component labels */
    double hubness_ms;       /* reverse degrees and scores: after the first selection on a graph, an
                                incremental refresh (the deltas of the lists that changed since, and
                                the nodes whose score inputs moved rescored) */
    double edges_ms;         /* the undirected k-NN edge list (its count is the budget's |E|) */
    double selection_ms;     /* budget-lowest selection, per-component quota, ordering */
    double bridge_mst_ms;    /* dense MRD + Prim over the selected anti-hubs */
    double repair_ms;        /* connectivity repair (0 when the bridges join every component) */
    double total_ms;
    uint64_t selected, bridges, repair;
    uint32_t knn_components;
    uint32_t hub_refreshed;  /* 1: the hubness stage was the incremental refresh (HubnessIndex::refresh,
                                src/hubness.cpp:523-544); 0: a full pass (rescore_all) */
    uint64_t rescored;       /* nodes whose score the hubness stage computed */
    uint64_t changed;        /* nodes whose list changed since the last scoring (n after a full
                                pass with no earlier state); the refresh runs when at most n / 16
                                changed, else a full pass is the cheaper one */
} cs_bridge_stats;
cs_status cs_bridge_stats_get(cs_graph* g, cs_bridge_stats* out);
/* The selected anti-hubs of the last cs_select_bridges (HubnessIndex::selected). */
cs_status cs_get_selected(cs_graph* g, uint32_t* out, uint64_t cap, uint64_t* out_count);

/* ---- extraction (new: the reference runs all of this on the host) ------------ */

/* Core distances for mpts (CoreSG::core_distances, src/coresg.cpp:68-70 ->
 * KnnGraph::core_dist, include/coresg/knn_graph.hpp:157-163).  out: n floats. */
cs_status cs_core_distances(cs_graph* g, uint32_t mpts, float* host_out);

/* CoreSG::edges(mpts) (src/coresg.cpp:391-406): the undirected k-NN edges in the
 * reference's enumeration order, reweighted by mrd_mpts, then the bridges.  Writes
 * min(count, cap) edges; *out_count gets the full count. */
cs_status cs_edges(cs_graph* g, uint32_t mpts, cs_edge* host_out, uint64_t cap,
                   uint64_t* out_count);

/* MST_mpts of the CORE-SG, the plain per-mpts path: edges(mpts) materialised on
 * device, then Boruvka rounds driven from the host, one launch sequence per mpts.
 * Same result as CoreSG::mst (src/coresg.cpp:408-410 -> mst_boruvka,
 * src/mst.cpp:79-151): the unique minimum spanning forest under (weight bits, edge
 * index).  Outputs (all optional): out_edges (n-1 cap) in ascending edge-index
 * order, out_labels (n; dense, numbered by smallest node), edge count, component
 * count, and the total weight as the correctly rounded exact sum. */
cs_status cs_extract(cs_graph* g, uint32_t mpts, cs_edge* out_edges, uint32_t* out_labels,
                     uint64_t* out_nedges, uint32_t* out_ncomp, double* out_weight);

/* The batched sweep: K MSTs (one per entry of mpts[]) from the one resident edge
 * list, reweighted on the fly and solved by one persistent cooperative launch per
 * pass of up to 32 MSTs (one warp lane per MST), replayed from CUDA graphs
 * (CoreSG::all_msts, src/coresg.cpp:412-417, which the reference runs as K
 * independent extractions).  Per-MST results as cs_extract, packed: out_edges
 * K*(n-1), out_labels K*n, and K-long count/weight arrays.  Any output may be NULL.
 * Sweeps of all contexts on one device run one at a time (the persistent kernel
 * takes every SM); the copies of the results to the host run outside that, so a
 * host that keeps two graphs on two contexts in flight overlaps one graph's
 * uploads and downloads with the other's sweep. */
cs_status cs_extract_sweep(cs_graph* g, const uint32_t* mpts, uint32_t K, cs_edge* out_edges,
                           uint32_t* out_labels, uint64_t* out_nedges, uint32_t* out_ncomp,
                           double* out_weight);

/* Sweep results kept on the device: runs the sweep and leaves the K trees in the
 * graph's result buffers (no host copy); *out_ms (optional) gets the device time of
 * the launch in milliseconds.  Fetch with cs_sweep_fetch. */
cs_status cs_extract_sweep_device(cs_graph* g, const uint32_t* mpts, uint32_t K, float* out_ms);
cs_status cs_sweep_fetch(cs_graph* g, uint32_t index, cs_edge* out_edges, uint32_t* out_labels,
                         uint64_t* out_nedges, uint32_t* out_ncomp, double* out_weight);
/* cs_sweep_fetch into caller DEVICE buffers on the graph's device (the tree:
 * nedges entries of d_out_edges; the labels: n entries of d_out_labels; either may be
 * NULL), copied device to device on the context stream, complete on return; the
 * scalars go to host memory.  For handing results to a collective (the multi-GPU
 * gather of a partitioned sweep) without a host round trip. */
cs_status cs_sweep_fetch_device(cs_graph* g, uint32_t index, cs_edge* d_out_edges, uint32_t* d_out_labels,
                                uint64_t* out_nedges, uint32_t* out_ncomp, double* out_weight);

/* Device times of the last sweep: the whole captured sequence and the persistent
 * Boruvka kernel alone (CUDA events on the context stream), in milliseconds. */
cs_status cs_sweep_timing(cs_graph* g, float* graph_ms, float* kernel_ms);
/* Per-round profile of the first pass of the last sweep, 7 words per Boruvka round:
 * device ns of phase A (offers), phase B (links) and the forest flatten, entries phase A
 * walked (edges, or the contracted tail's (MST, component pair) entries), roots phase B
 * walked, flags (bit 0: every node flattened; bits 1-2: what phase A walked -- 0 the
 * edges, 1 the edges while filling the tail table, 2 the tail entries), live pairs
 * phase A found.
 * Writes min(rounds, cap_rounds) rows; *out_rounds = rounds (the last round ends after
 * its phase A). */
cs_status cs_sweep_trace(cs_graph* g, uint64_t* out, uint32_t cap_rounds, uint32_t* out_rounds);

/* Sweep tuning knobs (no counterpart in the reference, whose Boruvka has none; the trees
 * are the same under every setting).  flatten_div: after every Boruvka round the roots that were
 * linked point at their final roots; from round 2 on, every node is flattened too when
 * the round's live (edge, MST) pairs exceed 32 n / flatten_div (0xFFFFFFFF: never);
 * block_threads: 128, 256 or 512.  0 picks the value cached by cs_autotune_sweep for
 * this (n, |E|, K, SM count), else the defaults (never, 512). */
cs_status cs_set_sweep_shape(cs_graph* g, uint32_t flatten_div, uint32_t block_threads);
/* The sweep's contracted tail: once a Boruvka round's root list holds at most
 * n / tail_div nodes, the next round reduces the live (edge, MST) pairs into a table of
 * (MST, root pair) -> lightest key and the rounds after it walk the table's entries
 * instead of the edges; the trees are the same either way.  tail_div: 0 never,
 * UINT32_MAX the default (4).  table_slots: a cap on the table's slots, a power of two
 * in [2^10, 2^26] (0: the default, min(4 n, |E|) rounded up, at most 2^26); a table
 * that fills past its probe limit leaves the sweep on its edge worklist.  Graphs of
 * 2^27 nodes or more never take the tail.  Plans are recaptured when these change. */
cs_status cs_set_sweep_tail(cs_graph* g, uint32_t tail_div, uint32_t table_slots);
/* Project-written autotuner: times every (block, flatten_div) pair on the resident
 * graph and caches the fastest for later sweeps of this shape. */
cs_status cs_autotune_sweep(cs_graph* g, const uint32_t* mpts, uint32_t K, uint32_t* out_flatten,
                            uint32_t* out_block);

/* ---- serving loop (no counterpart in the reference) -------------------------- */

/* A device-resident request loop over one cs_graph: extract(mpts) queries,
 * epsilon-cut label queries and insert batches are submitted from any host thread
 * and served in arrival order.  Consecutive queries are batched as they arrive:
 * every batch is one 32-lane graph-captured sweep (a query that arrives while a
 * batch is on the GPU joins the next one) -- over every mpts 1..k_max when k_max <=
 * 32, and then a later batch with no insert since is served from that sweep's
 * results without a sweep; over the batch's distinct mpts otherwise -- its
 * results are copied into device result slots in stream order (one slot per
 * distinct extract mpts, shared by its queries, and one per epsilon-cut), and a
 * completion thread copies the slots into the callers' host buffers on a second
 * stream while the next sweep runs.  Inserts that are queued back to back are
 * applied as one batch (CoreSG::insert of their rows in order, then the bridges are
 * re-selected).  In arrival order an insert is a barrier: queries before it see the
 * graph without its rows, queries after it see them; with inserts_first, queued
 * inserts go ahead of queued queries.  Admission is by free HBM: a result slot is allocated only while
 * cudaMemGetInfo leaves `reserve_bytes` free, otherwise the batch is cut short and
 * waits for slots in flight; an insert whose growth does not fit fails with
 * CS_ERR_OOM.  The graph must not be used through other entry points while a server
 * runs on it.  Results equal cs_extract on the graph state the request saw; an
 * epsilon-cut equals dbscan_labels_from_mst (src/eval.cpp:230-239) on that tree:
 * union of the tree edges with double(w) <= eps, dense labels by smallest node. */
typedef struct cs_server cs_server;

enum { CS_REQ_EXTRACT = 0, CS_REQ_EPS_LABELS = 1, CS_REQ_INSERT = 2 };

typedef struct {
    uint32_t max_batch;       /* distinct mpts per sweep, 1..32 (0: 32) */
    uint32_t max_slots;       /* result slots allocated at most (0: 64) */
    uint32_t inserts_first;   /* 0: arrival order, an insert is a barrier between the
                                 queries before and after it; 1: every queued insert
                                 is applied before the queued queries (a query sees
                                 at least the inserts submitted before it) */
    uint32_t reserved0;
    uint64_t reserve_bytes;   /* HBM left free by admission (0: 2 GiB) */
    cs_insert_params insert;  /* parameters of every insert (cs_insert_defaults if
                                 sample == 0) */
} cs_server_config;

typedef struct {
    int32_t kind;              /* CS_REQ_* */
    uint32_t mpts;             /* extract / epsilon-cut: 0..k_max (0 == 1) */
    double eps;                /* epsilon-cut threshold on the MRD merge heights */
    const float* rows;         /* insert: count rows of row_stride floats (copied at
                                  submit, the buffer is free on return) */
    uint64_t count;
    uint32_t row_stride;
    cs_edge* out_edges;        /* extract: the tree (optional); holds out_edges_cap edges */
    uint64_t out_edges_cap;
    uint32_t* out_labels;      /* extract: MST component labels (optional);
                                  epsilon-cut: the cut's labels (required) */
    uint64_t out_labels_cap;
} cs_request;

typedef struct {
    int32_t status;            /* the request's own status */
    uint32_t ncomp;            /* components of the MST / of the cut */
    uint64_t nedges;           /* tree edges (extract) */
    uint64_t n;                /* graph size the request saw */
    double weight;             /* exact tree weight (extract) */
    double queue_ms;           /* submit -> dispatched to the GPU */
    double latency_ms;         /* submit -> result in the caller's buffers */
    uint64_t batch;            /* sweep batch that served it (0: insert) */
    char error[160];           /* message when status != CS_OK */
} cs_result;

typedef struct {
    uint64_t submitted, completed, failed;
    uint64_t batches;          /* sweeps run */
    uint64_t queries;          /* extract + epsilon-cut requests served */
    uint64_t inserts, inserted_rows;
    uint64_t insert_batches;   /* knn inserts run (back-to-back inserts share one) */
    uint64_t slots, slot_bytes;  /* result slots allocated, bytes each */
    uint32_t max_batch_seen;   /* most requests served by one sweep */
    double sweep_ms;           /* device time of all sweeps */
    double insert_ms;          /* host time of all inserts */
    uint64_t reused_batches;   /* query batches served from the last sweep of every mpts
                                  (no insert since): no sweep run for them */
} cs_server_stats;

cs_status cs_server_create(cs_graph* g, const cs_server_config* cfg, cs_server** out);
/* Finishes every submitted request, then stops the threads and frees the slots. */
void cs_server_destroy(cs_server* s);
/* Queue a request; *out_ticket identifies it for cs_server_wait. */
cs_status cs_server_submit(cs_server* s, const cs_request* req, uint64_t* out_ticket);
/* Wait up to timeout_ms (UINT32_MAX: forever) for a ticket; on completion fills
 * *out and releases the ticket.  CS_ERR_TIMEOUT when it is still pending. */
cs_status cs_server_wait(cs_server* s, uint64_t ticket, uint32_t timeout_ms, cs_result* out);
cs_status cs_server_stats_get(cs_server* s, cs_server_stats* out);
/* Page-locked host memory for request buffers (the completion copies run
 * asynchronously only into pinned memory). */
void* cs_host_alloc(size_t bytes);
void cs_host_free(void* p);

/* ---- testing hooks (no counterpart in the reference) --------------------------
 * Failure paths made on purpose, without a GPU fault: a bounded wait that runs out
 * and a device allocation that fails.  Not for production use. */

/* Grid-barrier wait limit of later sweeps on g in nanoseconds (0: the default, 2 s),
 * and a delay block 0 of the persistent sweep kernel takes (a bounded sleep) before
 * its first grid barrier (0: none; at most 5 s).  With hold_ns above limit_ns the
 * other blocks' waits run out: the sweep returns CS_ERR_TIMEOUT, its results are not
 * valid, and the context and graph stay usable.  Plans are recaptured when these
 * change. */
cs_status cs_test_sweep_barrier(cs_graph* g, uint64_t limit_ns, uint64_t hold_ns);
/* Process-wide: after `after` further device allocations by the library succeed,
 * every later one fails with CS_ERR_OOM (no cudaMalloc is issued for it);
 * UINT64_MAX switches the injection off. */
void cs_test_fail_device_allocs(uint64_t after);

/* ---- allocation-free MST (no counterpart in the reference) ------------------- */

/* MST of a caller-provided edge list that allocates nothing, for callers that
 * cannot allocate device memory themselves or through a library: plugins whose
 * host application owns every device allocation, and code that must not touch the
 * allocation API.  Inputs and outputs are the caller's device buffers: d_u, d_v,
 * d_w (m edges, structure of arrays), d_out_edges (n-1 edges), d_out_labels (n,
 * optional); the scalars go to host memory (optional).  All scratch lives in one
 * fixed 12 MiB __device__ array of this library, held by every GPU that loads the
 * library until the process exits; limits: n <= 131072 nodes, m <= 1048576 edges,
 * larger sizes are rejected with CS_ERR_INVALID.  Edges must have both endpoints
 * below n and weights that are non-negative with the sign bit clear and not NaN
 * (+inf is allowed); a list that breaks this is rejected with CS_ERR_INVALID before
 * any Boruvka round runs.  Runs on the current device, in the current CUDA context,
 * and on `stream` (a cudaStream_t; NULL is the default stream); needs no cs_ctx;
 * errors via cs_last_error(NULL).  The array's device address belongs to the
 * current context, so every call looks it up (cudaGetSymbolAddress) with the
 * caller's device and context current.  The call synchronises `stream` (the host
 * reads a counter after every Boruvka round) and returns with the results written:
 * it blocks the host and must not be called while `stream` is capturing.  Every
 * call reuses the same array (its contents are re-initialised per call), so calls
 * that overlap on the GPU -- from two streams or two host threads on one device --
 * race: serialise them.  Same result as cs_extract on the same edges: the unique
 * minimum spanning forest under (weight bits, edge index), tree in ascending edge
 * index order, dense labels by smallest node, exact total weight. */
cs_status cs_mst_noalloc(const uint32_t* d_u, const uint32_t* d_v, const float* d_w, uint64_t m,
                         uint32_t n, cs_edge* d_out_edges, uint32_t* d_out_labels,
                         uint64_t* out_nedges, uint32_t* out_ncomp, double* out_weight,
                         void* stream);

#ifdef __cplusplus
}
#endif
#endif /* CORESG_B200_H */
