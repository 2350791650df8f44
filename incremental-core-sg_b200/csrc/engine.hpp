// Host-side internals of the B200 CORE-SG engine: contexts, resident graphs,
// device buffers and error plumbing shared by the .cu translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "coresg_b200.h"

namespace csb {

// ---- errors -------------------------------------------------------------------

struct Error : std::runtime_error {
    cs_status status;
    Error(cs_status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

[[noreturn]] void fail(cs_status s, const std::string& msg);
void check_cuda(cudaError_t e, const char* what, const char* file, int line);

#define CSB_CUDA(expr) ::csb::check_cuda((expr), #expr, __FILE__, __LINE__)
#define CSB_REQUIRE(cond, msg)                                   \
    do {                                                         \
        if (!(cond)) ::csb::fail(CS_ERR_INVALID, (msg));         \
    } while (0)

void set_thread_error(const std::string& m);
const char* thread_error();

// ---- device memory ----------------------------------------------------------

/// Owning device allocation that only grows.  cudaMalloc failures surface as
/// CS_ERR_OOM.
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void release();
    void ensure(size_t nbytes);  // contents not preserved when it grows
    void grow_keep(size_t nbytes, cudaStream_t s);  // contents preserved
    template <typename T>
    T* as() const { return static_cast<T*>(p); }
};

/// Pinned host staging that only grows.
struct PinnedBuf {
    void* p = nullptr;
    size_t bytes = 0;
    PinnedBuf() = default;
    PinnedBuf(const PinnedBuf&) = delete;
    PinnedBuf& operator=(const PinnedBuf&) = delete;
    ~PinnedBuf() { release(); }
    void release();
    void ensure(size_t nbytes);
    template <typename T>
    T* as() const { return static_cast<T*>(p); }
};

// ---- context ------------------------------------------------------------------

struct Ctx {
    int device = 0;
    int sm_count = 0;
    int cc_major = 0, cc_minor = 0;
    cudaStream_t stream = nullptr;
    std::recursive_mutex mu;
    std::string last_error;
    uint64_t launches = 0;  // engine kernel launches issued
    DevBuf scratch[8];      // per-call scratch, reused across calls
    PinnedBuf pinned[2];
    DevBuf status;          // device error word(s) written by bounded waits
    int live_graphs = 0;    // graphs created on this context and not yet destroyed
    bool destroy_pending = false;  // cs_ctx_destroy called while graphs were alive
    void bind() const;      // cudaSetDevice(device)
    void sync();            // stream synchronise + error check
};

// ---- resident CORE-SG -------------------------------------------------------------

struct SweepPlan;  // mst.cu

struct Graph {
    Ctx* ctx = nullptr;
    uint32_t dim = 0, k = 0, stride = 0;
    int metric = CS_METRIC_L2;
    uint64_t n = 0;       // nodes with points
    uint64_t knn_n = 0;   // nodes with k-NN arrays (== n once set)
    uint64_t cap_n = 0;   // allocated node capacity

    DevBuf pts;     // float [cap_n][stride]
    DevBuf ids;     // u32  [cap_n][k]
    DevBuf dists;   // f32  [cap_n][k]
    DevBuf flags;   // u8   [cap_n][k]
    DevBuf counts;  // u32  [cap_n]
    DevBuf bridges; // cs_edge [nb]
    uint64_t nb = 0;
    uint64_t n_repair = 0;

    // Derived undirected edge list (base weights), in the reference order:
    // k-NN edges node-major (src/knn_graph.cpp:132-200), then the bridges.
    bool edges_valid = false;
    bool knn_edges_valid = false;  // the k-NN part (first e_knn entries, node_off) is current
    bool knn_offsets_valid = false;  // node_off, e_knn and the emit mask are current (edges maybe not emitted)
    DevBuf emask;                    // per node, which list entries emit an undirected edge
    uint64_t e_knn = 0, e_total = 0;
    DevBuf eu, ev, ew;    // SoA u32/u32/f32 [e_total]
    DevBuf node_off;      // u32 [n+1] offsets of each node's emitted edges

    // Workspace of the plain per-mpts path (mst.cu), kept across calls.
    struct PlainWork {
        DevBuf eu, ev, ew, core, parent, best, touched, wl, bitmap, bins, ctr, tiles, lab, out, counts;
    } plain;

    // Scratch kept across calls (grow-only): NN-Descent (knn.cu), the insert path's
    // search and active sets (knn.cu), the bridge selection (bridges.cu).
    DevBuf knn_scratch[14];
    DevBuf insert_scratch[12];
    DevBuf bridge_scratch[23];

    // Stages of the last cs_insert.
    cs_insert_stats last_insert{};
    // Distance evaluations and device ms of the last cs_knn_build.
    uint64_t last_build_evals = 0;
    double last_build_ms = 0.0;

    // Hubness selection of the last cs_select_bridges, and the component count of
    // the k-NN graph it saw.
    std::vector<uint32_t> selected;
    uint32_t last_ncomp = 0;

    // Batched sweep state (sweep.cu): a chain of plans, one per pass of <= 32 MSTs.
    SweepPlan* plan = nullptr;
    uint32_t sweep_K = 0;                      // MSTs of the last sweep
    uint32_t sweep_block = 0;                  // 0 = autotuned/cached
    uint32_t sweep_flatten = 0xFFFFFFFEu;      // kFlattenAuto, or a divisor (0: never)
    // testing hook (cs_test_sweep_barrier): grid-barrier wait limit of the sweep
    // kernel (0: the default) and a delay block 0 takes before its first barrier
    uint64_t sweep_barrier_ns = 0, sweep_hold_ns = 0;
    uint32_t sweep_tail_div = 0xFFFFFFFFu;  // contracted tail divisor (0: never; all ones: the default)
    uint32_t sweep_tail_slots = 0;          // cap on the tail table's slots (0: the default)

    ~Graph();
    void invalidate_edges() { edges_valid = knn_edges_valid = knn_offsets_valid = false; }
    /// Only the bridges changed: the k-NN part of the edge list stays, and the next
    /// build re-emits the bridge tail alone.
    void invalidate_bridges() { edges_valid = false; }
    // Stages of the last cs_select_bridges.
    cs_bridge_stats last_bridges{};
    // Incremental hubness (bridges.cu): the lists as of the last scoring (snapshot and
    // counts), k_merge's flags of nodes whose membership changed since, the flags of
    // nodes whose reverse degree changed, a counter; valid after a full pass until the
    // k-NN arrays are replaced.
    bool hub_valid = false;
    // NN-Descent overflow tables known empty for nodes [0, cand_clean_n) of the buffer at
    // cand_clean_ptr with cand_clean_bytes (every completed session leaves them so)
    const void* cand_clean_ptr = nullptr;
    size_t cand_clean_bytes = 0;
    uint64_t cand_clean_n = 0;
    uint64_t hub_n = 0;  // nodes scored by the last pass
    DevBuf hub_prev_ids, hub_prev_cnt, hub_changed, hub_rd_dirty, hub_ctr, hub_list;
    void ensure_capacity(uint64_t need, bool keep);
};

constexpr uint32_t kFlattenAuto = 0xFFFFFFFEu;

/// Node count that per-graph scratch is sized for: the allocated capacity, which grows
/// 1.5x at a time, so scratch is reallocated together with the resident arrays and
/// not at every insert (a fresh device allocation of hundreds of MB took up to a
/// second on these GPUs).
inline uint64_t scratch_nodes(const Graph& g) { return g.cap_n > g.n ? g.cap_n : g.n; }
/// `count` items proportional to the node count, scaled to scratch_nodes.
inline uint64_t scratch_scale(const Graph& g, uint64_t count) {
    return g.n ? count * scratch_nodes(g) / g.n + (count * scratch_nodes(g) % g.n ? 1 : 0) : count;
}

// ---- module entry points (implemented in the .cu files) ----------------------------

// graph.cu
void graph_build_edges(Graph& g);  // cached base edge list (no-op when valid)
/// The undirected k-NN edge count (e_knn) and per-node offsets of the cached edge
/// list, without emitting the edges (no-op when current).
void graph_count_knn_edges(Graph& g);
/// Allocate the cached edge list and its enumeration scratch for scratch_nodes(g)
/// nodes now.
void edges_reserve(Graph& g);
/// Upload (or append) n rows of `row_stride` floats as padded points; new nodes
/// start with empty k-NN lists (Dataset::append + KnnGraph::grow).
void graph_set_points(Graph& g, const float* rows, uint64_t n, uint32_t row_stride, bool append);
uint64_t graph_materialize_edges(Graph& g, uint32_t mpts, bool reweight, DevBuf& u, DevBuf& v,
                                 DevBuf& w, DevBuf& core_out, DevBuf& tmp_mask, DevBuf& tmp_cnt,
                                 DevBuf& tmp_off);
void launch_core(const Graph& g, uint32_t mpts, float* core, cudaStream_t s);

// mst.cu, sweep.cu
struct MstHost {
    uint64_t nedges = 0;
    uint32_t ncomp = 0;
    double weight = 0.0;
};
void extract_plain(Graph& g, uint32_t mpts, cs_edge* out_edges, uint32_t* out_labels, MstHost* res);
void sweep_run(Graph& g, const uint32_t* mpts, uint32_t K, bool want_labels, float* out_ms);
/// Result `index` of the last sweep: scalars to *res; the tree and labels to host
/// buffers, or (device_out) to caller device buffers on the graph's device.
void sweep_fetch(Graph& g, uint32_t index, cs_edge* out_edges, uint32_t* out_labels, MstHost* res,
                 bool device_out = false);
void sweep_free(SweepPlan* p);
/// Device outputs of MST `index` of the last sweep, valid until the next sweep.
struct SweepOut {
    const cs_edge* edges = nullptr;             // [cap] tree edges, ascending edge index
    const uint32_t* labels = nullptr;           // [n] (null when the sweep ran without labels)
    const unsigned long long* count = nullptr;  // tree edges
    const unsigned long long* bins = nullptr;   // [256] exact-sum bins of the tree weights
    uint64_t cap = 0, n = 0;
};
SweepOut sweep_outputs(Graph& g, uint32_t index);
double exact_sum_from_bins(const uint64_t* bins256);
/// Dense labels (numbered by smallest node) of K union-find forests parent_all[K][n]
/// whose roots are their sets' smallest nodes; component counts -> ncomp[K].
void launch_labels(Ctx& c, uint32_t* parent_all, uint32_t n, uint32_t K, uint32_t* lab_all, uint32_t* bc,
                   unsigned long long* ncomp);
/// In-place exclusive scan of K rows of nt u32 tile counts; row totals -> totals[K].
void launch_scan_tiles(Ctx& c, uint32_t* tiles, uint32_t nt, uint32_t K, unsigned long long* totals);

// knn.cu
/// Allocate the NN-Descent and insert scratch for scratch_nodes(g) nodes now.
void knn_reserve(Graph& g);
void knn_descent(Graph& g, uint32_t sample, uint32_t iters, double delta, uint64_t seed,
                 bool random_fill, uint64_t* out_updates, uint32_t* out_rounds);
struct InsertStats {
    uint64_t active = 0, updates = 0;
    uint32_t rounds = 0;
    double search_ms = 0.0, refine_ms = 0.0;
    cs_insert_stats detail{};
};
void knn_insert(Graph& g, const float* rows, uint64_t count, uint32_t row_stride, const cs_insert_params& p,
                InsertStats* st);

// bridges.cu
/// Allocate the selection scratch for scratch_nodes(g) nodes now.
void bridges_reserve(Graph& g);
/// The changed-membership flags of the incremental hubness refresh, for
/// scratch_nodes(g) nodes (contents kept; new entries zero).  The NN-Descent merge
/// writes them.
void hub_track(Graph& g);
/// An upper bound of the selection size on a graph of up to scratch_nodes(g) nodes
/// whose k-NN graph has at most 4x the last seen component count (+ 64).
uint64_t selection_bound(const Graph& g);
void select_bridges(Graph& g, uint64_t* out_selected, uint64_t* out_bridges, uint64_t* out_repair,
                    uint32_t* out_components);
void mrd_rows(Ctx& c, const float* d_pts, uint32_t m, uint32_t stride, int metric,
              const float* d_core, uint32_t r0, uint32_t r1, float* d_out);

// scan.cu
/// Exclusive prefix sum of n u32 values into out (n+1 entries; out[n] = total).
void scan_u32(Ctx& c, const uint32_t* in, uint32_t* out, uint64_t n);
/// Allocate scan_u32's scratch for scans of up to n items now.
void scan_reserve(Ctx& c, uint64_t n);

// host <-> device through the context's pinned staging (context.cu)
void copy_h2d(Ctx& c, void* dst, const void* src, size_t bytes);
void copy_d2h(Ctx& c, void* dst, const void* src, size_t bytes);
/// Device -> page-locked host memory enqueued on the context stream without waiting
/// (true: the caller synchronises the stream before reading dst); any other host
/// memory is copied through the staging at once (false).
bool copy_d2h_enqueue(Ctx& c, void* dst, const void* src, size_t bytes);

/// Run `f` for a C entry point: lock the context, bind its device, translate
/// exceptions into a status plus the context's last error.
template <typename F>
cs_status guarded(Ctx* c, F&& f) {
    if (!c) {
        set_thread_error("null context or handle");
        return CS_ERR_INVALID;
    }
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    try {
        c->bind();
        f();
        return CS_OK;
    } catch (const Error& e) {
        c->last_error = e.what();
        set_thread_error(e.what());
        return e.status;
    } catch (const std::bad_alloc&) {
        c->last_error = "host allocation failed";
        set_thread_error(c->last_error);
        return CS_ERR_OOM;
    } catch (const std::exception& e) {
        c->last_error = e.what();
        set_thread_error(e.what());
        return CS_ERR_INVALID;
    }
}

/// Run f for an entry point that needs no device (host formatting): exceptions
/// become the status and the thread's last error.
template <typename F>
cs_status host_guarded(F&& f) {
    try {
        f();
        return CS_OK;
    } catch (const Error& e) {
        set_thread_error(e.what());
        return e.status;
    } catch (const std::bad_alloc&) {
        set_thread_error("host allocation failed");
        return CS_ERR_OOM;
    } catch (const std::exception& e) {
        set_thread_error(e.what());
        return CS_ERR_INVALID;
    }
}

void ctx_free(Ctx* c);

// launch bookkeeping
inline void count_launch(Ctx& c, uint64_t n = 1) { c.launches += n; }
void check_launch(Ctx& c, const char* what);

}  // namespace csb
