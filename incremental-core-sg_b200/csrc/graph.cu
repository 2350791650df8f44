// Resident CORE-SG: points, k-NN arrays and bridges in HBM; the undirected edge
// list in the reference's enumeration order; core distances; CoreSG::edges(mpts).
#include <algorithm>
#include <cmath>
#include <cstring>

#include "common.cuh"
#include "engine.hpp"

namespace csb {
namespace {

constexpr int kThreads = 256;

inline unsigned blocks_for(uint64_t work, int threads = kThreads) {
    uint64_t b = (work + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > (1u << 30)) b = 1u << 30;
    return static_cast<unsigned>(b);
}

/// Pad rows to `stride` floats (zero tail) and, for cosine, L2-normalise them in
/// double like Dataset::normalise (include/coresg/dataset.hpp:89-95).
__global__ void k_pad_rows(const float* __restrict__ src, uint64_t n, uint32_t dim,
                           uint32_t src_stride, uint32_t stride, int metric,
                           float* __restrict__ dst) {
    const uint64_t row = static_cast<uint64_t>(blockIdx.x) * (blockDim.x / 32) + (threadIdx.x >> 5);
    if (row >= n) return;
    const unsigned lane = threadIdx.x & 31u;
    const float* s = src + row * src_stride;
    float* d = dst + row * stride;
    float inv = 1.0f;
    if (metric == CS_METRIC_COSINE) {
        // sequential double sum, as the reference does, done by lane 0
        double acc = 0.0;
        if (lane == 0) {
            for (uint32_t i = 0; i < dim; ++i) acc += static_cast<double>(s[i]) * s[i];
        }
        acc = __shfl_sync(0xFFFFFFFFu, acc, 0);
        inv = acc > 0.0 ? static_cast<float>(1.0 / sqrt(acc)) : 1.0f;
        for (uint32_t i = lane; i < stride; i += 32) d[i] = i < dim ? (acc > 0.0 ? s[i] * inv : s[i]) : 0.0f;
        return;
    }
    for (uint32_t i = lane; i < stride; i += 32) d[i] = i < dim ? s[i] : 0.0f;
}

/// Per node p (one warp): which of its list entries collect_undirected emits
/// (src/knn_graph.cpp:132-200): q valid, q != p, and, when q < p, p not in N(q)
/// (prefiltered by d(p,q) > the last distance of q).  Bit j of mask word j/32.
__global__ void k_edge_mask(const uint32_t* __restrict__ ids, const float* __restrict__ dists,
                            const uint32_t* __restrict__ counts, uint32_t n, uint32_t k,
                            uint32_t words, uint32_t* __restrict__ mask, uint32_t* __restrict__ cnt) {
    const uint32_t p = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    if (p >= n) return;
    const unsigned lane = threadIdx.x & 31u;
    const uint32_t c = counts[p];
    uint32_t total = 0;
    for (uint32_t w = 0; w < words; ++w) {
        const uint32_t j = w * 32 + lane;
        bool emit = false;
        if (j < c) {
            const uint32_t q = ids[static_cast<uint64_t>(p) * k + j];
            if (q != kInvalid && q != p && q < n) {
                emit = true;
                if (q < p) {
                    const uint32_t cq = counts[q];
                    if (cq > 0) {
                        const float d = dists[static_cast<uint64_t>(p) * k + j];
                        const float last = dists[static_cast<uint64_t>(q) * k + cq - 1];
                        if (!(d > last)) {
                            const uint32_t* J = ids + static_cast<uint64_t>(q) * k;
                            for (uint32_t t = 0; t < cq; ++t) {
                                if (J[t] == p) {
                                    emit = false;
                                    break;
                                }
                            }
                        }
                    }
                }
            } else if (q != kInvalid && q != p) {
                // q >= n cannot be reweighted (no core distance); the reference
                // would index out of range.  Such entries never arise from a
                // consistent graph; they are skipped.
                emit = false;
            }
        }
        const unsigned bits = __ballot_sync(0xFFFFFFFFu, emit);
        if (lane == 0) mask[static_cast<uint64_t>(p) * words + w] = bits;
        total += __popc(bits);
    }
    if (lane == 0) cnt[p] = total;
}

/// Write the emitted edges of node p at off[p]..: (min, max, w) with w the base
/// distance, or mrd_mpts(p,q) = max(w, max(core[p], core[q])) when core != null
/// (KnnGraph::mutual_reachability_edges, src/knn_graph.cpp:219-235).
__global__ void k_edge_emit(const uint32_t* __restrict__ ids, const float* __restrict__ dists,
                            uint32_t n, uint32_t k, uint32_t words, const uint32_t* __restrict__ mask,
                            const uint32_t* __restrict__ off, const float* __restrict__ core,
                            uint32_t* __restrict__ eu, uint32_t* __restrict__ ev, float* __restrict__ ew) {
    const uint32_t p = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    if (p >= n) return;
    const unsigned lane = threadIdx.x & 31u;
    uint32_t pos = off[p];
    for (uint32_t w = 0; w < words; ++w) {
        const uint32_t bits = mask[static_cast<uint64_t>(p) * words + w];
        const uint32_t j = w * 32 + lane;
        if (bits >> lane & 1u) {
            const uint32_t q = ids[static_cast<uint64_t>(p) * k + j];
            float d = dists[static_cast<uint64_t>(p) * k + j];
            if (core) d = max_ref(d, max_ref(core[p], core[q]));
            const uint32_t at = pos + __popc(bits & ((1u << lane) - 1u));
            eu[at] = p < q ? p : q;
            ev[at] = p < q ? q : p;
            ew[at] = d;
        }
        pos += __popc(bits);
    }
}

/// Bridges appended after the k-NN edges, reweighted from their base distance
/// (src/coresg.cpp:400-405); canonical orientation as the Edge constructor.
__global__ void k_bridge_emit(const cs_edge* __restrict__ br, uint64_t nb, const float* __restrict__ core,
                              uint32_t* __restrict__ eu, uint32_t* __restrict__ ev, float* __restrict__ ew) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= nb) return;
    const cs_edge e = br[i];
    float w = e.w;
    if (core) w = max_ref(w, max_ref(core[e.u], core[e.v]));
    eu[i] = e.u < e.v ? e.u : e.v;
    ev[i] = e.u < e.v ? e.v : e.u;
    ew[i] = w;
}

__global__ void k_core(const float* __restrict__ dists, const uint32_t* __restrict__ counts,
                       uint32_t n, uint32_t k, uint32_t mpts, float* __restrict__ core) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < n) core[v] = core_of(dists, counts, k, v, mpts);
}

__global__ void k_aos(const uint32_t* __restrict__ eu, const uint32_t* __restrict__ ev,
                      const float* __restrict__ ew, uint64_t m, cs_edge* __restrict__ out) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= m) return;
    cs_edge e;
    e.u = eu[i];
    e.v = ev[i];
    e.w = ew[i];
    out[i] = e;
}

}  // namespace

void launch_core(const Graph& g, uint32_t mpts, float* core, cudaStream_t s) {
    k_core<<<blocks_for(g.n), kThreads, 0, s>>>(g.dists.as<float>(), g.counts.as<uint32_t>(),
                                               static_cast<uint32_t>(g.n), g.k, mpts, core);
    count_launch(*g.ctx);
}

/// Enumerate (and optionally reweight) the CORE-SG edges into u/v/w.  Returns the
/// total count (k-NN edges + bridges).  tmp buffers are caller scratch.
uint64_t graph_materialize_edges(Graph& g, uint32_t mpts, bool reweight, DevBuf& u, DevBuf& v,
                                 DevBuf& w, DevBuf& core_buf, DevBuf& tmp_mask, DevBuf& tmp_cnt,
                                 DevBuf& tmp_off) {
    Ctx& c = *g.ctx;
    const uint32_t n = static_cast<uint32_t>(g.n);
    const uint32_t words = (g.k + 31) / 32;
    const uint64_t ns = scratch_nodes(g);
    tmp_mask.ensure(ns * words * sizeof(uint32_t) + 4);
    tmp_cnt.ensure((ns + 1) * sizeof(uint32_t));
    tmp_off.ensure((ns + 1) * sizeof(uint32_t));
    float* core = nullptr;
    if (reweight) {
        core_buf.ensure(static_cast<size_t>(n) * sizeof(float) + 4);
        core = core_buf.as<float>();
        launch_core(g, mpts, core, c.stream);
    }
    const unsigned warps_per_block = kThreads / 32;
    const unsigned nb = std::max(1u, (n + warps_per_block - 1) / warps_per_block);
    if (n) {
        k_edge_mask<<<nb, kThreads, 0, c.stream>>>(g.ids.as<uint32_t>(), g.dists.as<float>(),
                                                   g.counts.as<uint32_t>(), n, g.k, words,
                                                   tmp_mask.as<uint32_t>(), tmp_cnt.as<uint32_t>());
        count_launch(c);
    }
    scan_u32(c, tmp_cnt.as<uint32_t>(), tmp_off.as<uint32_t>(), n);
    uint32_t e_knn = 0;
    CSB_CUDA(cudaMemcpyAsync(&e_knn, tmp_off.as<uint32_t>() + n, sizeof(uint32_t),
                             cudaMemcpyDeviceToHost, c.stream));
    CSB_CUDA(cudaStreamSynchronize(c.stream));
    const uint64_t total = static_cast<uint64_t>(e_knn) + g.nb;
    if (total > 0xFFFFFFFEull) fail(CS_ERR_UNSUPPORTED, "edge count exceeds 32-bit edge indices");
    // the graph's cached edge list is sized for its capacity (it is rebuilt after
    // every insert): the k-NN edges scaled to it, and the bridges
    const uint64_t room = &u == &g.eu ? std::max(scratch_scale(g, e_knn) + g.nb, total) : total;
    u.ensure(room * sizeof(uint32_t) + 4);
    v.ensure(room * sizeof(uint32_t) + 4);
    w.ensure(room * sizeof(float) + 4);
    if (n && e_knn) {
        k_edge_emit<<<nb, kThreads, 0, c.stream>>>(g.ids.as<uint32_t>(), g.dists.as<float>(), n, g.k,
                                                   words, tmp_mask.as<uint32_t>(),
                                                   tmp_off.as<uint32_t>(), core, u.as<uint32_t>(),
                                                   v.as<uint32_t>(), w.as<float>());
        count_launch(c);
    }
    if (g.nb) {
        k_bridge_emit<<<blocks_for(g.nb), kThreads, 0, c.stream>>>(
            g.bridges.as<cs_edge>(), g.nb, core, u.as<uint32_t>() + e_knn, v.as<uint32_t>() + e_knn,
            w.as<float>() + e_knn);
        count_launch(c);
    }
    check_launch(c, "edge enumeration");
    return total;
}

void edges_reserve(Graph& g) {
    Ctx& c = *g.ctx;
    const uint64_t ns = scratch_nodes(g), words = (g.k + 31) / 32;
    // a mask that grows loses its contents: offsets counted against it are stale
    const void* mask_before = g.emask.p;
    g.emask.ensure(ns * words * sizeof(uint32_t) + 4);
    if (g.emask.p != mask_before) g.invalidate_edges();
    c.scratch[1].ensure((ns + 1) * sizeof(uint32_t));
    // the cached list: at most k edges per node, and the bridges; growing it drops
    // the cached edges, which are enumerated again when next needed
    const uint64_t room = ns * g.k + selection_bound(g);
    if (g.node_off.bytes < (ns + 1) * sizeof(uint32_t) || g.eu.bytes < room * sizeof(uint32_t) + 4) {
        g.node_off.ensure((ns + 1) * sizeof(uint32_t));
        g.eu.ensure(room * sizeof(uint32_t) + 4);
        g.ev.ensure(room * sizeof(uint32_t) + 4);
        g.ew.ensure(room * sizeof(float) + 4);
        g.invalidate_edges();
    }
}

void graph_build_edges(Graph& g) {
    if (g.edges_valid) return;
    Ctx& c = *g.ctx;
    // every endpoint of the edge list is a node of the graph: the k-NN edges by
    // construction (k_edge_mask), the bridges checked here (they may predate a
    // cs_graph_set_points that shrank the graph); the sweep relies on it
    if (g.nb) {
        std::vector<cs_edge> br(g.nb);
        copy_d2h(c, br.data(), g.bridges.p, g.nb * sizeof(cs_edge));
        for (const cs_edge& e : br) {
            if (e.u >= g.n || e.v >= g.n) fail(CS_ERR_STATE, "bridge endpoint out of range for the current graph");
        }
    }
    // only the bridges changed since the last enumeration: the k-NN edges and their
    // node offsets stand, and the bridge tail is written after them again
    if (g.knn_edges_valid && g.eu.bytes / sizeof(uint32_t) >= g.e_knn + g.nb + 1 &&
        g.e_knn + g.nb <= 0xFFFFFFFEull) {
        if (g.nb) {
            k_bridge_emit<<<blocks_for(g.nb), kThreads, 0, c.stream>>>(
                g.bridges.as<cs_edge>(), g.nb, nullptr, g.eu.as<uint32_t>() + g.e_knn,
                g.ev.as<uint32_t>() + g.e_knn, g.ew.as<float>() + g.e_knn);
            count_launch(c);
            check_launch(c, "bridge edges");
        }
        g.e_total = g.e_knn + g.nb;
        g.edges_valid = true;
        return;
    }
    // the k-NN edges' per-node offsets (counted by a bridge selection already, or now),
    // then the edges themselves in the reference order, then the bridges
    graph_count_knn_edges(g);
    const uint32_t n = static_cast<uint32_t>(g.n);
    const uint64_t e_knn = g.e_knn, total = e_knn + g.nb;
    if (total > 0xFFFFFFFEull) fail(CS_ERR_UNSUPPORTED, "edge count exceeds 32-bit edge indices");
    const uint64_t room = std::max(scratch_scale(g, e_knn) + g.nb, total);
    g.eu.ensure(room * sizeof(uint32_t) + 4);
    g.ev.ensure(room * sizeof(uint32_t) + 4);
    g.ew.ensure(room * sizeof(float) + 4);
    const uint32_t words = (g.k + 31) / 32;
    const unsigned warps_per_block = kThreads / 32;
    const unsigned nb = std::max(1u, (n + warps_per_block - 1) / warps_per_block);
    if (n && e_knn) {
        k_edge_emit<<<nb, kThreads, 0, c.stream>>>(g.ids.as<uint32_t>(), g.dists.as<float>(), n, g.k, words,
                                                   g.emask.as<uint32_t>(), g.node_off.as<uint32_t>(), nullptr,
                                                   g.eu.as<uint32_t>(), g.ev.as<uint32_t>(), g.ew.as<float>());
        count_launch(c);
    }
    if (g.nb) {
        k_bridge_emit<<<blocks_for(g.nb), kThreads, 0, c.stream>>>(
            g.bridges.as<cs_edge>(), g.nb, nullptr, g.eu.as<uint32_t>() + e_knn, g.ev.as<uint32_t>() + e_knn,
            g.ew.as<float>() + e_knn);
        count_launch(c);
    }
    check_launch(c, "edge enumeration");
    g.e_total = total;
    g.edges_valid = g.knn_edges_valid = true;
}

void graph_count_knn_edges(Graph& g) {
    if (g.knn_edges_valid || g.knn_offsets_valid) return;
    Ctx& c = *g.ctx;
    const uint32_t n = static_cast<uint32_t>(g.n);
    const uint32_t words = (g.k + 31) / 32;
    const uint64_t ns = scratch_nodes(g);
    g.emask.ensure(ns * words * sizeof(uint32_t) + 4);
    c.scratch[1].ensure((ns + 1) * sizeof(uint32_t));
    g.node_off.ensure((ns + 1) * sizeof(uint32_t));
    const unsigned warps_per_block = kThreads / 32;
    const unsigned nb = std::max(1u, (n + warps_per_block - 1) / warps_per_block);
    if (n) {
        k_edge_mask<<<nb, kThreads, 0, c.stream>>>(g.ids.as<uint32_t>(), g.dists.as<float>(), g.counts.as<uint32_t>(),
                                                   n, g.k, words, g.emask.as<uint32_t>(), c.scratch[1].as<uint32_t>());
        count_launch(c);
    }
    scan_u32(c, c.scratch[1].as<uint32_t>(), g.node_off.as<uint32_t>(), n);
    uint32_t e_knn = 0;
    CSB_CUDA(cudaMemcpyAsync(&e_knn, g.node_off.as<uint32_t>() + n, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                             c.stream));
    CSB_CUDA(cudaStreamSynchronize(c.stream));
    g.e_knn = e_knn;
    g.knn_offsets_valid = true;
}

Graph::~Graph() {
    if (plan) sweep_free(plan);
}

void Graph::ensure_capacity(uint64_t need, bool keep) {
    if (need <= cap_n) return;
    uint64_t cap = std::max<uint64_t>(need, cap_n + cap_n / 2);
    cudaStream_t s = ctx->stream;
    if (keep) {
        pts.grow_keep(cap * stride * sizeof(float), s);
        ids.grow_keep(cap * k * sizeof(uint32_t), s);
        dists.grow_keep(cap * k * sizeof(float), s);
        flags.grow_keep(cap * k, s);
        counts.grow_keep(cap * sizeof(uint32_t), s);
    } else {
        pts.ensure(cap * stride * sizeof(float));
        ids.ensure(cap * k * sizeof(uint32_t));
        dists.ensure(cap * k * sizeof(float));
        flags.ensure(cap * k);
        counts.ensure(cap * sizeof(uint32_t));
    }
    cap_n = cap;
}

}  // namespace csb

// ============================================================================
// C API
// ============================================================================

using namespace csb;

extern "C" {

cs_status cs_graph_create(cs_ctx* ctx, uint32_t dim, uint32_t k_max, int32_t metric, cs_graph** out) {
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    return guarded(c, [&] {
        CSB_REQUIRE(out != nullptr, "cs_graph_create: null output");
        CSB_REQUIRE(dim > 0, "cs_graph_create: dim must be positive");
        CSB_REQUIRE(k_max > 0 && k_max <= static_cast<uint32_t>(kMaxK), "cs_graph_create: k_max must be in [1, 64]");
        if (metric != CS_METRIC_L2 && metric != CS_METRIC_COSINE)
            fail(CS_ERR_UNSUPPORTED, "cs_graph_create: only L2 and cosine run on the device");
        Graph* g = new Graph();
        g->ctx = c;
        ++c->live_graphs;
        g->dim = dim;
        g->k = k_max;
        g->stride = (dim + 7u) & ~7u;
        g->metric = metric;
        *out = reinterpret_cast<cs_graph*>(g);
    });
}

void cs_graph_destroy(cs_graph* gp) {
    Graph* g = reinterpret_cast<Graph*>(gp);
    if (!g) return;
    Ctx* c = g->ctx;
    bool free_ctx = false;
    {
        std::lock_guard<std::recursive_mutex> lk(c->mu);
        cudaSetDevice(c->device);  // no throw: may run at interpreter teardown
        delete g;
        cudaGetLastError();
        --c->live_graphs;
        free_ctx = c->destroy_pending && c->live_graphs == 0;
    }
    if (free_ctx) ctx_free(c);
}

}  // extern "C"

namespace csb {
void graph_set_points(Graph& gr, const float* rows, uint64_t n, uint32_t row_stride, bool append) {
    Graph* g = &gr;
    {
        CSB_REQUIRE(rows != nullptr || n == 0, "points: null rows");
        if (row_stride == 0) row_stride = g->dim;
        CSB_REQUIRE(row_stride >= g->dim, "points: row_stride < dim");
        const uint64_t first = append ? g->n : 0;
        const uint64_t total = first + n;
        CSB_REQUIRE(total < 0xFFFFFFFFull, "points: too many rows for 32-bit ids");
        Ctx& c = *g->ctx;
        g->ensure_capacity(total, append);
        if (n) {
            DevBuf& tmp = c.scratch[6];
            tmp.ensure(n * row_stride * sizeof(float));
            copy_h2d(c, tmp.p, rows, n * row_stride * sizeof(float));
            const unsigned wpb = kThreads / 32;
            k_pad_rows<<<static_cast<unsigned>((n + wpb - 1) / wpb), kThreads, 0, c.stream>>>(
                tmp.as<float>(), n, g->dim, row_stride, g->stride, g->metric,
                g->pts.as<float>() + first * g->stride);
            count_launch(c);
            check_launch(c, "pad rows");
        }
        if (!append) {
            g->knn_n = 0;
            g->hub_valid = false;  // new k-NN arrays: the next selection is a full one
        }
        // new nodes start with empty neighbourhoods (KnnGraph::grow)
        const uint64_t from = append ? g->knn_n : 0;
        if (total > from) {
            CSB_CUDA(cudaMemsetAsync(g->ids.as<uint32_t>() + from * g->k, 0xFF, (total - from) * g->k * 4, c.stream));
            CSB_CUDA(cudaMemsetAsync(g->flags.as<uint8_t>() + from * g->k, 0, (total - from) * g->k, c.stream));
            CSB_CUDA(cudaMemsetAsync(g->counts.as<uint32_t>() + from, 0, (total - from) * 4, c.stream));
            // +inf = 0x7f800000: write via a pattern fill of the float array
            std::vector<float> inf_row(static_cast<size_t>(g->k), INFINITY);
            // fill with a small kernel-free approach: copy one row then double
            float* base = g->dists.as<float>() + from * g->k;
            const uint64_t rows_n = total - from;
            CSB_CUDA(cudaMemcpyAsync(base, inf_row.data(), g->k * sizeof(float), cudaMemcpyHostToDevice, c.stream));
            uint64_t done = 1;
            while (done < rows_n) {
                const uint64_t m = std::min(done, rows_n - done);
                CSB_CUDA(cudaMemcpyAsync(base + done * g->k, base, m * g->k * sizeof(float),
                                         cudaMemcpyDeviceToDevice, c.stream));
                done += m;
            }
            CSB_CUDA(cudaStreamSynchronize(c.stream));
        }
        g->n = total;
        g->knn_n = total;
        if (!append) {
            g->nb = 0;
            g->n_repair = 0;
        }
        g->invalidate_edges();
    }
}
}  // namespace csb

extern "C" {

static cs_status set_points_impl(Graph* g, const float* rows, uint64_t n, uint32_t row_stride, bool append) {
    return guarded(g ? g->ctx : nullptr, [&] { graph_set_points(*g, rows, n, row_stride, append); });
}

cs_status cs_graph_set_points(cs_graph* gp, const float* rows, uint64_t n, uint32_t row_stride) {
    return set_points_impl(reinterpret_cast<Graph*>(gp), rows, n, row_stride, false);
}

cs_status cs_graph_append_points(cs_graph* gp, const float* rows, uint64_t n, uint32_t row_stride) {
    return set_points_impl(reinterpret_cast<Graph*>(gp), rows, n, row_stride, true);
}

cs_status cs_graph_set_knn(cs_graph* gp, const uint32_t* ids, const float* dists, const uint8_t* flags,
                           const uint32_t* counts, uint64_t n) {
    Graph* g = reinterpret_cast<Graph*>(gp);
    return guarded(g ? g->ctx : nullptr, [&] {
        CSB_REQUIRE(ids && dists && counts, "cs_graph_set_knn: null array");
        CSB_REQUIRE(n < 0xFFFFFFFFull, "cs_graph_set_knn: too many nodes");
        Ctx& c = *g->ctx;
        if (g->n == 0 && n > 0) {
            // extraction-only use: no points; allocate the graph arrays alone
            g->ensure_capacity(n, false);
            g->n = n;
        }
        CSB_REQUIRE(n == g->n, "cs_graph_set_knn: n differs from the resident point count");
        for (uint64_t i = 0; i < n; ++i) {
            if (counts[i] > g->k) fail(CS_ERR_INVALID, "cs_graph_set_knn: count exceeds k_max");
        }
        copy_h2d(c, g->ids.p, ids, n * g->k * sizeof(uint32_t));
        copy_h2d(c, g->dists.p, dists, n * g->k * sizeof(float));
        if (flags) copy_h2d(c, g->flags.p, flags, n * g->k);
        else CSB_CUDA(cudaMemsetAsync(g->flags.p, 0, n * g->k, c.stream));
        copy_h2d(c, g->counts.p, counts, n * sizeof(uint32_t));
        g->knn_n = n;
        g->hub_valid = false;
        g->invalidate_edges();
    });
}

cs_status cs_graph_get_knn(cs_graph* gp, uint32_t* ids, float* dists, uint8_t* flags, uint32_t* counts) {
    Graph* g = reinterpret_cast<Graph*>(gp);
    return guarded(g ? g->ctx : nullptr, [&] {
        Ctx& c = *g->ctx;
        if (ids) copy_d2h(c, ids, g->ids.p, g->n * g->k * sizeof(uint32_t));
        if (dists) copy_d2h(c, dists, g->dists.p, g->n * g->k * sizeof(float));
        if (flags) copy_d2h(c, flags, g->flags.p, g->n * g->k);
        if (counts) copy_d2h(c, counts, g->counts.p, g->n * sizeof(uint32_t));
    });
}

cs_status cs_graph_set_bridges(cs_graph* gp, const cs_edge* edges, uint64_t m) {
    Graph* g = reinterpret_cast<Graph*>(gp);
    return guarded(g ? g->ctx : nullptr, [&] {
        CSB_REQUIRE(edges != nullptr || m == 0, "cs_graph_set_bridges: null edges");
        for (uint64_t i = 0; i < m; ++i) {
            if (edges[i].u >= g->n || edges[i].v >= g->n)
                fail(CS_ERR_INVALID, "cs_graph_set_bridges: endpoint out of range");
        }
        g->bridges.ensure(std::max<uint64_t>(m, 1) * sizeof(cs_edge));
        copy_h2d(*g->ctx, g->bridges.p, edges, m * sizeof(cs_edge));
        g->nb = m;
        g->invalidate_bridges();
    });
}

cs_status cs_graph_get_bridges(cs_graph* gp, cs_edge* out, uint64_t cap, uint64_t* out_count) {
    Graph* g = reinterpret_cast<Graph*>(gp);
    return guarded(g ? g->ctx : nullptr, [&] {
        if (out_count) *out_count = g->nb;
        if (out && cap) copy_d2h(*g->ctx, out, g->bridges.p, std::min(cap, g->nb) * sizeof(cs_edge));
    });
}

cs_status cs_graph_info(cs_graph* gp, uint64_t* n, uint32_t* k_max, uint32_t* dim, uint32_t* stride,
                        uint64_t* knn_edges, uint64_t* bridges) {
    Graph* g = reinterpret_cast<Graph*>(gp);
    return guarded(g ? g->ctx : nullptr, [&] {
        if (knn_edges) {
            graph_build_edges(*g);
            *knn_edges = g->e_knn;
        }
        if (n) *n = g->n;
        if (k_max) *k_max = g->k;
        if (dim) *dim = g->dim;
        if (stride) *stride = g->stride;
        if (bridges) *bridges = g->nb;
    });
}

cs_status cs_graph_reserve(cs_graph* gp, uint64_t rows) {
    Graph* g = reinterpret_cast<Graph*>(gp);
    return guarded(g ? g->ctx : nullptr, [&] {
        CSB_REQUIRE(rows < 0xFFFFFFFFull, "cs_graph_reserve: too many rows for 32-bit ids");
        if (rows > g->cap_n) g->ensure_capacity(rows, true);
        knn_reserve(*g);
        bridges_reserve(*g);
        edges_reserve(*g);
    });
}

cs_status cs_core_distances(cs_graph* gp, uint32_t mpts, float* host_out) {
    Graph* g = reinterpret_cast<Graph*>(gp);
    return guarded(g ? g->ctx : nullptr, [&] {
        CSB_REQUIRE(host_out != nullptr, "cs_core_distances: null output");
        Ctx& c = *g->ctx;
        if (mpts > g->k) mpts = g->k;  // CoreSG::core_distances clamps to k_max
        DevBuf& tmp = c.scratch[5];
        tmp.ensure(std::max<uint64_t>(g->n, 1) * sizeof(float));
        if (g->n) launch_core(*g, mpts, tmp.as<float>(), c.stream);
        check_launch(c, "core distances");
        copy_d2h(c, host_out, tmp.p, g->n * sizeof(float));
    });
}

cs_status cs_edges(cs_graph* gp, uint32_t mpts, cs_edge* host_out, uint64_t cap, uint64_t* out_count) {
    Graph* g = reinterpret_cast<Graph*>(gp);
    return guarded(g ? g->ctx : nullptr, [&] {
        if (mpts == 0) mpts = 1;
        if (mpts > g->k) fail(CS_ERR_INVALID, "CoreSG::edges: mpts exceeds k_max");
        Ctx& c = *g->ctx;
        DevBuf u, v, w, core;
        const uint64_t m = graph_materialize_edges(*g, mpts, true, u, v, w, core, c.scratch[0],
                                                   c.scratch[1], c.scratch[2]);
        if (out_count) *out_count = m;
        if (host_out && cap) {
            const uint64_t wr = std::min(cap, m);
            DevBuf aos;
            aos.ensure(std::max<uint64_t>(wr, 1) * sizeof(cs_edge));
            k_aos<<<blocks_for(wr), kThreads, 0, c.stream>>>(u.as<uint32_t>(), v.as<uint32_t>(),
                                                              w.as<float>(), wr, aos.as<cs_edge>());
            count_launch(c);
            check_launch(c, "edges aos");
            copy_d2h(c, host_out, aos.p, wr * sizeof(cs_edge));
        }
    });
}

}  // extern "C"
