// Test infrastructure only: a C ABI over the reference implementation's own CPU
// code path (coresg::CoreSG and friends), compiled from the reference sources by
// oracle/Makefile.  Python tests, the golden-fixture script and bench.py's CPU
// legs load it with ctypes.  Nothing in the product links or loads this file.
//
// Every entry point forwards to the reference's public API; the only logic here
// is marshalling (and writing a CORESG01 file so CoreSG::load can adopt a given
// state, following the format of src/io.cpp:195-261).

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <memory>
#include <stdexcept>
#include <string>
#include <unistd.h>
#include <vector>

#include "coresg/coresg.hpp"
#include "coresg/eval.hpp"
#include "coresg/io.hpp"
#include "coresg/mst.hpp"
#include "coresg/nndescent.hpp"
#include "coresg/thread_pool.hpp"

using namespace coresg;

extern "C" float refd_metric_distance_l2(const float* a, const float* b, std::uint32_t stride);
extern "C" float refd_metric_distance(int metric, const float* a, const float* b, std::uint32_t stride);

namespace {

thread_local std::string g_err;

struct Handle {
    std::unique_ptr<CoreSG> sg;
    CoreSGStats stats;
};

CoreSGParams make_params(std::uint32_t k_max, std::uint32_t instances, std::uint32_t iters,
                         std::uint32_t sample, std::uint64_t seed, unsigned threads, int metric = 0) {
    // Mirrors coresg_cli build (apps/coresg_cli.cpp:81-177) with --gpu 0.
    CoreSGParams p;
    p.k_max = k_max;
    p.metric = static_cast<MetricKind>(metric);
    p.threads = threads;
    p.seed = seed;
    p.backend.prefer_gpu = false;
    p.incr.instances = instances;
    p.incr.instance_nnd.k = k_max;
    p.incr.instance_nnd.sample = sample;
    p.incr.instance_nnd.iters = iters;
    p.incr.refine_nnd.k = k_max;
    p.incr.refine_nnd.sample = sample;
    p.incr.refine_nnd.iters = 5;
    p.incr.refine_per_new = 2.0;
    return p;
}

double since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

template <typename T>
void put(std::ofstream& os, const T& v) {
    os.write(reinterpret_cast<const char*>(&v), sizeof(T));
}

template <typename T>
void put_vec(std::ofstream& os, const T* data, std::uint64_t count) {
    put(os, count);
    if (count) os.write(reinterpret_cast<const char*>(data), std::streamsize(count * sizeof(T)));
}

}  // namespace

extern "C" {

const char* ref_last_error() { return g_err.c_str(); }

float ref_metric_distance(const float* a, const float* b, std::uint32_t stride) {
    return refd_metric_distance_l2(a, b, stride);
}

/// metric_distance under metric code `metric` (MetricKind order: 0 L2, 1 cosine).
float ref_metric_distance_m(int metric, const float* a, const float* b, std::uint32_t stride) {
    return refd_metric_distance(metric, a, b, stride);
}

/// The padded rows Dataset::append stores for `n` rows of `dim` floats under
/// `metric` (cosine rows are L2-normalised, dataset.hpp normalise).
void ref_dataset_rows(const float* rows, std::uint64_t n, std::uint32_t dim, int metric, float* out_padded) {
    Dataset data(dim, static_cast<MetricKind>(metric));
    data.append(rows, static_cast<std::size_t>(n));
    std::memcpy(out_padded, data.data(), n * data.stride() * sizeof(float));
}

/// CoreSG::build over `n` rows of `dim` floats (reference path, CPU backend) under
/// metric code `metric`.
void* ref_build_m(const float* rows, std::uint64_t n, std::uint32_t dim, std::uint32_t k_max,
                  std::uint32_t instances, std::uint32_t iters, std::uint32_t sample,
                  std::uint64_t seed, std::uint32_t threads, int metric, double* times4) {
    try {
        auto h = std::make_unique<Handle>();
        h->sg = std::make_unique<CoreSG>(make_params(k_max, instances, iters, sample, seed, threads, metric));
        h->stats = h->sg->build(rows, static_cast<std::size_t>(n), dim);
        if (times4) {
            times4[0] = h->stats.knn_seconds;
            times4[1] = h->stats.hubness_seconds;
            times4[2] = h->stats.missing_seconds + h->stats.repair_seconds;
            times4[3] = h->stats.total_seconds;
        }
        return h.release();
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

/// CoreSG::build under L2.
void* ref_build(const float* rows, std::uint64_t n, std::uint32_t dim, std::uint32_t k_max,
                std::uint32_t instances, std::uint32_t iters, std::uint32_t sample,
                std::uint64_t seed, std::uint32_t threads, double* times4) {
    return ref_build_m(rows, n, dim, k_max, instances, iters, sample, seed, threads, 0, times4);
}

/// CoreSG::insert of `count` further rows.
int ref_insert(void* hp, const float* rows, std::uint64_t count, double* total_seconds) {
    try {
        Handle* h = static_cast<Handle*>(hp);
        CoreSGStats st = h->sg->insert(rows, static_cast<std::size_t>(count));
        if (total_seconds) *total_seconds = st.total_seconds;
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

/// Adopt a given state (padded points, k-NN arrays, bridges) through CoreSG::load,
/// which re-derives connectivity and hubness exactly as `coresg_cli extract` does.
void* ref_from_state_m(const float* padded, std::uint64_t n, std::uint32_t dim,
                       std::uint32_t stride, std::uint32_t k_max, const std::uint32_t* ids,
                       const float* dists, const std::uint8_t* flags, const std::uint32_t* counts,
                       const void* bridges, std::uint64_t n_bridges, std::uint64_t repair,
                       std::uint32_t threads, int metric) {
    char path[] = "/tmp/coresg_ref_XXXXXX";
    const int fd = mkstemp(path);
    if (fd < 0) {
        g_err = "mkstemp failed";
        return nullptr;
    }
    close(fd);
    try {
        {
            std::ofstream os(path, std::ios::binary);
            const char magic[8] = {'C', 'O', 'R', 'E', 'S', 'G', '0', '1'};
            os.write(magic, 8);
            put(os, k_max);
            put(os, dim);
            put(os, stride);
            put(os, std::uint32_t(metric));
            put(os, std::uint32_t(0));  // missing mode AntiHub
            put(os, std::uint64_t(n));
            put_vec(os, padded, n * stride);
            put_vec(os, ids, n * k_max);
            put_vec(os, dists, n * k_max);
            put_vec(os, flags, n * k_max);
            put_vec(os, counts, n);
            put_vec(os, static_cast<const Edge*>(bridges), n_bridges);
            put(os, std::uint64_t(repair));
        }
        auto h = std::make_unique<Handle>();
        h->sg = std::make_unique<CoreSG>(make_params(k_max, 1, 10, 16, 42, threads, metric));
        h->sg->load(path);
        std::remove(path);
        return h.release();
    } catch (const std::exception& e) {
        std::remove(path);
        g_err = e.what();
        return nullptr;
    }
}

/// ref_from_state_m under L2.
void* ref_from_state(const float* padded, std::uint64_t n, std::uint32_t dim,
                     std::uint32_t stride, std::uint32_t k_max, const std::uint32_t* ids,
                     const float* dists, const std::uint8_t* flags, const std::uint32_t* counts,
                     const void* bridges, std::uint64_t n_bridges, std::uint64_t repair,
                     std::uint32_t threads) {
    return ref_from_state_m(padded, n, dim, stride, k_max, ids, dists, flags, counts, bridges, n_bridges, repair,
                            threads, 0);
}

void ref_free(void* hp) { delete static_cast<Handle*>(hp); }

// coresg::write_edges_tsv / write_labels_tsv (src/io.cpp:131-145) on caller arrays
int ref_write_edges_tsv(const char* path, const void* edges, std::uint64_t m) {
    try {
        const auto* e = static_cast<const coresg::Edge*>(edges);
        coresg::write_edges_tsv(path, std::vector<coresg::Edge>(e, e + m));
        return 0;
    } catch (const std::exception& ex) {
        g_err = ex.what();
        return 1;
    }
}

int ref_write_labels_tsv(const char* path, const std::uint32_t* labels, std::uint64_t n) {
    try {
        coresg::write_labels_tsv(path, std::vector<coresg::idx_t>(labels, labels + n));
        return 0;
    } catch (const std::exception& ex) {
        g_err = ex.what();
        return 1;
    }
}

int ref_save(void* hp, const char* path) {
    try {
        static_cast<Handle*>(hp)->sg->save(path);
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

void* ref_load(const char* path, std::uint32_t threads) {
    try {
        auto h = std::make_unique<Handle>();
        h->sg = std::make_unique<CoreSG>(make_params(32, 1, 10, 16, 42, threads));
        h->sg->load(path);
        return h.release();
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

std::uint64_t ref_n(void* hp) { return static_cast<Handle*>(hp)->sg->knn().size(); }
std::uint32_t ref_k(void* hp) { return static_cast<Handle*>(hp)->sg->knn().k(); }
std::uint32_t ref_stride(void* hp) { return static_cast<Handle*>(hp)->sg->data().stride(); }

void ref_get_points(void* hp, float* padded) {
    const Dataset& d = static_cast<Handle*>(hp)->sg->data();
    std::memcpy(padded, d.data(), d.size() * d.stride() * sizeof(float));
}

void ref_get_knn(void* hp, std::uint32_t* ids, float* dists, std::uint8_t* flags,
                 std::uint32_t* counts) {
    const KnnGraph& g = static_cast<Handle*>(hp)->sg->knn();
    const std::size_t nk = std::size_t(g.size()) * g.k();
    if (ids) std::memcpy(ids, g.ids_storage().data(), nk * sizeof(std::uint32_t));
    if (dists) std::memcpy(dists, g.dist_storage().data(), nk * sizeof(float));
    if (flags) std::memcpy(flags, g.flag_storage().data(), nk);
    if (counts) std::memcpy(counts, g.count_storage().data(), g.size() * sizeof(std::uint32_t));
}

std::uint64_t ref_bridges(void* hp, void* out) {
    const std::vector<Edge>& m = static_cast<Handle*>(hp)->sg->missing_edges();
    if (out) std::memcpy(out, m.data(), m.size() * sizeof(Edge));
    return m.size();
}

std::uint64_t ref_repair_count(void* hp) { return static_cast<Handle*>(hp)->sg->repair_edge_count(); }

/// Anti-hub selection (HubnessIndex::selected), scores and reverse degrees.
std::uint64_t ref_selected(void* hp, std::uint32_t* out) {
    const std::vector<idx_t>& s = static_cast<Handle*>(hp)->sg->hubness().selected();
    if (out) std::memcpy(out, s.data(), s.size() * sizeof(std::uint32_t));
    return s.size();
}

void ref_scores(void* hp, double* score, std::int32_t* rdeg) {
    const HubnessIndex& hub = static_cast<Handle*>(hp)->sg->hubness();
    const idx_t n = static_cast<Handle*>(hp)->sg->knn().size();
    for (idx_t v = 0; v < n; ++v) {
        if (score) score[v] = hub.reverse_score(v);
        if (rdeg) rdeg[v] = static_cast<std::int32_t>(hub.reverse_degree(v));
    }
}

std::uint32_t ref_conn_labels(void* hp, std::uint32_t* labels) {
    const ConnectivityTracker& c = static_cast<Handle*>(hp)->sg->connectivity();
    if (labels) std::memcpy(labels, c.labels().data(), c.labels().size() * sizeof(std::uint32_t));
    return c.components();
}

/// CoreSG::core_distances(mpts).
void ref_core(void* hp, std::uint32_t mpts, float* out) {
    const std::vector<dist_t> c = static_cast<Handle*>(hp)->sg->core_distances(mpts);
    std::memcpy(out, c.data(), c.size() * sizeof(float));
}

/// CoreSG::edges(mpts): count, and the list itself when `out` is non-null.
std::uint64_t ref_edges(void* hp, std::uint32_t mpts, void* out) {
    try {
        const std::vector<Edge> e = static_cast<Handle*>(hp)->sg->edges(mpts);
        if (out) std::memcpy(out, e.data(), e.size() * sizeof(Edge));
        return e.size();
    } catch (const std::exception& e) {
        g_err = e.what();
        return ~std::uint64_t(0);
    }
}

/// MST over CoreSG::edges(mpts).
///   algo 0: CoreSG::mst (mst_from_edges with the CoreSG's own pool; all-in timing
///           covers edges() + the MST, like `coresg_cli extract`)
///   algo 1: mst_boruvka with a pool of `threads`
///   algo 2: mst_kruskal
/// `out_edges` receives the tree in the reference's discovery order.
int ref_mst(void* hp, std::uint32_t mpts, int algo, std::uint32_t threads, void* out_edges,
            std::uint32_t* out_labels, std::uint32_t* out_ncomp, std::uint64_t* out_nedges,
            double* out_weight, double* out_seconds_mst, double* out_seconds_all) {
    try {
        Handle* h = static_cast<Handle*>(hp);
        const idx_t n = h->sg->knn().size();
        MstResult r;
        const auto t0 = std::chrono::steady_clock::now();
        if (algo == 0) {
            r = h->sg->mst(mpts);
        } else {
            const std::vector<Edge> e = h->sg->edges(mpts);
            if (algo == 1) {
                ThreadPool pool(threads ? threads : 4);
                r = mst_boruvka(e, n, &pool);
            } else {
                r = mst_kruskal(e, n);
            }
        }
        const double all = since(t0);
        if (out_edges) std::memcpy(out_edges, r.edges.data(), r.edges.size() * sizeof(Edge));
        if (out_labels) std::memcpy(out_labels, r.component.data(), r.component.size() * sizeof(std::uint32_t));
        if (out_ncomp) *out_ncomp = r.num_components;
        if (out_nedges) *out_nedges = r.edges.size();
        if (out_weight) *out_weight = r.weight;
        if (out_seconds_mst) *out_seconds_mst = r.seconds;
        if (out_seconds_all) *out_seconds_all = all;
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

/// MST of an arbitrary edge list (coresg::Edge layout) with the reference's
/// Boruvka (algo 1, pool of `threads`) or Kruskal (algo 2).
int ref_mst_edges(const void* edges, std::uint64_t m, std::uint32_t n, int algo,
                  std::uint32_t threads, void* out_edges, std::uint32_t* out_labels,
                  std::uint32_t* out_ncomp, std::uint64_t* out_nedges, double* out_weight) {
    try {
        const Edge* e = static_cast<const Edge*>(edges);
        std::vector<Edge> list(e, e + m);
        MstResult r;
        if (algo == 1) {
            ThreadPool pool(threads ? threads : 4);
            r = mst_boruvka(list, n, &pool);
        } else {
            r = mst_kruskal(list, n);
        }
        if (out_edges) std::memcpy(out_edges, r.edges.data(), r.edges.size() * sizeof(Edge));
        if (out_labels) std::memcpy(out_labels, r.component.data(), r.component.size() * sizeof(std::uint32_t));
        if (out_ncomp) *out_ncomp = r.num_components;
        if (out_nedges) *out_nedges = r.edges.size();
        if (out_weight) *out_weight = r.weight;
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

/// mst_dense (Prim, lowest index wins ties) over an m x m row-major matrix.
std::uint64_t ref_mst_dense(const float* matrix, std::uint64_t m, void* out_edges) {
    MstResult r = mst_dense(matrix, static_cast<std::size_t>(m));
    if (out_edges) std::memcpy(out_edges, r.edges.data(), r.edges.size() * sizeof(Edge));
    return r.edges.size();
}

/// sampled_recall (src/eval.cpp:24-105) of a given graph.
double ref_sampled_recall(const float* rows, std::uint64_t n, std::uint32_t dim,
                          const std::uint32_t* ids, const float* dists,
                          const std::uint32_t* counts, std::uint32_t k, std::uint64_t queries,
                          std::uint64_t seed, std::uint32_t threads) {
    Dataset data(dim, MetricKind::L2);
    data.append(rows, static_cast<std::size_t>(n));
    KnnGraph g(static_cast<idx_t>(n), k);
    std::memcpy(g.ids_storage().data(), ids, n * k * sizeof(std::uint32_t));
    std::memcpy(g.dist_storage().data(), dists, n * k * sizeof(float));
    std::memcpy(g.count_storage().data(), counts, n * sizeof(std::uint32_t));
    ThreadPool pool(threads ? threads : 1);
    return sampled_recall(data, g, k, static_cast<std::size_t>(queries), seed, &pool).recall;
}

/// The reference's CPU NN-Descent alone (init_random + nndescent), as the CPU
/// backend runs one k-NN job (src/cpu_backend.cpp:47-59).
int ref_nndescent_m(const float* rows, std::uint64_t n, std::uint32_t dim, std::uint32_t k,
                    std::uint32_t sample, std::uint32_t iters, double delta, std::uint64_t seed,
                    std::uint32_t threads, int metric, std::uint32_t* ids, float* dists,
                    std::uint32_t* counts, std::uint64_t* evals, double* seconds) {
    try {
        Dataset data(dim, static_cast<MetricKind>(metric));
        data.append(rows, static_cast<std::size_t>(n));
        KnnGraph g(static_cast<idx_t>(n), k);
        ThreadPool pool(threads ? threads : 1);
        NNDescentParams p;
        p.k = k;
        p.sample = sample;
        p.iters = iters;
        p.delta = delta;
        p.seed = seed;
        const auto t0 = std::chrono::steady_clock::now();
        init_random(data.view(), data.metric(), &g, seed, &pool);
        NNDescentStats st = nndescent(data.view(), data.metric(), &g, p, &pool);
        if (seconds) *seconds = since(t0);
        if (evals) *evals = st.distance_evals;
        std::memcpy(ids, g.ids_storage().data(), n * k * sizeof(std::uint32_t));
        std::memcpy(dists, g.dist_storage().data(), n * k * sizeof(float));
        std::memcpy(counts, g.count_storage().data(), n * sizeof(std::uint32_t));
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

/// ref_nndescent_m under L2.
int ref_nndescent(const float* rows, std::uint64_t n, std::uint32_t dim, std::uint32_t k,
                  std::uint32_t sample, std::uint32_t iters, double delta, std::uint64_t seed,
                  std::uint32_t threads, std::uint32_t* ids, float* dists,
                  std::uint32_t* counts, std::uint64_t* evals, double* seconds) {
    return ref_nndescent_m(rows, n, dim, k, sample, iters, delta, seed, threads, 0, ids, dists, counts, evals,
                           seconds);
}

}  // extern "C"
