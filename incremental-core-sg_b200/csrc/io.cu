// CORESG01 persistence of a resident CORE-SG, byte-compatible with the reference's
// CoreSG::save / CoreSG::load (src/io.cpp:195-330): magic "CORESG01"; u32 k_max, dim,
// stride, metric, missing-edge mode; u64 n; u64 float count + the padded rows; then
// length-prefixed (u64) vectors of ids, dists, flags, counts and bridge edges; u64
// repair count.  Like the reference, connectivity and hubness are not stored: they
// are derived state (cs_select_bridges recomputes them).
#include <cstdio>
#include <cstring>
#include <vector>

#include "engine.hpp"

namespace csb {
namespace {

const char kMagic[8] = {'C', 'O', 'R', 'E', 'S', 'G', '0', '1'};

struct File {
    FILE* f = nullptr;
    explicit File(FILE* x) : f(x) {}
    ~File() {
        if (f) std::fclose(f);
    }
};

template <typename T>
void put(FILE* f, const T& v) {
    if (std::fwrite(&v, sizeof(T), 1, f) != 1) fail(CS_ERR_INVALID, "CORESG01: write failed");
}

void put_bytes(FILE* f, const void* p, size_t bytes) {
    if (bytes && std::fwrite(p, 1, bytes, f) != bytes) fail(CS_ERR_INVALID, "CORESG01: write failed");
}

template <typename T>
void get(FILE* f, T* v) {
    if (std::fread(v, sizeof(T), 1, f) != 1) fail(CS_ERR_INVALID, "truncated coresg file");
}

void get_bytes(FILE* f, void* p, size_t bytes) {
    if (bytes && std::fread(p, 1, bytes, f) != bytes) fail(CS_ERR_INVALID, "truncated coresg file");
}

template <typename T>
std::vector<T> get_vec(FILE* f, uint64_t expect) {
    uint64_t count = 0;
    get(f, &count);
    if (count != expect) fail(CS_ERR_INVALID, "CORESG01: vector length does not match the header");
    std::vector<T> v(count);
    get_bytes(f, v.data(), count * sizeof(T));
    return v;
}

}  // namespace
/// write_edges_tsv (src/io.cpp:131-138): a "u\tv\tweight" header, then one line per
/// edge with the weight in std::scientific at precision 9 (the float widened to
/// double, as the stream formats it: printf's %.9e).
void write_edges_tsv_file(const char* path, const cs_edge* edges, uint64_t m) {
    File file(std::fopen(path, "wb"));
    if (!file.f) fail(CS_ERR_INVALID, std::string("cannot write ") + path);
    std::vector<char> buf(size_t(1) << 20);
    std::setvbuf(file.f, buf.data(), _IOFBF, buf.size());
    std::fputs("u\tv\tweight\n", file.f);
    for (uint64_t i = 0; i < m; ++i)
        std::fprintf(file.f, "%u\t%u\t%.9e\n", edges[i].u, edges[i].v, static_cast<double>(edges[i].w));
    if (std::fflush(file.f) != 0) fail(CS_ERR_INVALID, std::string("cannot write ") + path);
}

/// write_labels_tsv (src/io.cpp:140-145): an "id\tlabel" header, then "i\tlabel[i]".
void write_labels_tsv_file(const char* path, const uint32_t* labels, uint64_t n) {
    File file(std::fopen(path, "wb"));
    if (!file.f) fail(CS_ERR_INVALID, std::string("cannot write ") + path);
    std::vector<char> buf(size_t(1) << 20);
    std::setvbuf(file.f, buf.data(), _IOFBF, buf.size());
    std::fputs("id\tlabel\n", file.f);
    for (uint64_t i = 0; i < n; ++i)
        std::fprintf(file.f, "%llu\t%u\n", static_cast<unsigned long long>(i), labels[i]);
    if (std::fflush(file.f) != 0) fail(CS_ERR_INVALID, std::string("cannot write ") + path);
}

}  // namespace csb

using namespace csb;

extern "C" {

cs_status cs_graph_save(cs_graph* gp, const char* path) {
    Graph* g = reinterpret_cast<Graph*>(gp);
    return guarded(g ? g->ctx : nullptr, [&] {
        CSB_REQUIRE(path != nullptr, "cs_graph_save: null path");
        Ctx& c = *g->ctx;
        const uint64_t n = g->n, nk = n * g->k;
        std::vector<float> pts(n * g->stride);
        std::vector<uint32_t> ids(nk), counts(n);
        std::vector<float> dists(nk);
        std::vector<uint8_t> flags(nk);
        std::vector<cs_edge> br(g->nb);
        if (n) {
            copy_d2h(c, pts.data(), g->pts.p, pts.size() * 4);
            copy_d2h(c, ids.data(), g->ids.p, nk * 4);
            copy_d2h(c, dists.data(), g->dists.p, nk * 4);
            copy_d2h(c, flags.data(), g->flags.p, nk);
            copy_d2h(c, counts.data(), g->counts.p, n * 4);
        }
        if (g->nb) copy_d2h(c, br.data(), g->bridges.p, g->nb * sizeof(cs_edge));
        File file(std::fopen(path, "wb"));
        if (!file.f) fail(CS_ERR_INVALID, std::string("cannot write ") + path);
        FILE* f = file.f;
        put_bytes(f, kMagic, 8);
        put(f, g->k);
        put(f, g->dim);
        put(f, g->stride);
        put(f, static_cast<uint32_t>(g->metric));
        put(f, static_cast<uint32_t>(0));  // MissingEdgeMode::AntiHub
        put(f, n);
        put(f, static_cast<uint64_t>(pts.size()));
        put_bytes(f, pts.data(), pts.size() * 4);
        put(f, nk);
        put_bytes(f, ids.data(), nk * 4);
        put(f, nk);
        put_bytes(f, dists.data(), nk * 4);
        put(f, nk);
        put_bytes(f, flags.data(), nk);
        put(f, n);
        put_bytes(f, counts.data(), n * 4);
        put(f, static_cast<uint64_t>(g->nb));
        put_bytes(f, br.data(), g->nb * sizeof(cs_edge));
        put(f, static_cast<uint64_t>(g->n_repair));
    });
}

cs_status cs_graph_load(cs_ctx* ctx, const char* path, cs_graph** out) {
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    return guarded(c, [&] {
        CSB_REQUIRE(path != nullptr && out != nullptr, "cs_graph_load: null argument");
        *out = nullptr;
        File file(std::fopen(path, "rb"));
        if (!file.f) fail(CS_ERR_INVALID, std::string("cannot open ") + path);
        FILE* f = file.f;
        char magic[8] = {0};
        get_bytes(f, magic, 8);
        if (std::memcmp(magic, kMagic, 8) != 0) fail(CS_ERR_INVALID, std::string(path) + " is not a coresg file");
        uint32_t k = 0, dim = 0, stride = 0, metric = 0, mode = 0;
        uint64_t n = 0, floats = 0;
        get(f, &k);
        get(f, &dim);
        get(f, &stride);
        get(f, &metric);
        get(f, &mode);
        get(f, &n);
        if (k == 0 || k > 64 || dim == 0 || stride != ((dim + 7u) & ~7u))
            fail(CS_ERR_UNSUPPORTED, "CORESG01: k_max/dim/stride outside the device path");
        if (metric != CS_METRIC_L2 && metric != CS_METRIC_COSINE)
            fail(CS_ERR_UNSUPPORTED, "CORESG01: metric not on the device path");
        get(f, &floats);
        if (floats != n * stride) fail(CS_ERR_INVALID, "CORESG01: payload size does not match n*stride");
        std::vector<float> pts(floats);
        get_bytes(f, pts.data(), floats * 4);
        const uint64_t nk = n * k;
        const std::vector<uint32_t> ids = get_vec<uint32_t>(f, nk);
        const std::vector<float> dists = get_vec<float>(f, nk);
        const std::vector<uint8_t> flags = get_vec<uint8_t>(f, nk);
        const std::vector<uint32_t> counts = get_vec<uint32_t>(f, n);
        uint64_t nb = 0;
        get(f, &nb);
        std::vector<cs_edge> br(nb);
        get_bytes(f, br.data(), nb * sizeof(cs_edge));
        uint64_t repair = 0;
        get(f, &repair);
        cs_graph* gh = nullptr;
        cs_status st = cs_graph_create(ctx, dim, k, static_cast<int32_t>(metric), &gh);
        if (st != CS_OK) fail(st, cs_last_error(ctx));
        // rows are stored padded (and already normalised for cosine): upload them as-is
        st = cs_graph_set_points(gh, pts.data(), n, stride);
        if (st == CS_OK) st = cs_graph_set_knn(gh, ids.data(), dists.data(), flags.data(), counts.data(), n);
        if (st == CS_OK) st = cs_graph_set_bridges(gh, br.data(), nb);
        if (st != CS_OK) {
            const std::string msg = cs_last_error(ctx);
            cs_graph_destroy(gh);
            fail(st, msg);
        }
        reinterpret_cast<Graph*>(gh)->n_repair = repair;
        *out = gh;
    });
}

cs_status cs_write_edges_tsv(const char* path, const cs_edge* edges, uint64_t m) {
    return host_guarded([&] {
        CSB_REQUIRE(path != nullptr && (edges != nullptr || m == 0), "cs_write_edges_tsv: null argument");
        write_edges_tsv_file(path, edges, m);
    });
}

cs_status cs_write_labels_tsv(const char* path, const uint32_t* labels, uint64_t n) {
    return host_guarded([&] {
        CSB_REQUIRE(path != nullptr && (labels != nullptr || n == 0), "cs_write_labels_tsv: null argument");
        write_labels_tsv_file(path, labels, n);
    });
}

cs_status cs_sweep_write_tsv(cs_graph* gp, uint32_t index, const char* edges_path, const char* labels_path) {
    Graph* g = reinterpret_cast<Graph*>(gp);
    return guarded(g ? g->ctx : nullptr, [&] {
        MstHost r;
        sweep_fetch(*g, index, nullptr, nullptr, &r);  // sizes: the sweep's node count is edges + components
        const uint64_t n = r.nedges + r.ncomp;
        std::vector<cs_edge> edges(edges_path ? r.nedges : 0);
        std::vector<uint32_t> labels(labels_path ? n : 0);
        sweep_fetch(*g, index, edges_path ? edges.data() : nullptr, labels_path ? labels.data() : nullptr, &r);
        if (edges_path) write_edges_tsv_file(edges_path, edges.data(), r.nedges);
        if (labels_path) write_labels_tsv_file(labels_path, labels.data(), n);
    });
}

}  // extern "C"
