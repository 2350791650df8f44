// Test infrastructure: the reference-side binding a maintainer adds to adopt the
// engine, compiled against the reference's own headers and objects by
// oracle/Makefile (target `binding`) so that the code shown in INTEGRATION.md is
// known to build, link and run.
//
//   B200Backend      a coresg::Backend (include/coresg/backend.hpp:72-92) with the
//                    KnnJob semantics of CudaBackend::run_knn_job
//                    (src/cuda_backend.cpp:60-109) and its mrd_block (:111-123),
//                    over cs_nndescent / cs_mrd_block; no CPU fallback: an OOM is
//                    recorded in the job, any other failure throws.
//   B200Extractor    the extraction hook of CoreSG::mst / all_msts
//                    (src/coresg.cpp:408-417): a device copy of the CoreSG's k-NN
//                    arrays and bridges, then cs_extract / cs_extract_sweep.
#include "b200_backend.hpp"

#include <stdexcept>
#include <string>

namespace coresg {
namespace {

class B200Backend : public Backend {
public:
    explicit B200Backend(const std::vector<int>& devices) {
        for (int id : devices) {
            cs_ctx* ctx = nullptr;
            if (cs_ctx_create(id, &ctx) != CS_OK)
                throw std::runtime_error(std::string("b200 device: ") + cs_last_error(nullptr));
            ctxs_.push_back(ctx);
            char name[256] = {0};
            size_t total = 0, free_b = 0;
            int32_t sms = 0, ma = 0, mi = 0;
            cs_device_props(id, name, sizeof name, &total, &free_b, &sms, &ma, &mi);
            DeviceInfo d;
            d.kind = DeviceKind::Cuda;
            d.id = id;
            d.name = name;
            d.total_memory = total;
            d.free_memory = free_b;
            d.multiprocessors = sms;
            d.cc_major = ma;
            d.cc_minor = mi;
            devices_.push_back(d);
        }
    }
    ~B200Backend() override {
        for (cs_ctx* c : ctxs_) cs_ctx_destroy(c);
    }

    std::string name() const override { return "b200"; }
    const std::vector<DeviceInfo>& devices() const override { return devices_; }
    unsigned parallelism() const override { return static_cast<unsigned>(ctxs_.size()); }

    void run_knn_job(unsigned slot, KnnJob& job) override {
        cs_nnd_config cfg{};
        cfg.n = static_cast<uint32_t>(job.local_n);
        cfg.dim = job.dim;
        cfg.stride = job.stride;
        cfg.k = job.graph.k();
        cfg.sample = job.params.sample;
        cfg.iters = job.params.iters;
        cfg.seed = job.params.seed + job.job_id * 0x9E3779B97F4A7C15ull;
        cfg.metric = job.metric == MetricKind::Cosine ? CS_METRIC_COSINE : CS_METRIC_L2;
        cfg.delta = static_cast<float>(job.params.delta);
        cfg.random_fill = 1;
        job.graph.grow(static_cast<idx_t>(job.local_n));
        uint64_t updates = 0;
        cs_ctx* ctx = ctxs_[slot < ctxs_.size() ? slot : 0];
        const cs_status st = cs_nndescent(ctx, &cfg, job.vectors.data(), job.graph.ids_storage().data(),
                                          job.graph.dist_storage().data(), job.graph.flag_storage().data(),
                                          job.graph.count_storage().data(), &updates);
        if (st == CS_ERR_OOM) {
            job.out_of_memory = true;
            job.error = cs_last_error(ctx);
            return;
        }
        if (st != CS_OK) throw std::runtime_error(std::string("b200 nndescent: ") + cs_last_error(ctx));
        job.ran_on = DeviceKind::Cuda;
        job.ran_on_device = devices_[slot < devices_.size() ? slot : 0].id;
        job.stats.rounds = job.params.iters;
        job.stats.updates = static_cast<std::size_t>(updates);
    }

    void mrd_block(unsigned slot, const float* pts, std::size_t m, std::uint32_t dim, std::uint32_t stride,
                   MetricKind metric, const float* core, std::size_t r0, std::size_t r1, float* out) override {
        cs_ctx* ctx = ctxs_[slot < ctxs_.size() ? slot : 0];
        const int32_t code = metric == MetricKind::Cosine ? CS_METRIC_COSINE : CS_METRIC_L2;
        if (cs_mrd_block(ctx, pts, m, dim, stride, code, core, r0, r1, out) != CS_OK)
            throw std::runtime_error(std::string("b200 mrd_block: ") + cs_last_error(ctx));
    }

    void trim() override {
        for (cs_ctx* c : ctxs_) cs_ctx_trim(c);
    }

private:
    std::vector<cs_ctx*> ctxs_;
    std::vector<DeviceInfo> devices_;
};

}  // namespace

std::unique_ptr<Backend> make_b200_backend(const std::vector<int>& ids) {
    return std::unique_ptr<Backend>(new B200Backend(ids));
}

B200Extractor::B200Extractor(int device) {
    if (cs_ctx_create(device, &ctx_) != CS_OK)
        throw std::runtime_error(std::string("b200 device: ") + cs_last_error(nullptr));
}

B200Extractor::~B200Extractor() {
    if (dev_) cs_graph_destroy(dev_);
    if (ctx_) cs_ctx_destroy(ctx_);
}

void B200Extractor::check(cs_status st, const char* what) const {
    if (st != CS_OK) throw std::runtime_error(std::string(what) + ": " + cs_last_error(ctx_));
}

void B200Extractor::sync(const CoreSG& sg) {
    const KnnGraph& knn = sg.knn();
    if (!dev_) {
        const int32_t metric = sg.data().metric() == MetricKind::Cosine ? CS_METRIC_COSINE : CS_METRIC_L2;
        check(cs_graph_create(ctx_, sg.data().dim(), knn.k(), metric, &dev_), "cs_graph_create");
    }
    check(cs_graph_set_knn(dev_, knn.ids_storage().data(), knn.dist_storage().data(), knn.flag_storage().data(),
                           knn.count_storage().data(), knn.size()),
          "cs_graph_set_knn");
    const std::vector<Edge>& missing = sg.missing_edges();
    check(cs_graph_set_bridges(dev_, reinterpret_cast<const cs_edge*>(missing.data()), missing.size()),
          "cs_graph_set_bridges");
    n_ = knn.size();
}

MstResult B200Extractor::mst(std::uint32_t mpts) const {
    MstResult r;
    r.edges.resize(n_ ? n_ - 1 : 0);
    r.component.resize(n_);
    uint64_t ne = 0;
    uint32_t nc = 0;
    check(cs_extract(dev_, mpts, reinterpret_cast<cs_edge*>(r.edges.data()), r.component.data(), &ne, &nc,
                     &r.weight),
          "cs_extract");
    r.edges.resize(ne);
    r.num_components = nc;
    return r;
}

std::vector<MstResult> B200Extractor::all_msts(const std::vector<std::uint32_t>& m) const {
    const std::size_t cap = n_ ? n_ - 1 : 0, K = m.size();
    std::vector<Edge> edges(K * cap);
    std::vector<idx_t> labels(K * n_);
    std::vector<uint64_t> ne(K);
    std::vector<uint32_t> nc(K);
    std::vector<double> w(K);
    check(cs_extract_sweep(dev_, m.data(), static_cast<uint32_t>(K), reinterpret_cast<cs_edge*>(edges.data()),
                           labels.data(), ne.data(), nc.data(), w.data()),
          "cs_extract_sweep");
    std::vector<MstResult> out(K);
    for (std::size_t j = 0; j < K; ++j) {
        out[j].edges.assign(edges.begin() + j * cap, edges.begin() + j * cap + ne[j]);
        out[j].component.assign(labels.begin() + j * n_, labels.begin() + (j + 1) * n_);
        out[j].num_components = nc[j];
        out[j].weight = w[j];
    }
    return out;
}

}  // namespace coresg
