// Test infrastructure: a C ABI over the compiled binding (b200_backend.cpp) for the
// Python tests.  Each entry drives the binding through the reference's own call
// path: k-NN jobs through coresg::JobScheduler::run_all (include/coresg/backend.hpp:
// 139-147) onto B200Backend::run_knn_job, dense MRD rows through
// JobScheduler::mrd_matrix, and MSTs of a CORE-SG that coresg::CoreSG::load read from
// a CORESG01 file through B200Extractor.
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "b200_backend.hpp"
#include "coresg/dataset.hpp"

using namespace coresg;

namespace {
thread_local std::string g_err;
}

extern "C" {

const char* bb_last_error() { return g_err.c_str(); }

/// One KnnJob over `n` rows of `dim` floats through JobScheduler + B200Backend on
/// `device`; the job's graph (metric units) into ids/dists/counts.  Returns 0, or 1
/// with bb_last_error(); *out_oom and *out_ran_on_cuda report the job's outcome.
int bb_knn_job(const float* rows, std::uint64_t n, std::uint32_t dim, std::uint32_t k, std::uint32_t sample,
               std::uint32_t iters, std::uint64_t seed, int metric, int device, std::uint32_t* ids, float* dists,
               std::uint32_t* counts, int* out_oom, int* out_ran_on_cuda) {
    try {
        Dataset data(dim, static_cast<MetricKind>(metric));
        data.append(rows, static_cast<std::size_t>(n));
        std::vector<KnnJob> jobs(1);
        KnnJob& job = jobs[0];
        job.vectors.assign(data.data(), data.data() + n * data.stride());
        job.dim = dim;
        job.stride = data.stride();
        job.local_n = static_cast<std::size_t>(n);
        job.metric = static_cast<MetricKind>(metric);
        job.params.k = k;
        job.params.sample = sample;
        job.params.iters = iters;
        job.params.seed = seed;
        job.graph.reset(static_cast<idx_t>(n), k);
        job.job_id = 0;
        std::unique_ptr<Backend> be = make_b200_backend({device});
        JobScheduler sched(be.get());
        sched.run_all(&jobs);
        std::memcpy(ids, job.graph.ids_storage().data(), n * k * sizeof(std::uint32_t));
        std::memcpy(dists, job.graph.dist_storage().data(), n * k * sizeof(float));
        std::memcpy(counts, job.graph.count_storage().data(), n * sizeof(std::uint32_t));
        if (out_oom) *out_oom = job.out_of_memory ? 1 : 0;
        if (out_ran_on_cuda) *out_ran_on_cuda = job.ran_on == DeviceKind::Cuda ? 1 : 0;
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

/// The m x m MRD matrix of `pts` (padded rows) through JobScheduler::mrd_matrix on a
/// B200Backend over `device`.
int bb_mrd_matrix(const float* pts, std::uint64_t m, std::uint32_t dim, std::uint32_t stride, const float* core,
                  int device, float* out) {
    try {
        std::unique_ptr<Backend> be = make_b200_backend({device});
        JobScheduler sched(be.get());
        sched.mrd_matrix(pts, static_cast<std::size_t>(m), dim, stride, MetricKind::L2, core, out);
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

/// CoreSG::load of a CORESG01 file, then B200Extractor on `device`: K MSTs, one at a
/// time (all = 0, B200Extractor::mst) or in one sweep (all = 1, all_msts).  Trees
/// into out_edges (K x (n-1) coresg::Edge), labels into out_labels (K x n), and the
/// per-MST edge counts, component counts and weights.
int bb_extract(const char* path, const std::uint32_t* mpts, std::uint32_t K, int all, int device, void* out_edges,
               std::uint32_t* out_labels, std::uint64_t* out_nedges, std::uint32_t* out_ncomp,
               double* out_weight) {
    try {
        CoreSGParams p;
        p.backend.prefer_gpu = false;
        CoreSG sg(p);
        sg.load(path);
        B200Extractor ext(device);
        ext.sync(sg);
        const std::size_t n = sg.knn().size(), cap = n ? n - 1 : 0;
        std::vector<MstResult> res;
        if (all) {
            res = ext.all_msts(std::vector<std::uint32_t>(mpts, mpts + K));
        } else {
            for (std::uint32_t j = 0; j < K; ++j) res.push_back(ext.mst(mpts[j]));
        }
        Edge* oe = static_cast<Edge*>(out_edges);
        for (std::uint32_t j = 0; j < K; ++j) {
            std::memcpy(oe + j * cap, res[j].edges.data(), res[j].edges.size() * sizeof(Edge));
            std::memcpy(out_labels + j * n, res[j].component.data(), n * sizeof(std::uint32_t));
            out_nedges[j] = res[j].edges.size();
            out_ncomp[j] = res[j].num_components;
            out_weight[j] = res[j].weight;
        }
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

}  // extern "C"
