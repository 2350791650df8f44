// Test and baseline infrastructure only.  A C ABI over the reference's own CUDA
// NN-Descent (coresg::cuda::nndescent_gpu, cuda/nndescent_kernels.cu:295-437),
// compiled from the reference's sources for sm_100a by oracle/Makefile (target
// `refgpu`), so that bench.py can time the reference's existing GPU kernel on the
// same B200 as the engine's build.  Nothing in the product links or loads it.
#include <cstdint>

#include "coresg/cuda_api.hpp"

extern "C" {

const char* refgpu_last_error() { return coresg::cuda::last_error(); }

/// nndescent_gpu on `device`: host buffers in and out, distances in metric units.
/// Returns 0, or 1 with refgpu_last_error().
int refgpu_nndescent(int device, std::uint32_t n, std::uint32_t dim, std::uint32_t stride, std::uint32_t k,
                     std::uint32_t sample, std::uint32_t iters, std::uint64_t seed, int metric, float delta,
                     const float* vectors, std::uint32_t* ids, float* dists, std::uint8_t* flags,
                     std::uint32_t* counts, std::uint64_t* out_updates) {
    coresg::cuda::NndConfig cfg;
    cfg.n = n;
    cfg.dim = dim;
    cfg.stride = stride;
    cfg.k = k;
    cfg.sample = sample;
    cfg.iters = iters;
    cfg.seed = seed;
    cfg.metric = metric;
    cfg.delta = delta;
    cfg.random_fill = true;
    return coresg::cuda::nndescent_gpu(device, cfg, vectors, ids, dists, flags, counts, out_updates) ? 0 : 1;
}

}  // extern "C"
