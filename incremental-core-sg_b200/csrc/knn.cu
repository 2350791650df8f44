// Dynamic NN-Descent on the device (placeholder until the kernels land).
#include "common.cuh"
#include "engine.hpp"

namespace csb {
void knn_descent(Graph& g, uint32_t, uint32_t, double, uint64_t, bool, uint64_t*, uint32_t*) {
    (void)g;
    fail(CS_ERR_UNSUPPORTED, "cs_knn_build: not built yet");
}
}  // namespace csb

using namespace csb;
extern "C" {
cs_status cs_nndescent(cs_ctx* ctx, const cs_nnd_config*, const float*, uint32_t*, float*, uint8_t*,
                       uint32_t*, uint64_t*) {
    return guarded(reinterpret_cast<Ctx*>(ctx), [&] { fail(CS_ERR_UNSUPPORTED, "cs_nndescent: not built yet"); });
}
cs_status cs_knn_build(cs_graph* gp, uint32_t sample, uint32_t iters, double delta, uint64_t seed,
                       uint64_t* out_updates, uint32_t* out_rounds) {
    Graph* g = reinterpret_cast<Graph*>(gp);
    return guarded(g ? g->ctx : nullptr, [&] { knn_descent(*g, sample, iters, delta, seed, true, out_updates, out_rounds); });
}
}
