// Anti-hub bridges on the device (placeholder until the kernels land).
#include "common.cuh"
#include "engine.hpp"

namespace csb {
void select_bridges(Graph& g, uint64_t*, uint64_t*, uint64_t*, uint32_t*) {
    (void)g;
    fail(CS_ERR_UNSUPPORTED, "cs_select_bridges: not built yet");
}
}  // namespace csb

using namespace csb;
extern "C" {
cs_status cs_mrd_block(cs_ctx* ctx, const float*, size_t, uint32_t, uint32_t, int32_t, const float*, size_t,
                       size_t, float*) {
    return guarded(reinterpret_cast<Ctx*>(ctx), [&] { fail(CS_ERR_UNSUPPORTED, "cs_mrd_block: not built yet"); });
}
cs_status cs_select_bridges(cs_graph* gp, uint64_t* a, uint64_t* b, uint64_t* c, uint32_t* d) {
    Graph* g = reinterpret_cast<Graph*>(gp);
    return guarded(g ? g->ctx : nullptr, [&] { select_bridges(*g, a, b, c, d); });
}
cs_status cs_get_selected(cs_graph* gp, uint32_t* out, uint64_t cap, uint64_t* out_count) {
    Graph* g = reinterpret_cast<Graph*>(gp);
    return guarded(g ? g->ctx : nullptr, [&] {
        if (out_count) *out_count = g->selected.size();
        for (uint64_t i = 0; out && i < cap && i < g->selected.size(); ++i) out[i] = g->selected[i];
    });
}
}
