// Anti-hub bridges on the device.
//
// Restates the bridge half of CoreSG::build/insert (src/coresg.cpp:472-516,
// :537-583) with CoreSGParams/HubnessParams defaults:
//
//   connectivity  lock-free union-find over the k-NN adjacency, roots linked
//                 larger-under-smaller, dense labels by first node
//                 (ConnectivityTracker::rebuild, src/connectivity.cpp:24-139)
//   hubness       reverse degrees by atomics, the arithmetic-mean reverse score in
//                 double with the degenerate rules (src/hubness.cpp:44-158, :302-352)
//   selection     the budget llround(d * ln|E|) capped by max_pair_ops (:16-40) lowest
//                 under (score, rdeg, id) -- found by two 64-bit radix selects, one over
//                 the score bits and one over (rdeg, id) among the score ties -- plus
//                 the 2 lowest of every component (the reference's bucket scan keeps
//                 exactly those, the order being strict); sorted by the same order
//                 (:424-521)
//   bridge MST    the m x m mutual-reachability matrix at k_max and Prim with the
//                 lowest index winning ties, in one CTA; edges re-stored with their
//                 base distance (mst_over_subset, src/coresg.cpp:97-141; mst_dense,
//                 src/mst.cpp:268-330)
//   repair        components left after the bridges are spanned through their
//                 4 lowest-scoring members (repair_connectivity, src/coresg.cpp:171-258)
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include "common.cuh"
#include "engine.hpp"

namespace csb {
namespace {

constexpr int kThreads = 256;
constexpr uint32_t kDenseLimit = 8192;  // CoreSGParams::dense_matrix_limit (coresg.hpp:88)

inline unsigned blocks_for(uint64_t work, int threads = kThreads) {
    uint64_t b = (work + threads - 1) / threads;
    return static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>(b, 1u << 30)));
}

__global__ void k_iota_u32(uint32_t* __restrict__ a, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = i;
}

/// Unite every node with its listed neighbours at list positions [j0, j1).
__global__ void k_conn_unite(const uint32_t* __restrict__ ids, const uint32_t* __restrict__ counts, uint32_t n,
                             uint32_t k, uint32_t j0, uint32_t j1, uint32_t* __restrict__ parent, int* status) {
    const uint32_t span = j1 - j0;
    const uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= static_cast<uint64_t>(n) * span) return;
    const uint32_t p = static_cast<uint32_t>(t / span), j = j0 + static_cast<uint32_t>(t % span);
    if (j >= counts[p]) return;
    const uint32_t q = ids[static_cast<uint64_t>(p) * k + j];
    if (q < n && q != p) uf_unite(parent, p, q, n, status);
}

/// Point every node at its root (no unions run meanwhile, so a chase that meets an
/// entry another thread rewrote still ends at the same root).  A chase longer than
/// n (a cycle, which the linking rule rules out) sets the status and stops.
__global__ void k_compress(uint32_t* __restrict__ parent, uint32_t n, int* status) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    uint32_t r = __ldcg(parent + v);
    if (r == v) return;
    for (uint32_t it = 0;; ++it) {
        const uint32_t p = __ldcg(parent + r);
        if (p == r) break;
        if (it > n) {
            atomicOr(status, kStatusUnionLimit);
            return;
        }
        r = p;
    }
    parent[v] = r;
}

__global__ void k_rdeg(const uint32_t* __restrict__ ids, const uint32_t* __restrict__ counts, uint32_t n, uint32_t k,
                       int* __restrict__ rdeg) {
    const uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= static_cast<uint64_t>(n) * k) return;
    const uint32_t p = static_cast<uint32_t>(t / k), j = static_cast<uint32_t>(t % k);
    if (j >= counts[p]) return;
    const uint32_t q = ids[t];
    if (q < n) atomicAdd(rdeg + q, 1);
}

/// compute_score, arithmetic mean (src/hubness.cpp:302-352), of node v; IEEE double
/// division.  Writes the score and v's selection keys.
__device__ __forceinline__ void score_node(uint32_t v, const uint32_t* __restrict__ ids,
                                           const uint32_t* __restrict__ counts, uint32_t n, uint32_t k,
                                           uint32_t k_for_score, const int* __restrict__ rdeg,
                                           double* __restrict__ score, unsigned long long* __restrict__ key_score,
                                           unsigned long long* __restrict__ key_tie) {
    const uint32_t deg = counts[v];
    const int rd = rdeg[v];
    long long sum = 0;
    for (uint32_t j = 0; j < deg; ++j) {
        const uint32_t q = ids[static_cast<uint64_t>(v) * k + j];
        if (q < n) sum += rdeg[q];
    }
    double s;
    if (rd > 0 && sum <= 0) s = static_cast<double>(k_for_score);
    else if (rd <= 0 && sum > 0) s = 0.0;
    else if (rd <= 0 && sum <= 0) s = 1.0;
    else if (deg == 0) s = 1.0;
    else {
        const double denom = __ddiv_rn(static_cast<double>(sum), static_cast<double>(deg));
        s = denom > 0.0 ? __ddiv_rn(static_cast<double>(rd), denom) : static_cast<double>(k_for_score);
    }
    score[v] = s;
    // scores are >= 0, so their bit patterns order like the values
    key_score[v] = static_cast<unsigned long long>(__double_as_longlong(s));
    key_tie[v] = (static_cast<unsigned long long>(static_cast<uint32_t>(rd)) << 32) | v;
}

__global__ void k_score(const uint32_t* __restrict__ ids, const uint32_t* __restrict__ counts, uint32_t n, uint32_t k,
                        uint32_t k_for_score, const int* __restrict__ rdeg, double* __restrict__ score,
                        unsigned long long* __restrict__ key_score, unsigned long long* __restrict__ key_tie) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    score_node(v, ids, counts, n, k, k_for_score, rdeg, score, key_score, key_tie);
}

// ---- incremental hubness refresh (HubnessIndex::refresh, src/hubness.cpp:523-544) ----
// After a full pass the graph keeps a snapshot of the lists it scored.  k_merge flags
// every node whose membership changed since (hub_changed); nodes added since the
// snapshot count as changed.  The refresh applies the reverse-degree deltas of the
// changed lists (on_edge_added / on_edge_removed, :242-279) and rescores exactly the
// nodes whose score inputs moved: a changed list, a changed own reverse degree, or a
// listed neighbour whose reverse degree changed (collect_rescore_set, :482-520, with the
// reverse neighbours found by scanning the lists against the dirty flags).

/// One node of k_hub_delta (warp-collective).
__device__ __forceinline__ void hub_delta_node(const uint32_t* __restrict__ ids, const uint32_t* __restrict__ counts,
                                               uint32_t n, uint32_t k, uint32_t n_prev, uint32_t p, unsigned lane,
                                               uint32_t* __restrict__ prev_ids, uint32_t* __restrict__ prev_cnt,
                                               int* __restrict__ rdeg, uint8_t* __restrict__ rd_dirty) {
    const bool fresh = p >= n_prev;
    const uint32_t cn = counts[p], co = fresh ? 0u : prev_cnt[p];
    const uint64_t base = static_cast<uint64_t>(p) * k;
    uint32_t nw[2], od[2];
    bool od_kept[2] = {false, false}, nw_known[2] = {false, false};
#pragma unroll
    for (int e = 0; e < 2; ++e) {
        const uint32_t j = lane + 32u * e;
        nw[e] = j < cn ? ids[base + j] : kInvalid;
        od[e] = j < co ? prev_ids[base + j] : kInvalid;
    }
    const int halves = k > 32 ? 2 : 1;
    for (int e2 = 0; e2 < halves; ++e2) {
        for (int src = 0; src < 32; ++src) {
            const uint32_t a = __shfl_sync(0xFFFFFFFFu, nw[e2], src);
            const uint32_t b = __shfl_sync(0xFFFFFFFFu, od[e2], src);
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                if (od[e] != kInvalid && od[e] == a) od_kept[e] = true;
                if (nw[e] != kInvalid && nw[e] == b) nw_known[e] = true;
            }
        }
    }
#pragma unroll
    for (int e = 0; e < 2; ++e) {
        if (od[e] != kInvalid && !od_kept[e] && od[e] < n) {
            atomicSub(rdeg + od[e], 1);
            rd_dirty[od[e]] = 1;
        }
        if (nw[e] != kInvalid && !nw_known[e] && nw[e] < n) {
            atomicAdd(rdeg + nw[e], 1);
            rd_dirty[nw[e]] = 1;
        }
        const uint32_t j = lane + 32u * e;
        if (j < k) prev_ids[base + j] = nw[e];
    }
    if (lane == 0) prev_cnt[p] = cn;
}

/// The nodes whose lists changed since the snapshot (flagged by k_merge, or added
/// since: v >= n_prev), compacted into list[0..*cnt) with one atomic per warp.
__global__ void k_hub_changed_list(uint32_t n, uint32_t n_prev, const uint8_t* __restrict__ changed,
                                   uint32_t* __restrict__ list, uint32_t* __restrict__ cnt) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    const bool want = v < n && (v >= n_prev || changed[v]);
    const uint32_t at = warp_append(want, cnt);
    if (want) list[at] = v;
}

/// Reverse-degree deltas of each listed node p's list against its snapshot, one warp
/// per node (grid-stride over list[0..*cnt)): an id that left the list loses one
/// reverse neighbour, an id that joined gains one; both get rd_dirty.  The snapshot
/// takes the new list.  k <= 64 (two entries a lane).
__global__ void k_hub_delta(const uint32_t* __restrict__ ids, const uint32_t* __restrict__ counts, uint32_t n,
                            uint32_t k, uint32_t n_prev, const uint32_t* __restrict__ list,
                            const uint32_t* __restrict__ cnt, uint32_t* __restrict__ prev_ids,
                            uint32_t* __restrict__ prev_cnt, int* __restrict__ rdeg, uint8_t* __restrict__ rd_dirty) {
    const unsigned lane = threadIdx.x & 31u;
    const uint32_t total = *cnt;
    for (uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < total; w += (gridDim.x * blockDim.x) >> 5) {
        hub_delta_node(ids, counts, n, k, n_prev, list[w], lane, prev_ids, prev_cnt, rdeg, rd_dirty);
    }
}


/// Rescore the nodes whose score inputs moved (see above); counts them into *rescored.
__global__ void k_score_refresh(const uint32_t* __restrict__ ids, const uint32_t* __restrict__ counts, uint32_t n,
                                uint32_t k, uint32_t k_for_score, uint32_t n_prev, const uint8_t* __restrict__ changed,
                                const uint8_t* __restrict__ rd_dirty, const int* __restrict__ rdeg,
                                double* __restrict__ score, unsigned long long* __restrict__ key_score,
                                unsigned long long* __restrict__ key_tie, unsigned long long* __restrict__ rescored) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    bool need = false;
    if (v < n) {
        need = v >= n_prev || changed[v] || rd_dirty[v];
        const uint32_t deg = counts[v];
        for (uint32_t j = 0; j < deg && !need; ++j) {
            const uint32_t q = ids[static_cast<uint64_t>(v) * k + j];
            need = q < n && rd_dirty[q];
        }
        if (need) score_node(v, ids, counts, n, k, k_for_score, rdeg, score, key_score, key_tie);
    }
    const unsigned b = __ballot_sync(0xFFFFFFFFu, need);
    if ((threadIdx.x & 31u) == 0 && b) atomicAdd(rescored, static_cast<unsigned long long>(__popc(b)));
}

/// Histogram of one 8-bit digit of key[] over the elements whose higher digits
/// equal `prefix` (and, when tie_key != null, whose tie_key equals tie_value).
__global__ void k_digit_hist(const unsigned long long* __restrict__ key, uint32_t n, int shift,
                             unsigned long long prefix, unsigned long long pmask,
                             const unsigned long long* __restrict__ filt, unsigned long long filt_value,
                             uint32_t* __restrict__ hist) {
    __shared__ uint32_t h[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) h[i] = 0;
    __syncthreads();
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t v = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; v < n; v += stride) {
        if (filt && filt[v] != filt_value) continue;
        const unsigned long long x = key[v];
        if ((x & pmask) != prefix) continue;
        atomicAdd(h + ((x >> shift) & 0xFFu), 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 256; i += blockDim.x) {
        if (h[i]) atomicAdd(hist + i, h[i]);
    }
}

/// Collect v with score < T, or score == T and tie <= T2 (selection of the budget).
__global__ void k_collect(const unsigned long long* __restrict__ ks, const unsigned long long* __restrict__ kt,
                          uint32_t n, unsigned long long T, unsigned long long T2, int use_ties,
                          uint8_t* __restrict__ chosen, uint32_t* __restrict__ out, uint32_t* __restrict__ cnt,
                          uint32_t cap) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const bool take = ks[v] < T || (use_ties && ks[v] == T && kt[v] <= T2);
    if (!take) return;
    chosen[v] = 1;
    const uint32_t pos = atomicAdd(cnt, 1u);
    if (pos < cap) out[pos] = v;
}

/// One quota round: per component, the lowest (score) then lowest (rdeg, id) among
/// the nodes not yet taken by an earlier quota round.  A warp whose candidate nodes
/// all lie in one component (the usual case: a k-NN graph has few components, and
/// one atomic per node on its key serialised) offers their minimum once.
__global__ void k_quota_score(const unsigned long long* __restrict__ ks, const uint32_t* __restrict__ comp, uint32_t n,
                              const uint8_t* __restrict__ qtaken, unsigned long long* __restrict__ best_s) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;  // every lane reaches the warp votes
    const unsigned lane = threadIdx.x & 31u;
    const bool ok = v < n && !qtaken[v];
    const uint32_t c = ok ? comp[v] : 0u;
    unsigned long long x = ok ? ks[v] : kNoKey;
    const unsigned live = __ballot_sync(0xFFFFFFFFu, ok);
    if (!live) return;
    const uint32_t c0 = __shfl_sync(0xFFFFFFFFu, c, __ffs(live) - 1);
    if (__all_sync(0xFFFFFFFFu, !ok || c == c0)) {
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long y = __shfl_xor_sync(0xFFFFFFFFu, x, o);
            x = y < x ? y : x;
        }
        if (lane == 0) atomicMin(best_s + c0, x);
    } else if (ok) {
        atomicMin(best_s + c, x);
    }
}
__global__ void k_quota_tie(const unsigned long long* __restrict__ ks, const unsigned long long* __restrict__ kt,
                            const uint32_t* __restrict__ comp, uint32_t n, const uint8_t* __restrict__ qtaken,
                            const unsigned long long* __restrict__ best_s, unsigned long long* __restrict__ best_t) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n || qtaken[v]) return;
    const uint32_t c = comp[v];
    if (ks[v] == best_s[c]) atomicMin(best_t + c, kt[v]);
}
__global__ void k_quota_take(const unsigned long long* __restrict__ best_t, uint32_t ncomp,
                             uint8_t* __restrict__ qtaken, uint8_t* __restrict__ chosen, uint32_t* __restrict__ out,
                             uint32_t* __restrict__ cnt, uint32_t cap) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncomp) return;
    const unsigned long long t = best_t[c];
    if (t == kNoKey) return;
    const uint32_t v = static_cast<uint32_t>(t);
    qtaken[v] = 1;
    if (!chosen[v]) {
        chosen[v] = 1;
        const uint32_t pos = atomicAdd(cnt, 1u);
        if (pos < cap) out[pos] = v;
    }
}

/// Gather the selected rows and their k_max core distances.
__global__ void k_gather(const float* __restrict__ pts, uint32_t stride, const float* __restrict__ dists,
                         const uint32_t* __restrict__ counts, uint32_t k, const uint32_t* __restrict__ sel, uint32_t m,
                         float* __restrict__ out_pts, float* __restrict__ out_core) {
    const uint32_t i = blockIdx.x;
    if (i >= m) return;
    const uint32_t v = sel[i];
    for (uint32_t d = threadIdx.x; d < stride; d += blockDim.x) out_pts[static_cast<uint64_t>(i) * stride + d] = pts[static_cast<uint64_t>(v) * stride + d];
    if (threadIdx.x == 0) out_core[i] = core_of(dists, counts, k, v, k);
}

/// Rows [r0, r1) of the m x m mutual-reachability matrix (mrd_block_kernel,
/// cuda/mrd_kernels.cu:30-87, with the CPU backend's association order so the
/// values equal src/cpu_backend.cpp:61-90 bit for bit).
__global__ void k_mrd(const float* __restrict__ pts, uint32_t m, uint32_t stride, int metric,
                      const float* __restrict__ core, uint32_t r0, uint32_t rows, float* __restrict__ out) {
    const uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= static_cast<uint64_t>(rows) * m) return;
    const uint32_t lr = static_cast<uint32_t>(t / m), j = static_cast<uint32_t>(t % m);
    const uint32_t i = r0 + lr;
    float v;
    if (i == j) {
        v = 0.0f;
    } else {
        const float d = finalize_rank(l2sqr_ref(pts + static_cast<uint64_t>(i) * stride, pts + static_cast<uint64_t>(j) * stride, stride), metric);
        v = max_ref(d, max_ref(core[i], core[j]));
    }
    out[t] = v;
}

/// Prim over the dense matrix in one CTA (mst_prim_virtual, src/mst.cpp:274-330):
/// start at 0, relax from the current row, pick the smallest best[] with the lowest
/// index winning ties; edges carry the base distance of their endpoints
/// (src/coresg.cpp:346-351) and global ids via `ids`.  The frontier (best, from,
/// in-tree: 9 bytes per node) lives in shared memory; a step's pick is one warp's
/// reduction of the warps' minima; the edges are recorded as local (from, pick) pairs
/// in pick order and their base distances computed by all threads after the loop.
__global__ void k_prim(const float* __restrict__ mat, uint32_t m, const float* __restrict__ pts, uint32_t stride,
                       int metric, const uint32_t* __restrict__ ids, cs_edge* __restrict__ out,
                       uint32_t* __restrict__ out_count) {
    extern __shared__ unsigned char prim_smem[];
    float* const best = reinterpret_cast<float*>(prim_smem);
    uint32_t* const from = reinterpret_cast<uint32_t*>(best + m);
    uint8_t* const in_tree = reinterpret_cast<uint8_t*>(from + m);
    __shared__ unsigned long long red[32];
    __shared__ uint32_t s_pick, s_cnt;
    const float inf = __int_as_float(0x7f800000);
    for (uint32_t j = threadIdx.x; j < m; j += blockDim.x) {
        best[j] = j == 0 ? 0.0f : inf;
        from[j] = kInvalid;
        in_tree[j] = j == 0 ? 1 : 0;
    }
    if (threadIdx.x == 0) s_cnt = 0;
    __syncthreads();
    uint32_t current = 0;
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (uint32_t step = 1; step < m; ++step) {
        const float* row = mat + static_cast<uint64_t>(current) * m;
        // relax, then argmin over (best bits, index): ties -> lowest index, and an
        // all-infinite frontier still picks its lowest index (the reference's rule)
        unsigned long long mine = kNoKey;
        for (uint32_t j = threadIdx.x; j < m; j += blockDim.x) {
            if (in_tree[j]) continue;
            const float w = row[j];
            float b = best[j];
            if (w < b) {
                b = w;
                best[j] = w;
                from[j] = current;
            }
            const unsigned long long key = (static_cast<unsigned long long>(__float_as_uint(b)) << 32) | j;
            mine = key < mine ? key : mine;
        }
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long other = __shfl_xor_sync(0xFFFFFFFFu, mine, o);
            mine = other < mine ? other : mine;
        }
        if (lane == 0) red[warp] = mine;
        __syncthreads();
        if (warp == 0) {
            unsigned long long v = lane < nw ? red[lane] : kNoKey;
            for (int o = 16; o > 0; o >>= 1) {
                const unsigned long long other = __shfl_xor_sync(0xFFFFFFFFu, v, o);
                v = other < v ? other : v;
            }
            if (lane == 0) {
                const uint32_t pick = v == kNoKey ? kInvalid : static_cast<uint32_t>(v);
                s_pick = pick;
                if (pick != kInvalid) {
                    in_tree[pick] = 1;
                    if (from[pick] != kInvalid && __uint_as_float(static_cast<uint32_t>(v >> 32)) < inf) {
                        out[s_cnt].u = from[pick];  // local indices until the pass below
                        out[s_cnt].v = pick;
                        ++s_cnt;
                    }
                }
            }
        }
        __syncthreads();
        if (s_pick == kInvalid) break;
        current = s_pick;
    }
    __syncthreads();
    const uint32_t cnt = s_cnt;
    for (uint32_t t = threadIdx.x; t < cnt; t += blockDim.x) {
        const uint32_t a = out[t].u, bb = out[t].v;
        const float base = finalize_rank(l2sqr_ref(pts + static_cast<uint64_t>(a) * stride, pts + static_cast<uint64_t>(bb) * stride, stride), metric);
        const uint32_t ga = ids[a], gb = ids[bb];
        cs_edge e;
        e.u = ga < gb ? ga : gb;
        e.v = ga < gb ? gb : ga;
        e.w = base;
        out[t] = e;
    }
    if (threadIdx.x == 0) *out_count = cnt;
}

/// Views of the graph's cached selection scratch (grow-only buffers).
struct Scratch {
    DevBuf &parent, &lab, &bc, &ncomp, &rdeg, &score, &ks, &kt, &hist, &chosen, &qtaken, &sel, &selcnt, &best_s,
        &best_t, &sub_pts, &sub_core, &mat, &pout, &pcnt;
    explicit Scratch(Graph& g)
        : parent(g.bridge_scratch[0]), lab(g.bridge_scratch[1]), bc(g.bridge_scratch[2]), ncomp(g.bridge_scratch[3]),
          rdeg(g.bridge_scratch[4]), score(g.bridge_scratch[5]), ks(g.bridge_scratch[6]), kt(g.bridge_scratch[7]),
          hist(g.bridge_scratch[8]), chosen(g.bridge_scratch[9]), qtaken(g.bridge_scratch[10]),
          sel(g.bridge_scratch[11]), selcnt(g.bridge_scratch[12]), best_s(g.bridge_scratch[13]),
          best_t(g.bridge_scratch[14]), sub_pts(g.bridge_scratch[15]), sub_core(g.bridge_scratch[16]),
          mat(g.bridge_scratch[17]), pout(g.bridge_scratch[21]), pcnt(g.bridge_scratch[22]) {}
};

/// The anti-hub budget: round(dim x ln |E|) with |E| the k-NN edge count, capped so
/// the bridge MST's m^2 x dim / 2 coordinate operations stay within 2e9
/// (m <= sqrt(4e9 / dim)), at least 2 and at most n (antihub_budget,
/// src/hubness.cpp:16-40, with its default multiplier 1, max_pair_ops 2e9 and
/// min_selected 2).
uint64_t antihub_budget(uint64_t num_edges, uint32_t dim, uint64_t n) {
    const double logs = num_edges > 1 ? std::log(static_cast<double>(num_edges)) : 0.0;
    double raw = 1.0 * static_cast<double>(dim) * logs;
    if (!(raw > 0.0)) raw = 0.0;
    uint64_t budget = static_cast<uint64_t>(std::llround(raw));
    const double m_max = std::sqrt(2.0 * 2e9 / static_cast<double>(dim));
    if (m_max >= 1.0 && static_cast<double>(budget) > m_max) budget = static_cast<uint64_t>(m_max);
    if (budget < 2) budget = 2;
    if (budget > n) budget = n;
    return budget;
}

/// The node-proportional selection scratch for `ns` nodes.
void size_bridge_scratch(Scratch& s, uint64_t ns, cudaStream_t st) {
    s.parent.ensure(ns * 4ull);
    s.lab.ensure(ns * 4ull);
    // the reverse degrees, scores and keys persist between selections (incremental
    // refresh): they keep their contents when they grow
    s.rdeg.grow_keep(ns * 4ull, st);
    s.score.grow_keep(ns * 8ull, st);
    s.ks.grow_keep(ns * 8ull, st);
    s.kt.grow_keep(ns * 8ull, st);
    s.chosen.ensure(ns + 16ull);
    s.qtaken.ensure(ns + 16ull);
}

/// out[i] = (key_a[idx[i]], key_b[idx[i]]): the sort keys of the selected ids.
__global__ void k_gather_keys(const uint32_t* __restrict__ idx, uint32_t m, const unsigned long long* __restrict__ a,
                              const unsigned long long* __restrict__ b, unsigned long long* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    out[2 * i] = a[idx[i]];
    out[2 * i + 1] = b[idx[i]];
}

/// out[i] = src[idx[i]].
__global__ void k_gather_u32(const uint32_t* __restrict__ idx, uint32_t m, const uint32_t* __restrict__ src,
                             uint32_t* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) out[i] = src[idx[i]];
}

/// Smallest threshold T over key[] (restricted by the filter) with
/// count(key <= T) >= rank (1-based), by 8-bit radix passes from the top.
unsigned long long radix_select(Ctx& c, Scratch& s, const unsigned long long* key, uint32_t n, uint64_t rank,
                                const unsigned long long* filt, unsigned long long filt_value) {
    unsigned long long prefix = 0, pmask = 0;
    uint64_t remaining = rank;
    uint32_t h[256];
    for (int shift = 56; shift >= 0; shift -= 8) {
        CSB_CUDA(cudaMemsetAsync(s.hist.p, 0, 256 * 4, c.stream));
        k_digit_hist<<<std::min<unsigned>(blocks_for(n), 4u * c.sm_count), kThreads, 0, c.stream>>>(
            key, n, shift, prefix, pmask, filt, filt_value, s.hist.as<uint32_t>());
        count_launch(c);
        CSB_CUDA(cudaMemcpyAsync(h, s.hist.p, sizeof(h), cudaMemcpyDeviceToHost, c.stream));
        CSB_CUDA(cudaStreamSynchronize(c.stream));
        uint32_t d = 0;
        uint64_t acc = 0;
        for (; d < 256; ++d) {
            if (acc + h[d] >= remaining) break;
            acc += h[d];
        }
        if (d == 256) fail(CS_ERR_STATE, "radix select: rank beyond the population");
        remaining -= acc;
        prefix |= static_cast<unsigned long long>(d) << shift;
        pmask |= 0xFFull << shift;
    }
    return prefix;
}

/// Dense MRD matrix + Prim over `m` selected nodes (device ids in d_sel); appends
/// the edges (global ids, base distances) to `out`.
void mst_over_subset(Graph& g, Scratch& s, const uint32_t* d_sel, uint32_t m, std::vector<cs_edge>* out) {
    Ctx& c = *g.ctx;
    if (m < 2) return;
    if (m > kDenseLimit) fail(CS_ERR_UNSUPPORTED, "bridge MST over more than 8192 nodes (streamed Prim) is not built");
    s.sub_pts.ensure(static_cast<uint64_t>(m) * g.stride * 4);
    s.sub_core.ensure(m * 4ull);
    s.mat.ensure(static_cast<uint64_t>(m) * m * 4);
    s.pout.ensure(m * sizeof(cs_edge) + 64);
    s.pcnt.ensure(64);
    k_gather<<<m, 128, 0, c.stream>>>(g.pts.as<float>(), g.stride, g.dists.as<float>(), g.counts.as<uint32_t>(), g.k, d_sel,
                                       m, s.sub_pts.as<float>(), s.sub_core.as<float>());
    const uint64_t cells = static_cast<uint64_t>(m) * m;
    k_mrd<<<blocks_for(cells), kThreads, 0, c.stream>>>(s.sub_pts.as<float>(), m, g.stride, g.metric, s.sub_core.as<float>(),
                                                       0, m, s.mat.as<float>());
    const size_t prim_smem = static_cast<size_t>(m) * 9;  // best, from, in-tree
    CSB_CUDA(cudaFuncSetAttribute(k_prim, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(prim_smem)));
    k_prim<<<1, 1024, prim_smem, c.stream>>>(s.mat.as<float>(), m, s.sub_pts.as<float>(), g.stride, g.metric, d_sel,
                                             s.pout.as<cs_edge>(), s.pcnt.as<uint32_t>());
    count_launch(c, 3);
    check_launch(c, "bridge MST");
    uint32_t cnt = 0;
    CSB_CUDA(cudaMemcpyAsync(&cnt, s.pcnt.p, 4, cudaMemcpyDeviceToHost, c.stream));
    CSB_CUDA(cudaStreamSynchronize(c.stream));
    std::vector<cs_edge> e(cnt);
    if (cnt) copy_d2h(c, e.data(), s.pout.p, cnt * sizeof(cs_edge));
    out->insert(out->end(), e.begin(), e.end());
}

// host-side union-find over component labels (a few thousand at most)
struct HostUF {
    std::vector<uint32_t> p;
    explicit HostUF(uint32_t n) : p(n) { std::iota(p.begin(), p.end(), 0u); }
    uint32_t find(uint32_t x) {
        while (p[x] != x) x = p[x] = p[p[x]];
        return x;
    }
    bool unite(uint32_t a, uint32_t b) {
        a = find(a);
        b = find(b);
        if (a == b) return false;
        if (a > b) std::swap(a, b);
        p[b] = a;
        return true;
    }
};

}  // namespace

void mrd_rows(Ctx& c, const float* d_pts, uint32_t m, uint32_t stride, int metric, const float* d_core, uint32_t r0,
              uint32_t r1, float* d_out) {
    const uint64_t cells = static_cast<uint64_t>(r1 - r0) * m;
    if (!cells) return;
    k_mrd<<<blocks_for(cells), kThreads, 0, c.stream>>>(d_pts, m, stride, metric, d_core, r0, r1 - r0, d_out);
    count_launch(c);
    check_launch(c, "mrd rows");
}

uint64_t selection_bound(const Graph& g) {
    const uint64_t ns = scratch_nodes(g);
    return antihub_budget(ns * g.k, g.dim, ns) + 2 * (4ull * g.last_ncomp + 64) + 8;
}

void bridges_reserve(Graph& g) {
    Scratch s(g);
    const uint64_t ns = scratch_nodes(g);
    size_bridge_scratch(s, ns, g.ctx->stream);
    // the rest of a selection on up to ns nodes: per-block label counts, the selected
    // list, the per-component quota keys, the bridge MST over the selected nodes and
    // the selection's sort keys
    const uint64_t m = selection_bound(g), comps = 4ull * g.last_ncomp + 64;
    const uint64_t md = std::min<uint64_t>(m, kDenseLimit);
    s.bc.ensure(blocks_for(ns) * 4ull + 64);
    s.ncomp.ensure(64);
    s.hist.ensure(256 * 4);
    s.sel.ensure(m * 4);
    s.selcnt.ensure(64);
    s.best_s.ensure(comps * 8);
    s.best_t.ensure(comps * 8);
    s.sub_pts.ensure(md * g.stride * 4);
    s.sub_core.ensure(md * 4);
    s.mat.ensure(md * md * 4);
    s.pout.ensure(md * sizeof(cs_edge) + 64);
    s.pcnt.ensure(64);
    g.ctx->scratch[6].ensure(m * 16 + 16);
    g.bridges.grow_keep(md * sizeof(cs_edge), g.ctx->stream);
    // the incremental hubness state (snapshot, flags, counter), kept when it grows
    g.hub_prev_ids.grow_keep(ns * g.k * 4ull, g.ctx->stream);
    g.hub_prev_cnt.grow_keep(ns * 4ull, g.ctx->stream);
    g.hub_rd_dirty.grow_keep(ns + 16ull, g.ctx->stream);
    g.hub_list.ensure(ns * 4ull + 16);
    g.hub_ctr.ensure(64);
    hub_track(g);
}

void hub_track(Graph& g) {
    const uint64_t ns = scratch_nodes(g) + 16;
    if (g.hub_changed.bytes >= ns && g.hub_changed.p) return;
    const size_t old = g.hub_changed.p ? g.hub_changed.bytes : 0;
    g.hub_changed.grow_keep(ns, g.ctx->stream);
    CSB_CUDA(cudaMemsetAsync(g.hub_changed.as<uint8_t>() + old, 0, g.hub_changed.bytes - old, g.ctx->stream));
}

/// The incremental hubness refresh runs when at most n / kRefreshShare lists changed
/// since the last scoring; beyond that a full pass is cheaper (measured: inserts of
/// 60k-180k rows into 2-3.6M nodes changed enough lists that the refresh rescored
/// 60-80 % of the nodes and took 0.6-2.0 ms against 0.5-0.85 ms for the full pass).
constexpr uint64_t kRefreshShare = 16;

/// Events recorded on a stream at stage boundaries; elapsed() gives the
/// milliseconds between consecutive marks once the last one has completed.
struct StageEvents {
    static constexpr int kMax = 12;
    cudaStream_t s;
    cudaEvent_t ev[kMax] = {};
    int n = 0;
    explicit StageEvents(cudaStream_t st) : s(st) {}
    ~StageEvents() {
        for (int i = 0; i < n; ++i) cudaEventDestroy(ev[i]);
    }
    void mark() {
        if (n == kMax) return;
        CSB_CUDA(cudaEventCreate(&ev[n]));
        CSB_CUDA(cudaEventRecord(ev[n], s));
        ++n;
    }
    void elapsed(double* out, int count) {
        if (n) CSB_CUDA(cudaEventSynchronize(ev[n - 1]));
        for (int i = 0; i < count; ++i) {
            float t = 0.0f;
            if (i + 1 < n) CSB_CUDA(cudaEventElapsedTime(&t, ev[i], ev[i + 1]));
            out[i] = t;
        }
    }
};

void select_bridges(Graph& g, uint64_t* out_selected, uint64_t* out_bridges, uint64_t* out_repair,
                    uint32_t* out_components) {
    Ctx& c = *g.ctx;
    const uint32_t n = static_cast<uint32_t>(g.n);
    const uint32_t k = g.k;
    CSB_REQUIRE(n > 0, "cs_select_bridges: empty graph");
    Scratch s(g);
    StageEvents ev(c.stream);
    ev.mark();
    int* status = c.status.as<int>();
    CSB_CUDA(cudaMemsetAsync(status, 0, 4, c.stream));
    const uint64_t nk = static_cast<uint64_t>(n) * k;
    // ---- connectivity
    const uint64_t ns = scratch_nodes(g);
    s.parent.ensure(ns * 4ull);
    s.lab.ensure(ns * 4ull);
    const uint32_t nb = blocks_for(n);
    s.bc.ensure(nb * 4ull + 64);
    s.ncomp.ensure(64);
    // the two nearest neighbours first (on clustered k-NN graphs they already join most
    // of each component), every node pointed at its root, then the other list
    // entries: their finds are one or two loads and most find the endpoints joined
    k_iota_u32<<<blocks_for(n), kThreads, 0, c.stream>>>(s.parent.as<uint32_t>(), n);
    const uint32_t j_first = std::min<uint32_t>(2, k);
    k_conn_unite<<<blocks_for(static_cast<uint64_t>(n) * j_first), kThreads, 0, c.stream>>>(
        g.ids.as<uint32_t>(), g.counts.as<uint32_t>(), n, k, 0, j_first, s.parent.as<uint32_t>(), status);
    k_compress<<<blocks_for(n), kThreads, 0, c.stream>>>(s.parent.as<uint32_t>(), n, status);
    count_launch(c, 3);
    if (k > j_first) {
        k_conn_unite<<<blocks_for(static_cast<uint64_t>(n) * (k - j_first)), kThreads, 0, c.stream>>>(
            g.ids.as<uint32_t>(), g.counts.as<uint32_t>(), n, k, j_first, k, s.parent.as<uint32_t>(), status);
        count_launch(c);
    }
    launch_labels(c, s.parent.as<uint32_t>(), n, 1, s.lab.as<uint32_t>(), s.bc.as<uint32_t>(),
                  s.ncomp.as<unsigned long long>());
    ev.mark();  // connectivity
    // ---- hubness
    // the scores persist between selections (incremental refresh), so these buffers
    // keep their contents when they grow (here, in a reserve, at a capacity step)
    s.rdeg.grow_keep(ns * 4ull, c.stream);
    s.score.grow_keep(ns * 8ull, c.stream);
    s.ks.grow_keep(ns * 8ull, c.stream);
    s.kt.grow_keep(ns * 8ull, c.stream);
    g.hub_prev_ids.grow_keep(ns * k * 4ull, c.stream);
    g.hub_prev_cnt.grow_keep(ns * 4ull, c.stream);
    g.hub_rd_dirty.grow_keep(ns + 16ull, c.stream);
    g.hub_list.ensure(ns * 4ull + 16);
    g.hub_ctr.ensure(64);
    hub_track(g);
    // the refresh pays when few lists changed: it rescores the changed nodes and every
    // node listing one whose reverse degree moved, which after a large insert is most
    // of the graph, and then a full pass (one streaming pass over the lists for the
    // reverse degrees, one for the scores) is cheaper.  The changed nodes are counted
    // first; above n / kRefreshShare the pass is a full one.
    bool refresh = g.hub_valid && g.hub_n <= n;
    uint64_t changed_nodes = n;
    CSB_CUDA(cudaMemsetAsync(g.hub_ctr.p, 0, 16, c.stream));
    uint32_t* list_cnt = g.hub_ctr.as<uint32_t>() + 2;
    if (refresh) {
        k_hub_changed_list<<<blocks_for(n), kThreads, 0, c.stream>>>(n, static_cast<uint32_t>(g.hub_n),
                                                                    g.hub_changed.as<uint8_t>(),
                                                                    g.hub_list.as<uint32_t>(), list_cnt);
        count_launch(c);
        uint32_t changed = 0;
        CSB_CUDA(cudaMemcpyAsync(&changed, list_cnt, 4, cudaMemcpyDeviceToHost, c.stream));
        CSB_CUDA(cudaStreamSynchronize(c.stream));
        refresh = static_cast<uint64_t>(changed) * kRefreshShare <= n;
        changed_nodes = changed;
    }
    if (refresh) {
        if (n > g.hub_n) {  // nodes added since: no reverse neighbours yet, no flags
            CSB_CUDA(cudaMemsetAsync(s.rdeg.as<int>() + g.hub_n, 0, (n - g.hub_n) * 4ull, c.stream));
            CSB_CUDA(cudaMemsetAsync(g.hub_rd_dirty.as<uint8_t>() + g.hub_n, 0, n - g.hub_n, c.stream));
        }
        k_hub_delta<<<static_cast<unsigned>(c.sm_count) * 16u, kThreads, 0, c.stream>>>(
            g.ids.as<uint32_t>(), g.counts.as<uint32_t>(), n, k, static_cast<uint32_t>(g.hub_n),
            g.hub_list.as<uint32_t>(), list_cnt, g.hub_prev_ids.as<uint32_t>(), g.hub_prev_cnt.as<uint32_t>(),
            s.rdeg.as<int>(), g.hub_rd_dirty.as<uint8_t>());
        count_launch(c);
        k_score_refresh<<<blocks_for(n), kThreads, 0, c.stream>>>(
            g.ids.as<uint32_t>(), g.counts.as<uint32_t>(), n, k, k, static_cast<uint32_t>(g.hub_n),
            g.hub_changed.as<uint8_t>(), g.hub_rd_dirty.as<uint8_t>(), s.rdeg.as<int>(), s.score.as<double>(),
            s.ks.as<unsigned long long>(), s.kt.as<unsigned long long>(), g.hub_ctr.as<unsigned long long>());
        count_launch(c);
    } else {
        CSB_CUDA(cudaMemsetAsync(s.rdeg.p, 0, n * 4ull, c.stream));
        k_rdeg<<<blocks_for(nk), kThreads, 0, c.stream>>>(g.ids.as<uint32_t>(), g.counts.as<uint32_t>(), n, k,
                                                          s.rdeg.as<int>());
        k_score<<<blocks_for(n), kThreads, 0, c.stream>>>(g.ids.as<uint32_t>(), g.counts.as<uint32_t>(), n, k, k,
                                                          s.rdeg.as<int>(), s.score.as<double>(),
                                                          s.ks.as<unsigned long long>(), s.kt.as<unsigned long long>());
        count_launch(c, 2);
        // the snapshot the next refresh compares against
        CSB_CUDA(cudaMemcpyAsync(g.hub_prev_ids.p, g.ids.p, nk * 4ull, cudaMemcpyDeviceToDevice, c.stream));
        CSB_CUDA(cudaMemcpyAsync(g.hub_prev_cnt.p, g.counts.p, n * 4ull, cudaMemcpyDeviceToDevice, c.stream));
    }
    CSB_CUDA(cudaMemsetAsync(g.hub_changed.p, 0, n, c.stream));
    CSB_CUDA(cudaMemsetAsync(g.hub_rd_dirty.p, 0, n, c.stream));
    g.hub_valid = true;
    g.hub_n = n;
    check_launch(c, "hubness");
    ev.mark();  // hubness
    unsigned long long ncomp64 = 0, rescored = n;
    CSB_CUDA(cudaMemcpyAsync(&ncomp64, s.ncomp.p, 8, cudaMemcpyDeviceToHost, c.stream));
    if (refresh) CSB_CUDA(cudaMemcpyAsync(&rescored, g.hub_ctr.p, 8, cudaMemcpyDeviceToHost, c.stream));
    int st = 0;
    CSB_CUDA(cudaMemcpyAsync(&st, status, 4, cudaMemcpyDeviceToHost, c.stream));
    CSB_CUDA(cudaStreamSynchronize(c.stream));
    if (st & kStatusUnionLimit) fail(CS_ERR_TIMEOUT, "connectivity: a union retry loop ran out");
    const uint32_t ncomp = static_cast<uint32_t>(ncomp64);
    g.last_ncomp = ncomp;
    // ---- budget: the undirected k-NN edge count (the edges themselves are emitted
    // when a sweep next needs them)
    graph_count_knn_edges(g);
    ev.mark();  // edge list
    const uint64_t budget = antihub_budget(g.e_knn, g.dim, n);
    // ---- selection: budget lowest under (score, rdeg, id)
    const uint32_t cap = static_cast<uint32_t>(budget + 2ull * ncomp + 8);
    s.hist.ensure(256 * 4);
    s.chosen.ensure(ns + 16ull);
    s.qtaken.ensure(ns + 16ull);
    s.sel.ensure(cap * 4ull);
    s.selcnt.ensure(64);
    CSB_CUDA(cudaMemsetAsync(s.chosen.p, 0, n, c.stream));
    CSB_CUDA(cudaMemsetAsync(s.qtaken.p, 0, n, c.stream));
    CSB_CUDA(cudaMemsetAsync(s.selcnt.p, 0, 64, c.stream));
    const unsigned long long* ks = s.ks.as<unsigned long long>();
    const unsigned long long* kt = s.kt.as<unsigned long long>();
    if (budget > 0) {
        const unsigned long long T = radix_select(c, s, ks, n, budget, nullptr, 0);
        // count strictly below T
        unsigned long long T2 = 0;
        int use_ties = 0;
        {
            // population of score < T = budget - (rank of the needed ties)
            uint64_t below = 0;
            // histogram-free count: reuse radix select on ks with rank = budget gives T;
            // the ties needed = budget - count(ks < T); count it with one more pass
            DevBuf& tmpc = s.pcnt;
            tmpc.ensure(64);
            CSB_CUDA(cudaMemsetAsync(tmpc.p, 0, 64, c.stream));
            k_collect<<<blocks_for(n), kThreads, 0, c.stream>>>(ks, kt, n, T, 0, 0, s.chosen.as<uint8_t>(),
                                                                 s.sel.as<uint32_t>(), tmpc.as<uint32_t>(), cap);
            count_launch(c);
            uint32_t hb = 0;
            CSB_CUDA(cudaMemcpyAsync(&hb, tmpc.p, 4, cudaMemcpyDeviceToHost, c.stream));
            CSB_CUDA(cudaStreamSynchronize(c.stream));
            below = hb;
            if (below < budget) {
                T2 = radix_select(c, s, kt, n, budget - below, ks, T);
                use_ties = 1;
            }
            // redo the collection with the tie rule into the real list
            CSB_CUDA(cudaMemsetAsync(s.chosen.p, 0, n, c.stream));
            k_collect<<<blocks_for(n), kThreads, 0, c.stream>>>(ks, kt, n, T, T2, use_ties, s.chosen.as<uint8_t>(),
                                                                 s.sel.as<uint32_t>(), s.selcnt.as<uint32_t>(), cap);
            count_launch(c);
        }
    }
    // ---- per-component quota (2 lowest of every component)
    s.best_s.ensure(std::max<uint32_t>(ncomp, 1) * 8ull);
    s.best_t.ensure(std::max<uint32_t>(ncomp, 1) * 8ull);
    for (int round = 0; round < 2 && ncomp > 0; ++round) {
        CSB_CUDA(cudaMemsetAsync(s.best_s.p, 0xFF, ncomp * 8ull, c.stream));
        CSB_CUDA(cudaMemsetAsync(s.best_t.p, 0xFF, ncomp * 8ull, c.stream));
        k_quota_score<<<blocks_for(n), kThreads, 0, c.stream>>>(ks, s.lab.as<uint32_t>(), n, s.qtaken.as<uint8_t>(),
                                                                s.best_s.as<unsigned long long>());
        k_quota_tie<<<blocks_for(n), kThreads, 0, c.stream>>>(ks, kt, s.lab.as<uint32_t>(), n, s.qtaken.as<uint8_t>(),
                                                              s.best_s.as<unsigned long long>(),
                                                              s.best_t.as<unsigned long long>());
        k_quota_take<<<blocks_for(ncomp), kThreads, 0, c.stream>>>(s.best_t.as<unsigned long long>(), ncomp,
                                                                   s.qtaken.as<uint8_t>(), s.chosen.as<uint8_t>(),
                                                                   s.sel.as<uint32_t>(), s.selcnt.as<uint32_t>(), cap);
        count_launch(c, 3);
    }
    check_launch(c, "selection");
    uint32_t m = 0;
    CSB_CUDA(cudaMemcpyAsync(&m, s.selcnt.p, 4, cudaMemcpyDeviceToHost, c.stream));
    CSB_CUDA(cudaStreamSynchronize(c.stream));
    if (m > cap) fail(CS_ERR_STATE, "selection overflow");
    // order the (few hundred) selected ids by (score, rdeg, id) on the host
    std::vector<uint32_t> sel(m);
    copy_d2h(c, sel.data(), s.sel.p, m * 4ull);
    if (m) {
        DevBuf& tmp = c.scratch[6];
        tmp.ensure(m * 16ull + 16);
        k_gather_keys<<<blocks_for(m), kThreads, 0, c.stream>>>(s.sel.as<uint32_t>(), m, ks, kt,
                                                                tmp.as<unsigned long long>());
        count_launch(c);
        std::vector<unsigned long long> keys(2ull * m);
        copy_d2h(c, keys.data(), tmp.p, m * 16ull);
        std::vector<uint32_t> order(m);
        for (uint32_t i = 0; i < m; ++i) order[i] = i;
        std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
            if (keys[2 * a] != keys[2 * b]) return keys[2 * a] < keys[2 * b];
            return keys[2 * a + 1] < keys[2 * b + 1];
        });
        std::vector<uint32_t> sorted(m);
        for (uint32_t i = 0; i < m; ++i) sorted[i] = sel[order[i]];
        sel.swap(sorted);
    }
    g.selected = sel;
    copy_h2d(c, s.sel.p, sel.data(), m * 4ull);
    ev.mark();  // selection
    // ---- bridge MST over the selected set
    std::vector<cs_edge> missing;
    mst_over_subset(g, s, s.sel.as<uint32_t>(), m, &missing);
    ev.mark();  // bridge MST
    // ---- repair_connectivity (only a k-NN graph of several components needs it)
    uint64_t added = 0;
    if (ncomp > 1) {
        // the component of every bridge endpoint, gathered on the device
        std::vector<uint32_t> ends(2 * missing.size()), end_lab(2 * missing.size());
        for (size_t i = 0; i < missing.size(); ++i) {
            ends[2 * i] = missing[i].u;
            ends[2 * i + 1] = missing[i].v;
        }
        if (!ends.empty()) {
            DevBuf& tmp = c.scratch[6];
            tmp.ensure(ends.size() * 8ull + 16);
            uint32_t* d_idx = tmp.as<uint32_t>();
            uint32_t* d_out = d_idx + ends.size();
            copy_h2d(c, d_idx, ends.data(), ends.size() * 4);
            k_gather_u32<<<blocks_for(ends.size()), kThreads, 0, c.stream>>>(
                d_idx, static_cast<uint32_t>(ends.size()), s.lab.as<uint32_t>(), d_out);
            count_launch(c);
            copy_d2h(c, end_lab.data(), d_out, ends.size() * 4);
        }
        HostUF uf(ncomp);
        for (size_t i = 0; i < missing.size(); ++i) uf.unite(end_lab[2 * i], end_lab[2 * i + 1]);
        // merged dense labels, numbered by first component (UnionFind::labels)
        std::vector<uint32_t> merged(ncomp), remap(ncomp, kInvalid);
        uint32_t nc2 = 0;
        for (uint32_t cc = 0; cc < ncomp; ++cc) {
            const uint32_t r = uf.find(cc);
            if (remap[r] == kInvalid) remap[r] = nc2++;
            merged[cc] = remap[r];
        }
        if (nc2 > 1) {
            std::vector<uint32_t> lab(n);
            copy_d2h(c, lab.data(), s.lab.p, n * 4ull);
            std::vector<double> score(n);
            copy_d2h(c, score.data(), s.score.p, n * 8ull);
            uint64_t per = 4;
            if (static_cast<uint64_t>(nc2) * per > 4096) per = std::max<uint64_t>(1, 4096 / nc2);
            std::vector<std::vector<uint32_t>> buckets(nc2);
            for (uint32_t v = 0; v < n; ++v) {
                std::vector<uint32_t>& b = buckets[merged[lab[v]]];
                if (b.size() < per) {
                    b.push_back(v);
                } else {
                    size_t worst = 0;
                    for (size_t t = 1; t < b.size(); ++t) {
                        if (score[b[t]] > score[b[worst]]) worst = t;
                    }
                    if (score[v] < score[b[worst]]) b[worst] = v;
                }
            }
            std::vector<uint32_t> reps;
            for (const auto& b : buckets) reps.insert(reps.end(), b.begin(), b.end());
            if (reps.size() > 4096) {
                std::partial_sort(reps.begin(), reps.begin() + 4096, reps.end(),
                                  [&](uint32_t a, uint32_t b) { return score[a] < score[b]; });
                reps.resize(4096);
            }
            if (reps.size() >= 2) {
                DevBuf d_reps;
                d_reps.ensure(reps.size() * 4);
                copy_h2d(c, d_reps.p, reps.data(), reps.size() * 4);
                std::vector<cs_edge> rep_mst;
                mst_over_subset(g, s, d_reps.as<uint32_t>(), static_cast<uint32_t>(reps.size()), &rep_mst);
                HostUF cuf(nc2);
                for (const cs_edge& e : rep_mst) {
                    if (cuf.unite(merged[lab[e.u]], merged[lab[e.v]])) {
                        missing.push_back(e);
                        ++added;
                    }
                }
            }
        }
    }
    ev.mark();  // repair
    // ---- install the bridges
    g.bridges.ensure(std::max<size_t>(missing.size(), 1) * sizeof(cs_edge));
    if (!missing.empty()) copy_h2d(c, g.bridges.p, missing.data(), missing.size() * sizeof(cs_edge));
    g.nb = missing.size();
    g.n_repair = added;
    g.invalidate_bridges();
    if (out_selected) *out_selected = m;
    if (out_bridges) *out_bridges = missing.size();
    if (out_repair) *out_repair = added;
    if (out_components) *out_components = ncomp;
    ev.mark();
    double ms[7] = {0};
    ev.elapsed(ms, 7);
    cs_bridge_stats& bs = g.last_bridges;
    bs = cs_bridge_stats{};
    bs.connectivity_ms = ms[0];
    bs.hubness_ms = ms[1];
    bs.edges_ms = ms[2];
    bs.selection_ms = ms[3];
    bs.bridge_mst_ms = ms[4];
    bs.repair_ms = ms[5];
    bs.total_ms = ms[0] + ms[1] + ms[2] + ms[3] + ms[4] + ms[5] + ms[6];
    bs.selected = m;
    bs.bridges = missing.size();
    bs.repair = added;
    bs.knn_components = ncomp;
    bs.hub_refreshed = refresh ? 1u : 0u;
    bs.rescored = rescored;
    bs.changed = changed_nodes;
}

}  // namespace csb

using namespace csb;

extern "C" {

cs_status cs_mrd_block(cs_ctx* ctx, const float* host_pts, size_t m, uint32_t dim, uint32_t stride, int32_t metric,
                       const float* host_core, size_t r0, size_t r1, float* host_out) {
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    return guarded(c, [&] {
        (void)dim;
        if (m == 0 || r1 <= r0) return;
        CSB_REQUIRE(host_pts && host_core && host_out, "cs_mrd_block: null buffer");
        CSB_REQUIRE(r1 <= m && stride % 8 == 0 && stride >= dim, "cs_mrd_block: bad range or stride");
        if (metric != CS_METRIC_L2 && metric != CS_METRIC_COSINE)
            fail(CS_ERR_UNSUPPORTED, "mrd_block_gpu: unsupported metric for the device path");
        DevBuf pts, core, out;
        pts.ensure(m * stride * 4);
        core.ensure(m * 4);
        out.ensure((r1 - r0) * m * 4);
        copy_h2d(*c, pts.p, host_pts, m * stride * 4);
        copy_h2d(*c, core.p, host_core, m * 4);
        mrd_rows(*c, pts.as<float>(), static_cast<uint32_t>(m), stride, metric, core.as<float>(),
                 static_cast<uint32_t>(r0), static_cast<uint32_t>(r1), out.as<float>());
        copy_d2h(*c, host_out, out.p, (r1 - r0) * m * 4);
    });
}

cs_status cs_select_bridges(cs_graph* gp, uint64_t* a, uint64_t* b, uint64_t* cc, uint32_t* d) {
    Graph* g = reinterpret_cast<Graph*>(gp);
    return guarded(g ? g->ctx : nullptr, [&] { select_bridges(*g, a, b, cc, d); });
}

cs_status cs_bridge_stats_get(cs_graph* gp, cs_bridge_stats* out) {
    Graph* g = reinterpret_cast<Graph*>(gp);
    return guarded(g ? g->ctx : nullptr, [&] {
        CSB_REQUIRE(out != nullptr, "cs_bridge_stats_get: null output");
        *out = g->last_bridges;
    });
}

cs_status cs_get_selected(cs_graph* gp, uint32_t* out, uint64_t cap, uint64_t* out_count) {
    Graph* g = reinterpret_cast<Graph*>(gp);
    return guarded(g ? g->ctx : nullptr, [&] {
        if (out_count) *out_count = g->selected.size();
        for (uint64_t i = 0; out && i < cap && i < g->selected.size(); ++i) out[i] = g->selected[i];
    });
}

}  // extern "C"
