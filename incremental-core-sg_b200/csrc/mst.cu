// MST_mpts extraction over the resident CORE-SG edge list.
//
// Result contract (both paths): the unique minimum spanning forest under the total
// order (weight bits, edge index) -- the order the reference's Boruvka selects by
// (pack_edge, src/mst.cpp:19-24; mst_boruvka :79-151) -- so the tree is the
// reference's tree edge for edge.  Components are labelled densely in order of their
// smallest node (UnionFind::labels, mst.cpp:48-59).  The weight is the correctly
// rounded exact sum of the tree weights (per-exponent integer bins), which is a
// function of the weight multiset alone.
//
// Boruvka round r, per MST:
//   A  every live edge i (implicit "all edges" in rounds 0-1, else the worklist)
//      finds the roots of its endpoints; if they differ it atomicMin's the packed
//      key (w' bits << 32 | i) into best[root] of both, appends itself to the next
//      worklist, and the first toucher of a root appends the root to `touched`.
//   B  every touched root takes its best edge, marks it in the tree bitmap (the
//      first marker adds its weight and unites the endpoints; a doubly chosen edge
//      is counted once) and resets best[root].
// Roots are linked larger-under-smaller, so after the last round find(v) is the
// smallest node of v's component, which is what the dense labelling needs.
//
// Plain path (cs_extract): edges(mpts) materialised per call exactly as
// CoreSG::edges does, then one kernel per phase with a host read of the counters
// after every phase A (the reference's round loop, moved to the device).  The
// batched sweep (cs_extract_sweep) is in sweep.cu; it shares the labelling and
// exact-sum helpers defined here.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>

#include "common.cuh"
#include "engine.hpp"

namespace csb {

struct MstView {
    uint32_t* parent;
    unsigned long long* best;
    uint32_t* touched;
    uint32_t* wl0;
    uint32_t* wl1;
    uint32_t* bitmap;
    unsigned long long* bins;
    uint32_t* ctr;  // [0] wc0 [1] wc1 [2] tc0 [3] tc1
    const float* core;
    uint32_t n;     // nodes (bounds every union-find chase)
};

namespace {

constexpr int kMaxRounds = 64;
constexpr int kThreads = 256;
constexpr int kTileWords = 2048;  // compaction tile: 256 threads x 8 words

inline unsigned blocks_for(uint64_t work, int threads = kThreads) {
    uint64_t b = (work + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > (1u << 30)) b = 1u << 30;
    return static_cast<unsigned>(b);
}

__device__ __forceinline__ uint32_t bin_of(uint32_t bits) {
    const uint32_t e = (bits >> 23) & 0xFFu;
    return e ? e : 1u;
}
__device__ __forceinline__ uint32_t mant_of(uint32_t bits) {
    const uint32_t e = (bits >> 23) & 0xFFu;
    return (bits & 0x7FFFFFu) | (e ? 0x800000u : 0u);
}

/// Phase A for one edge.  Must be called by all 32 lanes of a warp together
/// (`valid` false for padding lanes).
template <bool kReweight>
__device__ __forceinline__ void edge_step(const MstView& m, uint32_t i, bool valid, uint32_t u,
                                          uint32_t v, float w, uint32_t n, int r, bool write_wl) {
    bool live = false, t1 = false, t2 = false;
    uint32_t cu = 0, cv = 0;
    if (valid && u < n && v < n) {
        if (kReweight) w = max_ref(w, max_ref(__ldg(m.core + u), __ldg(m.core + v)));
        cu = uf_find(m.parent, u, n, nullptr);
        cv = uf_find(m.parent, v, n, nullptr);
        live = cu != cv;
        if (live) {
            const unsigned long long key = pack_key(w, i);
            t1 = atomicMin(m.best + cu, key) == kNoKey;
            t2 = atomicMin(m.best + cv, key) == kNoKey;
        }
    }
    if (write_wl) {
        const int o = (r + 1) & 1;
        const uint32_t slot = warp_append(live, m.ctr + o);
        if (live) (o ? m.wl1 : m.wl0)[slot] = i;
    }
    uint32_t* tc = m.ctr + 2 + (r & 1);
    const uint32_t s1 = warp_append(t1, tc);
    if (t1) m.touched[s1] = cu;
    const uint32_t s2 = warp_append(t2, tc);
    if (t2) m.touched[s2] = cv;
}

/// Phase B for one touched root.
__device__ __forceinline__ void root_step(const MstView& m, uint32_t c, const uint32_t* __restrict__ eu,
                                          const uint32_t* __restrict__ ev, unsigned long long* sbins,
                                          int* status) {
    const unsigned long long key = __ldcg(m.best + c);
    m.best[c] = kNoKey;
    if (key == kNoKey) return;
    const uint32_t i = static_cast<uint32_t>(key);
    const uint32_t bits = static_cast<uint32_t>(key >> 32);
    const uint32_t bit = 1u << (i & 31u);
    const uint32_t old = atomicOr(m.bitmap + (i >> 5), bit);
    if (!(old & bit)) {
        atomicAdd(sbins + bin_of(bits), static_cast<unsigned long long>(mant_of(bits)));
        uf_unite(m.parent, __ldg(eu + i), __ldg(ev + i), m.n, status);
    }
}

__device__ __forceinline__ void flush_bins(unsigned long long* sbins, unsigned long long* gbins) {
    __syncthreads();
    for (int b = threadIdx.x; b < 256; b += blockDim.x) {
        const unsigned long long x = sbins[b];
        if (x) {
            atomicAdd(gbins + b, x);
            sbins[b] = 0;
        }
    }
    __syncthreads();
}

// ---- plain path kernels -------------------------------------------------------------

__global__ void k_iota(uint32_t* __restrict__ parent, uint64_t total, uint32_t n) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < total) parent[i] = static_cast<uint32_t>(i % n);
}

__global__ void k_phase_a(MstView m, const uint32_t* __restrict__ eu, const uint32_t* __restrict__ ev,
                          const float* __restrict__ ew, uint32_t n, uint32_t count, int r) {
    const bool implicit = r <= 1;
    const uint64_t padded = (static_cast<uint64_t>(count) + 31) & ~31ull;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    const uint32_t* in = (r & 1) ? m.wl1 : m.wl0;
    for (uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < padded; t += stride) {
        const bool valid = t < count;
        uint32_t i = 0, u = 0, v = 0;
        float w = 0.0f;
        if (valid) {
            i = implicit ? static_cast<uint32_t>(t) : in[t];
            u = __ldg(eu + i);
            v = __ldg(ev + i);
            w = __ldg(ew + i);
        }
        edge_step<false>(m, i, valid, u, v, w, n, r, r >= 1);
    }
}

__global__ void k_phase_b(MstView m, const uint32_t* __restrict__ eu, const uint32_t* __restrict__ ev,
                          uint32_t count, int* status) {
    __shared__ unsigned long long sbins[256];
    for (int b = threadIdx.x; b < 256; b += blockDim.x) sbins[b] = 0;
    __syncthreads();
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < count; t += stride) {
        root_step(m, m.touched[t], eu, ev, sbins, status);
    }
    flush_bins(sbins, m.bins);
}

// ---- labels: dense, numbered by smallest node -------------------------------------------

__device__ __forceinline__ uint32_t block_prefix_flags(bool f, uint32_t* total) {
    __shared__ uint32_t wsum[32];
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const unsigned m = __ballot_sync(0xFFFFFFFFu, f);
    const uint32_t in_warp = __popc(m & ((1u << lane) - 1u));
    if (lane == 0) wsum[warp] = __popc(m);
    __syncthreads();
    uint32_t before = 0, all = 0;
    const unsigned nw = blockDim.x >> 5;
    for (unsigned w = 0; w < nw; ++w) {
        if (w < warp) before += wsum[w];
        all += wsum[w];
    }
    __syncthreads();
    if (total) *total = all;
    return before + in_warp;
}

__global__ void k_label_roots(uint32_t* __restrict__ parent_all, uint32_t n, uint32_t* __restrict__ lab_all,
                              uint32_t* __restrict__ bc, uint32_t nb) {
    const uint32_t j = blockIdx.y;
    uint32_t* parent = parent_all + static_cast<uint64_t>(j) * n;
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    bool root = false;
    if (v < n) {
        const uint32_t r = uf_find(parent, v, n, nullptr);
        lab_all[static_cast<uint64_t>(j) * n + v] = r;
        root = r == v;
    }
    uint32_t total;
    block_prefix_flags(root, &total);
    if (threadIdx.x == 0) bc[static_cast<uint64_t>(j) * nb + blockIdx.x] = total;
}

__global__ void k_label_dense(const uint32_t* __restrict__ parent_all, uint32_t n, uint32_t* __restrict__ lab_all,
                              const uint32_t* __restrict__ bc, uint32_t nb) {
    const uint32_t j = blockIdx.y;
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    const bool root = v < n && __ldcg(parent_all + static_cast<uint64_t>(j) * n + v) == v;
    const uint32_t pre = block_prefix_flags(root, nullptr);
    if (root) lab_all[static_cast<uint64_t>(j) * n + v] = bc[static_cast<uint64_t>(j) * nb + blockIdx.x] + pre;
}

__global__ void k_label_fill(const uint32_t* __restrict__ parent_all, uint32_t n, uint32_t* __restrict__ lab_all) {
    const uint32_t j = blockIdx.y;
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const uint64_t base = static_cast<uint64_t>(j) * n;
    if (__ldcg(parent_all + base + v) != v) lab_all[base + v] = lab_all[base + lab_all[base + v]];
}

/// Exclusive scan of `nt` u32 tile counts per MST (one block per MST); total -> tot[j].
__global__ void k_scan_tiles(uint32_t* __restrict__ tiles, uint32_t nt, unsigned long long* __restrict__ tot) {
    constexpr int kItems = 8;  // consecutive tiles per thread and pass
    const uint32_t j = blockIdx.x;
    uint32_t* t = tiles + static_cast<uint64_t>(j) * nt;
    __shared__ uint32_t wsum[32];
    __shared__ uint32_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (uint32_t base = 0; base < nt; base += blockDim.x * kItems) {
        const uint32_t first = base + threadIdx.x * kItems;
        uint32_t x[kItems], sum = 0;
#pragma unroll
        for (int s = 0; s < kItems; ++s) {
            x[s] = first + s < nt ? t[first + s] : 0u;
            sum += x[s];
        }
        uint32_t incl = sum;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= static_cast<unsigned>(o)) incl += y;
        }
        if (lane == 31) wsum[warp] = incl;
        __syncthreads();
        uint32_t before = 0, all = 0;
        for (unsigned w = 0; w < nw; ++w) {
            if (w < warp) before += wsum[w];
            all += wsum[w];
        }
        uint32_t run = carry + before + incl - sum;
#pragma unroll
        for (int s = 0; s < kItems; ++s) {
            if (first + s < nt) t[first + s] = run;
            run += x[s];
        }
        __syncthreads();
        if (threadIdx.x == 0) carry += all;
        __syncthreads();
    }
    if (threadIdx.x == 0) tot[j] = carry;
}

// ---- tree bitmap -> edge list (ascending edge index) -----------------------------------

__global__ void k_bits_tiles(const uint32_t* __restrict__ bitmap, uint32_t W, uint32_t nt,
                             uint32_t* __restrict__ tiles) {
    const uint32_t j = blockIdx.y;
    const uint32_t* bm = bitmap + static_cast<uint64_t>(j) * W;
    uint32_t s = 0;
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kTileWords + threadIdx.x * 8ull;
#pragma unroll
    for (int t = 0; t < 8; ++t) {
        if (base + t < W) s += __popc(__ldcg(bm + base + t));
    }
    __shared__ uint32_t red[kThreads];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = kThreads / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) tiles[static_cast<uint64_t>(j) * nt + blockIdx.x] = red[0];
}

__global__ void k_bits_emit(const uint32_t* __restrict__ bitmap, uint32_t W, uint32_t nt,
                            const uint32_t* __restrict__ tiles, const uint32_t* __restrict__ eu,
                            const uint32_t* __restrict__ ev, const float* __restrict__ ew,
                            const float* __restrict__ core, uint32_t n, uint64_t cap,
                            cs_edge* __restrict__ out, int* status) {
    const uint32_t j = blockIdx.y;
    const uint32_t* bm = bitmap + static_cast<uint64_t>(j) * W;
    const float* cj = core ? core + static_cast<uint64_t>(j) * n : nullptr;
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kTileWords + threadIdx.x * 8ull;
    uint32_t words[8];
    uint32_t s = 0;
#pragma unroll
    for (int t = 0; t < 8; ++t) {
        words[t] = (base + t < W) ? __ldcg(bm + base + t) : 0u;
        s += __popc(words[t]);
    }
    // block exclusive scan of s
    __shared__ uint32_t wsum[32];
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint32_t incl = s;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= static_cast<unsigned>(o)) incl += y;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    uint32_t before = 0;
    for (unsigned w = 0; w < nw && w < warp; ++w) before += wsum[w];
    uint64_t pos = tiles[static_cast<uint64_t>(j) * nt + blockIdx.x] + before + incl - s;
    cs_edge* o = out + static_cast<uint64_t>(j) * cap;
#pragma unroll
    for (int t = 0; t < 8; ++t) {
        uint32_t bits = words[t];
        while (bits) {
            const uint32_t b = __ffs(bits) - 1;
            bits &= bits - 1;
            const uint32_t i = static_cast<uint32_t>((base + t) * 32 + b);
            const uint32_t u = eu[i], v = ev[i];
            float w = ew[i];
            if (cj) w = max_ref(w, max_ref(cj[u], cj[v]));
            if (pos < cap) {
                cs_edge e;
                e.u = u;
                e.v = v;
                e.w = w;
                o[pos] = e;
            } else {
                atomicOr(status, kStatusCapacity);
            }
            ++pos;
        }
    }
}

}  // namespace

// ============================================================================
// exact weight from per-exponent bins
// ============================================================================

/// Correctly rounded double of sum_e bins[e] * 2^(e-150) (bins hold 24-bit
/// mantissas with the hidden bit; bin 255 non-empty means an infinite weight).
double exact_sum_from_bins(const uint64_t* bins) {
    if (bins[255]) return INFINITY;
    constexpr int L = 12;  // 384 bits; bins[e] (< 2^64) lands at bit e-1
    uint64_t limb[L] = {0};
    for (int e = 1; e < 255; ++e) {
        uint64_t x = bins[e];
        if (!x) continue;
        const int sh = e - 1;
        int li = sh / 32;
        const int off = sh % 32;
        unsigned __int128 y = static_cast<unsigned __int128>(x) << off;
        while (y && li < L) {
            const unsigned __int128 s = static_cast<unsigned __int128>(limb[li]) + static_cast<uint64_t>(y & 0xFFFFFFFFu);
            limb[li] = static_cast<uint64_t>(s & 0xFFFFFFFFu);
            y = (y >> 32) + (s >> 32);
            ++li;
        }
    }
    int top = -1;
    for (int li = L - 1; li >= 0 && top < 0; --li) {
        if (!limb[li]) continue;
        for (int b = 31; b >= 0; --b) {
            if (limb[li] >> b & 1u) {
                top = li * 32 + b;
                break;
            }
        }
    }
    if (top < 0) return 0.0;
    auto bit = [&](int p) -> unsigned { return p < 0 ? 0u : static_cast<unsigned>((limb[p / 32] >> (p % 32)) & 1u); };
    uint64_t mant = 0;
    const int low = top - 52;
    for (int p = top; p >= low && p >= 0; --p) mant = (mant << 1) | bit(p);
    if (low <= 0) return std::ldexp(static_cast<double>(mant), -149);
    const unsigned rb = bit(low - 1);
    unsigned sticky = 0;
    for (int p = low - 2; p >= 0 && !sticky; --p) sticky |= bit(p);
    if (rb && (sticky || (mant & 1u))) ++mant;
    return std::ldexp(static_cast<double>(mant), low - 149);
}

// ============================================================================
// shared finishing: labels + compaction for K MSTs
// ============================================================================

void launch_labels(Ctx& c, uint32_t* parent_all, uint32_t n, uint32_t K, uint32_t* lab_all,
                   uint32_t* bc, unsigned long long* ncomp) {
    const uint32_t nb = blocks_for(n);
    dim3 grid(nb, K);
    k_label_roots<<<grid, kThreads, 0, c.stream>>>(parent_all, n, lab_all, bc, nb);
    k_scan_tiles<<<K, 1024, 0, c.stream>>>(bc, nb, ncomp);
    k_label_dense<<<grid, kThreads, 0, c.stream>>>(parent_all, n, lab_all, bc, nb);
    k_label_fill<<<grid, kThreads, 0, c.stream>>>(parent_all, n, lab_all);
    count_launch(c, 4);
}

void launch_scan_tiles(Ctx& c, uint32_t* tiles, uint32_t nt, uint32_t K, unsigned long long* totals) {
    k_scan_tiles<<<K, 1024, 0, c.stream>>>(tiles, nt, totals);
    count_launch(c);
}

namespace {

void launch_compact(Ctx& c, const uint32_t* bitmap, uint32_t W, uint32_t K, uint32_t* tiles,
                    unsigned long long* nedges, const uint32_t* eu, const uint32_t* ev, const float* ew,
                    const float* core, uint32_t n, uint64_t cap, cs_edge* out, int* status) {
    const uint32_t nt = std::max<uint32_t>(1, (W + kTileWords - 1) / kTileWords);
    dim3 grid(nt, K);
    k_bits_tiles<<<grid, kThreads, 0, c.stream>>>(bitmap, W, nt, tiles);
    k_scan_tiles<<<K, 1024, 0, c.stream>>>(tiles, nt, nedges);
    k_bits_emit<<<grid, kThreads, 0, c.stream>>>(bitmap, W, nt, tiles, eu, ev, ew, core, n, cap, out, status);
    count_launch(c, 3);
}

void status_check(Ctx& c, const int* d_status) {
    int st = 0;
    CSB_CUDA(cudaMemcpyAsync(&st, d_status, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    CSB_CUDA(cudaStreamSynchronize(c.stream));
    if (st & kStatusBarrierTimeout) fail(CS_ERR_TIMEOUT, "MST sweep: a grid barrier wait ran out (device status 0x" + std::to_string(st) + ")");
    if (st & kStatusUnionLimit) fail(CS_ERR_TIMEOUT, "MST: a union retry loop ran out");
    if (st & kStatusRoundLimit) fail(CS_ERR_TIMEOUT, "MST: Boruvka round limit reached");
    if (st & kStatusCapacity) fail(CS_ERR_STATE, "MST: tree larger than n-1 edges (inconsistent state)");
}

}  // namespace

// ============================================================================
// plain per-mpts path
// ============================================================================

void extract_plain(Graph& g, uint32_t mpts, cs_edge* out_edges, uint32_t* out_labels, MstHost* res) {
    Ctx& c = *g.ctx;
    const uint32_t n = static_cast<uint32_t>(g.n);
    if (mpts == 0) mpts = 1;
    if (mpts > g.k) fail(CS_ERR_INVALID, "CoreSG::edges: mpts exceeds k_max");
    // edges(mpts), materialised and reweighted (the reference rebuilds them per call)
    Graph::PlainWork& pw = g.plain;
    DevBuf &eu = pw.eu, &ev = pw.ev, &ew = pw.ew, &core = pw.core;
    const uint64_t E = graph_materialize_edges(g, mpts, true, eu, ev, ew, core, c.scratch[0],
                                               c.scratch[1], c.scratch[2]);
    const uint32_t W = static_cast<uint32_t>((E + 31) / 32) + 1;
    DevBuf &parent = pw.parent, &best = pw.best, &touched = pw.touched, &wl = pw.wl, &bitmap = pw.bitmap,
           &bins = pw.bins, &ctr = pw.ctr, &tiles = pw.tiles, &lab = pw.lab, &outb = pw.out;
    parent.ensure(std::max<uint64_t>(n, 1) * 4);
    best.ensure(std::max<uint64_t>(n, 1) * 8);
    touched.ensure(std::max<uint64_t>(n, 1) * 4);
    wl.ensure(std::max<uint64_t>(E, 1) * 8);
    bitmap.ensure(static_cast<uint64_t>(W) * 4);
    bins.ensure(256 * 8 + 64);
    ctr.ensure(64);
    const uint32_t nbl = blocks_for(n);
    const uint32_t ntl = std::max<uint32_t>(1, (W + kTileWords - 1) / kTileWords);
    tiles.ensure((static_cast<uint64_t>(nbl) + ntl + 2) * 4 + 64);
    int* status = c.status.as<int>();
    CSB_CUDA(cudaMemsetAsync(status, 0, 4, c.stream));
    CSB_CUDA(cudaMemsetAsync(best.p, 0xFF, std::max<uint64_t>(n, 1) * 8, c.stream));
    CSB_CUDA(cudaMemsetAsync(bitmap.p, 0, static_cast<uint64_t>(W) * 4, c.stream));
    CSB_CUDA(cudaMemsetAsync(bins.p, 0, 256 * 8 + 64, c.stream));
    CSB_CUDA(cudaMemsetAsync(ctr.p, 0, 64, c.stream));
    if (n) {
        k_iota<<<blocks_for(n), kThreads, 0, c.stream>>>(parent.as<uint32_t>(), n, n);
        count_launch(c);
    }
    MstView m;
    m.parent = parent.as<uint32_t>();
    m.best = best.as<unsigned long long>();
    m.touched = touched.as<uint32_t>();
    m.wl0 = wl.as<uint32_t>();
    m.wl1 = wl.as<uint32_t>() + std::max<uint64_t>(E, 1);
    m.bitmap = bitmap.as<uint32_t>();
    m.bins = bins.as<unsigned long long>();
    m.ctr = ctr.as<uint32_t>();
    m.core = nullptr;
    m.n = static_cast<uint32_t>(n);
    const unsigned grid_cap = static_cast<unsigned>(c.sm_count) * 8u;
    uint32_t in_count = static_cast<uint32_t>(E);
    uint32_t hc[4];
    int r = 0;
    for (; r < kMaxRounds; ++r) {
        if (r <= 1) in_count = static_cast<uint32_t>(E);
        const unsigned gA = std::min<unsigned>(grid_cap, blocks_for(in_count));
        k_phase_a<<<gA, kThreads, 0, c.stream>>>(m, eu.as<uint32_t>(), ev.as<uint32_t>(), ew.as<float>(),
                                                  n, in_count, r);
        count_launch(c);
        check_launch(c, "boruvka phase A");
        // the host reads the round's counters, as the reference's round loop does
        CSB_CUDA(cudaMemcpyAsync(hc, m.ctr, sizeof(hc), cudaMemcpyDeviceToHost, c.stream));
        CSB_CUDA(cudaStreamSynchronize(c.stream));
        const uint32_t tcount = hc[2 + (r & 1)];
        if (tcount == 0) break;
        const unsigned gB = std::min<unsigned>(grid_cap, blocks_for(tcount));
        k_phase_b<<<gB, kThreads, 0, c.stream>>>(m, eu.as<uint32_t>(), ev.as<uint32_t>(), tcount, status);
        count_launch(c);
        check_launch(c, "boruvka phase B");
        in_count = hc[(r + 1) & 1];
        CSB_CUDA(cudaMemsetAsync(m.ctr + (r & 1), 0, 4, c.stream));
        CSB_CUDA(cudaMemsetAsync(m.ctr + 2 + ((r + 1) & 1), 0, 4, c.stream));
    }
    if (r == kMaxRounds) fail(CS_ERR_TIMEOUT, "MST: Boruvka round limit reached");

    DevBuf& counts = pw.counts;
    counts.ensure(64);
    unsigned long long* d_ncomp = counts.as<unsigned long long>();
    unsigned long long* d_nedges = d_ncomp + 1;
    lab.ensure(std::max<uint64_t>(n, 1) * 4);
    if (n) launch_labels(c, m.parent, n, 1, lab.as<uint32_t>(), tiles.as<uint32_t>(), d_ncomp);
    else CSB_CUDA(cudaMemsetAsync(d_ncomp, 0, 8, c.stream));
    const uint64_t cap = n ? n - 1 : 0;
    outb.ensure(std::max<uint64_t>(cap, 1) * sizeof(cs_edge));
    launch_compact(c, m.bitmap, W, 1, tiles.as<uint32_t>() + nbl + 1, d_nedges, eu.as<uint32_t>(),
                   ev.as<uint32_t>(), ew.as<float>(), nullptr, n, cap, outb.as<cs_edge>(), status);
    check_launch(c, "MST finish");
    status_check(c, status);
    unsigned long long hcount[2];
    uint64_t hbins[256];
    CSB_CUDA(cudaMemcpyAsync(hcount, counts.p, 16, cudaMemcpyDeviceToHost, c.stream));
    CSB_CUDA(cudaMemcpyAsync(hbins, bins.p, sizeof(hbins), cudaMemcpyDeviceToHost, c.stream));
    CSB_CUDA(cudaStreamSynchronize(c.stream));
    res->ncomp = static_cast<uint32_t>(hcount[0]);
    res->nedges = hcount[1];
    res->weight = exact_sum_from_bins(hbins);
    if (out_edges && res->nedges) copy_d2h(c, out_edges, outb.p, res->nedges * sizeof(cs_edge));
    if (out_labels && n) copy_d2h(c, out_labels, lab.p, static_cast<uint64_t>(n) * 4);
}

}  // namespace csb

// ============================================================================
// C API
// ============================================================================

using namespace csb;

extern "C" {

cs_status cs_extract(cs_graph* gp, uint32_t mpts, cs_edge* out_edges, uint32_t* out_labels,
                     uint64_t* out_nedges, uint32_t* out_ncomp, double* out_weight) {
    Graph* g = reinterpret_cast<Graph*>(gp);
    return guarded(g ? g->ctx : nullptr, [&] {
        MstHost r;
        extract_plain(*g, mpts, out_edges, out_labels, &r);
        if (out_nedges) *out_nedges = r.nedges;
        if (out_ncomp) *out_ncomp = r.ncomp;
        if (out_weight) *out_weight = r.weight;
    });
}

}  // extern "C"

// ============================================================================
// Allocation-free MST entry point (cs_mst_noalloc)
// ============================================================================
//
// For callers that cannot allocate device memory themselves or let a library do it:
// plugins whose host application owns every device allocation (a fixed memory pool
// or arena handed out by the host), and code that runs where the allocation API
// must not be touched.  The caller passes the edge list and the output buffers as
// device pointers; every intermediate the Boruvka rounds need lives in one
// file-scope __device__ array of fixed size, which each GPU that loads this library
// holds until the process exits.  No cudaMalloc, cudaFree, pinned allocation or
// context object is involved.
//
// The same kernels as the plain per-mpts path (k_iota, k_phase_a, k_phase_b, the
// label and compaction kernels) run on the caller's stream, so the result is the
// same tree: the unique minimum spanning forest under (weight bits, edge index).
namespace csb {
namespace {

constexpr uint32_t kNoAllocMaxNodes = 131072;   // n limit
constexpr uint64_t kNoAllocMaxEdges = 1048576;  // m limit
constexpr size_t kNoAllocScratchBytes = size_t(12) << 20;  // 12 MiB per GPU

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

/// Device address of the scratch array in the current context.  An address of a
/// __device__ variable belongs to one CUDA context (a caller that makes its own
/// context current, or resets the device, gets a different one), so it is looked up
/// on every call, with the caller's device current, and never cached.
unsigned char* noalloc_scratch() {
    void* ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || !ptr) {
        cudaGetLastError();
        fail(CS_ERR_CUDA, std::string("cs_mst_noalloc: cudaGetSymbolAddress of the scratch array failed: ") +
                              cudaGetErrorString(e));
    }
    return static_cast<unsigned char*>(ptr);
}

constexpr int kNoAllocBadEndpoint = 1;
constexpr int kNoAllocBadWeight = 2;

/// Input check of a caller's edge list: every endpoint below n, every weight
/// non-negative with the sign bit clear and not NaN (+inf is allowed: an empty
/// neighbourhood has an infinite core distance).  The packed (weight bits, index) key
/// orders weights only under those conditions, and the Boruvka kernels index node
/// arrays by the endpoints without range checks.
__global__ void k_noalloc_check(const uint32_t* __restrict__ eu, const uint32_t* __restrict__ ev,
                                const float* __restrict__ ew, uint64_t m, uint32_t n, int* bad) {
    int flags = 0;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < m;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        if (eu[i] >= n || ev[i] >= n) flags |= kNoAllocBadEndpoint;
        const uint32_t b = __float_as_uint(ew[i]);
        if ((b >> 31) || (b & 0x7FFFFFFFu) > 0x7F800000u) flags |= kNoAllocBadWeight;
    }
    flags = __reduce_or_sync(0xFFFFFFFFu, flags);
    if (flags && (threadIdx.x & 31u) == 0) atomicOr(bad, flags);
}

struct Carver {
    unsigned char* base;
    size_t off = 0;
    template <typename T>
    T* take(uint64_t count) {
        off = (off + 255) & ~size_t(255);
        T* p = reinterpret_cast<T*>(base + off);
        off += static_cast<size_t>(count) * sizeof(T);
        return p;
    }
};

/// Bytes the carve below needs for n nodes and m edges.
size_t noalloc_bytes(uint32_t n, uint64_t m) {
    const uint64_t W = m / 32 + 1;
    const uint64_t nbl = blocks_for(n), ntl = std::max<uint64_t>(1, (W + kTileWords - 1) / kTileWords);
    const uint64_t parts[] = {n * 4ull, n * 8ull, n * 4ull, std::max<uint64_t>(m, 1) * 4, std::max<uint64_t>(m, 1) * 4,
                              W * 4, 256 * 8, 64, 64, 64, (nbl + ntl + 2) * 4};
    size_t total = 0;
    for (uint64_t p : parts) total = ((total + 255) & ~size_t(255)) + p;
    return total;
}

static_assert(kNoAllocMaxNodes % 256 == 0, "limit");

}  // namespace
}  // namespace csb

extern "C" cs_status cs_mst_noalloc(const uint32_t* d_u, const uint32_t* d_v, const float* d_w, uint64_t m,
                                    uint32_t n, cs_edge* d_out_edges, uint32_t* d_out_labels, uint64_t* out_nedges,
                                    uint32_t* out_ncomp, double* out_weight, void* stream) {
    using namespace csb;
    try {
        if (n > kNoAllocMaxNodes)
            fail(CS_ERR_INVALID, "cs_mst_noalloc: n = " + std::to_string(n) + " exceeds the limit of " +
                                     std::to_string(kNoAllocMaxNodes) + " nodes");
        if (m > kNoAllocMaxEdges)
            fail(CS_ERR_INVALID, "cs_mst_noalloc: m = " + std::to_string(m) + " exceeds the limit of " +
                                     std::to_string(kNoAllocMaxEdges) + " edges");
        if (noalloc_bytes(n, m) > kNoAllocScratchBytes) fail(CS_ERR_INVALID, "cs_mst_noalloc: scratch too small");
        if (m > 0 && (!d_u || !d_v || !d_w)) fail(CS_ERR_INVALID, "cs_mst_noalloc: null edge array");
        if (n > 1 && !d_out_edges) fail(CS_ERR_INVALID, "cs_mst_noalloc: null output edge buffer");
        if (n == 0) {
            if (out_nedges) *out_nedges = 0;
            if (out_ncomp) *out_ncomp = 0;
            if (out_weight) *out_weight = 0.0;
            return CS_OK;
        }
        int device = 0;
        CSB_CUDA(cudaGetDevice(&device));
        Carver cv{noalloc_scratch()};
        const cudaStream_t s = static_cast<cudaStream_t>(stream);
        // a stack Ctx only carries the stream to the shared launch helpers; it owns
        // no device memory
        Ctx tmp;
        tmp.device = device;
        tmp.stream = s;
        const uint32_t W = static_cast<uint32_t>(m / 32) + 1;
        const uint32_t nbl = blocks_for(n);
        const uint32_t ntl = std::max<uint32_t>(1, (W + kTileWords - 1) / kTileWords);
        MstView mv;
        mv.parent = cv.take<uint32_t>(n);
        mv.best = cv.take<unsigned long long>(n);
        mv.touched = cv.take<uint32_t>(n);
        mv.wl0 = cv.take<uint32_t>(std::max<uint64_t>(m, 1));
        mv.wl1 = cv.take<uint32_t>(std::max<uint64_t>(m, 1));
        mv.bitmap = cv.take<uint32_t>(W);
        mv.bins = cv.take<unsigned long long>(256);
        mv.ctr = cv.take<uint32_t>(16);
        mv.core = nullptr;
        mv.n = static_cast<uint32_t>(n);
        int* status = cv.take<int>(16);
        unsigned long long* counts = cv.take<unsigned long long>(8);
        uint32_t* tiles = cv.take<uint32_t>(static_cast<uint64_t>(nbl) + ntl + 2);
        // the array keeps the previous call's contents: reset what must start empty
        CSB_CUDA(cudaMemsetAsync(mv.best, 0xFF, static_cast<size_t>(n) * 8, s));
        CSB_CUDA(cudaMemsetAsync(mv.bitmap, 0, static_cast<size_t>(W) * 4, s));
        CSB_CUDA(cudaMemsetAsync(mv.bins, 0, 256 * 8, s));
        CSB_CUDA(cudaMemsetAsync(mv.ctr, 0, 64, s));
        CSB_CUDA(cudaMemsetAsync(status, 0, 64, s));
        CSB_CUDA(cudaMemsetAsync(counts, 0, 64, s));
        int sms = 148;
        CSB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
        const unsigned grid_cap = static_cast<unsigned>(sms) * 8u;
        if (m > 0) {
            int bad = 0;
            k_noalloc_check<<<std::min<unsigned>(grid_cap, blocks_for(m)), kThreads, 0, s>>>(d_u, d_v, d_w, m, n,
                                                                                           status + 1);
            CSB_CUDA(cudaGetLastError());
            CSB_CUDA(cudaMemcpyAsync(&bad, status + 1, sizeof(int), cudaMemcpyDeviceToHost, s));
            CSB_CUDA(cudaStreamSynchronize(s));
            if (bad & kNoAllocBadEndpoint)
                fail(CS_ERR_INVALID, "cs_mst_noalloc: an edge endpoint is >= n = " + std::to_string(n));
            if (bad & kNoAllocBadWeight)
                fail(CS_ERR_INVALID, "cs_mst_noalloc: an edge weight is negative (sign bit set) or NaN");
        }
        k_iota<<<blocks_for(n), kThreads, 0, s>>>(mv.parent, n, n);
        uint32_t in_count = static_cast<uint32_t>(m);
        uint32_t hc[4];
        int r = 0;
        for (; r < kMaxRounds; ++r) {
            if (r <= 1) in_count = static_cast<uint32_t>(m);
            k_phase_a<<<std::min<unsigned>(grid_cap, blocks_for(in_count)), kThreads, 0, s>>>(mv, d_u, d_v, d_w, n,
                                                                                             in_count, r);
            CSB_CUDA(cudaGetLastError());
            CSB_CUDA(cudaMemcpyAsync(hc, mv.ctr, sizeof(hc), cudaMemcpyDeviceToHost, s));
            CSB_CUDA(cudaStreamSynchronize(s));
            const uint32_t tcount = hc[2 + (r & 1)];
            if (tcount == 0) break;
            k_phase_b<<<std::min<unsigned>(grid_cap, blocks_for(tcount)), kThreads, 0, s>>>(mv, d_u, d_v, tcount, status);
            CSB_CUDA(cudaGetLastError());
            in_count = hc[(r + 1) & 1];
            CSB_CUDA(cudaMemsetAsync(mv.ctr + (r & 1), 0, 4, s));
            CSB_CUDA(cudaMemsetAsync(mv.ctr + 2 + ((r + 1) & 1), 0, 4, s));
        }
        if (r == kMaxRounds) fail(CS_ERR_TIMEOUT, "cs_mst_noalloc: Boruvka round limit reached");
        if (d_out_labels) launch_labels(tmp, mv.parent, n, 1, d_out_labels, tiles, counts);
        launch_compact(tmp, mv.bitmap, W, 1, tiles + nbl + 1, counts + 1, d_u, d_v, d_w, nullptr, n, n - 1,
                       d_out_edges, status);
        CSB_CUDA(cudaGetLastError());
        int st = 0;
        unsigned long long hcount[2] = {0, 0};
        uint64_t hbins[256];
        CSB_CUDA(cudaMemcpyAsync(&st, status, sizeof(int), cudaMemcpyDeviceToHost, s));
        CSB_CUDA(cudaMemcpyAsync(hcount, counts, sizeof(hcount), cudaMemcpyDeviceToHost, s));
        CSB_CUDA(cudaMemcpyAsync(hbins, mv.bins, sizeof(hbins), cudaMemcpyDeviceToHost, s));
        CSB_CUDA(cudaStreamSynchronize(s));
        if (st & kStatusUnionLimit) fail(CS_ERR_TIMEOUT, "cs_mst_noalloc: a union retry loop ran out");
        if (st & kStatusCapacity) fail(CS_ERR_STATE, "cs_mst_noalloc: tree larger than n-1 edges");
        if (out_nedges) *out_nedges = hcount[1];
        if (out_ncomp) *out_ncomp = static_cast<uint32_t>(n - hcount[1]);
        if (out_weight) *out_weight = exact_sum_from_bins(hbins);
        return CS_OK;
    } catch (const Error& e) {
        set_thread_error(e.what());
        return e.status;
    } catch (const std::exception& e) {
        set_thread_error(e.what());
        return CS_ERR_INVALID;
    }
}
