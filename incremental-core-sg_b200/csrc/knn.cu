// Dynamic NN-Descent on the device.
//
// The reference's device descent (cuda/nndescent_kernels.cu:129-287) runs one CTA
// per node and inserts every accepted pair into the sorted lists under per-node
// spin locks.  Here a round is three warp-per-node kernels and no locks:
//
//   sample  take up to `sample` new and 3*sample old entries from the closest end
//           of the list, clear the taken new flags, and publish the node into its
//           samples' bounded reverse lists (Algorithm 1 lines 6-18 of the paper;
//           src/nndescent.cpp:199-260).
//   join    stage the rows of new = sampled new + reverse new and old = sampled old
//           + reverse old in shared memory, evaluate new x new and new x old with the
//           reference's L2 association order, and offer every pair that beats an
//           endpoint's current k-th distance as a packed 64-bit key
//           (rank-distance bits << 32 | id) into that endpoint's candidate slots with
//           one atomicMin -- the slot is picked by hashing the id, so a repeated
//           candidate collapses onto itself (src/nndescent.cpp:168-187, 264-283).
//   merge   one warp per node merges its list with its candidate slots by a bitonic
//           sort of the packed keys, drops ids already listed, keeps the top k,
//           flags the newcomers "new" and counts them as updates
//           (KnnGraph::insert_unlocked, src/knn_graph.cpp:37-81).
//
// The host stops when a round's updates <= delta * k * n (src/nndescent.cpp:309-341).
// Distances stay in rank space (squared L2) during the descent and are finalised
// with an IEEE sqrt at the end, so every stored distance equals the reference's
// metric_distance for that pair bit for bit.
#include <algorithm>
#include <cmath>

#include "common.cuh"
#include "engine.hpp"

namespace csb {
namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kSlots = 64;         // overflow table slots per node (two-choice hashed)
constexpr int kCap = 128;          // append buffer per node
constexpr int kMaxSample = 32;     // smpN ceiling (cuda/cuda_common.cuh:30)
constexpr int kMaxNewList = 2 * kMaxSample;
constexpr int kMaxOldList = 4 * kMaxSample;

inline unsigned blocks_for(uint64_t work, int threads = kThreads) {
    uint64_t b = (work + threads - 1) / threads;
    return static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>(b, 1u << 30)));
}

__device__ __forceinline__ uint32_t slot1(uint32_t id) { return (id * 2654435761u) >> 26; }  // 6 bits
__device__ __forceinline__ uint32_t slot2(uint32_t id) {
    const uint32_t a = ((id ^ 0x5BD1E995u) * 0x9E3779B1u) >> 26;
    return a == slot1(id) ? (a ^ 1u) : a;
}

/// Overflow table: atomicMin into the id's first slot; whichever key loses there
/// (the offer, or the key it displaced) gets one more atomicMin into its other
/// slot.  A key equal to the slot's content is already present and stops.
__device__ __forceinline__ void offer_table(unsigned long long* __restrict__ table, unsigned long long key) {
    const uint32_t id = static_cast<uint32_t>(key);
    const uint32_t s1 = slot1(id);
    const unsigned long long old = atomicMin(table + s1, key);
    if (old == key) return;
    const unsigned long long loser = old < key ? key : old;
    if (loser == kNoKey) return;
    const uint32_t lid = static_cast<uint32_t>(loser);
    const uint32_t alt = slot1(lid) == s1 ? slot2(lid) : slot1(lid);
    atomicMin(table + alt, loser);
}

/// Offer a packed (rank, id) key to node u: the first kCap offers of a round are
/// appended to u's buffer as they come, later ones go to the overflow table (so
/// the best of the overflow still has a slot).
struct CandStore {
    unsigned long long* buf;    // [n][kCap]
    uint32_t* cnt;              // [n]
    unsigned long long* table;  // [n][kSlots]
};
__device__ __forceinline__ void offer(const CandStore& cs, uint32_t u, unsigned long long key) {
    const uint32_t pos = atomicAdd(cs.cnt + u, 1u);
    if (pos < kCap) {
        cs.buf[static_cast<uint64_t>(u) * kCap + pos] = key;
    } else {
        offer_table(cs.table + static_cast<uint64_t>(u) * kSlots, key);
    }
}

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__device__ __forceinline__ unsigned long long make_key(float r, uint32_t id) {
    return (static_cast<unsigned long long>(__float_as_uint(r)) << 32) | id;
}

// ---- warp bitonic sort of I items per lane (element e = i*32 + lane) ---------------

template <int I>
__device__ __forceinline__ void warp_bitonic(unsigned long long (&key)[I], uint32_t (&pay)[I]) {
    const unsigned lane = threadIdx.x & 31u;
    constexpr int N = 32 * I;
#pragma unroll
    for (int size = 2; size <= N; size <<= 1) {
#pragma unroll
        for (int stride = size / 2; stride > 0; stride >>= 1) {
            if (stride >= 32) {
                const int d = stride / 32;
#pragma unroll
                for (int i = 0; i < I; ++i) {
                    if (i & d) continue;
                    const int j = i | d;
                    const unsigned e = static_cast<unsigned>(i) * 32u + lane;
                    const bool asc = (e & static_cast<unsigned>(size)) == 0;
                    if ((key[i] > key[j]) == asc) {
                        const unsigned long long tk = key[i];
                        key[i] = key[j];
                        key[j] = tk;
                        const uint32_t tp = pay[i];
                        pay[i] = pay[j];
                        pay[j] = tp;
                    }
                }
            } else {
#pragma unroll
                for (int i = 0; i < I; ++i) {
                    const unsigned e = static_cast<unsigned>(i) * 32u + lane;
                    const unsigned long long ok = __shfl_xor_sync(0xFFFFFFFFu, key[i], stride);
                    const uint32_t op = __shfl_xor_sync(0xFFFFFFFFu, pay[i], stride);
                    const bool lower = (lane & static_cast<unsigned>(stride)) == 0;
                    const bool asc = (e & static_cast<unsigned>(size)) == 0;
                    const bool want_min = lower == asc;
                    const bool take_other = want_min ? (ok < key[i]) : (ok > key[i]);
                    if (take_other) {
                        key[i] = ok;
                        pay[i] = op;
                    }
                }
            }
        }
    }
}

// ---- small kernels -----------------------------------------------------------------

/// Metric -> rank units for the stored distances (MetricOp::to_rank); +inf stays.
__global__ void k_to_rank(float* __restrict__ d, uint64_t total, int metric) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const float v = d[i];
    if (isfinite(v)) d[i] = to_rank(v, metric);
}

/// Rank -> metric units (MetricOp::finalize).
__global__ void k_finalize(float* __restrict__ d, uint64_t total, int metric) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const float v = d[i];
    if (isfinite(v)) d[i] = finalize_rank(fmaxf(v, 0.0f), metric);
}

/// thr[u] = the node's k-th rank distance, +inf while its list is short.
__global__ void k_threshold(const float* __restrict__ rank, const uint32_t* __restrict__ counts, uint32_t n,
                            uint32_t k, float* __restrict__ thr) {
    const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= n) return;
    thr[u] = counts[u] >= k ? rank[static_cast<uint64_t>(u) * k + k - 1] : __int_as_float(0x7f800000);
}

/// Random top-up candidates for short lists (init_random, src/nndescent.cpp:348-377):
/// `needed + needed/2 + 4` draws per node, in passes of 32 (one per lane), each
/// followed by a merge.
__global__ void k_random_push(const float* __restrict__ pts, uint32_t n, uint32_t stride,
                              const uint32_t* __restrict__ counts, uint32_t k, uint64_t seed, int pass,
                              CandStore cand) {
    const uint32_t p = blockIdx.x * kWarps + (threadIdx.x >> 5);
    if (p >= n || n < 2) return;
    const unsigned lane = threadIdx.x & 31u;
    const uint32_t c = counts[p];
    if (c >= k) return;
    const uint32_t needed = k - c;
    const uint32_t attempts = needed + needed / 2 + 4;
    const uint32_t t = static_cast<uint32_t>(pass) * 32u + lane;
    if (t >= attempts) return;
    const uint64_t h = mix64(seed ^ (0x9E3779B97F4A7C15ull * (p + 1ull)) ^ (0xC2B2AE3D27D4EB4Full * (t + 1ull)));
    const uint32_t cand_id = static_cast<uint32_t>((h >> 32) % n);
    if (cand_id == p) return;
    const float r = l2sqr_ref(pts + static_cast<uint64_t>(p) * stride, pts + static_cast<uint64_t>(cand_id) * stride, stride);
    offer(cand, p, make_key(r, cand_id));
}

/// Sampling + reverse publication (one warp per node).
__global__ void k_sample(uint32_t n, uint32_t k, uint32_t smp, const uint32_t* __restrict__ ids,
                         uint8_t* __restrict__ flags, const uint32_t* __restrict__ counts,
                         uint32_t* __restrict__ new_s, uint32_t* __restrict__ old_s,
                         uint32_t* __restrict__ ns, uint32_t* __restrict__ nold,
                         uint32_t* __restrict__ rnew, uint32_t* __restrict__ rold,
                         uint32_t* __restrict__ rnew_cnt, uint32_t* __restrict__ rold_cnt) {
    const uint32_t p = blockIdx.x * kWarps + (threadIdx.x >> 5);
    if (p >= n) return;
    const unsigned lane = threadIdx.x & 31u;
    const uint32_t c = counts[p];
    const uint32_t max_new = smp, max_old = 3 * smp;
    uint32_t taken_new = 0, taken_old = 0;
    for (uint32_t base = 0; base < c; base += 32) {
        const uint32_t j = base + lane;
        const bool in = j < c;
        uint32_t id = 0;
        bool is_new = false;
        if (in) {
            id = ids[static_cast<uint64_t>(p) * k + j];
            is_new = flags[static_cast<uint64_t>(p) * k + j] != 0;
        }
        const unsigned nm = __ballot_sync(0xFFFFFFFFu, in && is_new);
        const unsigned om = __ballot_sync(0xFFFFFFFFu, in && !is_new);
        const unsigned below = (1u << lane) - 1u;
        const uint32_t rank_new = taken_new + __popc(nm & below);
        const uint32_t rank_old = taken_old + __popc(om & below);
        if (in && is_new && rank_new < max_new && id < n) {
            new_s[static_cast<uint64_t>(p) * kMaxSample + rank_new] = id;
            flags[static_cast<uint64_t>(p) * k + j] = 0;  // "mark sampled new items as false"
            const uint32_t pos = atomicAdd(rnew_cnt + id, 1u);
            if (pos < smp) rnew[static_cast<uint64_t>(id) * kMaxSample + pos] = p;
        }
        if (in && !is_new && rank_old < max_old && id < n) {
            old_s[static_cast<uint64_t>(p) * 3 * kMaxSample + rank_old] = id;
            const uint32_t pos = atomicAdd(rold_cnt + id, 1u);
            if (pos < smp) rold[static_cast<uint64_t>(id) * kMaxSample + pos] = p;
        }
        taken_new = min(max_new, taken_new + __popc(nm));
        taken_old = min(max_old, taken_old + __popc(om));
        if (taken_new >= max_new && taken_old >= max_old) break;
    }
    if (lane == 0) {
        ns[p] = taken_new;
        nold[p] = taken_old;
    }
}

/// Local join (one warp per node; rows staged in shared memory).
__global__ void __launch_bounds__(kThreads) k_join(const float* __restrict__ pts, uint32_t n, uint32_t stride,
                                                   uint32_t smp, const uint32_t* __restrict__ new_s,
                                                   const uint32_t* __restrict__ old_s, const uint32_t* __restrict__ ns,
                                                   const uint32_t* __restrict__ nold,
                                                   const uint32_t* __restrict__ rnew, const uint32_t* __restrict__ rold,
                                                   const uint32_t* __restrict__ rnew_cnt,
                                                   const uint32_t* __restrict__ rold_cnt, const float* __restrict__ thr,
                                                   CandStore cand, int warps_per_block,
                                                   unsigned long long* __restrict__ evals) {
    extern __shared__ float smem[];
    const int w = threadIdx.x >> 5;
    if (w >= warps_per_block) return;
    const uint32_t p = blockIdx.x * warps_per_block + w;
    if (p >= n) return;
    const unsigned lane = threadIdx.x & 31u;
    constexpr int kRows = kMaxNewList + kMaxOldList;
    // per-warp shared layout: ids[kRows] | thr[kRows] | rows[kRows][stride]
    uint32_t* s_id = reinterpret_cast<uint32_t*>(smem) + static_cast<size_t>(w) * (2 * kRows + kRows * stride);
    float* s_thr = reinterpret_cast<float*>(s_id + kRows);
    float* s_row = s_thr + kRows;

    // assemble new = sampled new + reverse new, old = sampled old + reverse old
    const uint32_t sn = ns[p], so = nold[p];
    const uint32_t rn = min(rnew_cnt[p], smp), ro = min(rold_cnt[p], smp);
    const uint32_t nN = sn + rn, nO = so + ro;
    if (nN == 0) return;
    for (uint32_t t = lane; t < nN; t += 32) {
        s_id[t] = t < sn ? new_s[static_cast<uint64_t>(p) * kMaxSample + t]
                         : rnew[static_cast<uint64_t>(p) * kMaxSample + (t - sn)];
    }
    for (uint32_t t = lane; t < nO; t += 32) {
        s_id[nN + t] = t < so ? old_s[static_cast<uint64_t>(p) * 3 * kMaxSample + t]
                              : rold[static_cast<uint64_t>(p) * kMaxSample + (t - so)];
    }
    __syncwarp();
    const uint32_t nT = nN + nO;
    for (uint32_t t = lane; t < nT; t += 32) s_thr[t] = thr[s_id[t]];
    // stage rows with float4 loads
    const uint32_t q4 = stride / 4;
    for (uint32_t t = lane; t < nT * q4; t += 32) {
        const uint32_t row = t / q4, c4 = t % q4;
        const float4 v = reinterpret_cast<const float4*>(pts + static_cast<uint64_t>(s_id[row]) * stride)[c4];
        reinterpret_cast<float4*>(s_row + static_cast<size_t>(row) * stride)[c4] = v;
    }
    __syncwarp();
    // pairs: a in [0, nN), b in [0, nT), b > a when b < nN
    const uint32_t total = nN * nT;
    uint32_t my_evals = 0;
    for (uint32_t q = lane; q < total; q += 32) {
        const uint32_t a = q / nT, b = q % nT;
        if (b < nN && b <= a) continue;
        const uint32_t u1 = s_id[a], u2 = s_id[b];
        if (u1 == u2) continue;
        const float r = l2sqr_ref(s_row + static_cast<size_t>(a) * stride, s_row + static_cast<size_t>(b) * stride, stride);
        ++my_evals;
        if (r < s_thr[a]) offer(cand, u1, make_key(r, u2));
        if (r < s_thr[b]) offer(cand, u2, make_key(r, u1));
    }
    if (evals) {
        for (int o = 16; o > 0; o >>= 1) my_evals += __shfl_xor_sync(0xFFFFFFFFu, my_evals, o);
        if (lane == 0) atomicAdd(evals, static_cast<unsigned long long>(my_evals));
    }
}

/// Merge a node's offers into its sorted list (one warp per node).  The offers
/// (the append buffer, then the overflow table when it was used) are taken 32 at a
/// time: each chunk drops invalid keys, ids already listed, keys repeated inside the
/// chunk and keys not better than the current k-th entry, and if anything is left
/// the list (LI items per lane) and the chunk are sorted together by a warp bitonic
/// network of I = 2*LI... elements and the first k kept.  Newcomers carry the new
/// flag; the ones still listed at the end are the round's updates.
template <int LI, int I>
__global__ void k_merge(uint32_t n, uint32_t k, uint32_t* __restrict__ ids, float* __restrict__ rank,
                        uint8_t* __restrict__ flags, uint32_t* __restrict__ counts, float* __restrict__ thr,
                        CandStore cand, uint32_t* __restrict__ rnew_cnt, uint32_t* __restrict__ rold_cnt,
                        unsigned long long* __restrict__ updates) {
    static_assert(LI + 1 <= I, "merge layout");
    const uint32_t u = blockIdx.x * kWarps + (threadIdx.x >> 5);
    if (u >= n) return;
    const unsigned lane = threadIdx.x & 31u;
    unsigned long long key[I];
    uint32_t pay[I];  // bit 0: new flag, bit 1: came from an offer
    const uint32_t c = counts[u];
    const uint64_t base = static_cast<uint64_t>(u) * k;
#pragma unroll
    for (int i = 0; i < I; ++i) {
        const uint32_t j = static_cast<uint32_t>(i) * 32u + lane;
        if (i < LI && j < c) {
            key[i] = make_key(rank[base + j], ids[base + j]);
            pay[i] = flags[base + j] ? 1u : 0u;
        } else {
            key[i] = kNoKey;
            pay[i] = 0;
        }
    }
    const uint32_t offered = cand.cnt[u];
    const uint32_t nbuf = min(offered, static_cast<uint32_t>(kCap));
    const bool table_used = offered > static_cast<uint32_t>(kCap);
    const uint32_t total = nbuf + (table_used ? kSlots : 0);
    const unsigned long long* bufp = cand.buf + static_cast<uint64_t>(u) * kCap;
    unsigned long long* tabp = cand.table + static_cast<uint64_t>(u) * kSlots;
    // k-th key of the current list (element k-1)
    auto kth_of = [&]() -> unsigned long long {
        const uint32_t e = k - 1;
        unsigned long long x = kNoKey;
#pragma unroll
        for (int i = 0; i < I; ++i) {
            const unsigned long long y = __shfl_sync(0xFFFFFFFFu, key[i], e & 31u);
            if (static_cast<uint32_t>(i) == e / 32u) x = y;
        }
        return x;
    };
    unsigned long long kth = kth_of();
    for (uint32_t off = 0; off < total; off += 32) {
        const uint32_t t = off + lane;
        unsigned long long ck = kNoKey;
        if (t < total) {
            if (t < nbuf) {
                ck = bufp[t];
            } else {
                ck = tabp[t - nbuf];
                tabp[t - nbuf] = kNoKey;  // the table is reset as it is read
            }
        }
        const uint32_t cid = static_cast<uint32_t>(ck);
        // kth's rank bits compare like the key's (ids only break exact ties, where a
        // newcomer does not displace: the reference inserts behind equal distances)
        bool ok = ck != kNoKey && cid != u && cid < n &&
                  (kth == kNoKey || static_cast<uint32_t>(ck >> 32) < static_cast<uint32_t>(kth >> 32));
        // repeated inside the chunk: keep the lowest lane holding the key
        const unsigned same = __match_any_sync(0xFFFFFFFFu, ck);
        if (static_cast<int>(lane) != __ffs(same) - 1) ok = false;
        // already listed
#pragma unroll
        for (int i = 0; i < LI; ++i) {
            const uint32_t lid = static_cast<uint32_t>(key[i]);
            const bool lv = key[i] != kNoKey;
            for (int q = 0; q < 32; ++q) {
                const uint32_t other = __shfl_sync(0xFFFFFFFFu, lid, q);
                const bool ov = __shfl_sync(0xFFFFFFFFu, lv, q);
                if (ov && other == cid) ok = false;
            }
        }
        if (!__any_sync(0xFFFFFFFFu, ok)) continue;
        key[LI] = ok ? ck : kNoKey;
        pay[LI] = ok ? 3u : 0u;
#pragma unroll
        for (int i = LI + 1; i < I; ++i) {
            key[i] = kNoKey;
            pay[i] = 0;
        }
        warp_bitonic<I>(key, pay);
        // keep the first k; drop the rest
#pragma unroll
        for (int i = 0; i < I; ++i) {
            const uint32_t j = static_cast<uint32_t>(i) * 32u + lane;
            if (j >= k) {
                key[i] = kNoKey;
                pay[i] = 0;
            }
        }
        kth = kth_of();
    }
    uint32_t inserted = 0, cnt = 0;
#pragma unroll
    for (int i = 0; i < LI; ++i) {
        const uint32_t j = static_cast<uint32_t>(i) * 32u + lane;
        if (j < k) {
            const bool valid = key[i] != kNoKey;
            ids[base + j] = valid ? static_cast<uint32_t>(key[i]) : kInvalid;
            rank[base + j] = valid ? __uint_as_float(static_cast<uint32_t>(key[i] >> 32)) : __int_as_float(0x7f800000);
            flags[base + j] = valid ? static_cast<uint8_t>(pay[i] & 1u) : 0;
            cnt += valid;
            inserted += (valid && (pay[i] & 2u)) ? 1u : 0u;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        cnt += __shfl_xor_sync(0xFFFFFFFFu, cnt, o);
        inserted += __shfl_xor_sync(0xFFFFFFFFu, inserted, o);
    }
    if (lane == 0) {
        counts[u] = cnt;
        thr[u] = (cnt >= k && kth != kNoKey) ? __uint_as_float(static_cast<uint32_t>(kth >> 32))
                                             : __int_as_float(0x7f800000);
        cand.cnt[u] = 0;
        rnew_cnt[u] = 0;
        rold_cnt[u] = 0;
        if (inserted && updates) atomicAdd(updates, static_cast<unsigned long long>(inserted));
    }
}

struct KnnScratch {
    DevBuf thr, cand, cand_buf, cand_cnt, new_s, old_s, ns, nold, rnew, rold, rnew_cnt, rold_cnt, counters;
};

CandStore store_of(KnnScratch& s) {
    CandStore cs;
    cs.buf = s.cand_buf.as<unsigned long long>();
    cs.cnt = s.cand_cnt.as<uint32_t>();
    cs.table = s.cand.as<unsigned long long>();
    return cs;
}

void launch_merge(Ctx& c, Graph& g, KnnScratch& s, unsigned long long* updates) {
    const uint32_t n = static_cast<uint32_t>(g.n);
    const unsigned grid = static_cast<unsigned>((n + kWarps - 1) / kWarps);
    if (g.k <= 32) {
        k_merge<1, 2><<<grid, kThreads, 0, c.stream>>>(n, g.k, g.ids.as<uint32_t>(), g.dists.as<float>(),
                                                     g.flags.as<uint8_t>(), g.counts.as<uint32_t>(), s.thr.as<float>(),
                                                     store_of(s), s.rnew_cnt.as<uint32_t>(),
                                                     s.rold_cnt.as<uint32_t>(), updates);
    } else {
        k_merge<2, 4><<<grid, kThreads, 0, c.stream>>>(n, g.k, g.ids.as<uint32_t>(), g.dists.as<float>(),
                                                     g.flags.as<uint8_t>(), g.counts.as<uint32_t>(), s.thr.as<float>(),
                                                     store_of(s), s.rnew_cnt.as<uint32_t>(),
                                                     s.rold_cnt.as<uint32_t>(), updates);
    }
    count_launch(c);
}

}  // namespace

/// Dynamic NN-Descent over the graph's resident points and k-NN arrays (which are
/// the warm start; distances in metric units on entry and exit).
void knn_descent(Graph& g, uint32_t sample, uint32_t iters, double delta, uint64_t seed, bool random_fill,
                 uint64_t* out_updates, uint32_t* out_rounds) {
    Ctx& c = *g.ctx;
    const uint32_t n = static_cast<uint32_t>(g.n);
    if (g.k > 64) fail(CS_ERR_UNSUPPORTED, "NN-Descent: k > 64");
    if (out_updates) *out_updates = 0;
    if (out_rounds) *out_rounds = 0;
    if (n == 0) return;
    const uint32_t smp = std::min<uint32_t>(std::max<uint32_t>(sample, 1), kMaxSample);
    const uint32_t k = g.k;
    const uint64_t nk = static_cast<uint64_t>(n) * k;
    KnnScratch s;
    s.thr.ensure(n * 4ull);
    s.cand.ensure(n * 8ull * kSlots);
    s.cand_buf.ensure(n * 8ull * kCap);
    s.cand_cnt.ensure(n * 4ull);
    s.new_s.ensure(n * 4ull * kMaxSample);
    s.old_s.ensure(n * 4ull * 3 * kMaxSample);
    s.ns.ensure(n * 4ull);
    s.nold.ensure(n * 4ull);
    s.rnew.ensure(n * 4ull * kMaxSample);
    s.rold.ensure(n * 4ull * kMaxSample);
    s.rnew_cnt.ensure(n * 4ull);
    s.rold_cnt.ensure(n * 4ull);
    s.counters.ensure(64);
    unsigned long long* d_updates = s.counters.as<unsigned long long>();
    unsigned long long* d_evals = d_updates + 1;
    CSB_CUDA(cudaMemsetAsync(s.cand.p, 0xFF, n * 8ull * kSlots, c.stream));
    CSB_CUDA(cudaMemsetAsync(s.cand_cnt.p, 0, n * 4ull, c.stream));
    CSB_CUDA(cudaMemsetAsync(s.rnew_cnt.p, 0, n * 4ull, c.stream));
    CSB_CUDA(cudaMemsetAsync(s.rold_cnt.p, 0, n * 4ull, c.stream));
    CSB_CUDA(cudaMemsetAsync(s.counters.p, 0, 64, c.stream));
    k_to_rank<<<blocks_for(nk), kThreads, 0, c.stream>>>(g.dists.as<float>(), nk, g.metric);
    k_threshold<<<blocks_for(n), kThreads, 0, c.stream>>>(g.dists.as<float>(), g.counts.as<uint32_t>(), n, k,
                                                         s.thr.as<float>());
    count_launch(c, 2);
    const unsigned gw = static_cast<unsigned>((n + kWarps - 1) / kWarps);
    if (random_fill) {
        const uint32_t max_attempts = k + k / 2 + 4;
        for (int pass = 0; pass * 32u < max_attempts; ++pass) {
            k_random_push<<<gw, kThreads, 0, c.stream>>>(g.pts.as<float>(), n, g.stride, g.counts.as<uint32_t>(), k,
                                                          seed, pass, store_of(s));
            count_launch(c);
            launch_merge(c, g, s, nullptr);
        }
    }
    check_launch(c, "NN-Descent init");
    // join launch shape: as many warps per block as the staged rows allow
    constexpr int kRows = kMaxNewList + kMaxOldList;
    const size_t per_warp = (2 * kRows + static_cast<size_t>(kRows) * g.stride) * 4;
    int wpb = static_cast<int>(std::min<size_t>(kWarps, std::max<size_t>(1, (200u * 1024u) / per_warp)));
    const size_t smem = per_warp * wpb;
    CSB_CUDA(cudaFuncSetAttribute(k_join, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    const unsigned gj = static_cast<unsigned>((n + wpb - 1) / wpb);
    const double stop = delta * static_cast<double>(k) * static_cast<double>(n);
    uint64_t total = 0;
    uint32_t rounds = 0;
    for (uint32_t it = 0; it < iters; ++it) {
        CSB_CUDA(cudaMemsetAsync(d_updates, 0, 8, c.stream));
        k_sample<<<gw, kThreads, 0, c.stream>>>(n, k, smp, g.ids.as<uint32_t>(), g.flags.as<uint8_t>(),
                                                 g.counts.as<uint32_t>(), s.new_s.as<uint32_t>(), s.old_s.as<uint32_t>(),
                                                 s.ns.as<uint32_t>(), s.nold.as<uint32_t>(), s.rnew.as<uint32_t>(),
                                                 s.rold.as<uint32_t>(), s.rnew_cnt.as<uint32_t>(),
                                                 s.rold_cnt.as<uint32_t>());
        k_join<<<gj, wpb * 32, smem, c.stream>>>(g.pts.as<float>(), n, g.stride, smp, s.new_s.as<uint32_t>(),
                                                  s.old_s.as<uint32_t>(), s.ns.as<uint32_t>(), s.nold.as<uint32_t>(),
                                                  s.rnew.as<uint32_t>(), s.rold.as<uint32_t>(),
                                                  s.rnew_cnt.as<uint32_t>(), s.rold_cnt.as<uint32_t>(),
                                                  s.thr.as<float>(), store_of(s), wpb, d_evals);
        count_launch(c, 2);
        launch_merge(c, g, s, d_updates);
        check_launch(c, "NN-Descent round");
        unsigned long long upd = 0;
        CSB_CUDA(cudaMemcpyAsync(&upd, d_updates, 8, cudaMemcpyDeviceToHost, c.stream));
        CSB_CUDA(cudaStreamSynchronize(c.stream));
        total += upd;
        rounds = it + 1;
        if (static_cast<double>(upd) <= stop) break;
    }
    k_finalize<<<blocks_for(nk), kThreads, 0, c.stream>>>(g.dists.as<float>(), nk, g.metric);
    count_launch(c);
    check_launch(c, "NN-Descent finalize");
    c.sync();
    g.invalidate_edges();
    if (out_updates) *out_updates = total;
    if (out_rounds) *out_rounds = rounds;
}

}  // namespace csb

using namespace csb;

extern "C" {

cs_status cs_nndescent(cs_ctx* ctx, const cs_nnd_config* cfg, const float* host_vectors, uint32_t* ids, float* dists,
                       uint8_t* flags, uint32_t* counts, uint64_t* out_updates) {
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    return guarded(c, [&] {
        CSB_REQUIRE(cfg != nullptr, "cs_nndescent: null config");
        if (cfg->n == 0 || cfg->k == 0) return;
        CSB_REQUIRE(host_vectors && ids && dists && counts, "cs_nndescent: null buffer");
        if (cfg->metric != CS_METRIC_L2 && cfg->metric != CS_METRIC_COSINE)
            fail(CS_ERR_UNSUPPORTED, "nndescent_gpu: unsupported metric for the device path");
        CSB_REQUIRE(cfg->stride >= cfg->dim && cfg->stride % 8 == 0, "cs_nndescent: stride must be pad8(dim)");
        CSB_REQUIRE(cfg->k <= 64, "cs_nndescent: k > 64");
        Graph g;
        g.ctx = c;
        g.dim = cfg->dim;
        g.k = cfg->k;
        g.stride = cfg->stride;
        g.metric = cfg->metric;
        g.ensure_capacity(cfg->n, false);
        g.n = cfg->n;
        const uint64_t nk = static_cast<uint64_t>(cfg->n) * cfg->k;
        copy_h2d(*c, g.pts.p, host_vectors, static_cast<uint64_t>(cfg->n) * cfg->stride * 4);
        for (uint64_t i = 0; i < cfg->n; ++i) {
            if (counts[i] > cfg->k) fail(CS_ERR_INVALID, "cs_nndescent: count exceeds k");
        }
        copy_h2d(*c, g.ids.p, ids, nk * 4);
        copy_h2d(*c, g.dists.p, dists, nk * 4);
        if (flags) copy_h2d(*c, g.flags.p, flags, nk);
        else CSB_CUDA(cudaMemsetAsync(g.flags.p, 0, nk, c->stream));
        copy_h2d(*c, g.counts.p, counts, static_cast<uint64_t>(cfg->n) * 4);
        uint64_t upd = 0;
        knn_descent(g, cfg->sample, cfg->iters, cfg->delta, cfg->seed, cfg->random_fill != 0, &upd, nullptr);
        copy_d2h(*c, ids, g.ids.p, nk * 4);
        copy_d2h(*c, dists, g.dists.p, nk * 4);
        if (flags) copy_d2h(*c, flags, g.flags.p, nk);
        copy_d2h(*c, counts, g.counts.p, static_cast<uint64_t>(cfg->n) * 4);
        if (out_updates) *out_updates = upd;
    });
}

cs_status cs_knn_build(cs_graph* gp, uint32_t sample, uint32_t iters, double delta, uint64_t seed,
                       uint64_t* out_updates, uint32_t* out_rounds) {
    Graph* g = reinterpret_cast<Graph*>(gp);
    return guarded(g ? g->ctx : nullptr, [&] {
        CSB_REQUIRE(g->n > 0, "cs_knn_build: no points");
        // a fresh build: empty lists, then random fill (IncrementalKnn::build, one instance)
        const uint64_t nk = g->n * g->k;
        Ctx& c = *g->ctx;
        CSB_CUDA(cudaMemsetAsync(g->ids.p, 0xFF, nk * 4, c.stream));
        CSB_CUDA(cudaMemsetAsync(g->flags.p, 0, nk, c.stream));
        CSB_CUDA(cudaMemsetAsync(g->counts.p, 0, g->n * 4, c.stream));
        // +inf distances
        std::vector<float> inf_row(g->k, INFINITY);
        CSB_CUDA(cudaMemcpyAsync(g->dists.p, inf_row.data(), g->k * 4, cudaMemcpyHostToDevice, c.stream));
        for (uint64_t done = 1; done < g->n;) {
            const uint64_t m = std::min(done, g->n - done);
            CSB_CUDA(cudaMemcpyAsync(g->dists.as<float>() + done * g->k, g->dists.p, m * g->k * 4,
                                     cudaMemcpyDeviceToDevice, c.stream));
            done += m;
        }
        knn_descent(*g, sample, iters, delta, seed, true, out_updates, out_rounds);
    });
}

}  // extern "C"
