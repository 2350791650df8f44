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
#include <chrono>
#include <cmath>

#include <cub/device/device_radix_sort.cuh>

#include "common.cuh"
#include "engine.hpp"

namespace csb {
namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kSlots = 64;         // overflow table slots per node (two-choice hashed)
constexpr int kCap = 128;          // append buffer per node
constexpr int kMaxSample = 32;     // smpN ceiling (cuda/cuda_common.cuh:30)

inline unsigned blocks_for(uint64_t work, int threads = kThreads) {
    uint64_t b = (work + threads - 1) / threads;
    return static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>(b, 1u << 30)));
}

__device__ __forceinline__ uint32_t slot1(uint32_t id) { return (id * 2654435761u) >> 26; }  // 6 bits
__device__ __forceinline__ uint32_t slot2(uint32_t id) {
    const uint32_t a = ((id ^ 0x5BD1E995u) * 0x9E3779B1u) >> 26;
    return a == slot1(id) ? (a ^ 1u) : a;
}

/// Overflow table: the key is reduced (atomicMin) into both of its id's slots, so it
/// survives while it is the smallest of either slot.  Neither atomic returns a value,
/// so an offer never waits on the table (the overflow takes most of the offers of the
/// first rounds, when the lists are random); a key held by both slots is read twice
/// and the merge drops the second copy.
__device__ __forceinline__ void offer_table(unsigned long long* __restrict__ table, unsigned long long key) {
    const uint32_t id = static_cast<uint32_t>(key);
    atomicMin(table + slot1(id), key);
    atomicMin(table + slot2(id), key);
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

/// The last pass of warp_bitonic<I> alone: sorts ascending a sequence of 32 * I items
/// that is already bitonic (ascending, then descending).  log2(32 I) steps instead of
/// the full sort's log2(32 I) (log2(32 I) + 1) / 2.
template <int I>
__device__ __forceinline__ void warp_bitonic_merge(unsigned long long (&key)[I], uint32_t (&pay)[I]) {
    const unsigned lane = threadIdx.x & 31u;
    constexpr int N = 32 * I;
#pragma unroll
    for (int stride = N / 2; stride > 0; stride >>= 1) {
        if (stride >= 32) {
            const int d = stride / 32;
#pragma unroll
            for (int i = 0; i < I; ++i) {
                if (i & d) continue;
                const int j = i | d;
                if (key[i] > key[j]) {
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
                const unsigned long long ok = __shfl_xor_sync(0xFFFFFFFFu, key[i], stride);
                const uint32_t op = __shfl_xor_sync(0xFFFFFFFFu, pay[i], stride);
                const bool lower = (lane & static_cast<unsigned>(stride)) == 0;
                const bool take_other = lower ? (ok < key[i]) : (ok > key[i]);
                if (take_other) {
                    key[i] = ok;
                    pay[i] = op;
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
__global__ void k_random_push(const float* __restrict__ pts, uint32_t node_lo, uint32_t node_hi, uint32_t stride,
                              const uint32_t* __restrict__ counts, uint32_t k, uint64_t seed, int pass,
                              CandStore cand, uint32_t cand_lo, uint32_t cand_span) {
    const uint32_t p = node_lo + blockIdx.x * kWarps + (threadIdx.x >> 5);
    if (p >= node_hi || cand_span < 2) return;
    const unsigned lane = threadIdx.x & 31u;
    const uint32_t c = counts[p];
    if (c >= k) return;
    const uint32_t needed = k - c;
    const uint32_t attempts = needed + needed / 2 + 4;
    const uint32_t t = static_cast<uint32_t>(pass) * 32u + lane;
    if (t >= attempts) return;
    const uint64_t h = mix64(seed ^ (0x9E3779B97F4A7C15ull * (p + 1ull)) ^ (0xC2B2AE3D27D4EB4Full * (t + 1ull)));
    const uint32_t cand_id = cand_lo + static_cast<uint32_t>((h >> 32) % cand_span);
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
                         uint32_t* __restrict__ rnew_cnt, uint32_t* __restrict__ rold_cnt,
                         const uint32_t* __restrict__ active, uint32_t n_active) {
    const uint32_t w = blockIdx.x * kWarps + (threadIdx.x >> 5);
    if (w >= (active ? n_active : n)) return;
    const uint32_t p = active ? active[w] : w;
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

/// Staged row pitch in shared memory: four floats more than the row, so the float4
/// loads of 8 lanes reading 8 different rows fall into 8 different bank groups (a
/// pitch of 16 or 32 floats put them into two groups or one).
__host__ __device__ __forceinline__ uint32_t join_pitch(uint32_t stride) { return stride + 4; }

/// Local join (one warp per node; rows staged in shared memory, `rows` of them at
/// most: 2 x sample new + 4 x sample old).
__global__ void __launch_bounds__(kThreads) k_join(const float* __restrict__ pts, uint32_t n, uint32_t stride,
                                                   uint32_t smp, const uint32_t* __restrict__ new_s,
                                                   const uint32_t* __restrict__ old_s, const uint32_t* __restrict__ ns,
                                                   const uint32_t* __restrict__ nold,
                                                   const uint32_t* __restrict__ rnew, const uint32_t* __restrict__ rold,
                                                   const uint32_t* __restrict__ rnew_cnt,
                                                   const uint32_t* __restrict__ rold_cnt, const float* __restrict__ thr,
                                                   CandStore cand, int warps_per_block,
                                                   unsigned long long* __restrict__ evals,
                                                   const uint32_t* __restrict__ active, uint32_t n_active,
                                                   uint32_t rows) {
    extern __shared__ float smem[];
    const int w = threadIdx.x >> 5;
    if (w >= warps_per_block) return;
    const uint32_t slot = blockIdx.x * warps_per_block + w;
    if (slot >= (active ? n_active : n)) return;
    const uint32_t p = active ? active[slot] : slot;
    const unsigned lane = threadIdx.x & 31u;
    const uint32_t pitch = join_pitch(stride);
    // per-warp shared layout: ids[rows] | thr[rows] | rows[rows][pitch]
    uint32_t* s_id = reinterpret_cast<uint32_t*>(smem) + static_cast<size_t>(w) * rows * (2 + pitch);
    float* s_thr = reinterpret_cast<float*>(s_id + rows);
    float* s_row = s_thr + rows;

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
        reinterpret_cast<float4*>(s_row + static_cast<size_t>(row) * pitch)[c4] = v;
    }
    __syncwarp();
    // pairs: a in [0, nN) with every b > a in [0, nT) -- new x new once, new x old;
    // row a is read by the whole warp at once (a broadcast), the lanes take the b's.
    // Every lane's offer to u1 goes to the same node: one atomicAdd reserves the
    // warp's places in u1's append buffer (the lanes then fill them in lane order)
    // instead of one contended atomic per lane.
    // The offers of a chunk are written one chunk later: a chunk's places in the
    // append buffers are reserved with atomics whose results the stores need, and the
    // next chunk's distances run while those reservations are on their way (written
    // in the order: this chunk's distances, the previous chunk's stores, this chunk's
    // reservations, so a reservation's result register is only read a chunk later).
    uint32_t my_evals = 0;
    bool p1 = false, p2 = false;           // this lane has a pending row / column offer
    unsigned long long pk1 = 0, pk2 = 0;   // their keys
    uint32_t pu1 = 0, prank1 = 0, pu2 = 0; // row node and rank in its ballot; column node
    uint32_t res1 = 0, res2 = 0;           // reservation results (the row's: its leader lane)
    int pleader = -1;                      // lane holding the pending row reservation (-1: none)
    auto flush = [&]() {
        if (pleader >= 0) {  // warp-uniform
            const uint32_t base = __shfl_sync(0xFFFFFFFFu, res1, pleader);
            if (p1) {
                const uint32_t pos = base + prank1;
                if (pos < kCap) {
                    cand.buf[static_cast<uint64_t>(pu1) * kCap + pos] = pk1;
                } else {
                    offer_table(cand.table + static_cast<uint64_t>(pu1) * kSlots, pk1);
                }
            }
        }
        if (p2) {
            if (res2 < kCap) {
                cand.buf[static_cast<uint64_t>(pu2) * kCap + res2] = pk2;
            } else {
                offer_table(cand.table + static_cast<uint64_t>(pu2) * kSlots, pk2);
            }
        }
    };
    for (uint32_t a = 0; a < nN; ++a) {
        const float* ra = s_row + static_cast<size_t>(a) * pitch;
        const uint32_t u1 = s_id[a];
        const float ta = s_thr[a];
        for (uint32_t b0 = a + 1; b0 < nT; b0 += 32) {
            const uint32_t b = b0 + lane;
            const uint32_t u2 = b < nT ? s_id[b] : u1;
            const bool pair = b < nT && u1 != u2;
            float r = 0.0f;
            if (pair) {
                r = l2sqr_ref(ra, s_row + static_cast<size_t>(b) * pitch, stride);
                ++my_evals;
            }
            const bool to1 = pair && r < ta;
            const bool to2 = pair && r < s_thr[b];
            const unsigned m1 = __ballot_sync(0xFFFFFFFFu, to1);
            flush();
            // this chunk's reservations: one atomic for the row node (all lanes' offers
            // to it), one per lane for its column node
            const int leader = m1 ? __ffs(m1) - 1 : -1;
            if (static_cast<int>(lane) == leader) res1 = atomicAdd(cand.cnt + u1, static_cast<uint32_t>(__popc(m1)));
            if (to2) res2 = atomicAdd(cand.cnt + u2, 1u);
            p1 = to1;
            p2 = to2;
            pk1 = make_key(r, u2);
            pk2 = make_key(r, u1);
            pu1 = u1;
            pu2 = u2;
            prank1 = __popc(m1 & ((1u << lane) - 1u));
            pleader = leader;
        }
    }
    flush();
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
/// The nodes that took an offer this round (cand.cnt[u] != 0), compacted into a list:
/// the merge walks them alone instead of a warp for every node of the graph (an insert
/// round offers to a few hundred thousand nodes of a graph of millions).
__global__ void k_touched(uint32_t n, const uint32_t* __restrict__ cnt, uint32_t* __restrict__ list,
                          uint32_t* __restrict__ count) {
    const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
    const bool has = u < n && cnt[u] != 0;
    const uint32_t at = warp_append(has, count);  // every lane of the warp calls it
    if (has) list[at] = u;
}

template <int LI, int I>
__global__ void k_merge(uint32_t n, uint32_t k, uint32_t* __restrict__ ids, float* __restrict__ rank,
                        uint8_t* __restrict__ flags, uint32_t* __restrict__ counts, float* __restrict__ thr,
                        CandStore cand, const uint32_t* __restrict__ list, const uint32_t* __restrict__ list_count,
                        unsigned long long* __restrict__ updates, uint8_t* __restrict__ changed) {
    static_assert(LI + 1 <= I, "merge layout");
    const unsigned lane = threadIdx.x & 31u;
    // the nodes that took an offer (k_touched), a warp per node, grid-strided
    const uint32_t m_list = *list_count;
    for (uint32_t li = blockIdx.x * kWarps + (threadIdx.x >> 5); li < m_list; li += gridDim.x * kWarps) {
        const uint32_t u = list[li];
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
            if (inserted && updates) atomicAdd(updates, static_cast<unsigned long long>(inserted));
            // a newcomer in the list is a change of membership (none got in: the list
            // holds the same ids); the incremental hubness refresh reads the flag
            if (inserted) changed[u] = 1;
        }
    }
}

/// Seeds of new points by beam search over the base graph (IncrementalKnn::search_seeds,
/// src/incremental_knn.cpp:118-216, forward edges only): one warp per query, a pool of
/// 64 (rank, id) keys started from 32 random base entries, best-first expansion of the
/// closest unexpanded pool entry (its k-NN list is scored and merged into the pool by a
/// 128-element warp bitonic sort), at most max_expand expansions.  Reads the base
/// graph only; writes the best k pool keys of query t to seeds[t][*].
__global__ void k_search(const float* __restrict__ pts, uint32_t stride, const uint32_t* __restrict__ ids,
                         const uint32_t* __restrict__ counts, uint32_t k, uint32_t n_base, uint32_t first_new,
                         uint32_t count, uint64_t seed, uint32_t max_expand, const uint32_t* __restrict__ hints,
                         uint32_t n_hint, const uint32_t* __restrict__ rev_off,
                         const unsigned long long* __restrict__ rev_keys, uint32_t rev_cap, uint32_t width,
                         unsigned long long* __restrict__ seeds) {
    extern __shared__ float sq[];
    const uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned lane = threadIdx.x & 31u, wi = threadIdx.x >> 5;
    if (t >= count || n_base == 0) return;
    float* qrow = sq + static_cast<size_t>(wi) * stride;
    const uint32_t q = first_new + t;
    for (uint32_t d = lane; d < stride; d += 32) qrow[d] = pts[static_cast<uint64_t>(q) * stride + d];
    __syncwarp();
    unsigned long long key[4];
    uint32_t pay[4];  // bit 0: expanded
    {
        const uint64_t h = mix64(seed ^ (0x9E3779B97F4A7C15ull * (q + 1ull)) ^ (0xD6E8FEB86659FD93ull * (lane + 1ull)));
        const uint32_t e = static_cast<uint32_t>((h >> 32) % n_base);
        const float r = l2sqr_ref(qrow, pts + static_cast<uint64_t>(e) * stride, stride);
        unsigned long long ck = make_key(r, e);
        const unsigned same = __match_any_sync(0xFFFFFFFFu, ck);
        if (static_cast<int>(lane) != __ffs(same) - 1) ck = kNoKey;
        // the two closest of a strided scan of at most 256 hints (the selected
        // anti-hubs: a coarse index with a quota per component)
        unsigned long long hk = kNoKey;
        if (n_hint) {
            const uint32_t scan = min(n_hint, 256u), step = max(1u, n_hint / scan);
            const uint32_t off = static_cast<uint32_t>((h & 0xFFFFFFFFull) % n_hint);
            unsigned long long b0 = kNoKey, b1 = kNoKey;
            for (uint32_t t2 = lane; t2 < scan; t2 += 32) {
                const uint32_t e2 = hints[(off + static_cast<uint64_t>(t2) * step) % n_hint];
                if (e2 >= n_base) continue;
                const unsigned long long x =
                    make_key(l2sqr_ref(qrow, pts + static_cast<uint64_t>(e2) * stride, stride), e2);
                if (x < b0) {
                    b1 = b0;
                    b0 = x;
                } else if (x < b1) {
                    b1 = x;
                }
            }
            for (int r = 0; r < 2; ++r) {
                unsigned long long m = b0;
                for (int o = 16; o > 0; o >>= 1) {
                    const unsigned long long y = __shfl_xor_sync(0xFFFFFFFFu, m, o);
                    m = y < m ? y : m;
                }
                if (static_cast<uint32_t>(r) == lane) hk = m;
                if (b0 == m) {  // keys are unique per lane scan; pop the winner
                    b0 = b1;
                    b1 = kNoKey;
                }
            }
            // a hint already drawn as a random entry is not entered twice
            for (int s2 = 0; s2 < 32; ++s2) {
                const unsigned long long rk = __shfl_sync(0xFFFFFFFFu, ck, s2);
                if (hk != kNoKey && rk == hk) hk = kNoKey;
            }
        }
        key[0] = key[1] = kNoKey;
        key[2] = ck;
        key[3] = hk;
        pay[0] = pay[1] = pay[2] = pay[3] = 0;
        warp_bitonic<4>(key, pay);
        key[2] = key[3] = kNoKey;
    }
    for (uint32_t it = 0; it < max_expand; ++it) {
        unsigned long long best = kNoKey;
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            // only the ef best may be expanded: the search ends when the nearest
            // unexpanded candidate is behind them (the reference's beam rule)
            if (key[i] != kNoKey && !(pay[i] & 1u) && static_cast<uint32_t>(i) * 32u + lane < width &&
                key[i] < best)
                best = key[i];
        }
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long x = __shfl_xor_sync(0xFFFFFFFFu, best, o);
            best = x < best ? x : best;
        }
        if (best == kNoKey) break;
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            if (key[i] == best) pay[i] |= 1u;
        }
        const uint32_t c = static_cast<uint32_t>(best);
        const uint32_t cnt = counts[c];
        // the list, then the first rev_cap reverse neighbours (the undirected graph)
        const uint32_t r0 = rev_cap ? rev_off[c] : 0u;
        const uint32_t rc = rev_cap ? min(rev_cap, rev_off[c + 1] - r0) : 0u;
        for (uint32_t b = 0; b < cnt + rc; b += 32) {
            const uint32_t j = b + lane;
            uint32_t nb = kInvalid;
            if (j < cnt) nb = ids[static_cast<uint64_t>(c) * k + j];
            else if (j < cnt + rc) nb = static_cast<uint32_t>(rev_keys[r0 + (j - cnt)]);
            bool ok = nb < n_base;
            unsigned long long ck = kNoKey;
            if (ok) ck = make_key(l2sqr_ref(qrow, pts + static_cast<uint64_t>(nb) * stride, stride), nb);
            // a candidate behind the pool's last key cannot enter: most expansions
            // near convergence bring none, and skip the dedupe and the sort
            const unsigned long long worst = __shfl_sync(0xFFFFFFFFu, key[1], 31);
            ok = ok && ck < worst;
            if (!__any_sync(0xFFFFFFFFu, ok)) continue;
            // a node already in the pool has exactly this key there (the same
            // distance bits and id): a binary search over the sorted pool (element
            // e = i * 32 + lane, ascending, empty slots last) finds it
            {
                uint32_t lo = 0;
#pragma unroll
                for (uint32_t half = 32; half > 0; half >>= 1) {
                    const uint32_t e = lo + half - 1;
                    const unsigned long long v0 = __shfl_sync(0xFFFFFFFFu, key[0], e & 31u);
                    const unsigned long long v1 = __shfl_sync(0xFFFFFFFFu, key[1], e & 31u);
                    if ((e < 32 ? v0 : v1) < ck) lo += half;
                }
                const unsigned long long v0 = __shfl_sync(0xFFFFFFFFu, key[0], lo & 31u);
                const unsigned long long v1 = __shfl_sync(0xFFFFFFFFu, key[1], lo & 31u);
                if (lo < 64 && (lo < 32 ? v0 : v1) == ck) ok = false;
            }
            {  // forward and reverse entries can name the same node
                const unsigned same = __match_any_sync(0xFFFFFFFFu, nb);
                if (static_cast<int>(lane) != __ffs(same) - 1) ok = false;
            }
            if (!__any_sync(0xFFFFFFFFu, ok)) continue;
            // merge: the candidates sorted (32, one a lane) and placed descending behind
            // a block of empty slots make the 128 items bitonic; one merge pass sorts them
            {
                unsigned long long ckk[1] = {ok ? ck : kNoKey};
                uint32_t cp[1] = {0};
                warp_bitonic<1>(ckk, cp);
                key[2] = kNoKey;
                pay[2] = 0;
                key[3] = __shfl_sync(0xFFFFFFFFu, ckk[0], 31u - lane);
                pay[3] = 0;
            }
            warp_bitonic_merge<4>(key, pay);
            key[2] = key[3] = kNoKey;
        }
    }
    for (uint32_t e = lane; e < width; e += 32) {
        const int i = static_cast<int>(e / 32);
        // element e = i*32 + lane of the sorted pool
        unsigned long long x = kNoKey;
#pragma unroll
        for (int ii = 0; ii < 2; ++ii) {
            if (ii == i) x = key[ii];
        }
        seeds[static_cast<uint64_t>(t) * width + e] = x;
    }
}

/// Apply the seeds symmetrically: q <- s and s <- q (src/incremental_knn.cpp:1195-1200).
__global__ void k_apply_seeds(const unsigned long long* __restrict__ seeds, uint32_t count, uint32_t width,
                              uint32_t first_new, CandStore cand) {
    const uint64_t x = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (x >= static_cast<uint64_t>(count) * width) return;
    const unsigned long long key = seeds[x];
    if (key == kNoKey) return;
    const uint32_t q = first_new + static_cast<uint32_t>(x / width);
    const uint32_t s = static_cast<uint32_t>(key);
    const float r = __uint_as_float(static_cast<uint32_t>(key >> 32));
    offer(cand, q, make_key(r, s));
    offer(cand, s, make_key(r, q));
}

/// Position x of a ring sequence: source-major (x = i*k + j, discovery order) or
/// rank-major (x = j*ns + i: every source's nearest entry before any second one).
__device__ __forceinline__ void ring_pos(uint64_t x, uint32_t ns, uint32_t k, bool rank_major, uint32_t* i,
                                         uint32_t* j) {
    if (rank_major) {
        *i = static_cast<uint32_t>(x % ns);
        *j = static_cast<uint32_t>(x / ns);
    } else {
        *i = static_cast<uint32_t>(x / k);
        *j = static_cast<uint32_t>(x % k);
    }
}

/// One ring of refinement_set (src/incremental_knn.cpp:927-987): the sequence is
/// (src[i], j) over the list entries of the source nodes; a node joins the ring at its
/// first position in the sequence if unmarked.
__global__ void k_ring_first(const uint32_t* __restrict__ src, uint32_t ns, const uint32_t* __restrict__ ids,
                             const uint32_t* __restrict__ counts, uint32_t k, uint32_t n,
                             const uint8_t* __restrict__ mark, uint32_t* __restrict__ firstpos, bool rank_major) {
    const uint64_t x = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (x >= static_cast<uint64_t>(ns) * k) return;
    uint32_t i, j;
    ring_pos(x, ns, k, rank_major, &i, &j);
    const uint32_t v = src[i];
    if (j >= counts[v]) return;
    const uint32_t q = ids[static_cast<uint64_t>(v) * k + j];
    if (q < n && !mark[q]) atomicMin(firstpos + q, static_cast<uint32_t>(x));
}

__global__ void k_ring_flag(const uint32_t* __restrict__ src, uint32_t ns, const uint32_t* __restrict__ ids,
                            const uint32_t* __restrict__ counts, uint32_t k, uint32_t n,
                            const uint8_t* __restrict__ mark, const uint32_t* __restrict__ firstpos,
                            uint32_t* __restrict__ flag, bool rank_major) {
    const uint64_t x = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (x >= static_cast<uint64_t>(ns) * k) return;
    uint32_t i, j;
    ring_pos(x, ns, k, rank_major, &i, &j);
    const uint32_t v = src[i];
    uint32_t f = 0;
    if (j < counts[v]) {
        const uint32_t q = ids[static_cast<uint64_t>(v) * k + j];
        f = (q < n && !mark[q] && firstpos[q] == static_cast<uint32_t>(x)) ? 1u : 0u;
    }
    flag[x] = f;
}

__global__ void k_ring_emit(const uint32_t* __restrict__ src, uint32_t ns, const uint32_t* __restrict__ ids, uint32_t k,
                            const uint32_t* __restrict__ flag, const uint32_t* __restrict__ off, uint32_t limit,
                            uint8_t* __restrict__ mark, uint32_t* __restrict__ out, bool rank_major) {
    const uint64_t x = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (x >= static_cast<uint64_t>(ns) * k || !flag[x]) return;
    const uint32_t pos = off[x];
    if (pos >= limit) return;
    uint32_t i, j;
    ring_pos(x, ns, k, rank_major, &i, &j);
    const uint32_t q = ids[static_cast<uint64_t>(src[i]) * k + j];
    mark[q] = 1;
    out[pos] = q;
}

__global__ void k_iota_from(uint32_t* __restrict__ out, uint32_t first, uint32_t count, uint8_t* __restrict__ mark) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    out[t] = first + t;
    mark[first + t] = 1;
}

/// Keep the first `keep` entries of nodes [lo, hi) (owned_warm_fraction,
/// src/incremental_knn.cpp:808-840): the freed slots let the random fill put other
/// new points of the batch there.
__global__ void k_truncate(uint32_t* __restrict__ ids, float* __restrict__ rank, uint8_t* __restrict__ flags,
                           uint32_t* __restrict__ counts, float* __restrict__ thr, uint32_t k, uint32_t lo,
                           uint32_t hi, uint32_t keep) {
    const uint64_t x = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const uint64_t span = static_cast<uint64_t>(hi - lo) * k;
    if (x >= span) return;
    const uint32_t v = lo + static_cast<uint32_t>(x / k), j = static_cast<uint32_t>(x % k);
    if (j >= keep) {
        ids[static_cast<uint64_t>(v) * k + j] = kInvalid;
        rank[static_cast<uint64_t>(v) * k + j] = __int_as_float(0x7f800000);
        flags[static_cast<uint64_t>(v) * k + j] = 0;
    }
    if (j == 0) {
        counts[v] = min(counts[v], keep);
        thr[v] = __int_as_float(0x7f800000);
    }
}

/// Reverse adjacency of the base graph as sorted (target << 32 | source) keys; the
/// sort makes each node's reverse list ascending by source, so a capped prefix is
/// the same on every run (the reference reads its ReverseNeighbours table,
/// src/incremental_knn.cpp:185-189).
__global__ void k_rev_keys(const uint32_t* __restrict__ ids, const uint32_t* __restrict__ counts, uint32_t k,
                           uint32_t n_base, unsigned long long* __restrict__ keys, uint32_t* __restrict__ rdeg) {
    const uint64_t x = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (x >= static_cast<uint64_t>(n_base) * k) return;
    const uint32_t v = static_cast<uint32_t>(x / k), j = static_cast<uint32_t>(x % k);
    unsigned long long key = ~0ull;
    if (j < counts[v]) {
        const uint32_t t = ids[x];
        if (t < n_base) {
            key = (static_cast<unsigned long long>(t) << 32) | v;
            atomicAdd(rdeg + t, 1u);
        }
    }
    keys[x] = key;
}

/// Views of the graph's cached descent scratch (grow-only buffers).
struct KnnScratch {
    DevBuf &thr, &cand, &cand_buf, &cand_cnt, &new_s, &old_s, &ns, &nold, &rnew, &rold, &rnew_cnt, &rold_cnt, &counters,
        &touched;
    explicit KnnScratch(Graph& g)
        : thr(g.knn_scratch[0]), cand(g.knn_scratch[1]), cand_buf(g.knn_scratch[2]), cand_cnt(g.knn_scratch[3]),
          new_s(g.knn_scratch[4]), old_s(g.knn_scratch[5]), ns(g.knn_scratch[6]), nold(g.knn_scratch[7]),
          rnew(g.knn_scratch[8]), rold(g.knn_scratch[9]), rnew_cnt(g.knn_scratch[10]), rold_cnt(g.knn_scratch[11]),
          counters(g.knn_scratch[12]), touched(g.knn_scratch[13]) {}
};

/// The node-proportional NN-Descent scratch for `sn` nodes.
void size_descent_scratch(KnnScratch& s, uint64_t sn) {
    s.thr.ensure(sn * 4ull);
    s.cand.ensure(sn * 8ull * kSlots);
    s.cand_buf.ensure(sn * 8ull * kCap);
    s.cand_cnt.ensure(sn * 4ull);
    s.new_s.ensure(sn * 4ull * kMaxSample);
    s.old_s.ensure(sn * 4ull * 3 * kMaxSample);
    s.ns.ensure(sn * 4ull);
    s.nold.ensure(sn * 4ull);
    s.rnew.ensure(sn * 4ull * kMaxSample);
    s.rold.ensure(sn * 4ull * kMaxSample);
    s.rnew_cnt.ensure(sn * 4ull);
    s.rold_cnt.ensure(sn * 4ull);
    s.counters.ensure(64);
    s.touched.ensure(sn * 4ull);
}

/// The node-proportional insert scratch (reverse index, active-set marks) for `sn`
/// nodes.
void size_insert_scratch(Graph& g, uint64_t sn) {
    g.insert_scratch[2].ensure(sn * g.k * 8 + 8);  // reverse keys
    g.insert_scratch[3].ensure(sn * g.k * 8 + 8);  // their sort buffer
    g.insert_scratch[4].ensure(sn * 4ull + 8);     // reverse degrees
    g.insert_scratch[5].ensure(sn * 4ull + 8);     // reverse offsets
    g.insert_scratch[7].ensure(sn + 16ull);        // active-set marks
    g.insert_scratch[8].ensure(sn * 4ull);         // first positions
    g.insert_scratch[9].ensure(sn * 4 + 4);        // active set
}

CandStore store_of(KnnScratch& s) {
    CandStore cs;
    cs.buf = s.cand_buf.as<unsigned long long>();
    cs.cnt = s.cand_cnt.as<uint32_t>();
    cs.table = s.cand.as<unsigned long long>();
    return cs;
}

void launch_merge(Ctx& c, Graph& g, KnnScratch& s, unsigned long long* updates) {
    const uint32_t n = static_cast<uint32_t>(g.n);
    if (n == 0) return;
    // the nodes that took an offer, then the merge over them (a grid of a few waves)
    uint32_t* list_count = s.counters.as<uint32_t>() + 4;  // bytes 16-19: after the two 64-bit counters
    CSB_CUDA(cudaMemsetAsync(list_count, 0, 4, c.stream));
    k_touched<<<blocks_for(n), kThreads, 0, c.stream>>>(n, s.cand_cnt.as<uint32_t>(), s.touched.as<uint32_t>(),
                                                         list_count);
    const unsigned grid = static_cast<unsigned>(
        std::min<uint64_t>((n + kWarps - 1) / kWarps, static_cast<uint64_t>(std::max(c.sm_count, 1)) * 16));
    if (g.k <= 32) {
        k_merge<1, 2><<<grid, kThreads, 0, c.stream>>>(n, g.k, g.ids.as<uint32_t>(), g.dists.as<float>(),
                                                     g.flags.as<uint8_t>(), g.counts.as<uint32_t>(), s.thr.as<float>(),
                                                     store_of(s), s.touched.as<uint32_t>(), list_count, updates,
                                                     g.hub_changed.as<uint8_t>());
    } else {
        k_merge<2, 4><<<grid, kThreads, 0, c.stream>>>(n, g.k, g.ids.as<uint32_t>(), g.dists.as<float>(),
                                                     g.flags.as<uint8_t>(), g.counts.as<uint32_t>(), s.thr.as<float>(),
                                                     store_of(s), s.touched.as<uint32_t>(), list_count, updates,
                                                     g.hub_changed.as<uint8_t>());
    }
    count_launch(c, 2);
}

}  // namespace

/// One Dynamic NN-Descent session over a resident graph: scratch, rank-space
/// distances and thresholds on construction; rounds over all nodes or an active list;
/// metric units again on finish().
struct Descent {
    Graph& g;
    Ctx& c;
    KnnScratch s;
    uint32_t n, k, smp;
    int wpb = 1;
    uint32_t join_rows = 0;
    size_t smem = 0;
    unsigned long long* d_updates = nullptr;
    unsigned long long* d_evals = nullptr;

    Descent(Graph& graph, uint32_t sample) : g(graph), c(*graph.ctx), s(graph) {
        n = static_cast<uint32_t>(g.n);
        k = g.k;
        smp = std::min<uint32_t>(std::max<uint32_t>(sample, 1), kMaxSample);
        if (k > 64) fail(CS_ERR_UNSUPPORTED, "NN-Descent: k > 64");
        const uint64_t nk = static_cast<uint64_t>(n) * k;
        size_descent_scratch(s, scratch_nodes(g));
        hub_track(g);  // k_merge flags the nodes whose membership changes
        d_updates = s.counters.as<unsigned long long>();
        d_evals = d_updates + 1;
        // the overflow tables are empty after every completed session (the merge resets
        // each slot it reads), so only a new buffer, nodes added since, or a session that
        // did not complete need the memset (at millions of nodes a few GB per insert)
        {
            const uint64_t slot_bytes = 8ull * kSlots;
            uint64_t from = 0;
            if (g.cand_clean_ptr == s.cand.p && g.cand_clean_bytes == s.cand.bytes)
                from = std::min<uint64_t>(g.cand_clean_n, n);
            if (from < n)
                CSB_CUDA(cudaMemsetAsync(static_cast<char*>(s.cand.p) + from * slot_bytes, 0xFF,
                                         (n - from) * slot_bytes, c.stream));
            g.cand_clean_n = 0;  // until finish()
        }
        CSB_CUDA(cudaMemsetAsync(s.cand_cnt.p, 0, n * 4ull, c.stream));
        CSB_CUDA(cudaMemsetAsync(s.rnew_cnt.p, 0, n * 4ull, c.stream));
        CSB_CUDA(cudaMemsetAsync(s.rold_cnt.p, 0, n * 4ull, c.stream));
        CSB_CUDA(cudaMemsetAsync(s.counters.p, 0, 64, c.stream));
        k_to_rank<<<blocks_for(nk), kThreads, 0, c.stream>>>(g.dists.as<float>(), nk, g.metric);
        k_threshold<<<blocks_for(n), kThreads, 0, c.stream>>>(g.dists.as<float>(), g.counts.as<uint32_t>(), n, k,
                                                             s.thr.as<float>());
        count_launch(c, 2);
        // join launch shape: the staged rows of one node are at most 2 x sample new
        // and 4 x sample old; the warps per block that keep the most warps resident
        join_rows = 6 * smp;
        const size_t per_warp = static_cast<size_t>(join_rows) * (2 + join_pitch(g.stride)) * 4;
        int dev = 0, max_smem = 0;
        CSB_CUDA(cudaGetDevice(&dev));
        CSB_CUDA(cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        CSB_CUDA(cudaFuncSetAttribute(k_join, cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem));
        int best_resident = 0;
        for (int w = 1; w <= kWarps; ++w) {
            if (per_warp * w > static_cast<size_t>(max_smem)) break;
            int occ = 0;
            CSB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_join, w * 32, per_warp * w));
            if (occ * w > best_resident) {
                best_resident = occ * w;
                wpb = w;
            }
        }
        if (best_resident == 0) fail(CS_ERR_UNSUPPORTED, "NN-Descent: a join warp's rows do not fit in shared memory");
        smem = per_warp * wpb;
        check_launch(c, "NN-Descent setup");
    }

    /// init_random: top the short lists of nodes [lo, hi) up with random candidates
    /// drawn from [cand_lo, cand_lo + cand_span) (all nodes by default).
    void random_fill(uint64_t seed, uint32_t lo = 0, uint32_t hi = 0xFFFFFFFFu, uint32_t cand_lo = 0,
                     uint32_t cand_span = 0) {
        if (hi > n) hi = n;
        if (!cand_span) cand_span = n;
        const unsigned gw = static_cast<unsigned>(std::max<uint32_t>(1, (hi - lo + kWarps - 1) / kWarps));
        const uint32_t max_attempts = k + k / 2 + 4;
        for (int pass = 0; pass * 32u < max_attempts; ++pass) {
            k_random_push<<<gw, kThreads, 0, c.stream>>>(g.pts.as<float>(), lo, hi, g.stride, g.counts.as<uint32_t>(), k,
                                                          seed, pass, store_of(s), cand_lo, cand_span);
            count_launch(c);
            launch_merge(c, g, s, nullptr);
        }
        check_launch(c, "NN-Descent random fill");
    }

    /// Rounds over `active` (all nodes when null) with the delta stop rule.
    uint64_t rounds(const uint32_t* active, uint32_t n_active, uint32_t iters, double delta, uint32_t* out_rounds) {
        const uint32_t m = active ? n_active : n;
        const unsigned gw = static_cast<unsigned>(std::max<uint32_t>(1, (m + kWarps - 1) / kWarps));
        const unsigned gj = static_cast<unsigned>(std::max<uint32_t>(1, (m + wpb - 1) / wpb));
        const double stop = delta * static_cast<double>(k) * static_cast<double>(m);
        uint64_t total = 0;
        uint32_t done = 0;
        for (uint32_t it = 0; it < iters && m > 0; ++it) {
            CSB_CUDA(cudaMemsetAsync(d_updates, 0, 8, c.stream));
            // the reverse samples k_sample counts into start empty every round
            CSB_CUDA(cudaMemsetAsync(s.rnew_cnt.p, 0, n * 4ull, c.stream));
            CSB_CUDA(cudaMemsetAsync(s.rold_cnt.p, 0, n * 4ull, c.stream));
            k_sample<<<gw, kThreads, 0, c.stream>>>(n, k, smp, g.ids.as<uint32_t>(), g.flags.as<uint8_t>(),
                                                     g.counts.as<uint32_t>(), s.new_s.as<uint32_t>(),
                                                     s.old_s.as<uint32_t>(), s.ns.as<uint32_t>(), s.nold.as<uint32_t>(),
                                                     s.rnew.as<uint32_t>(), s.rold.as<uint32_t>(),
                                                     s.rnew_cnt.as<uint32_t>(), s.rold_cnt.as<uint32_t>(), active, m);
            k_join<<<gj, wpb * 32, smem, c.stream>>>(g.pts.as<float>(), n, g.stride, smp, s.new_s.as<uint32_t>(),
                                                      s.old_s.as<uint32_t>(), s.ns.as<uint32_t>(), s.nold.as<uint32_t>(),
                                                      s.rnew.as<uint32_t>(), s.rold.as<uint32_t>(),
                                                      s.rnew_cnt.as<uint32_t>(), s.rold_cnt.as<uint32_t>(),
                                                      s.thr.as<float>(), store_of(s), wpb, d_evals, active, m,
                                                      join_rows);
            count_launch(c, 2);
            launch_merge(c, g, s, d_updates);
            check_launch(c, "NN-Descent round");
            unsigned long long upd = 0;
            CSB_CUDA(cudaMemcpyAsync(&upd, d_updates, 8, cudaMemcpyDeviceToHost, c.stream));
            CSB_CUDA(cudaStreamSynchronize(c.stream));
            total += upd;
            done = it + 1;
            if (static_cast<double>(upd) <= stop) break;
        }
        if (out_rounds) *out_rounds = done;
        return total;
    }

    void finish() {
        const uint64_t nk = static_cast<uint64_t>(n) * k;
        k_finalize<<<blocks_for(nk), kThreads, 0, c.stream>>>(g.dists.as<float>(), nk, g.metric);
        count_launch(c);
        check_launch(c, "NN-Descent finalize");
        c.sync();
        g.invalidate_edges();
        // every offer of the session has been merged: the tables are empty again
        g.cand_clean_ptr = s.cand.p;
        g.cand_clean_bytes = s.cand.bytes;
        g.cand_clean_n = n;
    }
};

/// Dynamic NN-Descent over the graph's resident points and k-NN arrays (which are
/// the warm start; distances in metric units on entry and exit).
void knn_descent(Graph& g, uint32_t sample, uint32_t iters, double delta, uint64_t seed, bool random_fill,
                 uint64_t* out_updates, uint32_t* out_rounds) {
    if (out_updates) *out_updates = 0;
    if (out_rounds) *out_rounds = 0;
    if (g.n == 0) return;
    Ctx& c = *g.ctx;
    g.hub_valid = false;  // a full build: the next bridge selection scores every node
    Descent d(g, sample);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CSB_CUDA(cudaEventCreate(&e0));
    CSB_CUDA(cudaEventCreate(&e1));
    CSB_CUDA(cudaEventRecord(e0, c.stream));
    if (random_fill) d.random_fill(seed);
    const uint64_t upd = d.rounds(nullptr, 0, iters, delta, out_rounds);
    d.finish();
    CSB_CUDA(cudaEventRecord(e1, c.stream));
    unsigned long long evals = 0;
    CSB_CUDA(cudaMemcpyAsync(&evals, d.d_evals, 8, cudaMemcpyDeviceToHost, c.stream));
    CSB_CUDA(cudaStreamSynchronize(c.stream));
    float ms = 0.0f;
    CSB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    g.last_build_evals = evals;
    g.last_build_ms = ms;
    if (out_updates) *out_updates = upd;
}

/// One ring of refinement_set appended to `out` at `at` (at most `limit` nodes);
/// returns the ring's size.
uint32_t expand_ring(Ctx& c, Graph& g, const uint32_t* src, uint32_t ns, uint8_t* mark, uint32_t* firstpos,
                     DevBuf& flag, DevBuf& off, uint32_t* out, uint32_t limit, bool rank_major) {
    if (ns == 0 || limit == 0) return 0;
    const uint32_t n = static_cast<uint32_t>(g.n), k = g.k;
    const uint64_t seq = static_cast<uint64_t>(ns) * k;
    if (seq > 0xFFFFFFFEull) fail(CS_ERR_UNSUPPORTED, "insert: refinement ring too large");
    flag.ensure(seq * 4 + 4);
    off.ensure(seq * 4 + 8);
    CSB_CUDA(cudaMemsetAsync(firstpos, 0xFF, n * 4ull, c.stream));
    k_ring_first<<<blocks_for(seq), kThreads, 0, c.stream>>>(src, ns, g.ids.as<uint32_t>(), g.counts.as<uint32_t>(), k, n,
                                                            mark, firstpos, rank_major);
    k_ring_flag<<<blocks_for(seq), kThreads, 0, c.stream>>>(src, ns, g.ids.as<uint32_t>(), g.counts.as<uint32_t>(), k, n,
                                                           mark, firstpos, flag.as<uint32_t>(), rank_major);
    count_launch(c, 2);
    scan_u32(c, flag.as<uint32_t>(), off.as<uint32_t>(), seq);
    uint32_t total = 0;
    CSB_CUDA(cudaMemcpyAsync(&total, off.as<uint32_t>() + seq, 4, cudaMemcpyDeviceToHost, c.stream));
    CSB_CUDA(cudaStreamSynchronize(c.stream));
    k_ring_emit<<<blocks_for(seq), kThreads, 0, c.stream>>>(src, ns, g.ids.as<uint32_t>(), k, flag.as<uint32_t>(),
                                                           off.as<uint32_t>(), limit, mark, out, rank_major);
    count_launch(c);
    check_launch(c, "refinement ring");
    return std::min(total, limit);
}

void knn_reserve(Graph& g) {
    KnnScratch s(g);
    Ctx& c = *g.ctx;
    const uint64_t ns = scratch_nodes(g), nk = ns * g.k;
    size_descent_scratch(s, ns);
    size_insert_scratch(g, ns);
    // what an insert batch that keeps the graph within ns nodes needs besides: its
    // seeds, the anti-hub entry points, the flags and offsets of its rings (at most ns
    // nodes), the reverse index's sort and scan scratch, and the staged rows
    const uint64_t rows = ns > g.n ? ns - g.n : 0;
    const uint32_t width = std::min<uint32_t>(2 * g.k, 64);
    g.insert_scratch[0].ensure(rows * width * 8);
    g.insert_scratch[1].ensure(selection_bound(g) * 4);
    g.insert_scratch[10].ensure(nk * 4 + 4);
    g.insert_scratch[11].ensure(nk * 4 + 8);
    if (nk < 0x7FFFFFFFull) {
        // the widest sort (all 32 target bits) needs the most temporary storage
        cub::DoubleBuffer<unsigned long long> db(nullptr, nullptr);
        size_t tmp_bytes = 0;
        CSB_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tmp_bytes, db, static_cast<int>(nk), 32, 64, c.stream));
        g.insert_scratch[6].ensure(tmp_bytes + 16);
    }
    scan_reserve(c, nk);
    c.scratch[6].ensure(rows * g.dim * 4);
}

void knn_insert(Graph& g, const float* rows, uint64_t count, uint32_t row_stride, const cs_insert_params& p,
                InsertStats* st) {
    Ctx& c = *g.ctx;
    if (count == 0) return;
    CSB_REQUIRE(g.n > 0, "cs_insert: insert before build (CoreSG::insert requires a built graph)");
    const uint32_t first_new = static_cast<uint32_t>(g.n);
    graph_set_points(g, rows, count, row_stride, true);
    const uint32_t n = static_cast<uint32_t>(g.n), k = g.k, nn = static_cast<uint32_t>(count);
    // stage events: start, reverse index, search + seeds, instance, refinement, end
    cudaEvent_t ev[6];
    for (auto& e : ev) CSB_CUDA(cudaEventCreate(&e));
    cudaEvent_t &e0 = ev[0], &e1 = ev[2], &e2 = ev[5];
    Descent d(g, p.sample);
    CSB_CUDA(cudaEventRecord(e0, c.stream));
    // seeding search over the base graph (ef = 2k results, at most the 64-entry
    // pool; the selected anti-hubs as extra entry points), then the seeds both ways
    const uint32_t width = std::min<uint32_t>(2 * k, 64);
    DevBuf& seeds = g.insert_scratch[0];
    DevBuf& hints = g.insert_scratch[1];
    seeds.ensure(static_cast<uint64_t>(nn) * width * 8);
    const uint32_t n_hint = static_cast<uint32_t>(g.selected.size());
    if (n_hint) {
        hints.ensure(n_hint * 4ull);
        copy_h2d(c, hints.p, g.selected.data(), n_hint * 4ull);
    }
    DevBuf& rev_keys = g.insert_scratch[2];
    DevBuf& rev_alt = g.insert_scratch[3];
    DevBuf& rev_deg = g.insert_scratch[4];
    DevBuf& rev_off = g.insert_scratch[5];
    DevBuf& sort_tmp = g.insert_scratch[6];
    if (p.reverse_cap) {
        const uint64_t nk = static_cast<uint64_t>(first_new) * k;
        CSB_REQUIRE(nk < 0x7FFFFFFFull, "cs_insert: base graph too large for the reverse index");
        size_insert_scratch(g, scratch_nodes(g));
        CSB_CUDA(cudaMemsetAsync(rev_deg.p, 0, first_new * 4ull + 8, c.stream));
        k_rev_keys<<<blocks_for(nk), kThreads, 0, c.stream>>>(g.ids.as<uint32_t>(), g.counts.as<uint32_t>(), k,
                                                               first_new, rev_keys.as<unsigned long long>(),
                                                               rev_deg.as<uint32_t>());
        count_launch(c);
        // targets fit below bit end_bit; the invalid key ~0 has every target bit set,
        // above any valid target (< first_new < 2^(end_bit-32)), so it sorts last
        int end_bit = 33;
        while (end_bit < 64 && (1ull << (end_bit - 32)) <= first_new) ++end_bit;
        cub::DoubleBuffer<unsigned long long> db(rev_keys.as<unsigned long long>(), rev_alt.as<unsigned long long>());
        size_t tmp_bytes = 0;
        // keys are written in source order and the radix sort is stable, so sorting
        // the target bits alone leaves each node's reverse list ascending by source
        CSB_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tmp_bytes, db, static_cast<int>(nk), 32, end_bit, c.stream));
        sort_tmp.ensure(tmp_bytes + 16);
        CSB_CUDA(cub::DeviceRadixSort::SortKeys(sort_tmp.p, tmp_bytes, db, static_cast<int>(nk), 32, end_bit, c.stream));
        count_launch(c, static_cast<uint64_t>((end_bit - 32 + 7) / 8) + 1);  // histogram + one per digit
        if (db.Current() != rev_keys.as<unsigned long long>()) {
            std::swap(rev_keys.p, rev_alt.p);
            std::swap(rev_keys.bytes, rev_alt.bytes);
        }
        scan_u32(c, rev_deg.as<uint32_t>(), rev_off.as<uint32_t>(), first_new);
        check_launch(c, "insert reverse index");
    }
    CSB_CUDA(cudaEventRecord(ev[1], c.stream));
    const uint32_t max_expand = p.max_expand ? p.max_expand : 8 * k;
    const size_t qsmem = static_cast<size_t>(kWarps) * g.stride * 4;
    k_search<<<(nn + kWarps - 1) / kWarps, kThreads, qsmem, c.stream>>>(
        g.pts.as<float>(), g.stride, g.ids.as<uint32_t>(), g.counts.as<uint32_t>(), k, first_new, first_new, nn, p.seed,
        max_expand, hints.as<uint32_t>(), n_hint, rev_off.as<uint32_t>(), rev_keys.as<unsigned long long>(),
        p.reverse_cap, width, seeds.as<unsigned long long>());
    k_apply_seeds<<<blocks_for(static_cast<uint64_t>(nn) * width), kThreads, 0, c.stream>>>(
        seeds.as<unsigned long long>(), nn, width, first_new, store_of(d.s));
    count_launch(c, 2);
    launch_merge(c, g, d.s, nullptr);
    check_launch(c, "insert seeding");
    CSB_CUDA(cudaEventRecord(e1, c.stream));
    DevBuf& mark = g.insert_scratch[7];
    DevBuf& firstpos = g.insert_scratch[8];
    DevBuf& active = g.insert_scratch[9];
    DevBuf& flag = g.insert_scratch[10];
    DevBuf& off = g.insert_scratch[11];
    size_insert_scratch(g, scratch_nodes(g));
    // the active set of a pass: the new points, then two rings, capped.  For the
    // instance (make_anchored_instances, src/incremental_knn.cpp:652-705) ring one is
    // the seeds rank by rank and ring two their neighbours; for the refinement
    // (refinement_set) both rings are in discovery order.
    auto active_set = [&](uint64_t cap, bool seeds_by_rank) -> uint32_t {
        if (cap < nn) cap = nn;
        if (cap > n) cap = n;
        CSB_CUDA(cudaMemsetAsync(mark.p, 0, n, c.stream));
        k_iota_from<<<blocks_for(nn), kThreads, 0, c.stream>>>(active.as<uint32_t>(), first_new, nn, mark.as<uint8_t>());
        count_launch(c);
        uint32_t na = nn;
        const uint32_t r1 = expand_ring(c, g, active.as<uint32_t>(), nn, mark.as<uint8_t>(), firstpos.as<uint32_t>(),
                                        flag, off, active.as<uint32_t>() + na, static_cast<uint32_t>(cap - na),
                                        seeds_by_rank);
        na += r1;
        na += expand_ring(c, g, active.as<uint32_t>() + nn, r1, mark.as<uint8_t>(), firstpos.as<uint32_t>(), flag, off,
                          active.as<uint32_t>() + na, static_cast<uint32_t>(cap - na), false);
        return na;
    };
    // the instance: new points plus their context (context_per_new per point), taken
    // while the new points' lists still hold every seed
    uint32_t n_active = active_set(static_cast<uint64_t>((1.0 + p.context_per_new) * nn), true);
    // owned nodes keep the head of their seed lists; the rest is filled with random
    // points of the batch, so the batch's own neighbourhoods get built
    const uint32_t keep = p.owned_warm_fraction >= 1.0 ? k : static_cast<uint32_t>(p.owned_warm_fraction * k);
    if (keep < k) {
        k_truncate<<<blocks_for(static_cast<uint64_t>(nn) * k), kThreads, 0, c.stream>>>(
            g.ids.as<uint32_t>(), g.dists.as<float>(), g.flags.as<uint8_t>(), g.counts.as<uint32_t>(), d.s.thr.as<float>(),
            k, first_new, n, keep);
        count_launch(c);
        d.random_fill(p.seed ^ 0x5851F42D4C957F2Dull, first_new, n, first_new, nn);
    }
    uint32_t rounds = 0, r2 = 0;
    uint64_t upd = d.rounds(active.as<uint32_t>(), n_active, p.instance_iters, p.delta, &rounds);
    // merge_job: the truncation was local to the instance, the global lists keep
    // every seed -- offer them again next to what the instance found
    if (keep < k) {
        k_apply_seeds<<<blocks_for(static_cast<uint64_t>(nn) * width), kThreads, 0, c.stream>>>(
            seeds.as<unsigned long long>(), nn, width, first_new, store_of(d.s));
        count_launch(c);
        launch_merge(c, g, d.s, nullptr);
        check_launch(c, "insert seed merge");
    }
    CSB_CUDA(cudaEventRecord(ev[3], c.stream));
    const uint32_t n_instance = n_active;
    // the restricted refinement (refine_per_new, refine_max_fraction)
    uint64_t cap = n;
    if (p.refine_max_fraction > 0.0 && p.refine_max_fraction < 1.0) cap = static_cast<uint64_t>(p.refine_max_fraction * n);
    if (p.refine_per_new > 0.0) cap = std::min<uint64_t>(cap, static_cast<uint64_t>(p.refine_per_new * nn));
    uint32_t n_ref = 0;
    if (p.refine_iters) {
        n_ref = active_set(cap, false);
        upd += d.rounds(active.as<uint32_t>(), n_ref, p.refine_iters, p.delta, &r2);
        n_active = std::max(n_active, n_ref);
    }
    rounds += r2;
    CSB_CUDA(cudaEventRecord(ev[4], c.stream));
    d.finish();
    CSB_CUDA(cudaEventRecord(e2, c.stream));
    CSB_CUDA(cudaEventSynchronize(e2));
    float ms[5] = {0, 0, 0, 0, 0};
    for (int i = 0; i < 5; ++i) CSB_CUDA(cudaEventElapsedTime(&ms[i], ev[i], ev[i + 1]));
    float ms_search = 0.0f, ms_refine = 0.0f;
    CSB_CUDA(cudaEventElapsedTime(&ms_search, e0, e1));
    CSB_CUDA(cudaEventElapsedTime(&ms_refine, e1, e2));
    for (auto& e : ev) cudaEventDestroy(e);
    if (st) {
        st->active = n_active;
        st->updates = upd;
        st->rounds = rounds;
        st->search_ms = ms_search;
        st->refine_ms = ms_refine;
        cs_insert_stats& x = st->detail;
        x.new_points = nn;
        x.instance_nodes = n_instance;
        x.refine_nodes = n_ref;
        x.updates = upd;
        x.rounds = rounds;
        x.reverse_ms = ms[0];
        x.search_ms = ms[1];
        x.instance_ms = ms[2];
        x.refine_ms = ms[3];
        x.finish_ms = ms[4];
    }
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

void cs_insert_defaults(cs_insert_params* p) {
    if (!p) return;
    p->sample = 16;
    p->instance_iters = 10;
    p->refine_iters = 5;
    p->context_per_new = 2.0;
    p->owned_warm_fraction = 0.25;
    p->refine_per_new = 2.0;
    p->refine_max_fraction = 0.25;
    p->delta = 0.001;
    p->max_expand = 0;
    p->reverse_cap = 16;
    p->seed = 7;
    p->reselect_bridges = 1;
}

cs_status cs_insert_stats_get(cs_graph* gp, cs_insert_stats* out) {
    Graph* g = reinterpret_cast<Graph*>(gp);
    return guarded(g ? g->ctx : nullptr, [&] {
        CSB_REQUIRE(out != nullptr, "cs_insert_stats_get: null out");
        *out = g->last_insert;
    });
}

cs_status cs_insert(cs_graph* gp, const float* rows, uint64_t count, uint32_t row_stride,
                    const cs_insert_params* params, uint64_t* out_active, uint64_t* out_updates) {
    Graph* g = reinterpret_cast<Graph*>(gp);
    return guarded(g ? g->ctx : nullptr, [&] {
        CSB_REQUIRE(rows != nullptr || count == 0, "cs_insert: null rows");
        cs_insert_params p;
        cs_insert_defaults(&p);
        if (params) p = *params;
        InsertStats st;
        const auto t0 = std::chrono::steady_clock::now();
        knn_insert(*g, rows, count, row_stride, p, &st);
        const auto t1 = std::chrono::steady_clock::now();
        if (p.reselect_bridges && count) select_bridges(*g, nullptr, nullptr, nullptr, nullptr);
        const auto t2 = std::chrono::steady_clock::now();
        st.detail.bridges_ms = std::chrono::duration<double, std::milli>(t2 - t1).count();
        st.detail.total_ms = std::chrono::duration<double, std::milli>(t2 - t0).count();
        g->last_insert = st.detail;
        if (out_active) *out_active = st.active;
        if (out_updates) *out_updates = st.updates;
    });
}

cs_status cs_knn_build_stats(cs_graph* gp, uint64_t* out_evals, double* out_device_ms) {
    Graph* g = reinterpret_cast<Graph*>(gp);
    return guarded(g ? g->ctx : nullptr, [&] {
        if (out_evals) *out_evals = g->last_build_evals;
        if (out_device_ms) *out_device_ms = g->last_build_ms;
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
