// The batched mpts sweep: up to 32 MSTs of one CORE-SG in one persistent launch.
//
// CoreSG::all_msts (src/coresg.cpp:412-417) runs K independent extractions, each
// rebuilding edges(mpts) and a Boruvka (src/mst.cpp:79-151).  Here the K MSTs of a
// pass share everything that can be shared:
//
//   * the edge list is built once per CORE-SG (graph.cu) and reweighted on the fly,
//     w'_j = max(w, core_j(u), core_j(v)), with core_j read from a [n][32] table of
//     every node's core distances at the pass's mpts (one 128-byte row per node, built
//     from the k-NN distance rows in the captured pre graph);
//   * one warp handles one edge (or one node's emitted segment) for all MSTs at once:
//     lane j is MST j.  Per-node state is node-major -- parent[v][32], best[v][32] --
//     so a node's state for all 32 MSTs is one 128/256-byte line and every per-node
//     access of the warp is coalesced;
//   * membership of edge i in the 32 trees is one bit-packed word tree[i]; after round
//     2, when the tail is off or its table overflowed, a single worklist of edges still
//     live in any MST serves all of them, each entry carrying the edge (index,
//     endpoints, weight) and its live lanes as one bit word;
//   * rounds 0-2 walk each node's emitted segment (the node-major enumeration of
//     src/knn_graph.cpp:132-200; warps claim a few nodes at a time from a counter), so
//     the emitter-side atomicMin of every lane is aggregated over the segment in
//     registers and issued once;
//   * the contracted tail: once a round's root list is short, the next round (the table
//     round) reduces every live (edge, MST) pair into a hash table keyed by (MST, root
//     pair) -- of parallel edges between two components only the lightest can be a tree
//     edge -- and the compacted entries make its offers; later rounds walk the entries,
//     one thread each, re-keying them through the table under the current roots;
//   * between rounds the roots that phase B may have linked are pointed at their
//     final roots, so a root lookup takes at most two loads; while the live (edge,
//     MST) pairs outnumber the nodes enough, every node is flattened as well
//     (parent[v][j] = root) and a lookup is one coalesced load;
//   * worklist and root-list appends go 32 entries of a warp at a time (one
//     atomicAdd per chunk);
//   * the phases are separated by a bounded grid barrier of a cooperative launch, and
//     the state reset, the persistent kernel and the finishing kernels (labels, tree
//     compaction, exact weights) are each captured once into a CUDA graph.
//
// Per round r, lane j (MST j):
//   A  every live edge finds the roots of its endpoints; if they differ it offers the
//      key (w'_j bits << 32 | i) to best[root][j] of both with atomicMin (no result
//      is read back);
//   B  every root of the round's root list (every node in round 0; later the roots
//      that took an offer the round before -- a root without one is final) takes
//      best[root][j]; the first lane to set bit j of tree[i] unites the endpoints
//      (roots linked larger-under-smaller) and resets best; the roots that took an
//      offer form the next round's list.
// The result is the unique minimum spanning forest of each mpts under (weight bits,
// edge index), i.e. the reference Boruvka's tree (pack_edge, src/mst.cpp:19-24).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>

#include "common.cuh"
#include "engine.hpp"

namespace csb {
namespace {

constexpr int kLanes = 32;
constexpr int kMaxRounds = 64;
constexpr int kThreads = 256;
constexpr uint64_t kBarrierLimitNs = 2000000000ull;
constexpr uint32_t kChunkEdges = 256;  // tree compaction: edges per warp chunk
constexpr int kMaxBlock = 512;
// the contracted tail starts once a round's root list holds at most n / kTailDiv
// nodes (cs_set_sweep_tail changes it per graph)
constexpr uint32_t kTailDiv = 4;
// per round: globaltimer at the round's start, after phase A, after phase B, after
// the flatten; edges phase A walked; roots phase B walked; live (edge, MST) pairs
// phase A found; whether every node was flattened
constexpr int kTraceWords = 8;

inline unsigned blocks_for(uint64_t work, int threads = kThreads) {
    uint64_t b = (work + threads - 1) / threads;
    return static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>(b, 1u << 30)));
}

struct SweepArgs {
    uint32_t n, E, e_knn, K, k;
    uint32_t flatten_div;  // flatten every node when live pairs exceed 32 n / flatten_div (0: never)
    const uint32_t* eu;
    const uint32_t* ev;
    const float* ew;
    const uint32_t* node_off;  // [n+1] emitted-segment offsets
    const float* dists;        // [n][k]
    const uint32_t* counts;    // [n]
    const uint32_t* mpts;      // [K]
    uint32_t* parent;          // [n][32]
    unsigned long long* best;  // [n][32]
    uint32_t* tree;            // [E] bit j: edge in MST j
    uint4* wl;                 // [2][E] worklist entries: edge index, endpoints, base weight bits
    uint32_t* live;            // [2][E] per worklist entry, bit j: the edge is live in MST j
    uint32_t* rlist;           // [2][n] roots that took an offer in the previous round
    uint32_t* fl;              // [n] frozen root list: roots as of the last full flatten
    const float* core;         // [n][32] core distance of v at mpts[j]
    uint32_t* ctr;             // [0],[1] worklist counts; [2],[3] root-list counts; [4] rounds;
                               // [5],[6] "some edge offered" flags; [7] frozen-list count;
                               // [8] tail table overflow; [9],[10] tail entry counts;
                               // [11],[12] segment-walk node counters; [13],[14] phase B
                               // root counters
    uint32_t tail_roots;       // contract once a round's root list is at most this (0: never)
    uint32_t tail_cap;         // tail table slots (a power of two); each entry list holds as many
    ulonglong2* ttab;          // [tail_cap] tail table: (MST, root pair) -> smallest key
    ulonglong2* tl;            // [2][tail_cap] tail entries: (MST, root pair), key
    unsigned* bar;
    int* status;
    uint64_t limit_ns;
    uint64_t hold_ns;           // testing hook: block 0 reaches its first barrier this late
    unsigned long long* trace;  // [kMaxRounds][kTraceWords] per-round timestamps and sizes
};

/// find with path halving on forest j of the node-major parent array.  A forest of n
/// nodes has no chain longer than n; a chase that takes more steps (a cycle, which the
/// linking rule rules out) sets the status and stops instead of spinning.
__device__ __forceinline__ uint32_t find32(uint32_t* parent, uint32_t x, uint32_t j, uint32_t n, int* status) {
    for (uint32_t it = 0; it <= n; ++it) {
        const uint32_t p = __ldcg(parent + static_cast<uint64_t>(x) * kLanes + j);
        if (p == x) return x;
        const uint32_t gp = __ldcg(parent + static_cast<uint64_t>(p) * kLanes + j);
        if (gp == p) return p;
        parent[static_cast<uint64_t>(x) * kLanes + j] = gp;
        x = gp;
    }
    atomicOr(status, kStatusUnionLimit);
    return x;
}

/// Root of x in forest j without writing: the flatten passes use it, so that every
/// entry a flatten writes is its own node's, and only ever the final root (path
/// halving there would race with other nodes' flatten writes and could put back a
/// stale intermediate ancestor after the root was written).
__device__ __forceinline__ uint32_t root32(const uint32_t* parent, uint32_t x, uint32_t j, uint32_t n, int* status) {
    for (uint32_t it = 0; it <= n; ++it) {
        const uint32_t p = __ldcg(parent + static_cast<uint64_t>(x) * kLanes + j);
        if (p == x) return x;
        x = p;
    }
    atomicOr(status, kStatusUnionLimit);
    return x;
}

__device__ __forceinline__ bool unite32(uint32_t* parent, uint32_t a, uint32_t b, uint32_t j, uint32_t n,
                                        int* status) {
    for (int it = 0; it < (1 << 20); ++it) {
        a = find32(parent, a, j, n, status);
        b = find32(parent, b, j, n, status);
        if (a == b) return false;
        if (a > b) {
            const uint32_t t = a;
            a = b;
            b = t;
        }
        if (atomicCAS(parent + static_cast<uint64_t>(b) * kLanes + j, b, a) == b) return true;
    }
    atomicOr(status, kStatusUnionLimit);
    return false;
}

/// Append the entries of a warp's chunk whose bits are set in the warp-uniform
/// `mask` (bit t: the entry held by lane t) to list `which` of the double buffer
/// `lists` (cap entries each; counters[which] counts it): one atomicAdd reserves the
/// exact count, then every marked lane writes its own entry, in lane order.
__device__ __forceinline__ void chunk_append(uint32_t* lists, uint32_t* counters, int which, uint32_t cap,
                                             uint32_t mask, uint32_t mine) {
    if (!mask) return;
    // the list and its counter are derived here, next to their use
    uint32_t* const list = lists + static_cast<uint64_t>(which) * cap;
    uint32_t* const counter = counters + which;
    const unsigned lane = threadIdx.x & 31u;
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(counter, static_cast<uint32_t>(__popc(mask)));
    base = __shfl_sync(0xFFFFFFFFu, base, 0);
    if ((mask >> lane) & 1u) list[base + __popc(mask & ((1u << lane) - 1u))] = mine;
}

/// Append the edge entries of a warp's chunk whose bits are set in `mask` (lane t
/// holds entry `mine` with live lanes `my_live`) to worklist `which`: one atomicAdd
/// reserves the count, every marked lane writes its own entry, in lane order.
__device__ __forceinline__ void chunk_append_edges(const SweepArgs& a, int which, uint32_t mask, uint4 mine,
                                                   uint32_t my_live) {
    if (!mask) return;
    uint4* const list = a.wl + static_cast<uint64_t>(which) * a.E;
    uint32_t* const lives = a.live + static_cast<uint64_t>(which) * a.E;
    const unsigned lane = threadIdx.x & 31u;
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(a.ctr + which, static_cast<uint32_t>(__popc(mask)));
    base = __shfl_sync(0xFFFFFFFFu, base, 0);
    if ((mask >> lane) & 1u) {
        const uint32_t at = base + __popc(mask & ((1u << lane) - 1u));
        list[at] = mine;
        lives[at] = my_live;
    }
}

constexpr uint32_t kNodeChunk = 8;   // nodes a warp claims at a time in the segment walks
constexpr int kSegGroup = 6;      // emitted-segment entries in flight per warp (rounds 0-2)
constexpr int kWlGroupFlat = 4;   // worklist edges in flight per warp: one root load per endpoint,
constexpr int kWlGroupHop = 4;    // or two

/// Root of x in forest j in rounds 0 and 1: the identity in round 0; after round 0's
/// flatten every node holds its root.
__device__ __forceinline__ uint32_t root01(const SweepArgs& a, uint32_t x, unsigned lane, int r) {
    return r == 0 ? x : __ldcg(a.parent + static_cast<uint64_t>(x) * kLanes + lane);
}

/// Offer `key` to best[root][lane].  The old value is not needed (phase B finds the
/// offered roots through the root list), so the atomic is issued without a return.
__device__ __forceinline__ void offer_min(const SweepArgs& a, uint32_t root, unsigned lane, unsigned long long key) {
    atomicMin(a.best + static_cast<uint64_t>(root) * kLanes + lane, key);
}

/// Per-lane two-entry cache of pending offers (root -> smallest key).  Offers to a
/// root met again soon -- the few components of the late rounds, where every edge
/// offers to the same handful of roots -- are reduced in registers; an atomicMin is
/// issued on eviction and at the flush.
struct OfferCache {
    uint32_t r0 = kInvalid, r1 = kInvalid;
    unsigned long long k0 = kNoKey, k1 = kNoKey;
    __device__ __forceinline__ void offer(const SweepArgs& a, unsigned lane, uint32_t root, unsigned long long key) {
        if (root == r0) {
            k0 = key < k0 ? key : k0;
            return;
        }
        if (root == r1) {  // hit on the second entry: it becomes the first
            const unsigned long long k = key < k1 ? key : k1;
            r1 = r0;
            k1 = k0;
            r0 = root;
            k0 = k;
            return;
        }
        if (r1 != kInvalid) offer_min(a, r1, lane, k1);
        r1 = r0;
        k1 = k0;
        r0 = root;
        k0 = key;
    }
    __device__ __forceinline__ void flush(const SweepArgs& a, unsigned lane) {
        if (r0 != kInvalid) offer_min(a, r0, lane, k0);
        if (r1 != kInvalid) offer_min(a, r1, lane, k1);
        r0 = r1 = kInvalid;
        k0 = k1 = kNoKey;
    }
};

// ---- the contracted tail --------------------------------------------------------
// Once a round's root list is short, the live (edge, MST) pairs collapse onto few
// component pairs.  The table round reduces every live pair's key into a hash table
// keyed by (MST, smaller root, larger root): of the edges joining two components only
// the lightest can enter the tree (the others close a cycle with it and tree edges of
// those components, and are its heaviest edge), so the table's entries carry the rest
// of the forest.  From the next round on, phase A walks the entries -- one thread per
// (MST, component pair) -- instead of the edge worklist.

constexpr unsigned long long kTailEmpty = ~0ull;
constexpr int kTailProbes = 64;      // linear-probe limit; beyond it the table overflows
constexpr int kTailNodeBits = 27;    // root ids in a tail key: graphs of at most 2^27 nodes

/// Tail key of MST j's component pair {x, y}: j in the top 5 bits, the smaller root in
/// the next 27, the larger in the low 32.
__device__ __forceinline__ unsigned long long tail_key(unsigned j, uint32_t x, uint32_t y) {
    const uint32_t lo = x < y ? x : y, hi = x < y ? y : x;
    return (static_cast<unsigned long long>(j) << 59) | (static_cast<unsigned long long>(lo) << 32) | hi;
}

/// Slot of a tail key: the splitmix64 finaliser (Steele, Lea, Flood 2014) of the key.
__device__ __forceinline__ uint32_t tail_slot(unsigned long long k, uint32_t mask) {
    k ^= k >> 30;
    k *= 0xbf58476d1ce4e5b9ull;
    k ^= k >> 27;
    k *= 0x94d049bb133111ebull;
    k ^= k >> 31;
    return static_cast<uint32_t>(k) & mask;
}

/// Reduce `key` into the entry of tail key `tk`: linear probing from its slot; a slot
/// already holding tk takes an atomicMin, an empty one is claimed with atomicCAS.  A
/// probe sequence longer than `probes` sets the overflow flag: in the table round the
/// sweep then carries on over its edge worklist; the tail rounds probe the whole table,
/// which they size above their entry count, so they always find a slot.
__device__ __forceinline__ void tail_insert(const SweepArgs& a, uint32_t mask, unsigned long long tk,
                                            unsigned long long key, uint32_t probes = kTailProbes) {
    uint32_t s = tail_slot(tk, mask);
    for (uint32_t p = 0; p < probes; ++p) {
        unsigned long long* slot = &a.ttab[s].x;
        unsigned long long cur = __ldcg(slot);
        if (cur == kTailEmpty) cur = atomicCAS(slot, kTailEmpty, tk);
        if (cur == kTailEmpty || cur == tk) {
            atomicMin(&a.ttab[s].y, key);
            return;
        }
        s = (s + 1) & mask;
    }
    a.ctr[8] = 1u;
}

constexpr int kTailBuf = 160;  // per-warp staging of table inserts: < 32 left + 4 edges x 32 lanes

/// The table round's inserts.  Each lane reduces consecutive live pairs that join the
/// same two components (edges of one emitter into one neighbouring component) in a
/// one-entry register cache.  What a lane evicts is staged in its warp's shared-memory
/// buffer, and after every group of edges the staged entries are inserted 32 at a
/// time, one per lane, so their table round trips overlap instead of stalling the
/// walk once per evicting edge.
struct TailStage {
    unsigned long long tk = kTailEmpty, key = kNoKey;  // this lane's cache
    ulonglong2* buf;                                   // the warp's kTailBuf entries
    uint32_t cnt = 0;                                  // staged entries (warp-uniform)
    /// Warp-collective: the lanes with `has` reduce (k, v) into their cache.
    __device__ __forceinline__ void add(bool has, unsigned long long k, unsigned long long v) {
        const unsigned lane = threadIdx.x & 31u;
        const bool ev = has && k != tk && tk != kTailEmpty;
        const unsigned em = __ballot_sync(0xFFFFFFFFu, ev);
        if (ev) buf[cnt + __popc(em & ((1u << lane) - 1u))] = make_ulonglong2(tk, key);
        cnt += static_cast<uint32_t>(__popc(em));
        if (has) {
            if (k == tk) {
                key = v < key ? v : key;
            } else {
                tk = k;
                key = v;
            }
        }
    }
    /// Warp-collective: insert staged entries 32 at a time while at least `keep_below`
    /// remain (32: leave fewer than 32 staged; 1: insert all).
    __device__ __forceinline__ void drain(const SweepArgs& a, uint32_t mask, uint32_t keep_below) {
        const unsigned lane = threadIdx.x & 31u;
        if (cnt < keep_below) return;
        __syncwarp();
        while (cnt >= keep_below && cnt > 0) {
            const uint32_t m = cnt < 32u ? cnt : 32u;
            if (lane < m) {
                const ulonglong2 e = buf[cnt - m + lane];
                tail_insert(a, mask, e.x, e.y);
            }
            cnt -= m;
        }
        __syncwarp();
    }
    /// Warp-collective: stage every lane's cached entry and insert everything.
    __device__ __forceinline__ void flush(const SweepArgs& a, uint32_t mask) {
        const unsigned lane = threadIdx.x & 31u;
        const bool ev = tk != kTailEmpty;
        const unsigned em = __ballot_sync(0xFFFFFFFFu, ev);
        if (ev) buf[cnt + __popc(em & ((1u << lane) - 1u))] = make_ulonglong2(tk, key);
        cnt += static_cast<uint32_t>(__popc(em));
        tk = kTailEmpty;
        key = kNoKey;
        drain(a, mask, 1u);
    }
};

/// Block-collective append of the entries whose threads have `keep` set to entry list
/// `which`: the warps' counts are scanned in shared memory and one atomicAdd per block
/// reserves them.  Every thread of the block calls it the same number of times;
/// `scan` holds kMaxBlock / 32 + 1 words.
__device__ __forceinline__ void tail_append(const SweepArgs& a, int which, bool keep, ulonglong2 e,
                                            uint32_t* scan) {
    const unsigned lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    if (!__syncthreads_or(keep)) return;  // block-uniform
    const unsigned km = __ballot_sync(0xFFFFFFFFu, keep);
    if (lane == 0) scan[w] = static_cast<uint32_t>(__popc(km));
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t tot = 0;
        for (unsigned i = 0; i < (blockDim.x >> 5); ++i) {
            const uint32_t c = scan[i];
            scan[i] = tot;
            tot += c;
        }
        scan[kMaxBlock / 32] = tot ? atomicAdd(a.ctr + 9 + which, tot) : 0u;
    }
    __syncthreads();
    if (keep)
        a.tl[static_cast<uint64_t>(which) * a.tail_cap + scan[kMaxBlock / 32] + scan[w] +
             __popc(km & ((1u << lane) - 1u))] = e;
    __syncthreads();  // the scan words are reused by the next call
}


/// Smallest 64-bit key over the lanes of `grp` (every lane of the group calls it).
__device__ __forceinline__ unsigned long long group_min_key(unsigned grp, unsigned long long key) {
    const uint32_t hi = __reduce_min_sync(grp, static_cast<uint32_t>(key >> 32));
    const uint32_t lo = __reduce_min_sync(grp, static_cast<uint32_t>(key >> 32) == hi ? static_cast<uint32_t>(key)
                                                                                       : 0xFFFFFFFFu);
    return (static_cast<unsigned long long>(hi) << 32) | lo;
}

/// Warp-collective offer of `key` to best[root][j] by the lanes with `has`: the lanes
/// offering to the same (root, MST) are reduced first and their leader issues one
/// atomicMin (the few roots of the late rounds take most of the warp's offers).
__device__ __forceinline__ void offer_grouped(const SweepArgs& a, bool has, uint32_t root, unsigned j,
                                              unsigned long long key) {
    const unsigned lane = threadIdx.x & 31u;
    if (!__any_sync(0xFFFFFFFFu, has)) return;
    // roots are below 2^27, so (root << 5 | j) never equals a lane's placeholder
    const unsigned long long gk = has ? ((static_cast<unsigned long long>(root) << 5) | j) : (kTailEmpty - lane);
    const unsigned grp = __match_any_sync(0xFFFFFFFFu, gk);
    // the reductions only where some group has two lanes (a reduction over 32 one-lane
    // groups costs one pass per group)
    const unsigned long long m = __any_sync(0xFFFFFFFFu, grp != (1u << lane)) ? group_min_key(grp, key) : key;
    if (has && lane == static_cast<unsigned>(__ffs(grp) - 1)) offer_min(a, root, j, m);
}

/// After the table round's phase A: the table's `slots` slots (a power of two, at
/// least 1024, so every warp chunk is full) are compacted into entry list `which`, and
/// every entry offers its key to both of its roots (the roots of this round: the
/// table's keys were read after the last links).
__device__ __forceinline__ void tail_compact(const SweepArgs& a, uint32_t slots, int which, uint32_t* scan) {
    // block-uniform trip count: slots and the grid's thread count are multiples of the
    // block size (powers of two of at least 1024 over 128, 256 or 512)
    for (uint32_t base = blockIdx.x * blockDim.x; base < slots; base += gridDim.x * blockDim.x) {
        const ulonglong2 e = __ldcg(a.ttab + base + threadIdx.x);
        const bool has = e.x != kTailEmpty;
        const unsigned j = static_cast<unsigned>(e.x >> 59);
        const uint32_t x = static_cast<uint32_t>(e.x >> 32) & ((1u << kTailNodeBits) - 1u);
        const uint32_t y = static_cast<uint32_t>(e.x);
        offer_grouped(a, has, x, j, e.y);
        offer_grouped(a, has, y, j, e.y);
        tail_append(a, which, has, e, scan);
    }
}

/// Phase A of a tail round: one thread per entry (MST j, roots x < y as of the round
/// the entry was kept, the lightest key between them).  The current roots are read
/// without writing (the chase from a root of an earlier round through the links made
/// since: tail rounds do not flatten).  An entry whose roots still differ goes into the
/// tail table under its current roots (entries of a warp with the same roots reduced to
/// their lightest first), so the entries that the round's links made parallel collapse
/// into one; the compacted table then makes the offers and the next entry list.  The
/// table has more slots than the list has entries, so a probe of the whole table always
/// finds one.
__device__ __forceinline__ bool tail_round(const SweepArgs& a, int r, uint32_t gw, uint32_t nw, uint32_t tmask,
                                           uint32_t& live_pairs) {
    const unsigned lane = threadIdx.x & 31u;
    const int par = r & 1;
    const uint32_t cnt = __ldcg(a.ctr + 9 + par);
    const ulonglong2* in = a.tl + static_cast<uint64_t>(par) * a.tail_cap;
    bool offered = false;
    for (uint32_t base = gw * 32u; base < cnt; base += nw * 32u) {
        const uint32_t t = base + lane;
        bool keep = false;
        ulonglong2 e = make_ulonglong2(kTailEmpty, kNoKey);
        if (t < cnt) {
            e = __ldcg(in + t);
            const unsigned j = static_cast<unsigned>(e.x >> 59);
            const uint32_t x = static_cast<uint32_t>(e.x >> 32) & ((1u << kTailNodeBits) - 1u);
            const uint32_t y = static_cast<uint32_t>(e.x);
            const uint32_t rx = root32(a.parent, x, j, a.n, a.status);
            const uint32_t ry = root32(a.parent, y, j, a.n, a.status);
            keep = rx != ry;
            if (keep) e.x = tail_key(j, rx, ry);
        }
        const unsigned grp = __match_any_sync(0xFFFFFFFFu, keep ? e.x : kTailEmpty - lane);
        const unsigned long long m = __any_sync(0xFFFFFFFFu, grp != (1u << lane)) ? group_min_key(grp, e.y) : e.y;
        live_pairs += keep ? 1u : 0u;
        offered = offered || keep;
        if (keep && lane == static_cast<unsigned>(__ffs(grp) - 1)) tail_insert(a, tmask, e.x, m, tmask + 1u);
    }
    return offered;
}

/// Phase A of rounds 0-2 for one bridge edge (i, u, v, w), all lanes (warp-collective;
/// from round 1 on every node holds its root).  kList: a live edge is appended with
/// its live lanes to worklist `which`; kTable: the live lanes' keys go to the tail
/// table instead of the offers.  Returns whether this lane found the edge live.
template <bool kList, bool kTable>
__device__ __forceinline__ bool bridge_lanes(const SweepArgs& a, uint32_t i, uint32_t u, uint32_t v, float w, int r,
                                             bool act, OfferCache& oc, TailStage& ts, uint32_t tmask, int which) {
    const unsigned lane = threadIdx.x & 31u;
    bool live = false;
    uint32_t ru = 0, rv = 0;
    unsigned long long key = kNoKey;
    if (act && u < a.n && v < a.n) {
        const float cu = __ldg(a.core + static_cast<uint64_t>(u) * kLanes + lane);
        const float cv = __ldg(a.core + static_cast<uint64_t>(v) * kLanes + lane);
        ru = root01(a, u, lane, r);
        rv = root01(a, v, lane, r);
        live = ru != rv;
        if (live) {
            key = pack_key(max_ref(w, max_ref(cu, cv)), i);
            if (!kTable) {
                oc.offer(a, lane, ru, key);
                oc.offer(a, lane, rv, key);
            }
        }
    }
    if (kTable) {
        ts.add(live, tail_key(lane, ru, rv), key);
        ts.drain(a, tmask, 32u);
    }
    if (kList) {
        const unsigned L = __ballot_sync(0xFFFFFFFFu, live);
        if (L && lane == 0) {
            const uint32_t at = atomicAdd(a.ctr + which, 1u);
            a.wl[static_cast<uint64_t>(which) * a.E + at] = make_uint4(i, u, v, __float_as_uint(w));
            a.live[static_cast<uint64_t>(which) * a.E + at] = L;
        }
    }
    return live;
}

/// Rounds 0-2, one chunk of node p's emitted segment (m <= 32 edges b, b+1, ...; lane
/// t holds edge b+t's other endpoint and base weight).  kSegGroup edges' core and root
/// loads are issued together.  Offering rounds fold every live edge's key into p's
/// minimum `seg` (offered once per node by the caller) and offer it to the other
/// endpoint's root; the table round (kTable) puts the keys in the tail table instead.
/// kList stores the edges' live lanes and returns the bits of the edges that stay live.
template <int R, bool kList, bool kTable>
__device__ __forceinline__ uint32_t seg_chunk(const SweepArgs& a, uint32_t rp, float cp, bool act, uint32_t m,
                                              uint32_t b, uint32_t my_q, float my_w, unsigned long long& seg,
                                              OfferCache& oc, TailStage& ts, uint32_t tmask, uint32_t& live_pairs,
                                              uint32_t& my_live) {
    const unsigned lane = threadIdx.x & 31u;
    uint32_t pmask = 0;
    for (uint32_t t = 0; t < m; t += kSegGroup) {
        float cq[kSegGroup];
        uint32_t rq[kSegGroup];
#pragma unroll
        for (int x = 0; x < kSegGroup; ++x) {
            const uint32_t q = __shfl_sync(0xFFFFFFFFu, my_q, (t + x) & 31u);
            const bool ok = act && t + x < m;  // endpoints are nodes (graph_build_edges)
            cq[x] = ok ? __ldg(a.core + static_cast<uint64_t>(q) * kLanes + lane) : 0.0f;
            rq[x] = R == 0 ? q : (ok ? __ldcg(a.parent + static_cast<uint64_t>(q) * kLanes + lane) : rp);
        }
#pragma unroll
        for (int x = 0; x < kSegGroup; ++x) {
            const float w = __shfl_sync(0xFFFFFFFFu, my_w, (t + x) & 31u);
            const bool lv = act && t + x < m && rp != rq[x];
            live_pairs += lv ? 1u : 0u;
            unsigned long long key = kNoKey;
            if (lv) {
                key = pack_key(max_ref(w, max_ref(cp, cq[x])), b + t + x);
                if (!kTable) {
                    seg = key < seg ? key : seg;
                    // round 0: every receiver is its own root and differs edge to edge,
                    // so the cache would only delay the atomic; later it merges offers
                    if (R == 0) {
                        offer_min(a, rq[x], lane, key);
                    } else {
                        oc.offer(a, lane, rq[x], key);
                    }
                } else {
                    seg = 0;  // marks that p had a live pair
                }
            }
            if (kTable) {
                ts.add(lv, tail_key(lane, rp, rq[x]), key);
                if (x == kSegGroup / 2 - 1) ts.drain(a, tmask, 32u);  // the buffer holds 4 edges' evictions
            }
            // kList records the live lanes (the lane holding the edge keeps them); the
            // ballot is taken next to its value
            if (kList && t + x < m) {
                const unsigned L = __ballot_sync(0xFFFFFFFFu, lv);
                if (lane == t + x) my_live = L;
                if (L) pmask |= 1u << (t + x);
            }
        }
        if (kTable) ts.drain(a, tmask, 32u);
    }
    return pmask;
}

/// Rounds 0-2: the k-NN edges node by node over the emitted segments (32 edges of a
/// segment loaded at once); the emitter's offers are reduced in registers and issued
/// once.  R = 0: every node is its own root; R = 1: every node holds its root (rounds 1
/// and 2: rounds 0 and 1 flatten every node).  kList builds worklist `which`; kTable
/// fills the tail table (round 2 as the table round).
template <int R, bool kList, bool kTable>
__device__ __forceinline__ bool seg_round(const SweepArgs& a, uint32_t* work, bool act, OfferCache& oc,
                                          TailStage& ts, uint32_t tmask, int which, uint32_t& live_pairs) {
    static_assert(kTailBuf >= 32 + 32 * (kSegGroup - kSegGroup / 2) && kTailBuf >= 32 + 32 * (kSegGroup / 2),
                  "half a group's staged inserts must fit the warp's buffer");
    const unsigned lane = threadIdx.x & 31u;
    bool offered = false;
    // warps claim kNodeChunk consecutive nodes at a time from the phase's counter, so a
    // phase ends when the work does rather than when the slowest fixed share does
    for (;;) {
        uint32_t c0 = 0;
        if (lane == 0) c0 = atomicAdd(work, kNodeChunk);
        c0 = __shfl_sync(0xFFFFFFFFu, c0, 0);
        if (c0 >= a.n) break;
        const uint32_t c1 = min(c0 + kNodeChunk, a.n);
        for (uint32_t p = c0; p < c1; ++p) {
            const uint32_t beg = __ldg(a.node_off + p), end = __ldg(a.node_off + p + 1);
            if (beg == end) continue;
            const float cp = act ? __ldg(a.core + static_cast<uint64_t>(p) * kLanes + lane) : 0.0f;
            const uint32_t rp = act ? root01(a, p, lane, R) : p;
            unsigned long long seg = kNoKey;
            for (uint32_t b = beg; b < end; b += 32) {
                const uint32_t m = min(32u, end - b);
                uint32_t my_q = 0, my_x = 0, my_y = 0, my_live = 0;
                float my_w = 0.0f;
                if (lane < m) {
                    my_x = __ldg(a.eu + b + lane);
                    my_y = __ldg(a.ev + b + lane);
                    my_q = my_x == p ? my_y : my_x;
                    my_w = __ldg(a.ew + b + lane);
                }
                const uint32_t pmask =
                    seg_chunk<R, kList, kTable>(a, rp, cp, act, m, b, my_q, my_w, seg, oc, ts, tmask, live_pairs, my_live);
                if (kList)
                    chunk_append_edges(a, which, pmask, make_uint4(b + lane, my_x, my_y, __float_as_uint(my_w)), my_live);
            }
            if (seg != kNoKey) {
                if (!kTable) offer_min(a, rp, lane, seg);
                offered = true;
            }
        }
    }
    return offered;
}

/// Phase A of rounds 0-2: the emitted segments, then the bridges one warp per edge.
template <int R, bool kList, bool kTable>
__device__ __forceinline__ bool seg_phase(const SweepArgs& a, int r, uint32_t gw, uint32_t nw, bool act,
                                          OfferCache& oc, TailStage& ts, uint32_t tmask, uint32_t& live_pairs) {
    const int which = (r + 1) & 1;
    bool offered = seg_round<R, kList, kTable>(a, a.ctr + 11 + (r & 1), act, oc, ts, tmask, which, live_pairs);
    for (uint32_t i = a.e_knn + gw; i < a.E; i += nw) {
        const bool o = bridge_lanes<kList, kTable>(a, i, __ldg(a.eu + i), __ldg(a.ev + i), __ldg(a.ew + i), r, act, oc,
                                                   ts, tmask, which);
        offered = offered || o;
    }
    if (kTable) ts.flush(a, tmask);
    return offered;
}

/// Rounds >= 2: the worklist of edges live in some MST, 32 entries per warp loaded
/// at once (each entry carries the edge -- index, endpoints, weight -- and its live
/// lanes, so no gather by edge index precedes the root loads), a group of them in
/// flight.  With
/// kFlat every node was flattened after the last round and a root lookup is one
/// load.  Otherwise it is two: a node holds its root as of the last full flatten (or
/// a later root that phase B's path halving wrote), which is a node of the frozen
/// root list or a final root, and the flatten after every phase B points each node
/// of the frozen list at its current root.  Nothing is written back, so the second
/// loads of a group are issued together after the first ones.  With kTable (the table
/// round) every live pair's key is reduced into the tail table (slot mask tmask)
/// instead: no offers and no next worklist, the table's entries make both.
template <bool kFlat, bool kTable>
__device__ __forceinline__ bool wl_round(const SweepArgs& a, int r, uint32_t gw, uint32_t nw, bool act,
                                         OfferCache& oc, uint32_t& live_pairs, uint32_t tmask,
                                         ulonglong2* stage) {
    constexpr int G = kFlat ? kWlGroupFlat : kWlGroupHop;
    const unsigned lane = threadIdx.x & 31u;
    const int par = r & 1;
    bool offered = false;
    const uint32_t cnt = __ldcg(a.ctr + par);
    const uint4* in = a.wl + static_cast<uint64_t>(par) * a.E;
    const uint32_t* in_live = a.live + static_cast<uint64_t>(par) * a.E;
    static_assert(kTailBuf >= 32 + 32 * G, "a group's staged inserts must fit the warp's buffer");
    TailStage tc;
    tc.buf = stage + (threadIdx.x >> 5) * kTailBuf;
    for (uint32_t base = gw * 32u; base < cnt; base += nw * 32u) {
        const uint32_t m = min(32u, cnt - base);
        uint4 my_e = make_uint4(0u, 0u, 0u, 0u);
        uint32_t my_l = 0;
        if (lane < m) {
            my_e = __ldcg(in + base + lane);
            my_l = __ldcg(in_live + base + lane);
        }
        const uint32_t my_i = my_e.x, my_u = my_e.y, my_v = my_e.z;
        const float my_w = __uint_as_float(my_e.w);
        uint32_t pmask = 0;  // entries of this chunk that stay live
        uint32_t my_new = 0;  // this lane's entry's live lanes after the round
        for (uint32_t t = 0; t < m; t += G) {
            float cu[G], cv[G];
            uint32_t ru[G], rv[G];
            uint32_t okm = 0;
#pragma unroll
            for (int x = 0; x < G; ++x) {
                const uint32_t src = (t + x) & 31u;
                const uint32_t u = __shfl_sync(0xFFFFFFFFu, my_u, src);
                const uint32_t v = __shfl_sync(0xFFFFFFFFu, my_v, src);
                const uint32_t l = __shfl_sync(0xFFFFFFFFu, my_l, src);
                const bool ok = act && t + x < m && ((l >> lane) & 1u);
                okm |= ok ? 1u << x : 0u;
                cu[x] = ok ? __ldg(a.core + static_cast<uint64_t>(u) * kLanes + lane) : 0.0f;
                cv[x] = ok ? __ldg(a.core + static_cast<uint64_t>(v) * kLanes + lane) : 0.0f;
                ru[x] = ok ? __ldcg(a.parent + static_cast<uint64_t>(u) * kLanes + lane) : 0u;
                rv[x] = ok ? __ldcg(a.parent + static_cast<uint64_t>(v) * kLanes + lane) : 0u;
            }
            if (!kFlat) {
#pragma unroll
                for (int x = 0; x < G; ++x) {
                    const uint32_t src = (t + x) & 31u;
                    const uint32_t u = __shfl_sync(0xFFFFFFFFu, my_u, src);
                    const uint32_t v = __shfl_sync(0xFFFFFFFFu, my_v, src);
                    const bool ok = (okm >> x) & 1u;
                    if (ok && ru[x] != u) ru[x] = __ldcg(a.parent + static_cast<uint64_t>(ru[x]) * kLanes + lane);
                    if (ok && rv[x] != v) rv[x] = __ldcg(a.parent + static_cast<uint64_t>(rv[x]) * kLanes + lane);
                }
            }
#pragma unroll
            for (int x = 0; x < G; ++x) {
                const uint32_t src = (t + x) & 31u;
                const uint32_t i = __shfl_sync(0xFFFFFFFFu, my_i, src);
                const float w = __shfl_sync(0xFFFFFFFFu, my_w, src);
                const bool lv = ((okm >> x) & 1u) && ru[x] != rv[x];
                live_pairs += lv ? 1u : 0u;
                unsigned long long key = kNoKey;
                if (lv) {
                    key = pack_key(max_ref(w, max_ref(cu[x], cv[x])), i);
                    if (!kTable) {
                        oc.offer(a, lane, ru[x], key);
                        oc.offer(a, lane, rv[x], key);
                    }
                    offered = true;
                }
                if (kTable) tc.add(lv, tail_key(lane, ru[x], rv[x]), key);
                if (!kTable && t + x < m) {  // ballot next to the value it reads
                    const unsigned L = __ballot_sync(0xFFFFFFFFu, lv);
                    if (lane == t + x) my_new = L;
                    if (L) pmask |= 1u << (t + x);
                }
            }
            if (kTable) tc.drain(a, tmask, 32u);
        }
        if (!kTable) chunk_append_edges(a, (r + 1) & 1, pmask, my_e, my_new);
    }
    if (kTable) tc.flush(a, tmask);
    return offered;
}

/// Point node c's entry of forest `lane` at its root, if it is not there already
/// (only ever the final root is written, so concurrent chases stay correct).
__device__ __forceinline__ void point_at_root(uint32_t* parent, uint32_t c, unsigned lane, uint32_t n, int* status) {
    uint32_t* const pc = parent + static_cast<uint64_t>(c) * kLanes + lane;
    const uint32_t p = __ldcg(pc);
    if (p == c) return;
    const uint32_t f = root32(parent, p, lane, n, status);
    if (f != p) *pc = f;
}

// two blocks of kMaxBlock threads per SM: at most 64 registers a thread
__global__ void __launch_bounds__(kMaxBlock, 2) k_sweep(SweepArgs a) {
    __shared__ ulonglong2 s_stage[(kMaxBlock / 32) * kTailBuf];  // the table round's insert staging
    __shared__ uint32_t s_scan[kMaxBlock / 32 + 1];               // the tail lists' block appends
    const unsigned lane = threadIdx.x & 31u;
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    const uint32_t gt = blockIdx.x * blockDim.x + threadIdx.x, nt = gridDim.x * blockDim.x;
    const bool act = lane < a.K;
    bool flat = true;  // parents are the identity at the start
    // 0: phase A walks the edges; 1: the table round (phase A walks the edges into the
    // tail table, whose entries then make the offers); 2: phase A walks the tail
    // entries.  Grid-uniform: every change follows a value read after a grid barrier.
    int mode = 0;
    bool tail_ok = a.tail_roots != 0;
    uint32_t tmask = 0;
    int r = 0;
    for (; r < kMaxRounds; ++r) {
        const int par = r & 1, nxt = (r + 1) & 1;
        const int rmode = mode;
        unsigned long long* tr = a.trace + static_cast<uint64_t>(r) * kTraceWords;
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            a.ctr[2 + nxt] = 0;  // the root list phase B of this round writes
            a.ctr[5 + nxt] = 0;  // next round's offer flag
            tr[0] = global_ns();  // the other words start zeroed (pre graph)
            tr[4] = r <= 2 ? a.E : __ldcg(a.ctr + (mode == 2 ? 9 + par : par));
            tr[5] = r == 0 ? a.n : __ldcg(a.ctr + 2 + par);
            tr[7] = static_cast<unsigned>(mode) << 1;  // the flatten bit joins at the round's end
        }
        OfferCache oc;
        bool offered = false;
        uint32_t live_pairs = 0;
        // ---- phase A
        TailStage ts;
        ts.buf = s_stage + (threadIdx.x >> 5) * kTailBuf;
        if (r == 0) {
            offered = seg_phase<0, false, false>(a, r, gw, nw, act, oc, ts, 0u, live_pairs);
        } else if (r == 1) {
            offered = seg_phase<1, false, false>(a, r, gw, nw, act, oc, ts, 0u, live_pairs);
        } else if (r == 2 && mode == 1) {
            offered = seg_phase<1, false, true>(a, r, gw, nw, act, oc, ts, tmask, live_pairs);
        } else if (r == 2) {
            offered = seg_phase<1, true, false>(a, r, gw, nw, act, oc, ts, 0u, live_pairs);
        } else if (mode == 2) {
            offered = tail_round(a, r, gw, nw, tmask, live_pairs);
        } else if (mode == 1) {
            offered = flat ? wl_round<true, true>(a, r, gw, nw, act, oc, live_pairs, tmask, s_stage)
                           : wl_round<false, true>(a, r, gw, nw, act, oc, live_pairs, tmask, s_stage);
        } else {
            offered = flat ? wl_round<true, false>(a, r, gw, nw, act, oc, live_pairs, 0u, s_stage)
                           : wl_round<false, false>(a, r, gw, nw, act, oc, live_pairs, 0u, s_stage);
        }
        oc.flush(a, lane);
        {
            unsigned long long lp = live_pairs;
            for (int o = 16; o > 0; o >>= 1) lp += __shfl_xor_sync(0xFFFFFFFFu, lp, o);
            if (lane == 0 && lp) atomicAdd(tr + 6, lp);
        }
        if (__any_sync(0xFFFFFFFFu, offered) && lane == 0) a.ctr[5 + par] = 1u;
        if (a.hold_ns && r == 0 && blockIdx.x == 0) {
            // testing hook: block 0 arrives late (a bounded sleep), so the other
            // blocks' barrier waits run out when hold_ns exceeds the limit
            if (threadIdx.x == 0) {
                const uint64_t t0 = global_ns();
                while (global_ns() - t0 < a.hold_ns) __nanosleep(1000);
            }
            __syncthreads();
        }
        if (!grid_barrier(a.bar, a.bar + 1, a.status, a.limit_ns)) return;
        if (blockIdx.x == 0 && threadIdx.x == 0) tr[1] = global_ns();
        if (__ldcg(a.ctr + 5 + par) == 0u) break;
        if (mode == 1) {
            if (__ldcg(a.ctr + 8) != 0u) {
                // the table overflowed: phase A again over the same worklist, with its
                // offers and the next worklist; no tail
                mode = 0;
                tail_ok = false;
                uint32_t again = 0;
                if (r == 2) {
                    // the walk's node counter starts again
                    if (blockIdx.x == 0 && threadIdx.x == 0) a.ctr[11 + par] = 0;
                    if (!grid_barrier(a.bar, a.bar + 1, a.status, a.limit_ns)) return;
                    seg_phase<1, true, false>(a, r, gw, nw, act, oc, ts, 0u, again);
                } else if (flat) {
                    wl_round<true, false>(a, r, gw, nw, act, oc, again, 0u, s_stage);
                } else {
                    wl_round<false, false>(a, r, gw, nw, act, oc, again, 0u, s_stage);
                }
                oc.flush(a, lane);
            } else {
                // the table's entries become the first tail list, and each offers its
                // key to both of its roots
                tail_compact(a, tmask + 1u, nxt, s_scan);
            }
            if (!grid_barrier(a.bar, a.bar + 1, a.status, a.limit_ns)) return;
        } else if (mode == 2) {
            // the re-keyed entries: the next list, and the round's offers
            tail_compact(a, tmask + 1u, nxt, s_scan);
            if (!grid_barrier(a.bar, a.bar + 1, a.status, a.limit_ns)) return;
        }
        // ---- phase B: every root that took an offer (all nodes in round 0) links
        // along its best edge; the roots that took one form the next round's list
        // (a root without an offer has no outgoing live edge: its tree is final)
        {
            const uint32_t rc = r == 0 ? a.n : __ldcg(a.ctr + 2 + par);
            const uint32_t* rin = a.rlist + static_cast<uint64_t>(par) * a.n;
            // chunks of 32 roots claimed from the phase's counter
            for (;;) {
                uint32_t base = 0;
                if (lane == 0) base = atomicAdd(a.ctr + 13 + par, 32u);
                base = __shfl_sync(0xFFFFFFFFu, base, 0);
                if (base >= rc) break;
                const uint32_t m = min(32u, rc - base);
                const uint32_t my_c = lane < m ? (r == 0 ? base + lane : __ldcg(rin + base + lane)) : 0u;
                uint32_t keep = 0;  // roots of this chunk that took an offer
                for (uint32_t t = 0; t < m; ++t) {
                    const uint32_t c = __shfl_sync(0xFFFFFFFFu, my_c, t);
                    unsigned long long* slot = a.best + static_cast<uint64_t>(c) * kLanes + lane;
                    const unsigned long long key = act ? __ldcg(slot) : kNoKey;
                    const bool has = key != kNoKey;
                    if (__ballot_sync(0xFFFFFFFFu, has)) keep |= 1u << t;
                    if (has) {
                        *slot = kNoKey;
                        const uint32_t i = static_cast<uint32_t>(key);
                        // the tree bit by a reduction (nothing to wait for); both roots of
                        // an edge they both took call the union, and the second finds
                        // them united already
                        atomicOr(a.tree + i, 1u << lane);
                        unite32(a.parent, __ldg(a.eu + i), __ldg(a.ev + i), lane, a.n, a.status);
                    }
                }
                chunk_append(a.rlist, a.ctr + 2, (r + 1) & 1, a.n, keep, my_c);
            }
        }
        if (mode != 0) {
            // the next round is a tail round: it re-keys its entries through the table,
            // cleared here for them, at least twice as many slots as entries
            const uint32_t cn = __ldcg(a.ctr + 9 + nxt);
            uint32_t slots = 1024;
            while (slots < a.tail_cap && static_cast<uint64_t>(slots) < 2ull * cn) slots <<= 1;
            tmask = slots - 1u;
            for (uint32_t t = gt; t < slots; t += nt) a.ttab[t] = make_ulonglong2(kTailEmpty, kNoKey);
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            a.ctr[par] = 0;       // this round's worklist, consumed
            a.ctr[9 + par] = 0;   // and its tail entries
            a.ctr[11 + par] = 0;  // and phase A's node counter
        }
        if (!grid_barrier(a.bar, a.bar + 1, a.status, a.limit_ns)) return;
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            tr[2] = global_ns();
            a.ctr[13 + par] = 0;  // phase B's root counter, consumed
        }
        // ---- flatten.  Step 1 points at its final root every node of the list whose
        // roots phase B may have linked: in rounds 0 and 1 the list phase B walked
        // (every node with an edge, so that is a full flatten), later the frozen root
        // list (roots as of the last full flatten; it holds every root of this round).
        // Round 1 freezes round 2's root list.  The tail rounds skip it: their lookups
        // chase from roots without writing (the table round's flatten leaves the first
        // tail round one load from each root).
        if (mode != 2) {
            const uint32_t cnt = r == 0 ? a.n : __ldcg(a.ctr + (r == 1 ? 2 + par : 7));
            const uint32_t* lst = r == 1 ? a.rlist + static_cast<uint64_t>(par) * a.n : a.fl;
            for (uint32_t t = gw; t < cnt; t += nw) {
                if (act) point_at_root(a.parent, r == 0 ? t : __ldcg(lst + t), lane, a.n, a.status);
            }
            if (r == 1) {
                const uint32_t nc = __ldcg(a.ctr + 2 + nxt);
                const uint32_t* src = a.rlist + static_cast<uint64_t>(nxt) * a.n;
                for (uint32_t t = gt; t < nc; t += nt) a.fl[t] = __ldcg(src + t);
                if (gt == 0) a.ctr[7] = nc;
            }
            if (!grid_barrier(a.bar, a.bar + 1, a.status, a.limit_ns)) return;
        }
        // ---- step 2, from round 2 on: every node, when this round's live (edge, MST)
        // pairs say the next round's second root loads would cost more than a pass over
        // the nodes; it freezes the next round's root list.  After step 1 a node's entry
        // is a frozen-list node or a final root, whose entry is its root: two loads.
        const uint64_t pairs = __ldcg(tr + 6);
        const bool full = mode == 0 && r >= 2 && a.flatten_div != 0 &&
                          pairs > static_cast<uint64_t>(a.n) * kLanes / a.flatten_div;
        if (full) {
            for (uint32_t v = gw; v < a.n; v += nw) {
                if (act) {
                    uint32_t* const pv = a.parent + static_cast<uint64_t>(v) * kLanes + lane;
                    const uint32_t p = __ldcg(pv);
                    if (p != v) {
                        const uint32_t f = __ldcg(a.parent + static_cast<uint64_t>(p) * kLanes + lane);
                        if (f != p) *pv = f;
                    }
                }
            }
            const uint32_t nc = __ldcg(a.ctr + 2 + nxt);
            const uint32_t* src = a.rlist + static_cast<uint64_t>(nxt) * a.n;
            for (uint32_t t = gt; t < nc; t += nt) a.fl[t] = __ldcg(src + t);
            if (gt == 0) a.ctr[7] = nc;
            if (!grid_barrier(a.bar, a.bar + 1, a.status, a.limit_ns)) return;
        }
        flat = r <= 1 || full;
        if (mode == 1) mode = 2;
        // ---- arm the table round when the next round's root list is short (the
        // tail's keys hold root ids below 2^27; the host sets tail_roots only then).
        // This round's live pairs bound the next round's, so the table gets at least
        // twice as many slots when the buffer allows.
        if (mode == 0 && tail_ok && r >= 1 && __ldcg(a.ctr + 2 + nxt) <= a.tail_roots) {
            uint32_t slots = 1024;
            while (slots < a.tail_cap && static_cast<uint64_t>(slots) < 2 * pairs) slots <<= 1;
            tmask = slots - 1u;
            for (uint32_t t = gt; t < slots; t += nt) a.ttab[t] = make_ulonglong2(kTailEmpty, kNoKey);
            mode = 1;
            if (!grid_barrier(a.bar, a.bar + 1, a.status, a.limit_ns)) return;
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            tr[3] = global_ns();
            tr[7] = (flat ? 1u : 0u) | (static_cast<unsigned>(rmode) << 1);
        }
    }
    if (r == kMaxRounds) {
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(a.status, kStatusRoundLimit);
        return;
    }
    // final flatten: parent[v][j] = root (the component's smallest node)
    for (uint32_t v = gw; v < a.n; v += nw) {
        if (act) a.parent[static_cast<uint64_t>(v) * kLanes + lane] = root32(a.parent, v, lane, a.n, a.status);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) a.ctr[4] = static_cast<uint32_t>(r + 1);
}

/// The per-sweep node tables in one pass: core[v][j] = core distance of v at mpts[j]
/// (core_dist, include/coresg/knn_graph.hpp:157-163; +inf for an empty list; lanes
/// >= K hold 0), and parent[v][j] = v (every node its own root).
__global__ void k_core32(const float* __restrict__ dists, const uint32_t* __restrict__ counts, uint32_t k,
                         const uint32_t* __restrict__ mpts, uint32_t K, uint32_t n, float* __restrict__ core,
                         uint32_t* __restrict__ parent) {
    const uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= static_cast<uint64_t>(n) * kLanes) return;
    const uint32_t v = static_cast<uint32_t>(t / kLanes), j = static_cast<uint32_t>(t % kLanes);
    float x = 0.0f;
    if (j < K) {
        const uint32_t c = counts[v], m = mpts[j];
        x = c == 0 ? __int_as_float(0x7f800000) : dists[static_cast<uint64_t>(v) * k + (m < c ? m : c) - 1];
    }
    core[t] = x;
    parent[t] = v;
}

// ---- labels, numbered by each component's smallest node --------------------------------
// roots after the final flatten: parent[v][j] == v.  One warp per chunk of 32 nodes,
// lane j counts MST j's roots; the counts are scanned per MST; then lane j numbers its
// roots and every node takes its root's number (written MST-major through a shared
// transpose so the stores are coalesced).

__global__ void k_lab_count(const uint32_t* __restrict__ parent, uint32_t n, uint32_t K, uint32_t nchunks,
                            uint32_t* __restrict__ cc) {
    const uint32_t chunk = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned lane = threadIdx.x & 31u;
    if (chunk >= nchunks) return;
    uint32_t cnt = 0;
    for (uint32_t t = 0; t < 32; ++t) {
        const uint32_t v = chunk * 32 + t;
        if (v < n && lane < K && parent[static_cast<uint64_t>(v) * kLanes + lane] == v) ++cnt;
    }
    if (lane < K) cc[static_cast<uint64_t>(lane) * nchunks + chunk] = cnt;
}

__global__ void k_lab_roots(const uint32_t* __restrict__ parent, uint32_t n, uint32_t K, uint32_t nchunks,
                            const uint32_t* __restrict__ cc, uint32_t* __restrict__ rootlab) {
    const uint32_t chunk = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned lane = threadIdx.x & 31u;
    if (chunk >= nchunks || lane >= K) return;
    uint32_t next = cc[static_cast<uint64_t>(lane) * nchunks + chunk];
    for (uint32_t t = 0; t < 32; ++t) {
        const uint32_t v = chunk * 32 + t;
        if (v < n && parent[static_cast<uint64_t>(v) * kLanes + lane] == v) rootlab[static_cast<uint64_t>(v) * kLanes + lane] = next++;
    }
}

__global__ void k_lab_write(const uint32_t* __restrict__ parent, uint32_t n, uint32_t K, uint32_t nchunks,
                            const uint32_t* __restrict__ rootlab, uint32_t* __restrict__ lab) {
    __shared__ uint32_t tile[kThreads / 32][32][33];
    const uint32_t chunk = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    if (chunk >= nchunks) return;
    for (uint32_t t = 0; t < 32; ++t) {
        const uint32_t v = chunk * 32 + t;
        uint32_t x = 0;
        if (v < n && lane < K) x = rootlab[static_cast<uint64_t>(parent[static_cast<uint64_t>(v) * kLanes + lane]) * kLanes + lane];
        tile[w][t][lane] = x;  // [node][mst]
    }
    __syncwarp();
    const uint32_t v = chunk * 32 + lane;
    for (uint32_t j = 0; j < K; ++j) {
        if (v < n) lab[static_cast<uint64_t>(j) * n + v] = tile[w][lane][j];
    }
}

// ---- trees: bit-packed membership -> per-MST edge lists in ascending edge index ----------

/// tc[j][c] = edges of chunk c in MST j.  Lane j counts MST j: the warp walks only the
/// group's edges that are in some tree (a few of 32), each one broadcast.
__global__ void k_tree_count(const uint32_t* __restrict__ tree, uint32_t E, uint32_t K, uint32_t nchunks,
                             uint32_t* __restrict__ tc) {
    const uint32_t chunk = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned lane = threadIdx.x & 31u;
    if (chunk >= nchunks) return;
    uint32_t cnt = 0;
    for (uint32_t g = 0; g < kChunkEdges / 32; ++g) {
        const uint32_t i = chunk * kChunkEdges + g * 32 + lane;
        const uint32_t m = i < E ? tree[i] : 0u;
        unsigned nz = __ballot_sync(0xFFFFFFFFu, m != 0u);
        while (nz) {
            const int t = __ffs(nz) - 1;
            nz &= nz - 1;
            cnt += (__shfl_sync(0xFFFFFFFFu, m, t) >> lane) & 1u;
        }
    }
    if (lane < K) tc[static_cast<uint64_t>(lane) * nchunks + chunk] = cnt;
}

/// Per-MST edge lists: chunk c of MST j starts at tc[j][c]; edges in ascending index.
/// The MRD weight max(w, core_u, core_v) is taken from the sweep's core table (the
/// value k_core32 wrote, so the weight is the one the sweep ranked): each edge reads
/// the rows of its endpoints eight MSTs at a time (two 16-byte loads per row), all of
/// a group's loads before its ballots.
__global__ void k_tree_emit(const uint32_t* __restrict__ tree, uint32_t E, uint32_t K, uint32_t nchunks,
                            const uint32_t* __restrict__ tc, const uint32_t* __restrict__ eu,
                            const uint32_t* __restrict__ ev, const float* __restrict__ ew,
                            const float* __restrict__ core, uint64_t cap, cs_edge* __restrict__ out, int* status) {
    const uint32_t chunk = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned lane = threadIdx.x & 31u;
    if (chunk >= nchunks) return;
    uint32_t off = lane < K ? tc[static_cast<uint64_t>(lane) * nchunks + chunk] : 0u;
    for (uint32_t g = 0; g < kChunkEdges / 32; ++g) {
        const uint32_t i = chunk * kChunkEdges + g * 32 + lane;
        const uint32_t m = i < E ? tree[i] : 0u;
        uint32_t u = 0, v = 0;
        float w = 0.0f;
        if (m) {
            u = eu[i];
            v = ev[i];
            w = ew[i];
        }
        const float4* const ru = reinterpret_cast<const float4*>(core + static_cast<uint64_t>(u) * kLanes);
        const float4* const rv = reinterpret_cast<const float4*>(core + static_cast<uint64_t>(v) * kLanes);
        const unsigned any = __reduce_or_sync(0xFFFFFFFFu, m);  // MSTs some edge of the group is in
        for (uint32_t j0 = 0; j0 < K; j0 += 8) {
            if (!((any >> j0) & 0xFFu)) continue;  // warp-uniform
            const uint32_t mb = (m >> j0) & 0xFFu;
            float4 a0 = make_float4(0.f, 0.f, 0.f, 0.f), a1 = a0, b0 = a0, b1 = a0;
            if (mb) {
                a0 = __ldg(ru + j0 / 4);
                a1 = __ldg(ru + j0 / 4 + 1);
                b0 = __ldg(rv + j0 / 4);
                b1 = __ldg(rv + j0 / 4 + 1);
            }
            const float cu[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
            const float cv[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
            for (int x = 0; x < 8; ++x) {
                const uint32_t j = j0 + x;  // < 32; bits at and above K are never set
                if (!((any >> j) & 1u)) continue;  // warp-uniform: no lane has the bit
                const bool has = (mb >> x) & 1u;
                const unsigned b = __ballot_sync(0xFFFFFFFFu, has);
                if (!b) continue;
                const uint32_t base = __shfl_sync(0xFFFFFFFFu, off, j);
                if (has) {
                    const uint64_t pos = base + __popc(b & ((1u << lane) - 1u));
                    if (pos < cap) {
                        cs_edge e;
                        e.u = u;
                        e.v = v;
                        e.w = max_ref(w, max_ref(cu[x], cv[x]));
                        out[static_cast<uint64_t>(j) * cap + pos] = e;
                    } else {
                        atomicOr(status, kStatusCapacity);
                    }
                }
                if (lane == j) off += __popc(b);
            }
        }
    }
}

/// Exact weight bins of each tree (per-exponent mantissa sums), one MST per block row.
/// A warp's lanes of the same bin add their mantissas first (each < 2^24, so 32 of
/// them fit 32 bits) and one lane adds the sum to the block's bin.
__global__ void k_tree_weight(const cs_edge* __restrict__ out, uint64_t cap, const unsigned long long* __restrict__ nedges,
                              unsigned long long* __restrict__ bins) {
    __shared__ unsigned long long sb[256];
    const uint32_t j = blockIdx.y;
    const unsigned lane = threadIdx.x & 31u;
    for (int b = threadIdx.x; b < 256; b += blockDim.x) sb[b] = 0;
    __syncthreads();
    const uint64_t ne = nedges[j] < cap ? nedges[j] : cap;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    // whole warps step together, so the warp intrinsics see every lane of the warp
    for (uint64_t t0 = static_cast<uint64_t>(blockIdx.x) * blockDim.x + (threadIdx.x & ~31u); t0 < ne; t0 += stride) {
        const uint64_t t = t0 + lane;
        const bool ok = t < ne;
        uint32_t bin = 0, mant = 0;
        if (ok) {
            const uint32_t bits = __float_as_uint(out[static_cast<uint64_t>(j) * cap + t].w);
            const uint32_t e = (bits >> 23) & 0xFFu;
            bin = e ? e : 1u;
            mant = (bits & 0x7FFFFFu) | (e ? 0x800000u : 0u);
        }
        const unsigned act = __ballot_sync(0xFFFFFFFFu, ok);
        if (ok) {
            const unsigned grp = __match_any_sync(act, bin);
            const uint32_t sum = __reduce_add_sync(grp, mant);
            if (lane == static_cast<unsigned>(__ffs(grp) - 1)) atomicAdd(sb + bin, static_cast<unsigned long long>(sum));
        }
    }
    __syncthreads();
    for (int b = threadIdx.x; b < 256; b += blockDim.x) {
        if (sb[b]) atomicAdd(bins + static_cast<uint64_t>(j) * 256 + b, sb[b]);
    }
}

}  // namespace

// ============================================================================
// plans: buffers + the three captured graphs of one (graph, K<=32, shape)
// ============================================================================

struct SweepPlan {
    uint32_t n = 0, E = 0, e_knn = 0, K = 0, block = 0, grid = 0, flatten_div = 4;
    uint32_t tail_roots = 0, tail_cap = 0;  // contracted tail: trigger and table slots
    uint32_t tail_div = 0, tail_slots = 0;  // the graph's knobs they were made from
    bool labels = false;
    uint64_t limit_ns = 0, hold_ns = 0;  // grid-barrier limit and test hold captured in the graph
    uint32_t ncn = 0, nce = 0;  // node chunks, edge chunks
    DevBuf mpts, parent, best, tree, live, wl, rlist, fl, core, ctr, bar, status, cc, tcnt, rootlab, lab, out, counts, bins,
        trace, ttab, tl;
    cudaGraphExec_t exec_pre = nullptr, exec_main = nullptr, exec_post = nullptr;
    std::vector<uint32_t> host_mpts;
    const void* key_ptrs[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    cudaEvent_t ev_k0 = nullptr, ev_k1 = nullptr;
    cudaStream_t side = nullptr;                         // the labels' branch of the post graph
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    float last_graph_ms = 0.0f, last_kernel_ms = 0.0f;
    uint32_t last_rounds = 0;
    SweepPlan* next = nullptr;  // the following pass of a sweep with K > 32
    ~SweepPlan() {
        if (exec_pre) cudaGraphExecDestroy(exec_pre);
        if (exec_main) cudaGraphExecDestroy(exec_main);
        if (exec_post) cudaGraphExecDestroy(exec_post);
        if (ev_k0) cudaEventDestroy(ev_k0);
        if (ev_k1) cudaEventDestroy(ev_k1);
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_join) cudaEventDestroy(ev_join);
        if (side) cudaStreamDestroy(side);
        delete next;
    }
};

void sweep_free(SweepPlan* p) { delete p; }

namespace {

std::mutex g_tune_mu;

/// Sweeps on one device run one at a time, across contexts.  The persistent kernel
/// takes every SM, so a second sweep in flight gains nothing; interleaved, each
/// context's post-processing waited behind the other's whole kernel (two contexts'
/// steps finished together, after both sweeps).  Serialised, one context's copies
/// (its inputs going up, its trees coming down) overlap another context's sweep.
std::mutex& device_sweep_mutex(int device) {
    static std::mutex mus[64];
    return mus[static_cast<unsigned>(device) % 64u];
}
std::map<std::tuple<uint32_t, uint32_t, uint32_t, int>, std::pair<uint32_t, uint32_t>> g_tuned;  // -> (block, flatten_div)

SweepArgs args_of(Graph& g, SweepPlan& p) {
    SweepArgs a;
    a.n = p.n;
    a.E = p.E;
    a.e_knn = p.e_knn;
    a.K = p.K;
    a.k = g.k;
    a.flatten_div = p.flatten_div;
    a.eu = g.eu.as<uint32_t>();
    a.ev = g.ev.as<uint32_t>();
    a.ew = g.ew.as<float>();
    a.node_off = g.node_off.as<uint32_t>();
    a.dists = g.dists.as<float>();
    a.counts = g.counts.as<uint32_t>();
    a.mpts = p.mpts.as<uint32_t>();
    a.parent = p.parent.as<uint32_t>();
    a.best = p.best.as<unsigned long long>();
    a.tree = p.tree.as<uint32_t>();
    a.live = p.live.as<uint32_t>();
    a.wl = p.wl.as<uint4>();
    a.rlist = p.rlist.as<uint32_t>();
    a.fl = p.fl.as<uint32_t>();
    a.trace = p.trace.as<unsigned long long>();
    a.core = p.core.as<float>();
    a.ctr = p.ctr.as<uint32_t>();
    a.bar = p.bar.as<unsigned>();
    a.status = p.status.as<int>();
    a.limit_ns = p.limit_ns;
    a.hold_ns = p.hold_ns;
    a.tail_roots = p.tail_roots;
    a.tail_cap = p.tail_cap;
    a.ttab = p.ttab.as<ulonglong2>();
    a.tl = p.tl.as<ulonglong2>();
    return a;
}

/// pre: reset the per-sweep state.
void enqueue_pre(Graph& g, SweepPlan& p) {
    Ctx& c = *g.ctx;
    const uint64_t n = std::max<uint32_t>(p.n, 1), E = std::max<uint32_t>(p.E, 1);
    CSB_CUDA(cudaMemsetAsync(p.status.p, 0, 64, c.stream));
    CSB_CUDA(cudaMemsetAsync(p.bar.p, 0, 64, c.stream));
    CSB_CUDA(cudaMemsetAsync(p.ctr.p, 0, 64, c.stream));
    CSB_CUDA(cudaMemsetAsync(p.trace.p, 0, kMaxRounds * kTraceWords * 8, c.stream));
    CSB_CUDA(cudaMemsetAsync(p.best.p, 0xFF, n * kLanes * 8, c.stream));
    CSB_CUDA(cudaMemsetAsync(p.tree.p, 0, E * 4, c.stream));

    CSB_CUDA(cudaMemsetAsync(p.bins.p, 0, static_cast<uint64_t>(p.K) * 256 * 8, c.stream));
    k_core32<<<blocks_for(n * kLanes), kThreads, 0, c.stream>>>(g.dists.as<float>(), g.counts.as<uint32_t>(), g.k,
                                                                 p.mpts.as<uint32_t>(), p.K, p.n, p.core.as<float>(),
                                                                 p.parent.as<uint32_t>());
    count_launch(c);
}

void enqueue_main(Graph& g, SweepPlan& p) {
    Ctx& c = *g.ctx;
    SweepArgs a = args_of(g, p);
    void* params[] = {&a};
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(p.grid);
    cfg.blockDim = dim3(p.block);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = c.stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    CSB_CUDA(cudaLaunchKernelExC(&cfg, reinterpret_cast<const void*>(k_sweep), params));
    count_launch(c);
}

/// Swaps the context's stream for another until the scope ends.
struct StreamSwap {
    Ctx& c;
    cudaStream_t saved;
    StreamSwap(Ctx& ctx, cudaStream_t s) : c(ctx), saved(ctx.stream) { c.stream = s; }
    ~StreamSwap() { c.stream = saved; }
};

/// post: labels (optional), tree lists, exact weight bins.  The labels and the tree
/// lists read the same finished forest and write different outputs, so the labels run
/// on a side stream forked from the context stream and joined back at the end.
void enqueue_post(Graph& g, SweepPlan& p) {
    Ctx& c = *g.ctx;
    const unsigned wpb = kThreads / 32;
    unsigned long long* nedges = p.counts.as<unsigned long long>();
    unsigned long long* ncomp = nedges + 32;
    if (p.labels) {
        CSB_CUDA(cudaEventRecord(p.ev_fork, c.stream));
        CSB_CUDA(cudaStreamWaitEvent(p.side, p.ev_fork, 0));
        StreamSwap on_side(c, p.side);
        const unsigned gb = static_cast<unsigned>((p.ncn + wpb - 1) / wpb);
        k_lab_count<<<gb, kThreads, 0, c.stream>>>(p.parent.as<uint32_t>(), p.n, p.K, p.ncn, p.cc.as<uint32_t>());
        count_launch(c);
        launch_scan_tiles(c, p.cc.as<uint32_t>(), p.ncn, p.K, ncomp);
        k_lab_roots<<<gb, kThreads, 0, c.stream>>>(p.parent.as<uint32_t>(), p.n, p.K, p.ncn, p.cc.as<uint32_t>(),
                                                  p.rootlab.as<uint32_t>());
        k_lab_write<<<gb, kThreads, 0, c.stream>>>(p.parent.as<uint32_t>(), p.n, p.K, p.ncn, p.rootlab.as<uint32_t>(),
                                                  p.lab.as<uint32_t>());
        count_launch(c, 2);
        CSB_CUDA(cudaEventRecord(p.ev_join, c.stream));
    }
    const unsigned ge = static_cast<unsigned>((p.nce + wpb - 1) / wpb);
    k_tree_count<<<ge, kThreads, 0, c.stream>>>(p.tree.as<uint32_t>(), p.E, p.K, p.nce, p.tcnt.as<uint32_t>());
    count_launch(c);
    launch_scan_tiles(c, p.tcnt.as<uint32_t>(), p.nce, p.K, nedges);
    const uint64_t cap = p.n ? p.n - 1 : 0;
    k_tree_emit<<<ge, kThreads, 0, c.stream>>>(p.tree.as<uint32_t>(), p.E, p.K, p.nce, p.tcnt.as<uint32_t>(),
                                              g.eu.as<uint32_t>(), g.ev.as<uint32_t>(), g.ew.as<float>(),
                                              p.core.as<float>(), cap, p.out.as<cs_edge>(), p.status.as<int>());
    dim3 gw(std::max<unsigned>(1, std::min<unsigned>(64, blocks_for(cap))), p.K);
    k_tree_weight<<<gw, kThreads, 0, c.stream>>>(p.out.as<cs_edge>(), cap, nedges, p.bins.as<unsigned long long>());
    count_launch(c, 2);
    if (p.labels) CSB_CUDA(cudaStreamWaitEvent(c.stream, p.ev_join, 0));
}

using Enqueue = void (*)(Graph&, SweepPlan&);

bool capture_part(Graph& g, SweepPlan& p, Enqueue f, cudaGraphExec_t* out) {
    Ctx& c = *g.ctx;
    *out = nullptr;
    if (cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    const uint64_t before = c.launches;
    bool ok = true;
    try {
        f(g, p);
    } catch (...) {
        ok = false;
    }
    c.launches = before;  // counted when replayed
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(c.stream, &graph);
    ok = ok && e == cudaSuccess && graph;
    if (ok) ok = cudaGraphInstantiate(out, graph, 0) == cudaSuccess;
    if (graph) cudaGraphDestroy(graph);
    if (!ok) {
        cudaGetLastError();
        *out = nullptr;
    }
    return ok;
}

uint64_t kernels_pre() { return 1; }
uint64_t kernels_post(const SweepPlan& p) { return (p.labels ? 4 : 0) + 4; }

/// A plan for the graph's current shape.  `reuse` (a plan that no longer matches)
/// gives its buffers, which only grow, so a graph that grows by inserts recaptures
/// its graphs without reallocating every buffer; it is consumed either way.
SweepPlan* make_plan(Graph& g, uint32_t K, uint32_t block, uint32_t flatten_div, bool labels, SweepPlan* reuse) {
    Ctx& c = *g.ctx;
    SweepPlan* p = reuse ? reuse : new SweepPlan();
    if (reuse) {
        if (p->exec_pre) cudaGraphExecDestroy(p->exec_pre);
        if (p->exec_main) cudaGraphExecDestroy(p->exec_main);
        if (p->exec_post) cudaGraphExecDestroy(p->exec_post);
        if (p->ev_k0) cudaEventDestroy(p->ev_k0);
        if (p->ev_k1) cudaEventDestroy(p->ev_k1);
        if (p->ev_fork) cudaEventDestroy(p->ev_fork);
        if (p->ev_join) cudaEventDestroy(p->ev_join);
        p->exec_pre = p->exec_main = p->exec_post = nullptr;
        p->ev_k0 = p->ev_k1 = p->ev_fork = p->ev_join = nullptr;
        delete p->next;
        p->next = nullptr;
    }
    try {
        p->n = static_cast<uint32_t>(g.n);
        p->E = static_cast<uint32_t>(g.e_total);
        p->e_knn = static_cast<uint32_t>(g.e_knn);
        p->K = K;
        p->block = block;
        p->flatten_div = flatten_div;
        p->labels = labels;
        p->limit_ns = g.sweep_barrier_ns ? g.sweep_barrier_ns : kBarrierLimitNs;
        p->hold_ns = g.sweep_hold_ns;
        p->key_ptrs[0] = g.eu.p;
        p->key_ptrs[1] = g.ev.p;
        p->key_ptrs[2] = g.ew.p;
        p->key_ptrs[3] = g.dists.p;
        p->key_ptrs[4] = g.counts.p;
        p->key_ptrs[5] = g.node_off.p;
        const uint64_t n = std::max<uint32_t>(p->n, 1), E = std::max<uint32_t>(p->E, 1);
        p->ncn = static_cast<uint32_t>((n + 31) / 32);
        p->nce = static_cast<uint32_t>((E + kChunkEdges - 1) / kChunkEdges);
        // buffers sized for the graph's capacity (grown inserts reuse them)
        const uint64_t nc = std::max<uint64_t>(scratch_nodes(g), n), Ec = std::max<uint64_t>(scratch_scale(g, E), E);
        p->mpts.ensure(32 * 4);
        p->parent.ensure(nc * kLanes * 4);
        p->best.ensure(nc * kLanes * 8);
        p->tree.ensure(Ec * 4);
        p->live.ensure(2 * Ec * 4);
        p->wl.ensure(2 * Ec * 16);
        p->rlist.ensure(2 * nc * 4);
        p->fl.ensure(nc * 4);
        p->core.ensure(nc * kLanes * 4);
        p->ctr.ensure(64);
        p->trace.ensure(kMaxRounds * kTraceWords * 8);
        p->bar.ensure(64);
        p->status.ensure(64);
        // the contracted tail: a table of min(4 n, |E|) slots rounded up to a power of
        // two, at least 2^10 and at most 2^26 (1 GB; the table round holds about 1.6
        // entries per node, so up to ~20M nodes the table stays under half full, and a
        // fuller one overflows and the sweep keeps its worklist), and two entry lists as
        // long; graphs of 2^27 nodes or more keep the edge worklist to the end
        p->tail_div = g.sweep_tail_div;
        p->tail_slots = g.sweep_tail_slots;
        const uint32_t tdiv = g.sweep_tail_div == 0xFFFFFFFFu ? kTailDiv : g.sweep_tail_div;
        const uint32_t tmax = g.sweep_tail_slots ? g.sweep_tail_slots : (1u << 26);
        p->tail_cap = 1024;
        while (p->tail_cap < std::min<uint64_t>(4 * nc, Ec) && p->tail_cap < tmax) p->tail_cap <<= 1;
        p->tail_roots = (tdiv != 0 && nc < (1ull << kTailNodeBits)) ? static_cast<uint32_t>(n / tdiv) : 0u;
        p->ttab.ensure(static_cast<uint64_t>(p->tail_cap) * 16);
        p->tl.ensure(2ull * p->tail_cap * 16);
        p->cc.ensure(static_cast<uint64_t>(K) * p->ncn * 4 + 64);
        p->tcnt.ensure(static_cast<uint64_t>(K) * p->nce * 4 + 64);
        if (labels) {
            p->rootlab.ensure(nc * kLanes * 4);
            p->lab.ensure(static_cast<uint64_t>(K) * nc * 4);
        }
        p->out.ensure(static_cast<uint64_t>(K) * std::max<uint64_t>(nc - 1, 1) * sizeof(cs_edge));
        p->counts.ensure(64 * 8);
        p->bins.ensure(static_cast<uint64_t>(K) * 256 * 8);
        CSB_CUDA(cudaEventCreate(&p->ev_k0));
        CSB_CUDA(cudaEventCreate(&p->ev_k1));
        if (!p->side) CSB_CUDA(cudaStreamCreateWithFlags(&p->side, cudaStreamNonBlocking));
        CSB_CUDA(cudaEventCreateWithFlags(&p->ev_fork, cudaEventDisableTiming));
        CSB_CUDA(cudaEventCreateWithFlags(&p->ev_join, cudaEventDisableTiming));
        int occ = 0;
        CSB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_sweep, static_cast<int>(block), 0));
        if (occ < 1) fail(CS_ERR_UNSUPPORTED, "sweep kernel does not fit on an SM");
        p->grid = static_cast<uint32_t>(c.sm_count) * static_cast<uint32_t>(occ);
        capture_part(g, *p, enqueue_pre, &p->exec_pre);
        capture_part(g, *p, enqueue_main, &p->exec_main);
        capture_part(g, *p, enqueue_post, &p->exec_post);
    } catch (...) {
        delete p;
        throw;
    }
    return p;
}

void status_check(Ctx& c, const int* d_status) {
    int st = 0;
    CSB_CUDA(cudaMemcpyAsync(&st, d_status, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    CSB_CUDA(cudaStreamSynchronize(c.stream));
    if (st & kStatusBarrierTimeout) fail(CS_ERR_TIMEOUT, "MST sweep: a grid barrier wait ran out");
    if (st & kStatusUnionLimit) fail(CS_ERR_TIMEOUT, "MST sweep: a union retry loop ran out");
    if (st & kStatusRoundLimit) fail(CS_ERR_TIMEOUT, "MST sweep: Boruvka round limit reached");
    if (st & kStatusCapacity) fail(CS_ERR_STATE, "MST sweep: tree larger than n-1 edges (inconsistent state)");
}

/// Run one pass (K <= 32): replay pre / main / post with events around main.
void run_pass(Graph& g, SweepPlan& p) {
    Ctx& c = *g.ctx;
    CSB_CUDA(cudaMemcpyAsync(p.mpts.p, p.host_mpts.data(), p.K * 4, cudaMemcpyHostToDevice, c.stream));
    if (p.exec_pre) {
        CSB_CUDA(cudaGraphLaunch(p.exec_pre, c.stream));
        count_launch(c, kernels_pre());
    } else {
        enqueue_pre(g, p);
    }
    CSB_CUDA(cudaEventRecord(p.ev_k0, c.stream));
    if (p.exec_main) {
        CSB_CUDA(cudaGraphLaunch(p.exec_main, c.stream));
        count_launch(c, 1);
    } else {
        enqueue_main(g, p);
    }
    CSB_CUDA(cudaEventRecord(p.ev_k1, c.stream));
    if (p.exec_post) {
        CSB_CUDA(cudaGraphLaunch(p.exec_post, c.stream));
        count_launch(c, kernels_post(p));
    } else {
        enqueue_post(g, p);
    }
}

bool plan_matches(const SweepPlan* p, const Graph& g, uint32_t K, uint32_t block, uint32_t fdiv, bool labels) {
    return p && p->n == g.n && p->E == g.e_total && p->e_knn == g.e_knn && p->K == K && p->block == block &&
           p->flatten_div == fdiv && p->labels == labels &&
           p->limit_ns == (g.sweep_barrier_ns ? g.sweep_barrier_ns : kBarrierLimitNs) && p->hold_ns == g.sweep_hold_ns &&
           p->tail_div == g.sweep_tail_div && p->tail_slots == g.sweep_tail_slots &&
           p->key_ptrs[0] == g.eu.p && p->key_ptrs[1] == g.ev.p &&
           p->key_ptrs[2] == g.ew.p && p->key_ptrs[3] == g.dists.p && p->key_ptrs[4] == g.counts.p &&
           p->key_ptrs[5] == g.node_off.p;
}

}  // namespace

void sweep_run(Graph& g, const uint32_t* mpts, uint32_t K, bool want_labels, float* out_ms) {
    if (K == 0) fail(CS_ERR_INVALID, "sweep: K must be positive");
    for (uint32_t j = 0; j < K; ++j) {
        if (mpts[j] > g.k) fail(CS_ERR_INVALID, "sweep: mpts exceeds k_max");
    }
    if (g.n == 0) fail(CS_ERR_STATE, "sweep: empty graph");
    Ctx& c = *g.ctx;
    std::unique_lock<std::mutex> device_lock(device_sweep_mutex(c.device));
    graph_build_edges(g);
    uint32_t B = g.sweep_block, F = g.sweep_flatten;
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tuned.find(std::make_tuple(static_cast<uint32_t>(g.n), static_cast<uint32_t>(g.e_total), K, c.sm_count));
        if (it != g_tuned.end()) {
            if (!B) B = it->second.first;
            if (F == kFlattenAuto) F = it->second.second;
        }
    }
    if (!B) B = 512;
    if (F == kFlattenAuto) F = 0;  // the frozen root list alone was fastest at n = 1M
    // passes of at most 32 MSTs, chained plans
    SweepPlan** slot = &g.plan;
    for (uint32_t off = 0; off < K; off += kLanes) {
        const uint32_t Kp = std::min<uint32_t>(kLanes, K - off);
        if (!plan_matches(*slot, g, Kp, B, F, want_labels)) {
            SweepPlan* old = *slot;
            SweepPlan* nxt = old ? old->next : nullptr;
            if (old) old->next = nullptr;
            *slot = nxt;  // keeps the chain owned if the plan cannot be made
            SweepPlan* np = make_plan(g, Kp, B, F, want_labels, old);
            np->next = nxt;
            *slot = np;
        }
        (*slot)->host_mpts.assign(mpts + off, mpts + off + Kp);
        for (auto& m : (*slot)->host_mpts) {
            if (m == 0) m = 1;  // CoreSG::edges treats mpts 0 as 1
        }
        slot = &(*slot)->next;
    }
    // drop plans of passes this sweep does not use
    sweep_free(*slot);
    *slot = nullptr;
    g.sweep_K = K;
    cudaEvent_t e0, e1;
    CSB_CUDA(cudaEventCreate(&e0));
    CSB_CUDA(cudaEventCreate(&e1));
    CSB_CUDA(cudaEventRecord(e0, c.stream));
    for (SweepPlan* p = g.plan; p; p = p->next) run_pass(g, *p);
    CSB_CUDA(cudaEventRecord(e1, c.stream));
    CSB_CUDA(cudaEventSynchronize(e1));
    // the device's turn ends with the last kernel: the status and round counts below are
    // small reads that can wait behind other contexts' copies
    device_lock.unlock();
    float ms = 0.0f;
    CSB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    float kms = 0.0f;
    for (SweepPlan* p = g.plan; p; p = p->next) {
        float x = 0.0f;
        CSB_CUDA(cudaEventElapsedTime(&x, p->ev_k0, p->ev_k1));
        kms += x;
        status_check(c, p->status.as<int>());
        uint32_t rounds = 0;
        CSB_CUDA(cudaMemcpyAsync(&rounds, p->ctr.as<uint32_t>() + 4, 4, cudaMemcpyDeviceToHost, c.stream));
        CSB_CUDA(cudaStreamSynchronize(c.stream));
        p->last_rounds = rounds;
    }
    g.plan->last_graph_ms = ms;
    g.plan->last_kernel_ms = kms;
    if (out_ms) *out_ms = ms;
}

void sweep_fetch(Graph& g, uint32_t index, cs_edge* out_edges, uint32_t* out_labels, MstHost* res,
                 bool device_out) {
    if (!g.plan) fail(CS_ERR_STATE, "sweep_fetch: no sweep has run");
    if (index >= g.sweep_K) fail(CS_ERR_INVALID, "sweep_fetch: index out of range");
    SweepPlan* p = g.plan;
    uint32_t j = index;
    while (j >= p->K) {
        j -= p->K;
        p = p->next;
    }
    if (out_labels && !p->labels) fail(CS_ERR_STATE, "sweep_fetch: the sweep ran without labels");
    Ctx& c = *g.ctx;
    unsigned long long ne = 0;
    uint64_t bins[256];
    CSB_CUDA(cudaMemcpyAsync(&ne, p->counts.as<unsigned long long>() + j, 8, cudaMemcpyDeviceToHost, c.stream));
    CSB_CUDA(cudaMemcpyAsync(bins, p->bins.as<unsigned long long>() + static_cast<uint64_t>(j) * 256, sizeof(bins),
                             cudaMemcpyDeviceToHost, c.stream));
    CSB_CUDA(cudaStreamSynchronize(c.stream));
    const uint64_t cap = p->n ? p->n - 1 : 0;
    if (ne > cap) fail(CS_ERR_STATE, "sweep_fetch: the last sweep did not complete");
    res->nedges = ne;
    res->ncomp = static_cast<uint32_t>(p->n - ne);
    res->weight = exact_sum_from_bins(bins);
    const cs_edge* src_e = p->out.as<cs_edge>() + j * cap;
    const uint32_t* src_l = p->labels ? p->lab.as<uint32_t>() + static_cast<uint64_t>(j) * p->n : nullptr;
    if (device_out) {
        // the caller's device buffers on this device, copied on the context stream
        if (out_edges && ne)
            CSB_CUDA(cudaMemcpyAsync(out_edges, src_e, ne * sizeof(cs_edge), cudaMemcpyDeviceToDevice, c.stream));
        if (out_labels && p->n)
            CSB_CUDA(cudaMemcpyAsync(out_labels, src_l, static_cast<uint64_t>(p->n) * 4, cudaMemcpyDeviceToDevice,
                                     c.stream));
        CSB_CUDA(cudaStreamSynchronize(c.stream));
        return;
    }
    if (out_edges && ne) copy_d2h(c, out_edges, src_e, ne * sizeof(cs_edge));
    if (out_labels && p->n) copy_d2h(c, out_labels, src_l, static_cast<uint64_t>(p->n) * 4);
}

SweepOut sweep_outputs(Graph& g, uint32_t index) {
    if (!g.plan) fail(CS_ERR_STATE, "sweep: no sweep has run");
    if (index >= g.sweep_K) fail(CS_ERR_INVALID, "sweep: index out of range");
    SweepPlan* p = g.plan;
    uint32_t j = index;
    while (j >= p->K) {
        j -= p->K;
        p = p->next;
    }
    SweepOut o;
    o.n = p->n;
    o.cap = p->n ? p->n - 1 : 0;
    o.edges = p->out.as<cs_edge>() + j * o.cap;
    o.labels = p->labels ? p->lab.as<uint32_t>() + static_cast<uint64_t>(j) * p->n : nullptr;
    o.count = p->counts.as<unsigned long long>() + j;
    o.bins = p->bins.as<unsigned long long>() + static_cast<uint64_t>(j) * 256;
    return o;
}

}  // namespace csb

// ============================================================================
// C API
// ============================================================================

using namespace csb;

extern "C" {

cs_status cs_extract_sweep(cs_graph* gp, const uint32_t* mpts, uint32_t K, cs_edge* out_edges,
                           uint32_t* out_labels, uint64_t* out_nedges, uint32_t* out_ncomp,
                           double* out_weight) {
    Graph* g = reinterpret_cast<Graph*>(gp);
    return guarded(g ? g->ctx : nullptr, [&] {
        CSB_REQUIRE(mpts != nullptr, "cs_extract_sweep: null mpts");
        sweep_run(*g, mpts, K, out_labels != nullptr, nullptr);
        Ctx& c = *g->ctx;
        const uint64_t cap = g->n ? g->n - 1 : 0;
        // per pass: every tree's edge count and weight bins in one read; then each tree
        // with its labels, waited for before the next (a deeper queue of copies on the
        // context stream made other contexts' small reads, taken while they hold the
        // device's sweep turn, wait behind hundreds of MB)
        uint32_t base = 0;
        for (SweepPlan* p = g->plan; p; base += p->K, p = p->next) {
            std::vector<unsigned long long> cnt(p->K);
            std::vector<uint64_t> bins(static_cast<size_t>(p->K) * 256);
            CSB_CUDA(cudaMemcpyAsync(cnt.data(), p->counts.p, p->K * 8ull, cudaMemcpyDeviceToHost, c.stream));
            CSB_CUDA(cudaMemcpyAsync(bins.data(), p->bins.p, bins.size() * 8, cudaMemcpyDeviceToHost, c.stream));
            CSB_CUDA(cudaStreamSynchronize(c.stream));
            for (uint32_t jj = 0; jj < p->K; ++jj) {
                const uint32_t j = base + jj;
                const uint64_t ne = cnt[jj];
                if (ne > cap) fail(CS_ERR_STATE, "cs_extract_sweep: the sweep did not complete");
                if (out_nedges) out_nedges[j] = ne;
                if (out_ncomp) out_ncomp[j] = static_cast<uint32_t>(p->n - ne);
                if (out_weight) out_weight[j] = exact_sum_from_bins(bins.data() + static_cast<size_t>(jj) * 256);
                bool pending = false;
                if (out_edges && ne)
                    pending |= copy_d2h_enqueue(c, out_edges + j * cap, p->out.as<cs_edge>() + jj * cap,
                                                ne * sizeof(cs_edge));
                if (out_labels && p->n)
                    pending |= copy_d2h_enqueue(c, out_labels + static_cast<uint64_t>(j) * p->n,
                                                p->lab.as<uint32_t>() + static_cast<uint64_t>(jj) * p->n,
                                                static_cast<uint64_t>(p->n) * 4);
                if (pending) CSB_CUDA(cudaStreamSynchronize(c.stream));
            }
        }
    });
}

cs_status cs_extract_sweep_device(cs_graph* gp, const uint32_t* mpts, uint32_t K, float* out_ms) {
    Graph* g = reinterpret_cast<Graph*>(gp);
    return guarded(g ? g->ctx : nullptr, [&] {
        CSB_REQUIRE(mpts != nullptr, "cs_extract_sweep_device: null mpts");
        sweep_run(*g, mpts, K, true, out_ms);
    });
}

cs_status cs_sweep_fetch(cs_graph* gp, uint32_t index, cs_edge* out_edges, uint32_t* out_labels,
                         uint64_t* out_nedges, uint32_t* out_ncomp, double* out_weight) {
    Graph* g = reinterpret_cast<Graph*>(gp);
    return guarded(g ? g->ctx : nullptr, [&] {
        MstHost r;
        sweep_fetch(*g, index, out_edges, out_labels, &r, false);
        if (out_nedges) *out_nedges = r.nedges;
        if (out_ncomp) *out_ncomp = r.ncomp;
        if (out_weight) *out_weight = r.weight;
    });
}

cs_status cs_sweep_fetch_device(cs_graph* gp, uint32_t index, cs_edge* d_out_edges, uint32_t* d_out_labels,
                                uint64_t* out_nedges, uint32_t* out_ncomp, double* out_weight) {
    Graph* g = reinterpret_cast<Graph*>(gp);
    return guarded(g ? g->ctx : nullptr, [&] {
        MstHost r;
        sweep_fetch(*g, index, d_out_edges, d_out_labels, &r, true);
        if (out_nedges) *out_nedges = r.nedges;
        if (out_ncomp) *out_ncomp = r.ncomp;
        if (out_weight) *out_weight = r.weight;
    });
}

cs_status cs_sweep_trace(cs_graph* gp, uint64_t* out, uint32_t cap_rounds, uint32_t* out_rounds) {
    Graph* g = reinterpret_cast<Graph*>(gp);
    return guarded(g ? g->ctx : nullptr, [&] {
        if (!g->plan) fail(CS_ERR_STATE, "cs_sweep_trace: no sweep has run");
        SweepPlan& p = *g->plan;
        const uint32_t rounds = std::min<uint32_t>(p.last_rounds, kMaxRounds);
        std::vector<unsigned long long> t(static_cast<size_t>(kMaxRounds) * kTraceWords);
        copy_d2h(*g->ctx, t.data(), p.trace.p, t.size() * 8);
        for (uint32_t r = 0; r < rounds && r < cap_rounds && out; ++r) {
            const unsigned long long* x = t.data() + static_cast<size_t>(r) * kTraceWords;
            uint64_t* o = out + static_cast<size_t>(r) * 7;
            const bool last = r + 1 == rounds;
            o[0] = x[1] > x[0] ? x[1] - x[0] : 0;                      // phase A
            o[1] = (!last && x[2] > x[1]) ? x[2] - x[1] : 0;           // phase B
            o[2] = (!last && x[3] > x[2]) ? x[3] - x[2] : 0;           // flatten
            o[3] = x[4];
            o[4] = x[5];
            o[5] = last ? (x[7] & ~1ull) : x[7];
            o[6] = x[6];
        }
        if (out_rounds) *out_rounds = rounds;
    });
}

cs_status cs_sweep_timing(cs_graph* gp, float* graph_ms, float* kernel_ms) {
    Graph* g = reinterpret_cast<Graph*>(gp);
    return guarded(g ? g->ctx : nullptr, [&] {
        if (!g->plan) fail(CS_ERR_STATE, "cs_sweep_timing: no sweep has run");
        if (graph_ms) *graph_ms = g->plan->last_graph_ms;
        if (kernel_ms) *kernel_ms = g->plan->last_kernel_ms;
    });
}

cs_status cs_set_sweep_shape(cs_graph* gp, uint32_t flatten_div, uint32_t block_threads) {
    Graph* g = reinterpret_cast<Graph*>(gp);
    return guarded(g ? g->ctx : nullptr, [&] {
        CSB_REQUIRE(block_threads == 0 || block_threads == 128 || block_threads == 256 || block_threads == 512,
                    "cs_set_sweep_shape: block must be 128, 256 or 512");
        g->sweep_block = block_threads;
        g->sweep_flatten = flatten_div == 0 ? kFlattenAuto : (flatten_div == 0xFFFFFFFFu ? 0 : flatten_div);
    });
}

cs_status cs_set_sweep_tail(cs_graph* gp, uint32_t tail_div, uint32_t table_slots) {
    Graph* g = reinterpret_cast<Graph*>(gp);
    return guarded(g ? g->ctx : nullptr, [&] {
        CSB_REQUIRE(table_slots == 0 || (table_slots >= 1024 && table_slots <= (1u << 26) &&
                                         (table_slots & (table_slots - 1)) == 0),
                    "cs_set_sweep_tail: table_slots must be 0 or a power of two in [2^10, 2^26]");
        g->sweep_tail_div = tail_div;
        g->sweep_tail_slots = table_slots;
    });
}

cs_status cs_test_sweep_barrier(cs_graph* gp, uint64_t limit_ns, uint64_t hold_ns) {
    Graph* g = reinterpret_cast<Graph*>(gp);
    return guarded(g ? g->ctx : nullptr, [&] {
        CSB_REQUIRE(hold_ns <= 5000000000ull, "cs_test_sweep_barrier: hold above 5 s");
        g->sweep_barrier_ns = limit_ns;
        g->sweep_hold_ns = hold_ns;
    });
}

cs_status cs_autotune_sweep(cs_graph* gp, const uint32_t* mpts, uint32_t K, uint32_t* out_flatten,
                            uint32_t* out_block) {
    Graph* g = reinterpret_cast<Graph*>(gp);
    return guarded(g ? g->ctx : nullptr, [&] {
        CSB_REQUIRE(mpts != nullptr && K > 0, "cs_autotune_sweep: empty mpts");
        const uint32_t saved_b = g->sweep_block, saved_f = g->sweep_flatten;
        float best_ms = 1e30f;
        uint32_t best_b = 512, best_f = 0;
        const uint32_t blocks[] = {256, 512};
        const uint32_t flats[] = {0, 1, 2, 4, 16};
        for (uint32_t B : blocks) {
            for (uint32_t F : flats) {
                g->sweep_block = B;
                g->sweep_flatten = F;
                float ms = 0.0f, tot = 0.0f;
                sweep_run(*g, mpts, K, true, &ms);  // plan + warm
                for (int rep = 0; rep < 2; ++rep) {
                    sweep_run(*g, mpts, K, true, &ms);
                    tot += ms;
                }
                if (tot < best_ms) {
                    best_ms = tot;
                    best_b = B;
                    best_f = F;
                }
            }
        }
        g->sweep_block = saved_b;
        g->sweep_flatten = saved_f;
        {
            std::lock_guard<std::mutex> lk(g_tune_mu);
            g_tuned[std::make_tuple(static_cast<uint32_t>(g->n), static_cast<uint32_t>(g->e_total), K, g->ctx->sm_count)] =
                std::make_pair(best_b, best_f);
        }
        if (out_flatten) *out_flatten = best_f;
        if (out_block) *out_block = best_b;
    });
}

}  // extern "C"
