// Device helpers shared by the engine's kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace csb {

constexpr uint32_t kInvalid = 0xFFFFFFFFu;
constexpr uint64_t kNoKey = 0xFFFFFFFFFFFFFFFFull;
constexpr int kMaxK = 64;

// Device status word bits (Ctx::status).  A bounded wait that runs out sets one and
// the kernel returns; the host turns it into CS_ERR_TIMEOUT.
constexpr int kStatusBarrierTimeout = 1;
constexpr int kStatusUnionLimit = 2;
constexpr int kStatusRoundLimit = 4;
constexpr int kStatusCapacity = 8;

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }

/// Squared L2 in the association order of the reference's l2sqr_avx2
/// (include/coresg/distance.hpp:191-211): lane l of acc0 takes element i+l of every
/// 16-wide block and of the 8-wide tail block, lane l of acc1 element i+8+l of every
/// 16-wide block, one fused multiply-add each; then hsum256(acc0+acc1)
/// (:180-189) = ((v0+v4)+(v1+v5)) + ((v2+v6)+(v3+v7)).  Rows are padded to a
/// multiple of 8 floats, so no scalar tail exists.  Explicit _rn intrinsics keep
/// the compiler from contracting or reassociating.
__device__ __forceinline__ float l2sqr_ref(const float* __restrict__ a, const float* __restrict__ b,
                                           uint32_t stride) {
    float acc0[8], acc1[8];
#pragma unroll
    for (int l = 0; l < 8; ++l) {
        acc0[l] = 0.0f;
        acc1[l] = 0.0f;
    }
    uint32_t i = 0;
    for (; i + 16 <= stride; i += 16) {
        const float4* pa = reinterpret_cast<const float4*>(a + i);
        const float4* pb = reinterpret_cast<const float4*>(b + i);
        float x[16], y[16];
        *reinterpret_cast<float4*>(x + 0) = pa[0];
        *reinterpret_cast<float4*>(x + 4) = pa[1];
        *reinterpret_cast<float4*>(x + 8) = pa[2];
        *reinterpret_cast<float4*>(x + 12) = pa[3];
        *reinterpret_cast<float4*>(y + 0) = pb[0];
        *reinterpret_cast<float4*>(y + 4) = pb[1];
        *reinterpret_cast<float4*>(y + 8) = pb[2];
        *reinterpret_cast<float4*>(y + 12) = pb[3];
#pragma unroll
        for (int l = 0; l < 8; ++l) {
            const float d0 = __fsub_rn(x[l], y[l]);
            const float d1 = __fsub_rn(x[8 + l], y[8 + l]);
            acc0[l] = __fmaf_rn(d0, d0, acc0[l]);
            acc1[l] = __fmaf_rn(d1, d1, acc1[l]);
        }
    }
    if (i + 8 <= stride) {
        const float4* pa = reinterpret_cast<const float4*>(a + i);
        const float4* pb = reinterpret_cast<const float4*>(b + i);
        float x[8], y[8];
        *reinterpret_cast<float4*>(x + 0) = pa[0];
        *reinterpret_cast<float4*>(x + 4) = pa[1];
        *reinterpret_cast<float4*>(y + 0) = pb[0];
        *reinterpret_cast<float4*>(y + 4) = pb[1];
#pragma unroll
        for (int l = 0; l < 8; ++l) {
            const float d0 = __fsub_rn(x[l], y[l]);
            acc0[l] = __fmaf_rn(d0, d0, acc0[l]);
        }
    }
    float v[8];
#pragma unroll
    for (int l = 0; l < 8; ++l) v[l] = __fadd_rn(acc0[l], acc1[l]);
    const float lo0 = __fadd_rn(v[0], v[4]);
    const float lo1 = __fadd_rn(v[1], v[5]);
    const float lo2 = __fadd_rn(v[2], v[6]);
    const float lo3 = __fadd_rn(v[3], v[7]);
    return __fadd_rn(__fadd_rn(lo0, lo1), __fadd_rn(lo2, lo3));
}

/// MetricOp::finalize (include/coresg/distance.hpp:259-276): IEEE sqrt for L2,
/// half the squared distance for cosine on normalised rows.
__device__ __forceinline__ float finalize_rank(float r, int metric) {
    return metric == 1 ? __fmul_rn(0.5f, r) : __fsqrt_rn(r);
}
/// MetricOp::to_rank.
__device__ __forceinline__ float to_rank(float v, int metric) {
    return metric == 1 ? __fmul_rn(2.0f, v) : __fmul_rn(v, v);
}

/// std::max(a, b) == (a < b) ? b : a  (the reference's reweighting uses std::max).
__device__ __forceinline__ float max_ref(float a, float b) { return (a < b) ? b : a; }

/// pack_edge (src/mst.cpp:19-24): weight bits << 32 | edge index, so an integer
/// minimum is the (weight, index) minimum for non-negative weights.
__device__ __forceinline__ uint64_t pack_key(float w, uint32_t idx) {
    uint32_t b = __float_as_uint(w);
    if (w < 0.0f) b = ~b;
    return (static_cast<uint64_t>(b) << 32) | idx;
}

/// Core distance (KnnGraph::core_dist, include/coresg/knn_graph.hpp:157-163).
__device__ __forceinline__ float core_of(const float* dists, const uint32_t* counts, uint32_t k,
                                         uint32_t v, uint32_t mpts) {
    const uint32_t c = counts[v];
    if (c == 0) return __int_as_float(0x7f800000);
    uint32_t pos = mpts == 0 ? 0 : mpts - 1;
    if (pos >= c) pos = c - 1;
    return dists[static_cast<uint64_t>(v) * k + pos];
}

// ---- union-find over a device parent array -------------------------------------
// Roots are linked larger-under-smaller, so a root is always the smallest node of
// its set (the same rule as the reference's AtomicUnionFind,
// src/connectivity.cpp:20-61).  Path halving writes only non-root entries, unions
// write only roots (by CAS), so concurrent finds and unions are safe.

/// A set of n nodes has no chain longer than n: a chase that takes more steps (a
/// cycle, which the linking rule rules out) stops and sets kStatusUnionLimit in
/// `status` (when given) instead of spinning.
__device__ __forceinline__ uint32_t uf_find(uint32_t* parent, uint32_t x, uint32_t n, int* status) {
    for (uint32_t it = 0; it <= n; ++it) {
        const uint32_t p = __ldcg(parent + x);
        if (p == x) return x;
        const uint32_t gp = __ldcg(parent + p);
        if (gp == p) return p;
        parent[x] = gp;  // halving; benign race
        x = gp;
    }
    if (status) atomicOr(status, kStatusUnionLimit);
    return x;
}

/// Unite the sets of a and b.  Returns true when this call linked two roots.
/// The CAS retry loop is bounded; running out sets kStatusUnionLimit.
__device__ __forceinline__ bool uf_unite(uint32_t* parent, uint32_t a, uint32_t b, uint32_t n, int* status) {
    for (int it = 0; it < (1 << 20); ++it) {
        a = uf_find(parent, a, n, status);
        b = uf_find(parent, b, n, status);
        if (a == b) return false;
        if (a > b) {
            const uint32_t t = a;
            a = b;
            b = t;
        }
        if (atomicCAS(parent + b, b, a) == b) return true;
    }
    atomicOr(status, kStatusUnionLimit);
    return false;
}

// ---- bounded grid barrier for cooperative (co-resident) launches ------------------

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

/// Sense-free generation barrier over all blocks of a cooperative launch.  Each
/// wait is bounded by `limit_ns`; on expiry the status word gets
/// kStatusBarrierTimeout and every block leaves at its next barrier.  Returns false
/// when the kernel must stop.
__device__ __forceinline__ bool grid_barrier(unsigned* count, unsigned* gen, int* status,
                                             uint64_t limit_ns) {
    // every thread first waits for its own writes and reductions to be performed
    // GPU-wide: an atomic whose result is unused is issued as a reduction and may
    // otherwise still be in flight when the barrier releases
    __threadfence();
    __syncthreads();
    __shared__ int s_ok;
    if (threadIdx.x == 0) {
        const unsigned nblocks = gridDim.x * gridDim.y * gridDim.z;
        const unsigned my_gen = atomicAdd(gen, 0u);
        __threadfence();
        const unsigned arrived = atomicAdd(count, 1u);
        if (arrived == nblocks - 1) {
            atomicExch(count, 0u);
            __threadfence();
            atomicAdd(gen, 1u);
        } else {
            const uint64_t t0 = global_ns();
            unsigned spins = 0;
            while (atomicAdd(gen, 0u) == my_gen) {
                if (((++spins) & 63u) == 0 && global_ns() - t0 > limit_ns) {
                    atomicOr(status, kStatusBarrierTimeout);
                    break;
                }
                if (__ldcg(status) & kStatusBarrierTimeout) break;
                __nanosleep(32);
            }
        }
        __threadfence();
        s_ok = (__ldcg(status) & (kStatusBarrierTimeout | kStatusUnionLimit | kStatusRoundLimit)) == 0;
    }
    __syncthreads();
    return s_ok != 0;
}

// ---- warp helpers --------------------------------------------------------------

/// Warp-aggregated append: every lane with `pred` gets a unique slot in
/// list[0..*counter).  Returns the slot (or kInvalid when !pred).  All lanes of
/// the warp must call it.
__device__ __forceinline__ uint32_t warp_append(bool pred, uint32_t* counter) {
    const unsigned mask = __ballot_sync(0xFFFFFFFFu, pred);
    if (mask == 0) return kInvalid;
    const unsigned lane = lane_id();
    const int leader = __ffs(mask) - 1;
    uint32_t base = 0;
    if (static_cast<int>(lane) == leader) base = atomicAdd(counter, static_cast<uint32_t>(__popc(mask)));
    base = __shfl_sync(0xFFFFFFFFu, base, leader);
    if (!pred) return kInvalid;
    return base + __popc(mask & ((1u << lane) - 1u));
}

}  // namespace csb
