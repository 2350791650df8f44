// Device-wide exclusive prefix sum over u32 counts (three passes: tile sums, a
// single-block scan of the tile sums, tile rescan plus offset).
#include "common.cuh"
#include "engine.hpp"

namespace csb {
namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kTile = kScanThreads * kScanItems;

template <typename T>
__device__ T block_exclusive_scan(T x, T* total) {
    __shared__ T warp_sums[kScanThreads / 32];
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    T incl = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const T y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= static_cast<unsigned>(o)) incl += y;
    }
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        T s = lane < kScanThreads / 32 ? warp_sums[lane] : T(0);
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const T y = __shfl_up_sync(0xFFFFFFFFu, s, o);
            if (lane >= static_cast<unsigned>(o)) s += y;
        }
        if (lane < kScanThreads / 32) warp_sums[lane] = s;
    }
    __syncthreads();
    const T warp_off = warp ? warp_sums[warp - 1] : T(0);
    if (total) *total = warp_sums[kScanThreads / 32 - 1];
    __syncthreads();
    return warp_off + incl - x;
}

__global__ void k_tile_sums(const uint32_t* __restrict__ in, uint64_t n, uint64_t* __restrict__ sums) {
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kTile;
    uint64_t s = 0;
    for (int t = 0; t < kScanItems; ++t) {
        const uint64_t i = base + static_cast<uint64_t>(t) * kScanThreads + threadIdx.x;
        if (i < n) s += in[i];
    }
    uint64_t total;
    block_exclusive_scan<uint64_t>(s, &total);
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

__global__ void k_scan_sums(uint64_t* __restrict__ sums, uint64_t nb, uint64_t* __restrict__ total) {
    __shared__ uint64_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (uint64_t base = 0; base < nb; base += kScanThreads) {
        const uint64_t i = base + threadIdx.x;
        const uint64_t x = i < nb ? sums[i] : 0;
        uint64_t chunk;
        const uint64_t ex = block_exclusive_scan<uint64_t>(x, &chunk);
        if (i < nb) sums[i] = carry + ex;
        __syncthreads();
        if (threadIdx.x == 0) carry += chunk;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

__global__ void k_tile_apply(const uint32_t* __restrict__ in, uint64_t n,
                             const uint64_t* __restrict__ sums, uint32_t* __restrict__ out,
                             const uint64_t* __restrict__ total) {
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kTile;
    // each thread owns kScanItems consecutive elements
    const uint64_t my = base + static_cast<uint64_t>(threadIdx.x) * kScanItems;
    uint32_t v[kScanItems];
    uint64_t s = 0;
#pragma unroll
    for (int t = 0; t < kScanItems; ++t) {
        v[t] = (my + t < n) ? in[my + t] : 0u;
        s += v[t];
    }
    uint64_t ex = block_exclusive_scan<uint64_t>(s, nullptr) + sums[blockIdx.x];
#pragma unroll
    for (int t = 0; t < kScanItems; ++t) {
        if (my + t < n) out[my + t] = static_cast<uint32_t>(ex);
        ex += v[t];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = static_cast<uint32_t>(*total);
}

}  // namespace

void scan_reserve(Ctx& c, uint64_t n) { c.scratch[7].ensure(((n + kTile - 1) / kTile + 2) * sizeof(uint64_t)); }

void scan_u32(Ctx& c, const uint32_t* in, uint32_t* out, uint64_t n) {
    const uint64_t nb = (n + kTile - 1) / kTile;
    DevBuf& tmp = c.scratch[7];
    tmp.ensure((nb + 2) * sizeof(uint64_t));
    uint64_t* sums = tmp.as<uint64_t>();
    uint64_t* total = sums + nb + 1;
    if (nb == 0) {
        CSB_CUDA(cudaMemsetAsync(out, 0, sizeof(uint32_t), c.stream));
        return;
    }
    k_tile_sums<<<static_cast<unsigned>(nb), kScanThreads, 0, c.stream>>>(in, n, sums);
    k_scan_sums<<<1, kScanThreads, 0, c.stream>>>(sums, nb, total);
    k_tile_apply<<<static_cast<unsigned>(nb), kScanThreads, 0, c.stream>>>(in, n, sums, out, total);
    count_launch(c, 3);
    check_launch(c, "scan_u32");
    uint64_t host_total = 0;
    CSB_CUDA(cudaMemcpyAsync(&host_total, total, sizeof(uint64_t), cudaMemcpyDeviceToHost, c.stream));
    CSB_CUDA(cudaStreamSynchronize(c.stream));
    if (host_total > 0xFFFFFFFEull) fail(CS_ERR_UNSUPPORTED, "edge count exceeds 32-bit edge indices");
}

}  // namespace csb
