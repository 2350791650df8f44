// Contexts, device query, error plumbing, device/pinned buffers and staging copies.
#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>

#include "common.cuh"
#include "engine.hpp"

namespace csb {

namespace {
thread_local std::string t_error;
// device allocations made by DevBuf in this process: count and bytes
std::atomic<uint64_t> g_dev_allocs{0}, g_dev_alloc_bytes{0};
void count_alloc(size_t nbytes) {
    g_dev_allocs.fetch_add(1, std::memory_order_relaxed);
    g_dev_alloc_bytes.fetch_add(nbytes, std::memory_order_relaxed);
}
// testing hook (cs_test_fail_device_allocs): device allocations still allowed before
// every further one fails; UINT64_MAX = no injection
std::atomic<uint64_t> g_fail_after{UINT64_MAX};
/// True when this allocation must fail by injection (no cudaMalloc is issued).
bool injected_alloc_failure() {
    uint64_t v = g_fail_after.load(std::memory_order_relaxed);
    while (v != UINT64_MAX) {
        if (v == 0) return true;
        if (g_fail_after.compare_exchange_weak(v, v - 1, std::memory_order_relaxed)) return false;
    }
    return false;
}
}  // namespace

void set_thread_error(const std::string& m) { t_error = m; }
const char* thread_error() { return t_error.c_str(); }

void fail(cs_status s, const std::string& msg) { throw Error(s, msg); }

void check_cuda(cudaError_t e, const char* what, const char* file, int line) {
    if (e == cudaSuccess) return;
    const bool oom = e == cudaErrorMemoryAllocation;
    std::string msg = std::string(what) + " -> " + cudaGetErrorString(e) + " (" + file + ":" +
                      std::to_string(line) + ")";
    if (!oom) cudaGetLastError();  // clear sticky-free errors so the context stays usable
    throw Error(oom ? CS_ERR_OOM : CS_ERR_CUDA, msg);
}

void check_launch(Ctx& c, const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        fail(e == cudaErrorMemoryAllocation ? CS_ERR_OOM : CS_ERR_CUDA,
             std::string(what) + ": launch failed: " + cudaGetErrorString(e));
    }
    (void)c;
}

void DevBuf::release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
}

void DevBuf::ensure(size_t nbytes) {
    if (nbytes <= bytes && p) return;
    // a buffer that grows again (resident arrays after inserts) takes a quarter of
    // headroom, so a run of small growths does not reallocate every time
    if (p) nbytes = std::max(nbytes, bytes + bytes / 4);
    release();
    if (nbytes == 0) nbytes = 16;
    if (injected_alloc_failure())
        fail(CS_ERR_OOM, "cudaMalloc of " + std::to_string(nbytes) + " bytes failed: injected by cs_test_fail_device_allocs");
    void* q = nullptr;
    const cudaError_t e = cudaMalloc(&q, nbytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        fail(CS_ERR_OOM, "cudaMalloc of " + std::to_string(nbytes) + " bytes failed: " +
                             cudaGetErrorString(e));
    }
    count_alloc(nbytes);
    p = q;
    bytes = nbytes;
}

void DevBuf::grow_keep(size_t nbytes, cudaStream_t s) {
    if (nbytes <= bytes && p) return;
    if (injected_alloc_failure())
        fail(CS_ERR_OOM, "cudaMalloc of " + std::to_string(nbytes) + " bytes failed: injected by cs_test_fail_device_allocs");
    void* q = nullptr;
    const cudaError_t e = cudaMalloc(&q, nbytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        fail(CS_ERR_OOM, "cudaMalloc of " + std::to_string(nbytes) + " bytes failed: " +
                             cudaGetErrorString(e));
    }
    if (p && bytes) {
        CSB_CUDA(cudaMemcpyAsync(q, p, bytes, cudaMemcpyDeviceToDevice, s));
        CSB_CUDA(cudaStreamSynchronize(s));
    }
    count_alloc(nbytes);
    release();
    p = q;
    bytes = nbytes;
}

void PinnedBuf::release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    bytes = 0;
}

void PinnedBuf::ensure(size_t nbytes) {
    if (nbytes <= bytes && p) return;
    release();
    void* q = nullptr;
    const cudaError_t e = cudaMallocHost(&q, std::max<size_t>(nbytes, 64));
    if (e != cudaSuccess) {
        cudaGetLastError();
        fail(CS_ERR_OOM, std::string("cudaMallocHost failed: ") + cudaGetErrorString(e));
    }
    p = q;
    bytes = std::max<size_t>(nbytes, 64);
}

void Ctx::bind() const { CSB_CUDA(cudaSetDevice(device)); }

void Ctx::sync() { CSB_CUDA(cudaStreamSynchronize(stream)); }

/// Host -> device through pinned staging, in 64 MiB chunks so the staging stays
/// bounded; two staging halves let the memcpy into one overlap the DMA of the other.
/// Whether a host pointer is page-locked (cudaHostAlloc / cudaHostRegister memory):
/// such a buffer is copied by the DMA engine directly, without the staging copy.
static bool host_pinned(const void* p) {
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeHost;
}

void copy_h2d(Ctx& c, void* dst, const void* src, size_t bytes) {
    if (!bytes) return;
    if (host_pinned(src)) {
        CSB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c.stream));
        CSB_CUDA(cudaStreamSynchronize(c.stream));
        return;
    }
    // pageable: two staging halves, the host copy of one overlapping the DMA of the other
    const size_t chunk = size_t(32) << 20;
    PinnedBuf& st = c.pinned[0];
    st.ensure(2 * std::min(bytes, chunk));
    const size_t half = st.bytes / 2;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    CSB_CUDA(cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming));
    CSB_CUDA(cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming));
    int slot = 0;
    bool used[2] = {false, false};
    for (size_t off = 0; off < bytes; off += half) {
        const size_t b = std::min(half, bytes - off);
        if (used[slot]) CSB_CUDA(cudaEventSynchronize(ev[slot]));
        char* stage = static_cast<char*>(st.p) + slot * half;
        std::memcpy(stage, static_cast<const char*>(src) + off, b);
        CSB_CUDA(cudaMemcpyAsync(static_cast<char*>(dst) + off, stage, b, cudaMemcpyHostToDevice, c.stream));
        CSB_CUDA(cudaEventRecord(ev[slot], c.stream));
        used[slot] = true;
        slot ^= 1;
    }
    CSB_CUDA(cudaStreamSynchronize(c.stream));
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
}

bool copy_d2h_enqueue(Ctx& c, void* dst, const void* src, size_t bytes) {
    if (!bytes) return false;
    if (host_pinned(dst)) {
        CSB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c.stream));
        return true;
    }
    copy_d2h(c, dst, src, bytes);
    return false;
}

void copy_d2h(Ctx& c, void* dst, const void* src, size_t bytes) {
    if (!bytes) return;
    if (host_pinned(dst)) {
        CSB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c.stream));
        CSB_CUDA(cudaStreamSynchronize(c.stream));
        return;
    }
    // pageable: two staging halves, the DMA of the next chunk overlapping the host
    // copy of the current one
    const size_t chunk = size_t(32) << 20;
    PinnedBuf& st = c.pinned[1];
    st.ensure(2 * std::min(bytes, chunk));
    const size_t half = st.bytes / 2;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    CSB_CUDA(cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming));
    CSB_CUDA(cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming));
    const size_t nchunks = (bytes + half - 1) / half;
    auto issue = [&](size_t k) {
        const size_t off = k * half, b = std::min(half, bytes - off);
        char* stage = static_cast<char*>(st.p) + (k & 1) * half;
        CSB_CUDA(cudaMemcpyAsync(stage, static_cast<const char*>(src) + off, b, cudaMemcpyDeviceToHost, c.stream));
        CSB_CUDA(cudaEventRecord(ev[k & 1], c.stream));
    };
    issue(0);
    for (size_t k = 0; k < nchunks; ++k) {
        if (k + 1 < nchunks) issue(k + 1);  // its half was drained by the host copy of chunk k-1
        CSB_CUDA(cudaEventSynchronize(ev[k & 1]));
        const size_t off = k * half, b = std::min(half, bytes - off);
        std::memcpy(static_cast<char*>(dst) + off, static_cast<char*>(st.p) + (k & 1) * half, b);
    }
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
}

}  // namespace csb

using namespace csb;

extern "C" {

cs_status cs_device_count(int32_t* out) {
    int n = 0;
    const cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) {
        cudaGetLastError();
        if (out) *out = 0;
        set_thread_error(std::string("cudaGetDeviceCount: ") + cudaGetErrorString(e));
        return (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) ? CS_OK : CS_ERR_CUDA;
    }
    if (out) *out = n;
    return CS_OK;
}

cs_status cs_device_props(int32_t device, char* name, size_t name_len, size_t* total_mem,
                          size_t* free_mem, int32_t* sm_count, int32_t* cc_major, int32_t* cc_minor) {
    try {
        cudaDeviceProp p;
        CSB_CUDA(cudaGetDeviceProperties(&p, device));
        if (name && name_len) {
            std::strncpy(name, p.name, name_len - 1);
            name[name_len - 1] = 0;
        }
        if (total_mem) *total_mem = p.totalGlobalMem;
        if (sm_count) *sm_count = p.multiProcessorCount;
        if (cc_major) *cc_major = p.major;
        if (cc_minor) *cc_minor = p.minor;
        if (free_mem) {
            int prev = 0;
            CSB_CUDA(cudaGetDevice(&prev));
            CSB_CUDA(cudaSetDevice(device));
            size_t f = 0, t = 0;
            CSB_CUDA(cudaMemGetInfo(&f, &t));
            *free_mem = f;
            CSB_CUDA(cudaSetDevice(prev));
        }
        return CS_OK;
    } catch (const Error& e) {
        set_thread_error(e.what());
        return e.status;
    }
}

const char* cs_last_error(const cs_ctx* ctx) {
    const Ctx* c = reinterpret_cast<const Ctx*>(ctx);
    if (!c) return thread_error();
    return c->last_error.c_str();
}

cs_status cs_ctx_create(int32_t device, cs_ctx** out) {
    if (!out) {
        set_thread_error("cs_ctx_create: null output");
        return CS_ERR_INVALID;
    }
    *out = nullptr;
    Ctx* c = new Ctx();
    try {
        c->device = device;
        CSB_CUDA(cudaSetDevice(device));
        cudaDeviceProp p;
        CSB_CUDA(cudaGetDeviceProperties(&p, device));
        c->sm_count = p.multiProcessorCount;
        c->cc_major = p.major;
        c->cc_minor = p.minor;
        if (p.major < 10) {
            fail(CS_ERR_UNSUPPORTED, "device is sm_" + std::to_string(p.major) +
                                         std::to_string(p.minor) +
                                         "; this library is built for sm_100a only");
        }
        CSB_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        c->status.ensure(64);
        CSB_CUDA(cudaMemsetAsync(c->status.p, 0, 64, c->stream));
        CSB_CUDA(cudaStreamSynchronize(c->stream));
        *out = reinterpret_cast<cs_ctx*>(c);
        return CS_OK;
    } catch (const Error& e) {
        set_thread_error(e.what());
        if (c->stream) cudaStreamDestroy(c->stream);
        delete c;
        return e.status;
    }
}

}  // extern "C"

namespace csb {
/// Free a context's resources.  Never throws (it runs at interpreter teardown too,
/// when the runtime may already be gone).
void ctx_free(Ctx* c) {
    if (cudaSetDevice(c->device) == cudaSuccess && c->stream) cudaStreamSynchronize(c->stream);
    for (auto& b : c->scratch) b.release();
    c->status.release();
    for (auto& b : c->pinned) b.release();
    if (c->stream) cudaStreamDestroy(c->stream);
    c->stream = nullptr;
    cudaGetLastError();
    delete c;
}
}  // namespace csb

extern "C" {

void cs_ctx_destroy(cs_ctx* ctx) {
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (!c) return;
    {
        std::lock_guard<std::recursive_mutex> lk(c->mu);
        if (c->live_graphs > 0) {
            c->destroy_pending = true;  // freed with its last graph
            return;
        }
    }
    ctx_free(c);
}

cs_status cs_ctx_trim(cs_ctx* ctx) {
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    return guarded(c, [&] {
        c->sync();
        for (auto& b : c->scratch) b.release();
        for (auto& b : c->pinned) b.release();
    });
}

void* cs_ctx_stream(const cs_ctx* ctx) {
    const Ctx* c = reinterpret_cast<const Ctx*>(ctx);
    return c ? static_cast<void*>(c->stream) : nullptr;
}

uint64_t cs_ctx_launches(const cs_ctx* ctx) {
    const Ctx* c = reinterpret_cast<const Ctx*>(ctx);
    return c ? c->launches : 0;
}

void cs_device_allocs(uint64_t* out_count, uint64_t* out_bytes) {
    if (out_count) *out_count = g_dev_allocs.load(std::memory_order_relaxed);
    if (out_bytes) *out_bytes = g_dev_alloc_bytes.load(std::memory_order_relaxed);
}

void cs_test_fail_device_allocs(uint64_t after) { g_fail_after.store(after, std::memory_order_relaxed); }

}  // extern "C"
