// Serving loop over a device-resident CORE-SG (cs_server_*).
//
// Two host threads per server:
//   scheduler   takes requests in arrival order.  A run of consecutive queries
//               (extract / epsilon-cut) becomes one batch: one 32-lane sweep over
//               its distinct mpts values (the plan is captured once and replayed;
//               unused lanes repeat a value), after which each distinct extract
//               mpts has its tree, labels and exact-sum bins copied into one result
//               slot in HBM that its queries share, in stream order, and every
//               epsilon-cut is labelled on the device into a slot of its own.
//               Inserts queued back to back are applied as one batch; in arrival
//               order they are a barrier between batches (CoreSG::insert,
//               src/coresg.cpp:325-389), with inserts_first they go ahead of the
//               queued queries.
//   completion  waits for a batch's event and copies its slots into the callers'
//               host buffers on its own stream, while the scheduler already runs
//               the next sweep on the context stream.
// Slots are allocated on demand while free HBM stays above the reserve (admission
// by free memory) and are recycled when their copies finish.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <thread>
#include <unordered_map>

#include "common.cuh"
#include "engine.hpp"

namespace csb {
namespace {

constexpr int kThreads = 256;
constexpr uint32_t kSweepLanes = 32;
constexpr uint64_t kMetaWords = 260;  // [0] tree edges, [1] cut components, [2..257] bins, [258] status

inline unsigned blocks_for(uint64_t work) { return static_cast<unsigned>((work + kThreads - 1) / kThreads); }

double now_ms() {
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

__global__ void k_cut_init(uint32_t* __restrict__ parent, uint32_t n) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < n) parent[v] = v;
}

/// dbscan_labels_from_mst (src/eval.cpp:230-239): unite the tree edges whose weight,
/// widened to double, is <= eps.  Roots stay the smallest node of their set.
__global__ void k_cut_unite(const cs_edge* __restrict__ tree, const unsigned long long* __restrict__ count,
                            uint64_t cap, double eps, uint32_t* __restrict__ parent, int* __restrict__ status) {
    const uint64_t x = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (x >= cap || x >= *count) return;
    const cs_edge e = tree[x];
    if (static_cast<double>(e.w) <= eps) uf_unite(parent, e.u, e.v, static_cast<uint32_t>(cap + 1), status);
}

struct Slot {
    DevBuf edges;   // cs_edge [n-1]
    DevBuf labels;  // u32 [n]
    DevBuf meta;    // u64 [kMetaWords]
    uint64_t n = 0; // nodes the slot can hold
    size_t bytes() const { return edges.bytes + labels.bytes + meta.bytes; }
};

size_t slot_bytes_for(uint64_t n) {
    return std::max<uint64_t>(n ? n - 1 : 0, 1) * sizeof(cs_edge) + std::max<uint64_t>(n, 1) * 4 + kMetaWords * 8;
}

struct Req {
    uint64_t ticket = 0;
    cs_request r{};
    std::vector<float> rows;  // insert rows, copied at submit
    cs_result res{};
    double t_submit = 0.0;
    bool done = false;
    bool waited = false;      // a waiter holds the ticket
    Slot* slot = nullptr;
    uint32_t lane = 0;
};

struct Batch {
    uint64_t id = 0;
    std::vector<Req*> reqs;
    std::vector<Slot*> slots;  // owned until the batch's copies finish
    cudaEvent_t ready = nullptr;
    uint64_t n = 0;
};

void set_error(Req* q, cs_status st, const std::string& msg) {
    q->res.status = st;
    std::snprintf(q->res.error, sizeof(q->res.error), "%s", msg.c_str());
}

}  // namespace

struct Server {
    Graph* g = nullptr;
    Ctx* c = nullptr;
    cs_server_config cfg{};
    std::mutex mu;
    std::condition_variable cv;
    std::deque<Req*> queue;
    std::unordered_map<uint64_t, Req*> tickets;
    std::deque<Batch*> inflight;
    std::vector<Slot*> free_slots;
    std::vector<Slot*> all_slots;
    uint64_t next_ticket = 1, next_batch = 1;
    bool stop_sched = false, stop_comp = false;
    cs_server_stats st{};
    std::thread sched, comp;
    cudaStream_t copy_stream = nullptr;
    DevBuf cut_parent, cut_tiles;
    // scheduler thread only: bumped by every insert batch; the graph version the last
    // sweep of every mpts 1..k_max solved (its results stay in the sweep plan until
    // the next sweep)
    uint64_t graph_version = 0, swept_version = ~0ull;

    void finish(Req* q) {  // under mu
        q->res.latency_ms = now_ms() - q->t_submit;
        q->done = true;
        ++st.completed;
        if (q->res.status != CS_OK) ++st.failed;
        q->rows.clear();
        q->rows.shrink_to_fit();
    }

    /// A slot for `n` nodes, or null when none is free and memory does not admit a
    /// new one (the caller waits for the batches in flight).  Under mu.
    Slot* try_slot(uint64_t n) {
        // a free slot that holds n nodes is reused as it is: slots are sized for the
        // graph's capacity (cs_graph_reserve) or with a quarter of headroom, so a graph
        // that grows by inserts keeps its slots
        for (size_t i = 0; i < free_slots.size(); ++i) {
            if (free_slots[i]->n >= n) {
                Slot* s = free_slots[i];
                free_slots.erase(free_slots.begin() + static_cast<long>(i));
                return s;
            }
        }
        // slots too small for the grown graph are released before new ones are made
        for (Slot* s : free_slots) {
            all_slots.erase(std::find(all_slots.begin(), all_slots.end(), s));
            delete s;
        }
        free_slots.clear();
        if (all_slots.size() >= cfg.max_slots) return nullptr;
        const uint64_t cap = std::max<uint64_t>(n + n / 4, scratch_nodes(*g));
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return nullptr;
        const size_t need = slot_bytes_for(cap);
        if (free_b < need + cfg.reserve_bytes) return nullptr;
        Slot* s = new Slot;
        try {
            s->edges.ensure(std::max<uint64_t>(cap ? cap - 1 : 0, 1) * sizeof(cs_edge));
            s->labels.ensure(std::max<uint64_t>(cap, 1) * 4);
            s->meta.ensure(kMetaWords * 8);
        } catch (const Error&) {
            delete s;
            return nullptr;
        }
        s->n = cap;
        all_slots.push_back(s);
        st.slots = all_slots.size();
        st.slot_bytes = s->bytes();
        return s;
    }

    void release_free_slots() {  // under mu
        for (Slot* s : free_slots) {
            all_slots.erase(std::find(all_slots.begin(), all_slots.end(), s));
            delete s;
        }
        free_slots.clear();
        st.slots = all_slots.size();
    }

    void run_inserts(std::vector<Req*>& batch);
    void run_batch(std::vector<Req*>& take);
    void sched_loop();
    void comp_loop();
};

void Server::run_inserts(std::vector<Req*>& batch) {
    const double t0 = now_ms();
    ++graph_version;  // the last sweep's results no longer describe the graph
    uint64_t rows_total = 0;
    {
        std::lock_guard<std::mutex> lk(mu);
        for (Req* q : batch) {
            q->res.queue_ms = t0 - q->t_submit;
            rows_total += q->r.count;
        }
    }
    cs_status status = CS_OK;
    std::string msg;
    {
        std::lock_guard<std::recursive_mutex> ck(c->mu);
        try {
            c->bind();
            // admission: the growth of the resident arrays and the descent scratch
            const uint64_t n1 = g->n + rows_total;
            const uint64_t need = n1 * (static_cast<uint64_t>(g->stride) * 4 + g->k * 9ull + 2600) +
                                  rows_total * 64ull * 8;
            size_t free_b = 0, total_b = 0;
            CSB_CUDA(cudaMemGetInfo(&free_b, &total_b));
            if (free_b < need + cfg.reserve_bytes) {
                // let the batches in flight finish and give back the idle slots
                std::unique_lock<std::mutex> lk(mu);
                cv.wait(lk, [&] { return inflight.empty(); });
                release_free_slots();
                lk.unlock();
                CSB_CUDA(cudaMemGetInfo(&free_b, &total_b));
                if (free_b < need + cfg.reserve_bytes)
                    fail(CS_ERR_OOM, "insert not admitted: free HBM below the batch's growth plus the reserve");
            }
            // back-to-back inserts are one batch: their rows in submission order
            const uint32_t dim = g->dim;
            const float* rows = nullptr;
            uint32_t stride = dim;
            std::vector<float> joined;
            if (batch.size() == 1) {
                rows = batch[0]->rows.data();
                stride = batch[0]->r.row_stride;
            } else {
                joined.resize(rows_total * dim);
                uint64_t at = 0;
                for (Req* q : batch) {
                    for (uint64_t i = 0; i < q->r.count; ++i, ++at)
                        std::memcpy(joined.data() + at * dim, q->rows.data() + i * q->r.row_stride, dim * 4);
                }
                rows = joined.data();
            }
            if (rows_total) {
                InsertStats ist;
                knn_insert(*g, rows, rows_total, stride, cfg.insert, &ist);
                if (cfg.insert.reselect_bridges) select_bridges(*g, nullptr, nullptr, nullptr, nullptr);
            }
        } catch (const Error& e) {
            status = e.status;
            msg = e.what();
        } catch (const std::exception& e) {
            status = CS_ERR_INVALID;
            msg = e.what();
        }
    }
    std::lock_guard<std::mutex> lk(mu);
    st.insert_ms += now_ms() - t0;
    if (status == CS_OK) {
        st.inserts += batch.size();
        st.inserted_rows += rows_total;
        ++st.insert_batches;
    }
    for (Req* q : batch) {
        if (status != CS_OK) set_error(q, status, msg);
        q->res.n = g->n;
        finish(q);
    }
    cv.notify_all();
}

void Server::run_batch(std::vector<Req*>& take) {
    const uint64_t n = g->n;
    // result slots, admitted by free memory: one per distinct extract mpts (its
    // queries share the tree) and one per epsilon-cut.  A batch that cannot get a
    // slot it needs is cut short there and the rest goes back to the queue head.
    std::vector<Slot*> slots;
    std::vector<std::pair<uint32_t, Slot*>> trees;  // extract mpts -> shared slot
    size_t got = 0;
    {
        std::unique_lock<std::mutex> lk(mu);
        while (got < take.size()) {
            Req* q = take[got];
            const uint32_t m = std::max<uint32_t>(q->r.mpts, 1);
            if (q->r.kind == CS_REQ_EXTRACT) {
                auto it = std::find_if(trees.begin(), trees.end(), [&](const auto& t) { return t.first == m; });
                if (it != trees.end()) {
                    q->slot = it->second;
                    ++got;
                    continue;
                }
            }
            Slot* sl = try_slot(n);
            if (sl) {
                slots.push_back(sl);
                if (q->r.kind == CS_REQ_EXTRACT) trees.emplace_back(m, sl);
                q->slot = sl;
                ++got;
                continue;
            }
            if (got > 0) break;  // serve what fits now
            if (inflight.empty()) break;
            cv.wait(lk);         // a completed batch returns its slots
        }
        if (got == 0) {
            set_error(take[0], CS_ERR_OOM, "query not admitted: no result slot fits in free HBM");
            take[0]->res.n = n;
            finish(take[0]);
            for (size_t i = take.size(); i-- > 1;) queue.push_front(take[i]);
            take.resize(1);
            cv.notify_all();
            return;
        }
        for (size_t i = take.size(); i-- > got;) queue.push_front(take[i]);
        take.resize(got);
        const double t = now_ms();
        for (Req* q : take) q->res.queue_ms = t - q->t_submit;
    }
    // lanes.  With k_max <= 32 a sweep solves every mpts 1..k_max (lane = mpts - 1):
    // it costs what a padded sweep of the requested values costs, and until an insert
    // changes the graph, later batches are served from its results without a sweep.
    // Otherwise: the distinct mpts in order of first appearance, padded to 32.
    const bool every_mpts = g->k <= kSweepLanes;
    std::vector<uint32_t> lanes;
    if (every_mpts) {
        for (uint32_t m = 1; m <= g->k; ++m) lanes.push_back(m);
        for (Req* q : take) q->lane = std::max<uint32_t>(q->r.mpts, 1) - 1;
    } else {
        for (Req* q : take) {
            const uint32_t m = std::max<uint32_t>(q->r.mpts, 1);
            auto it = std::find(lanes.begin(), lanes.end(), m);
            q->lane = static_cast<uint32_t>(it - lanes.begin());
            if (it == lanes.end()) lanes.push_back(m);
        }
    }
    while (lanes.size() < kSweepLanes) lanes.push_back(lanes.back());
    const bool reuse = every_mpts && swept_version == graph_version && g->plan != nullptr;
    Batch* b = new Batch;
    b->n = n;
    b->reqs = take;
    b->slots = slots;
    cs_status status = CS_OK;
    std::string msg;
    float ms = 0.0f;
    {
        std::lock_guard<std::recursive_mutex> ck(c->mu);
        try {
            c->bind();
            if (!reuse) {
                swept_version = ~0ull;  // until this sweep has completed
                sweep_run(*g, lanes.data(), kSweepLanes, true, &ms);
                if (every_mpts) swept_version = graph_version;
            }
            // every slot is filled once: a shared tree slot by its first query, with
            // the edges / labels any of its queries asked for
            for (size_t i = 0; i < take.size(); ++i) {
                Req* q = take[i];
                Slot* sl = q->slot;
                bool first = true;
                for (size_t j = 0; j < i; ++j) first = first && take[j]->slot != sl;
                if (!first) continue;
                const SweepOut o = sweep_outputs(*g, q->lane);
                unsigned long long* meta = sl->meta.as<unsigned long long>();
                CSB_CUDA(cudaMemsetAsync(meta, 0, kMetaWords * 8, c->stream));
                CSB_CUDA(cudaMemcpyAsync(meta, o.count, 8, cudaMemcpyDeviceToDevice, c->stream));
                CSB_CUDA(cudaMemcpyAsync(meta + 2, o.bins, 256 * 8, cudaMemcpyDeviceToDevice, c->stream));
                if (q->r.kind == CS_REQ_EXTRACT) {
                    bool edges = false, labels = false;
                    for (size_t j = i; j < take.size(); ++j) {
                        if (take[j]->slot != sl) continue;
                        edges = edges || take[j]->r.out_edges;
                        labels = labels || take[j]->r.out_labels;
                    }
                    if (edges && o.cap)
                        CSB_CUDA(cudaMemcpyAsync(sl->edges.p, o.edges, o.cap * sizeof(cs_edge), cudaMemcpyDeviceToDevice,
                                                 c->stream));
                    if (labels && n)
                        CSB_CUDA(cudaMemcpyAsync(sl->labels.p, o.labels, n * 4, cudaMemcpyDeviceToDevice, c->stream));
                } else if (n) {  // epsilon-cut of this tree, labelled into the slot
                    cut_parent.ensure(n * 4);
                    cut_tiles.ensure((blocks_for(n) + 2) * 4ull + 64);
                    k_cut_init<<<blocks_for(n), kThreads, 0, c->stream>>>(cut_parent.as<uint32_t>(),
                                                                          static_cast<uint32_t>(n));
                    if (o.cap)
                        k_cut_unite<<<blocks_for(o.cap), kThreads, 0, c->stream>>>(
                            o.edges, o.count, o.cap, q->r.eps, cut_parent.as<uint32_t>(),
                            reinterpret_cast<int*>(meta + 258));
                    count_launch(*c, 2);
                    launch_labels(*c, cut_parent.as<uint32_t>(), static_cast<uint32_t>(n), 1, sl->labels.as<uint32_t>(),
                                  cut_tiles.as<uint32_t>(), meta + 1);
                }
            }
            check_launch(*c, "serving batch");
            CSB_CUDA(cudaEventCreateWithFlags(&b->ready, cudaEventDisableTiming));
            CSB_CUDA(cudaEventRecord(b->ready, c->stream));
        } catch (const Error& e) {
            status = e.status;
            msg = e.what();
        } catch (const std::exception& e) {
            status = CS_ERR_INVALID;
            msg = e.what();
        }
    }
    std::lock_guard<std::mutex> lk(mu);
    if (status != CS_OK) {
        for (Req* q : take) {
            set_error(q, status, msg);
            q->res.n = n;
            q->slot = nullptr;
            finish(q);
        }
        for (Slot* sl : slots) free_slots.push_back(sl);
        if (b->ready) cudaEventDestroy(b->ready);
        delete b;
        cv.notify_all();
        return;
    }
    b->id = next_batch++;
    if (reuse) {
        ++st.reused_batches;
    } else {
        ++st.batches;
    }
    st.queries += take.size();
    st.max_batch_seen = std::max<uint32_t>(st.max_batch_seen, static_cast<uint32_t>(take.size()));
    st.sweep_ms += ms;
    inflight.push_back(b);
    cv.notify_all();
}

void Server::sched_loop() {
    cudaSetDevice(c->device);
    for (;;) {
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [&] { return stop_sched || !queue.empty(); });
        if (queue.empty()) {
            if (stop_sched) return;
            continue;
        }
        // inserts: the run at the head of the queue (arrival order: a barrier after
        // the sweeps already dispatched), or every queued one (inserts_first)
        std::vector<Req*> ins;
        if (cfg.inserts_first) {
            for (auto it = queue.begin(); it != queue.end();) {
                if ((*it)->r.kind == CS_REQ_INSERT) {
                    ins.push_back(*it);
                    it = queue.erase(it);
                } else {
                    ++it;
                }
            }
        } else {
            while (!queue.empty() && queue.front()->r.kind == CS_REQ_INSERT) {
                ins.push_back(queue.front());
                queue.pop_front();
            }
        }
        if (!ins.empty()) {
            lk.unlock();
            run_inserts(ins);
            continue;
        }
        // the run of queries at the head: at most max_batch distinct mpts and
        // max_slots slots (a distinct extract mpts or an epsilon-cut takes one)
        std::vector<Req*> take;
        std::vector<uint32_t> distinct, trees;
        uint32_t need = 0;
        while (!queue.empty() && queue.front()->r.kind != CS_REQ_INSERT) {
            Req* q = queue.front();
            const uint32_t m = std::max<uint32_t>(q->r.mpts, 1);
            const bool new_m = std::find(distinct.begin(), distinct.end(), m) == distinct.end();
            const bool new_slot =
                q->r.kind != CS_REQ_EXTRACT || std::find(trees.begin(), trees.end(), m) == trees.end();
            if ((new_m && distinct.size() >= cfg.max_batch) || (new_slot && need >= cfg.max_slots)) break;
            if (new_m) distinct.push_back(m);
            if (new_slot) {
                ++need;
                if (q->r.kind == CS_REQ_EXTRACT) trees.push_back(m);
            }
            take.push_back(q);
            queue.pop_front();
        }
        lk.unlock();
        run_batch(take);
    }
}

void Server::comp_loop() {
    cudaSetDevice(c->device);
    std::vector<unsigned long long> meta;
    for (;;) {
        Batch* b = nullptr;
        {
            std::unique_lock<std::mutex> lk(mu);
            cv.wait(lk, [&] { return stop_comp || !inflight.empty(); });
            if (inflight.empty()) return;
            b = inflight.front();
        }
        cudaError_t err = cudaEventSynchronize(b->ready);
        const size_t nq = b->reqs.size();
        meta.assign(nq * kMetaWords, 0);
        for (size_t i = 0; i < nq && err == cudaSuccess; ++i)
            err = cudaMemcpyAsync(meta.data() + i * kMetaWords, b->reqs[i]->slot->meta.p, kMetaWords * 8,
                                  cudaMemcpyDeviceToHost, copy_stream);
        if (err == cudaSuccess) err = cudaStreamSynchronize(copy_stream);
        for (size_t i = 0; i < nq && err == cudaSuccess; ++i) {
            Req* q = b->reqs[i];
            const unsigned long long* m = meta.data() + i * kMetaWords;
            q->res.n = b->n;
            q->res.batch = b->id;
            const int dstatus = static_cast<int>(m[258]);
            if (dstatus & kStatusUnionLimit) {
                set_error(q, CS_ERR_TIMEOUT, "epsilon-cut: a union retry loop ran out");
                continue;
            }
            if (q->r.kind == CS_REQ_EXTRACT) {
                q->res.nedges = m[0];
                q->res.ncomp = static_cast<uint32_t>(b->n - m[0]);
                q->res.weight = exact_sum_from_bins(reinterpret_cast<const uint64_t*>(m + 2));
                if (q->r.out_edges && m[0]) {
                    if (q->r.out_edges_cap < m[0]) {
                        set_error(q, CS_ERR_INVALID, "out_edges_cap is smaller than the tree");
                        continue;
                    }
                    err = cudaMemcpyAsync(q->r.out_edges, q->slot->edges.p, m[0] * sizeof(cs_edge),
                                          cudaMemcpyDeviceToHost, copy_stream);
                }
                if (err == cudaSuccess && q->r.out_labels && b->n) {
                    if (q->r.out_labels_cap < b->n) {
                        set_error(q, CS_ERR_INVALID, "out_labels_cap is smaller than n");
                        continue;
                    }
                    err = cudaMemcpyAsync(q->r.out_labels, q->slot->labels.p, b->n * 4, cudaMemcpyDeviceToHost,
                                          copy_stream);
                }
            } else {
                q->res.ncomp = static_cast<uint32_t>(m[1]);
                if (q->r.out_labels_cap < b->n) {
                    set_error(q, CS_ERR_INVALID, "out_labels_cap is smaller than n");
                    continue;
                }
                if (b->n)
                    err = cudaMemcpyAsync(q->r.out_labels, q->slot->labels.p, b->n * 4, cudaMemcpyDeviceToHost,
                                          copy_stream);
            }
        }
        if (err == cudaSuccess) err = cudaStreamSynchronize(copy_stream);
        std::lock_guard<std::mutex> lk(mu);
        for (Req* q : b->reqs) {
            if (err != cudaSuccess && q->res.status == CS_OK)
                set_error(q, CS_ERR_CUDA, std::string("result copy: ") + cudaGetErrorString(err));
            q->slot = nullptr;
            finish(q);
        }
        for (Slot* sl : b->slots) free_slots.push_back(sl);
        inflight.pop_front();
        cudaEventDestroy(b->ready);
        delete b;
        cv.notify_all();
    }
}

}  // namespace csb

using namespace csb;

extern "C" {

cs_status cs_server_create(cs_graph* gp, const cs_server_config* cfg, cs_server** out) {
    Graph* g = reinterpret_cast<Graph*>(gp);
    return guarded(g ? g->ctx : nullptr, [&] {
        CSB_REQUIRE(out != nullptr, "cs_server_create: null out");
        *out = nullptr;
        CSB_REQUIRE(g->n > 0, "cs_server_create: the graph is empty");
        Server* s = new Server;
        s->g = g;
        s->c = g->ctx;
        if (cfg) s->cfg = *cfg;
        if (s->cfg.max_batch == 0 || s->cfg.max_batch > kSweepLanes) s->cfg.max_batch = kSweepLanes;
        if (s->cfg.max_slots == 0) s->cfg.max_slots = 64;
        if (s->cfg.reserve_bytes == 0) s->cfg.reserve_bytes = 2ull << 30;
        if (s->cfg.insert.sample == 0) cs_insert_defaults(&s->cfg.insert);
        if (cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking) != cudaSuccess) {
            delete s;
            fail(CS_ERR_CUDA, "cs_server_create: stream creation failed");
        }
        s->sched = std::thread([s] { s->sched_loop(); });
        s->comp = std::thread([s] { s->comp_loop(); });
        *out = reinterpret_cast<cs_server*>(s);
    });
}

void cs_server_destroy(cs_server* sp) {
    Server* s = reinterpret_cast<Server*>(sp);
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop_sched = true;
    }
    s->cv.notify_all();
    s->sched.join();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop_comp = true;
    }
    s->cv.notify_all();
    s->comp.join();
    {
        std::lock_guard<std::recursive_mutex> ck(s->c->mu);
        cudaSetDevice(s->c->device);
        for (auto& kv : s->tickets) delete kv.second;
        s->tickets.clear();
        for (Slot* sl : s->all_slots) delete sl;
        s->all_slots.clear();
        s->free_slots.clear();
        s->cut_parent.release();
        s->cut_tiles.release();
        cudaStreamDestroy(s->copy_stream);
    }
    delete s;
}

cs_status cs_server_submit(cs_server* sp, const cs_request* req, uint64_t* out_ticket) {
    Server* s = reinterpret_cast<Server*>(sp);
    if (!s || !req || !out_ticket) {
        set_thread_error("cs_server_submit: null argument");
        return CS_ERR_INVALID;
    }
    std::string err;
    if (req->kind == CS_REQ_EXTRACT || req->kind == CS_REQ_EPS_LABELS) {
        if (req->mpts > s->g->k) err = "cs_server_submit: mpts exceeds k_max";
        if (req->kind == CS_REQ_EPS_LABELS && !req->out_labels) err = "cs_server_submit: an epsilon-cut needs out_labels";
    } else if (req->kind == CS_REQ_INSERT) {
        if (req->count && (!req->rows || req->row_stride < s->g->dim))
            err = "cs_server_submit: insert rows must be count x row_stride >= dim floats";
    } else {
        err = "cs_server_submit: unknown request kind";
    }
    if (!err.empty()) {
        set_thread_error(err);
        return CS_ERR_INVALID;
    }
    Req* q = new (std::nothrow) Req;
    if (!q) return CS_ERR_OOM;
    q->r = *req;
    if (req->kind == CS_REQ_INSERT && req->count) {
        try {
            q->rows.assign(req->rows, req->rows + req->count * req->row_stride);
        } catch (const std::bad_alloc&) {
            delete q;
            set_thread_error("cs_server_submit: host allocation failed");
            return CS_ERR_OOM;
        }
        q->r.rows = nullptr;
    }
    q->res.status = CS_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop_sched) {
            delete q;
            set_thread_error("cs_server_submit: the server is stopping");
            return CS_ERR_STATE;
        }
        q->ticket = s->next_ticket++;
        q->t_submit = now_ms();
        s->tickets[q->ticket] = q;
        s->queue.push_back(q);
        ++s->st.submitted;
        *out_ticket = q->ticket;
    }
    s->cv.notify_all();
    return CS_OK;
}

cs_status cs_server_wait(cs_server* sp, uint64_t ticket, uint32_t timeout_ms, cs_result* out) {
    Server* s = reinterpret_cast<Server*>(sp);
    if (!s) {
        set_thread_error("cs_server_wait: null server");
        return CS_ERR_INVALID;
    }
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->tickets.find(ticket);
    if (it == s->tickets.end() || it->second->waited) {
        set_thread_error("cs_server_wait: unknown ticket");
        return CS_ERR_INVALID;
    }
    Req* q = it->second;
    auto ready = [&] { return q->done; };
    if (timeout_ms == 0xFFFFFFFFu) {
        s->cv.wait(lk, ready);
    } else if (!s->cv.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) {
        set_thread_error("cs_server_wait: still pending");
        return CS_ERR_TIMEOUT;
    }
    if (out) *out = q->res;
    s->tickets.erase(ticket);
    delete q;
    return CS_OK;
}

cs_status cs_server_stats_get(cs_server* sp, cs_server_stats* out) {
    Server* s = reinterpret_cast<Server*>(sp);
    if (!s || !out) {
        set_thread_error("cs_server_stats_get: null argument");
        return CS_ERR_INVALID;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    *out = s->st;
    return CS_OK;
}

void* cs_host_alloc(size_t bytes) {
    void* p = nullptr;
    if (cudaHostAlloc(&p, bytes ? bytes : 1, cudaHostAllocPortable) != cudaSuccess) return nullptr;
    return p;
}

void cs_host_free(void* p) {
    if (p) cudaFreeHost(p);
}

}  // extern "C"
