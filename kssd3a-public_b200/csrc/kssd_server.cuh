// Continuous-batching query server over a resident index (part of the kssdgpu.cu
// translation unit: it launches the batched counting kernel defined there).
//
// Requests are single query samples (sorted comblco keys).  submit() checks and
// copies the keys into the request and queues it.  A worker thread owns a pool of
// device slots whose buffers are reserved when the server is created: as many slots
// as the configured device-memory budget holds (at most the configured count), so
// the budget bounds the work in flight.  A free slot admits the oldest queued
// requests up to its query and key capacity, uploads them from pinned staging, runs
// the batched counting kernel with global accumulators over dense
// [query][reference] rows, compacts the nonzero cells into sparse hits on the device
// (re-zeroing the rows for the next batch) and copies the hits back.  Requests that
// arrive while batches run are admitted into the next free slot at once, so several
// batches overlap on the device.  A batch whose hits overflow the hit capacity is
// split: its requests go back to the front of the queue and run one per batch; only
// a request that overflows alone fails.  Every request's hits are the nonzero
// counter cells of kssdgpu_count_block for that query alone, sorted by reference id.
#pragma once

#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <thread>
#include <unordered_map>

namespace {

__global__ void k_server_compact(unsigned long long *__restrict__ rc, unsigned long long *__restrict__ ro,
                                 unsigned long long *__restrict__ urc, unsigned long long *__restrict__ uro, int nq,
                                 int nref, kssdgpu_hit_t *__restrict__ hits, unsigned int *__restrict__ count,
                                 unsigned int cap)
{
    // one CTA per query row: coalesced scan, nonzero cells appended, row re-zeroed
    for (int q = blockIdx.x; q < nq; q += gridDim.x) {
        const size_t row = (size_t)q * nref;
        for (int r = threadIdx.x; r < nref; r += blockDim.x) {
            const unsigned long long c = rc[row + r];
            const unsigned long long uc = urc ? urc[row + r] : 0ull;
            if (!c && !uc)
                continue;
            const unsigned long long o = ro[row + r];
            const unsigned long long uo = uro ? uro[row + r] : 0ull;
            rc[row + r] = 0;
            ro[row + r] = 0;
            if (urc) {
                urc[row + r] = 0;
                uro[row + r] = 0;
            }
            const unsigned int at = atomicAdd(count, 1u);
            if (at < cap) {
                kssdgpu_hit_t h;
                h.query = (uint32_t)q;
                h.ref = (uint32_t)r;
                h.num_ctx = (uint32_t)c;
                h.num_mut2_ctx = (uint32_t)(c >> 32);
                h.diff_obj = (uint32_t)o;
                h.diff_obj_section = (uint32_t)(o >> 32);
                h.u_num_ctx = (uint32_t)uc;
                h.u_num_mut2_ctx = (uint32_t)(uc >> 32);
                h.u_diff_obj = (uint32_t)uo;
                h.u_diff_obj_section = (uint32_t)(uo >> 32);
                hits[at] = h;
            }
        }
    }
}

struct ServerRequest {
    uint64_t ticket = 0;
    std::vector<uint64_t> keys;
    std::vector<kssdgpu_hit_t> hits;
    double t_submit = 0, t_done = 0;
    int status = KSSDGPU_OK;
    std::string error;
    bool done = false;
    bool solo = false;  // re-run alone after its batch overflowed the hit capacity
};

double now_ms()
{
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct ServerSlot {
    uint64_t *d_keys = nullptr, *d_offs = nullptr;
    unsigned long long *d_rc = nullptr, *d_ro = nullptr, *d_urc = nullptr, *d_uro = nullptr;
    kssdgpu_hit_t *d_hits = nullptr;
    unsigned int *d_count = nullptr, *d_work = nullptr;
    uint64_t *h_keys = nullptr, *h_offs = nullptr;
    WorkItem *d_items = nullptr, *h_items = nullptr;
    unsigned int *h_count = nullptr;
    kssdgpu_hit_t *h_hits = nullptr;
    cudaStream_t st = nullptr;
    cudaEvent_t ev = nullptr;
    std::vector<std::shared_ptr<ServerRequest>> batch;
    bool busy = false;
};

}  // namespace

struct kssdgpu_server {
    kssdgpu_index *ix = nullptr;
    kssdgpu_server_config_t cfg{};
    unsigned hit_cap = 0;
    std::vector<ServerSlot> slots;
    uint64_t slot_bytes = 0;  // device memory reserved per slot
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<std::shared_ptr<ServerRequest>> pending;
    std::unordered_map<uint64_t, std::shared_ptr<ServerRequest>> live;
    uint64_t next_ticket = 1;
    bool stop = false;
    std::thread worker;
    // statistics (under mu)
    std::vector<double> latencies;
    uint64_t batches = 0, queries = 0, max_inflight = 0, overlapped = 0, splits = 0;
    int fatal = KSSDGPU_OK;
    std::string fatal_msg;
};

namespace {

// chunks of a full batch: every query may end in a partial chunk
size_t server_item_cap(const kssdgpu_server_config_t &c)
{
    return (size_t)(c.max_batch_keys / kChunkKeys) + (size_t)c.max_batch_queries + 1;
}

// Device bytes one slot reserves: keys, offsets, work items, dense counter rows
// (twice with unique contexts), hits and two counters.
uint64_t server_slot_bytes(const kssdgpu_server_config_t &c, int nref, unsigned hit_cap)
{
    const uint64_t cells = (uint64_t)c.max_batch_queries * (uint64_t)nref;
    return c.max_batch_keys * 8 + ((uint64_t)c.max_batch_queries + 1) * 8 + server_item_cap(c) * sizeof(WorkItem) +
           cells * 16 * ((c.flags & KSSDGPU_UNIQUE) ? 2 : 1) + (uint64_t)hit_cap * sizeof(kssdgpu_hit_t) + 8;
}

bool any_busy(const kssdgpu_server *s)
{
    for (const auto &sl : s->slots)
        if (sl.busy)
            return true;
    return false;
}

int server_slot_alloc(kssdgpu_server *s, ServerSlot &sl)
{
    const auto &c = s->cfg;
    const size_t cells = (size_t)c.max_batch_queries * s->ix->nref;
    const bool uq = (c.flags & KSSDGPU_UNIQUE) != 0;
    CUDA_TRY(cudaMalloc(&sl.d_keys, std::max<uint64_t>(c.max_batch_keys, 1) * 8));
    CUDA_TRY(cudaMalloc(&sl.d_offs, ((size_t)c.max_batch_queries + 1) * 8));
    CUDA_TRY(cudaMalloc(&sl.d_items, server_item_cap(c) * sizeof(WorkItem)));
    CUDA_TRY(cudaMalloc(&sl.d_rc, cells * 8));
    CUDA_TRY(cudaMalloc(&sl.d_ro, cells * 8));
    CUDA_TRY(cudaMemset(sl.d_rc, 0, cells * 8));
    CUDA_TRY(cudaMemset(sl.d_ro, 0, cells * 8));
    if (uq) {
        CUDA_TRY(cudaMalloc(&sl.d_urc, cells * 8));
        CUDA_TRY(cudaMalloc(&sl.d_uro, cells * 8));
        CUDA_TRY(cudaMemset(sl.d_urc, 0, cells * 8));
        CUDA_TRY(cudaMemset(sl.d_uro, 0, cells * 8));
    }
    CUDA_TRY(cudaMalloc(&sl.d_hits, (size_t)s->hit_cap * sizeof(kssdgpu_hit_t)));
    CUDA_TRY(cudaMalloc(&sl.d_count, sizeof(unsigned int)));
    CUDA_TRY(cudaMalloc(&sl.d_work, sizeof(unsigned int)));
    CUDA_TRY(cudaMallocHost(&sl.h_keys, std::max<uint64_t>(c.max_batch_keys, 1) * 8));
    CUDA_TRY(cudaMallocHost(&sl.h_offs, ((size_t)c.max_batch_queries + 1) * 8));
    CUDA_TRY(cudaMallocHost(&sl.h_items, server_item_cap(c) * sizeof(WorkItem)));
    CUDA_TRY(cudaMallocHost(&sl.h_count, sizeof(unsigned int)));
    CUDA_TRY(cudaMallocHost(&sl.h_hits, (size_t)s->hit_cap * sizeof(kssdgpu_hit_t)));
    CUDA_TRY(cudaStreamCreateWithFlags(&sl.st, cudaStreamNonBlocking));
    CUDA_TRY(cudaEventCreateWithFlags(&sl.ev, cudaEventDisableTiming));
    return KSSDGPU_OK;
}

void server_slot_free(ServerSlot &sl)
{
    cudaFree(sl.d_keys);
    cudaFree(sl.d_offs);
    cudaFree(sl.d_items);
    cudaFree(sl.d_rc);
    cudaFree(sl.d_ro);
    cudaFree(sl.d_urc);
    cudaFree(sl.d_uro);
    cudaFree(sl.d_hits);
    cudaFree(sl.d_count);
    cudaFree(sl.d_work);
    cudaFreeHost(sl.h_keys);
    cudaFreeHost(sl.h_offs);
    cudaFreeHost(sl.h_items);
    cudaFreeHost(sl.h_count);
    cudaFreeHost(sl.h_hits);
    if (sl.st)
        cudaStreamDestroy(sl.st);
    if (sl.ev)
        cudaEventDestroy(sl.ev);
    sl = ServerSlot();
}

// Launch one admitted batch on a slot (worker thread; mu not held).
int server_launch(kssdgpu_server *s, ServerSlot &sl)
{
    const int nq = (int)sl.batch.size();
    uint64_t nk = 0;
    size_t nitems = 0;
    sl.h_offs[0] = 0;
    for (int i = 0; i < nq; ++i) {
        const auto &k = sl.batch[i]->keys;
        if (!k.empty())
            std::memcpy(sl.h_keys + nk, k.data(), k.size() * 8);
        // key-range chunks: a large request spreads over many SMs
        for (uint64_t c = nk; c < nk + k.size(); c += kChunkKeys)
            sl.h_items[nitems++] = WorkItem{(uint32_t)i, 0u, c, std::min<uint64_t>(nk + k.size(), c + kChunkKeys)};
        nk += k.size();
        sl.h_offs[i + 1] = nk;
    }
    if (nk)
        CUDA_TRY(cudaMemcpyAsync(sl.d_keys, sl.h_keys, nk * 8, cudaMemcpyHostToDevice, sl.st));
    CUDA_TRY(cudaMemcpyAsync(sl.d_offs, sl.h_offs, ((size_t)nq + 1) * 8, cudaMemcpyHostToDevice, sl.st));
    if (nitems)
        CUDA_TRY(cudaMemcpyAsync(sl.d_items, sl.h_items, nitems * sizeof(WorkItem), cudaMemcpyHostToDevice, sl.st));
    CUDA_TRY(cudaMemsetAsync(sl.d_count, 0, sizeof(unsigned int), sl.st));
    CountParams P{};
    P.table = s->ix->table;
    P.mask = s->ix->mask;
    P.post = s->ix->post;
    P.qkeys = sl.d_keys;
    P.qoffs = sl.d_offs;
    P.nq = nq;
    P.nref = s->ix->nref;
    P.obj_bits = s->ix->obj_bits;
    P.ignoreconflict = (s->cfg.flags & KSSDGPU_IGNORECONFLICT) ? 1 : 0;
    P.out_ctx = sl.d_rc;
    P.out_obj = sl.d_ro;
    P.out_uctx = sl.d_urc;
    P.out_uobj = sl.d_uro;
    P.work = sl.d_work;
    P.order = nullptr;
    P.chunk_keys = (uint32_t)kChunkKeys;
    P.items = sl.d_items;
    P.nitems = (int)nitems;
    P.err = s->ix->err;
    P.bloom = s->ix->count_filter ? s->ix->bloom : nullptr;
    P.bloom_mask = s->ix->bloom_mask;
    P.bloom_stripes = s->ix->bloom_stripes;
    P.bloom_bounds = s->ix->bloom_bounds;
    int rc = (s->cfg.flags & KSSDGPU_UNIQUE) ? launch_batched<false, true, false>(s->ix, P, 0, sl.st)
                                             : launch_batched<false, false, false>(s->ix, P, 0, sl.st);
    if (rc)
        return rc;
    k_server_compact<<<std::min(nq, s->ix->sms * 8), 256, 0, sl.st>>>(sl.d_rc, sl.d_ro, sl.d_urc, sl.d_uro, nq,
                                                                      s->ix->nref, sl.d_hits, sl.d_count, s->hit_cap);
    count_launch();
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(sl.h_count, sl.d_count, sizeof(unsigned int), cudaMemcpyDeviceToHost, sl.st));
    CUDA_TRY(cudaEventRecord(sl.ev, sl.st));
    sl.busy = true;
    return KSSDGPU_OK;
}

// Collect a finished slot: copy the hits back and hand them to their requests.
int server_finish(kssdgpu_server *s, ServerSlot &sl)
{
    const unsigned n = *sl.h_count;
    int status = KSSDGPU_OK;
    std::string msg;
    if (n > s->hit_cap && sl.batch.size() > 1) {
        // split: the requests go back to the front of the queue, in order, to run
        // alone (the compaction re-zeroed every row, so the slot is clean)
        {
            std::lock_guard<std::mutex> lock(s->mu);
            for (auto it = sl.batch.rbegin(); it != sl.batch.rend(); ++it) {
                (*it)->solo = true;
                s->pending.push_front(*it);
            }
            s->splits++;
        }
        sl.batch.clear();
        sl.busy = false;
        s->cv_work.notify_one();
        return KSSDGPU_OK;
    }
    if (n > s->hit_cap) {
        status = KSSDGPU_ERR_CAPACITY;
        msg = "query produced more nonzero cells (" + std::to_string(n) + ") than the server's hit capacity (" +
              std::to_string(s->hit_cap) + ")";
    } else if (n) {
        const cudaError_t e = cudaMemcpyAsync(sl.h_hits, sl.d_hits, (size_t)n * sizeof(kssdgpu_hit_t),
                                              cudaMemcpyDeviceToHost, sl.st);
        const cudaError_t e2 = e == cudaSuccess ? cudaStreamSynchronize(sl.st) : e;
        if (e2 != cudaSuccess) {
            status = KSSDGPU_ERR_CUDA;
            msg = cudaGetErrorString(e2);
        }
    }
    std::vector<std::vector<kssdgpu_hit_t>> per(sl.batch.size());
    if (status == KSSDGPU_OK)
        for (unsigned i = 0; i < n; ++i)
            per[sl.h_hits[i].query].push_back(sl.h_hits[i]);
    const double t = now_ms();
    {
        std::lock_guard<std::mutex> lock(s->mu);
        for (size_t i = 0; i < sl.batch.size(); ++i) {
            auto &r = sl.batch[i];
            auto &h = per[i];
            std::sort(h.begin(), h.end(), [](const kssdgpu_hit_t &a, const kssdgpu_hit_t &b) { return a.ref < b.ref; });
            for (auto &x : h)
                x.query = 0;
            r->hits = std::move(h);
            r->status = status;
            r->error = msg;
            r->t_done = t;
            r->done = true;
            r->keys.clear();
            r->keys.shrink_to_fit();
            s->latencies.push_back(t - r->t_submit);
        }
        s->batches++;
        s->queries += sl.batch.size();
    }
    s->cv_done.notify_all();
    sl.batch.clear();
    sl.busy = false;
    return KSSDGPU_OK;
}

void server_loop(kssdgpu_server *s)
{
    cudaSetDevice(s->ix->device);
    for (;;) {
        bool progressed = false;
        // collect finished batches
        for (auto &sl : s->slots)
            if (sl.busy && cudaEventQuery(sl.ev) == cudaSuccess) {
                server_finish(s, sl);
                progressed = true;
            }
        // admit into free slots
        for (auto &sl : s->slots) {
            if (sl.busy)
                continue;
            {
                std::lock_guard<std::mutex> lock(s->mu);
                uint64_t keys = 0;
                while (!s->pending.empty() && sl.batch.size() < (size_t)s->cfg.max_batch_queries &&
                       keys + s->pending.front()->keys.size() <= s->cfg.max_batch_keys) {
                    const bool solo = s->pending.front()->solo;
                    if (solo && !sl.batch.empty())
                        break;  // a split request runs in a batch of its own
                    keys += s->pending.front()->keys.size();
                    sl.batch.push_back(std::move(s->pending.front()));
                    s->pending.pop_front();
                    if (solo)
                        break;
                }
                if (!sl.batch.empty()) {
                    uint64_t inflight = sl.batch.size();
                    for (const auto &o : s->slots)
                        if (o.busy)
                            inflight += o.batch.size();
                    if (any_busy(s))
                        s->overlapped++;
                    s->max_inflight = std::max<uint64_t>(s->max_inflight, inflight);
                }
            }
            if (sl.batch.empty())
                continue;
            const int rc = server_launch(s, sl);
            if (rc) {
                std::lock_guard<std::mutex> lock(s->mu);
                s->fatal = rc;
                s->fatal_msg = g_last_error;
                for (auto &r : sl.batch) {
                    r->status = rc;
                    r->error = g_last_error;
                    r->done = true;
                    r->t_done = now_ms();
                }
                sl.batch.clear();
                sl.busy = false;
                s->cv_done.notify_all();
            }
            progressed = true;
        }
        std::unique_lock<std::mutex> lock(s->mu);
        if (s->stop && s->pending.empty() && !any_busy(s))
            break;
        if (!progressed) {
            if (any_busy(s)) {
                lock.unlock();
                std::this_thread::sleep_for(std::chrono::microseconds(20));
            } else {
                // idle: wait for a submission (bounded, so stop is always seen)
                s->cv_work.wait_for(lock, std::chrono::milliseconds(5));
            }
        }
    }
}

}  // namespace

extern "C" {

int kssdgpu_server_create(kssdgpu_index_t *ix, const kssdgpu_server_config_t *cfg, kssdgpu_server_t **out)
{
    if (!ix || !cfg || !out)
        return fail(KSSDGPU_ERR_ARG, "null argument");
    if (cfg->max_batch_queries <= 0 || cfg->max_batch_keys == 0 || cfg->slots < 0)
        return fail(KSSDGPU_ERR_ARG, "server batch capacity and slot count must be positive");
    CUDA_TRY(cudaSetDevice(ix->device));
    const uint64_t dense = (uint64_t)cfg->max_batch_queries * (uint64_t)ix->nref;
    const unsigned hit_cap = (unsigned)std::min<uint64_t>(dense, cfg->max_hits ? cfg->max_hits : (1ull << 22));
    const uint64_t per_slot = server_slot_bytes(*cfg, ix->nref, hit_cap);
    uint64_t budget = cfg->device_budget;
    if (!budget) {
        size_t free_b = 0, total_b = 0;
        CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
        budget = free_b / 2;
    }
    const uint64_t fit = budget / std::max<uint64_t>(per_slot, 1);
    const int want = cfg->slots ? cfg->slots : 4;
    if (fit < 1)
        return fail(KSSDGPU_ERR_CAPACITY, "one server slot needs " + std::to_string(per_slot) +
                                              " bytes of device memory, above the budget of " + std::to_string(budget));
    auto *s = new kssdgpu_server();
    s->ix = ix;
    s->cfg = *cfg;
    s->hit_cap = hit_cap;
    s->slot_bytes = per_slot;
    s->slots.resize((size_t)std::min<uint64_t>((uint64_t)want, fit));
    for (auto &sl : s->slots) {
        const int rc = server_slot_alloc(s, sl);
        if (rc) {
            for (auto &x : s->slots)
                server_slot_free(x);
            delete s;
            return rc;
        }
    }
    s->worker = std::thread(server_loop, s);
    *out = s;
    return KSSDGPU_OK;
}

int kssdgpu_server_submit(kssdgpu_server_t *s, const uint64_t *keys, uint64_t n_keys, uint64_t *ticket)
{
    if (!s || !ticket || (n_keys && !keys))
        return fail(KSSDGPU_ERR_ARG, "invalid submit arguments");
    if (n_keys > s->cfg.max_batch_keys)
        return fail(KSSDGPU_ERR_CAPACITY, "query has more keys than a server slot admits (" +
                                              std::to_string(s->cfg.max_batch_keys) + ")");
    for (uint64_t i = 1; i < n_keys; ++i)
        if (keys[i - 1] > keys[i])
            return fail(KSSDGPU_ERR_UNSORTED, "query keys are not sorted ascending (position " + std::to_string(i) + ")");
    auto r = std::make_shared<ServerRequest>();
    r->keys.assign(keys, keys + n_keys);
    {
        std::lock_guard<std::mutex> lock(s->mu);
        if (s->fatal)
            return fail(s->fatal, "server stopped after a device error: " + s->fatal_msg);
        r->ticket = s->next_ticket++;
        r->t_submit = now_ms();
        s->live[r->ticket] = r;
        s->pending.push_back(r);
        *ticket = r->ticket;
    }
    s->cv_work.notify_one();
    return KSSDGPU_OK;
}

int kssdgpu_server_wait(kssdgpu_server_t *s, uint64_t ticket, int timeout_ms, uint32_t *n_hits, double *latency_ms)
{
    if (!s)
        return fail(KSSDGPU_ERR_ARG, "null server");
    std::unique_lock<std::mutex> lock(s->mu);
    auto it = s->live.find(ticket);
    if (it == s->live.end())
        return fail(KSSDGPU_ERR_ARG, "unknown ticket");
    auto r = it->second;
    const auto pred = [&] { return r->done; };
    if (timeout_ms < 0)
        s->cv_done.wait(lock, pred);
    else if (!s->cv_done.wait_for(lock, std::chrono::milliseconds(timeout_ms), pred))
        return fail(KSSDGPU_ERR_TIMEOUT, "request not finished within the wait limit");
    if (r->status)
        return fail(r->status, r->error);
    if (n_hits)
        *n_hits = (uint32_t)r->hits.size();
    if (latency_ms)
        *latency_ms = r->t_done - r->t_submit;
    return KSSDGPU_OK;
}

int kssdgpu_server_take(kssdgpu_server_t *s, uint64_t ticket, kssdgpu_hit_t *hits, uint32_t cap)
{
    if (!s)
        return fail(KSSDGPU_ERR_ARG, "null server");
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->live.find(ticket);
    if (it == s->live.end())
        return fail(KSSDGPU_ERR_ARG, "unknown ticket");
    auto r = it->second;
    if (!r->done)
        return fail(KSSDGPU_ERR_ARG, "request not finished");
    if (r->hits.size() > cap)
        return fail(KSSDGPU_ERR_CAPACITY, "hit buffer too small");
    if (!r->hits.empty() && hits)
        std::memcpy(hits, r->hits.data(), r->hits.size() * sizeof(kssdgpu_hit_t));
    s->live.erase(it);
    return KSSDGPU_OK;
}

int kssdgpu_server_stats(kssdgpu_server_t *s, kssdgpu_server_stats_t *out)
{
    if (!s || !out)
        return fail(KSSDGPU_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> lock(s->mu);
    std::vector<double> l = s->latencies;
    std::sort(l.begin(), l.end());
    auto pct = [&](double p) { return l.empty() ? 0.0 : l[std::min(l.size() - 1, (size_t)(p * (l.size() - 1) + 0.5))]; };
    out->completed = l.size();
    out->batches = s->batches;
    out->pending = s->pending.size();
    out->max_inflight = s->max_inflight;
    out->overlapped_batches = s->overlapped;
    out->p50_ms = pct(0.50);
    out->p99_ms = pct(0.99);
    out->max_ms = l.empty() ? 0.0 : l.back();
    out->mean_ms = 0;
    for (double x : l)
        out->mean_ms += x;
    if (!l.empty())
        out->mean_ms /= (double)l.size();
    out->reserved_bytes = s->slot_bytes * s->slots.size();
    out->slots = s->slots.size();
    out->splits = s->splits;
    return KSSDGPU_OK;
}

int kssdgpu_server_reset_stats(kssdgpu_server_t *s)
{
    if (!s)
        return fail(KSSDGPU_ERR_ARG, "null server");
    std::lock_guard<std::mutex> lock(s->mu);
    s->latencies.clear();
    s->batches = s->queries = s->max_inflight = s->overlapped = s->splits = 0;
    return KSSDGPU_OK;
}

void kssdgpu_server_destroy(kssdgpu_server_t *s)
{
    if (!s)
        return;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->worker.joinable())
        s->worker.join();
    cudaSetDevice(s->ix->device);
    for (auto &sl : s->slots) {
        if (sl.st)
            cudaStreamSynchronize(sl.st);
        server_slot_free(sl);
    }
    delete s;
}

}  // extern "C"
