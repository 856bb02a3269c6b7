// gxy_server.cu -- serving loop over resident position tables.
//
// Requests (a query against one resident table, one or both strands) are
// copied in by gxy_server_submit and queued.  max_streams dispatcher threads
// each own a worker stream; a free dispatcher forms a batch from the queue,
// admitting requests in arrival order while the device-memory budget
// (max_device_bytes, and the device's actually free memory) and the unit
// limits allow, runs it through the same pipeline as gxy_batch_search, and
// hands each request its HSPs.  Requests that arrive while batches run are
// admitted by the next free dispatcher, so batches overlap on the device.
// Every unit's result is computed exactly as a lone search() would compute it
// (units never share diagonal state), so a request's HSPs are the same alone
// and in any mix.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <thread>
#include <vector>

#include "gxy_engine.cuh"

namespace gxy {
namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    uint64_t id = 0;
    uint32_t table = 0;
    std::vector<uint8_t> codes, valid, mask;
    uint64_t len = 0;
    uint64_t bytes = 0;                 // admission estimate
    Clock::time_point submitted;
    Clock::time_point done_at;
    bool done = false;
    bool canceled = false;
    gxy_status status = GXY_OK;
    gxy_status fault = GXY_OK;          // injected failure (test hook), GXY_OK when none
    std::vector<gxy_hsp> plus, minus;
};

}  // namespace
}  // namespace gxy

using namespace gxy;

struct gxy_server {
    gxy_ctx* ctx = nullptr;
    std::vector<const gxy_table*> tables;
    gxy_search_params params{};
    gxy_server_opts opts{};
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request*> pending;
    std::map<uint64_t, Request*> requests;
    std::vector<std::thread> threads;
    bool stop = false;
    uint64_t next_id = 1;
    uint64_t bytes_in_use = 0;
    uint64_t units_in_flight = 0;
    uint32_t big_in_flight = 0;
    uint32_t started = 0;               // dispatchers past their start-up (worker and warm buffers)
    gxy_server_stats st{};
    // Free device memory: cudaMemGetInfo once at creation (it can take tens
    // of milliseconds while the device works, so it stays off the dispatch
    // path), then less whatever the allocation pool has reserved since --
    // a host-side counter.
    size_t free_at_create = 0;
    uint64_t pool_at_create = 0;
    cudaMemPool_t pool = nullptr;
    // Other processes on a shared GPU allocate too, which the pool counter
    // cannot see: a monitor thread re-reads the free memory whenever the
    // server has been idle for kMemRefreshMs, off the dispatch path.
    std::thread monitor;
    std::condition_variable cv_stop;
    std::map<uint64_t, gxy_status> future_faults;   // injected faults of ids not yet submitted
};

static constexpr int kMemRefreshMs = 500;

namespace {

// Runs one batch of requests on worker W.  Called without the server lock.
gxy_status run_batch(gxy_server* s, Worker* W, std::vector<Request*>& batch) {
    cudaStream_t stream = W->st;
    {
        std::lock_guard<std::mutex> g(s->mu);
        for (Request* q : batch)
            if (q->fault != GXY_OK) {
                set_error("injected fault");
                return q->fault;
            }
    }
    const Pattern& pat = s->tables[0]->pat;
    std::vector<gxy_dseq*> owned;
    auto cleanup = [&]() {
        // Only this worker's stream used them: no device-wide sync.
        for (gxy_dseq* d : owned) dseq_destroy_async(d, stream);
    };
    std::vector<SeqView> tsegs, qsegs;
    std::vector<int> tseg_of(s->tables.size(), -1);
    std::vector<UnitPlan> plan;
    std::vector<std::pair<size_t, int>> unit_owner;   // (request index, strand)
    const int strands = s->opts.both_strands ? 2 : 1;
    uint64_t max_cols = 0;
    for (size_t r = 0; r < batch.size(); r++) {
        Request* q = batch[r];
        const gxy_table* t = s->tables[q->table];
        if (tseg_of[q->table] < 0) {
            tseg_of[q->table] = (int)tsegs.size();
            tsegs.push_back(table_view(t));
        }
        gxy_dseq* d = nullptr;
        gxy_status e = dseq_alloc(s->ctx, q->len, &d, stream);
        if (e != GXY_OK) {
            cleanup();
            return e;
        }
        owned.push_back(d);
        gxy_packed_seq h{q->codes.data(), q->valid.data(), q->mask.data(), q->len};
        e = dseq_fill_host(d, &h, stream);
        if (e != GXY_OK) {
            cleanup();
            return e;
        }
        max_cols = std::max<uint64_t>(max_cols, std::min<uint64_t>(t->hi - t->lo, q->len));
        for (int sd = 0; sd < strands; sd++) {
            const gxy_dseq* qs = d;
            if (sd == 1) {
                gxy_dseq* rc = nullptr;
                e = dseq_alloc(s->ctx, q->len, &rc, stream);
                if (e != GXY_OK) {
                    cleanup();
                    return e;
                }
                owned.push_back(rc);
                launch_reverse_complement(d->codes, d->valid, d->mask, d->len, rc->codes, rc->valid, rc->mask,
                                          stream);
                qs = rc;
            }
            UnitPlan u;
            u.tseg = (uint32_t)tseg_of[q->table];
            u.qseg = (uint32_t)qsegs.size();
            qsegs.push_back(view_of(qs, 0, qs->len));
            u.starts = t->starts;
            u.positions = t->positions;
            u.occ = t->occ;
            u.nwin = n_windows(q->len, pat.len, s->params.step);
            u.primary_lo = u.primary_hi = 0;
            u.avg_bucket = t->num_words ? (double)t->npos / (double)t->num_words : 0.0;
            plan.push_back(u);
            unit_owner.push_back({r, sd});
        }
    }
    gxy_status e = check_params(&s->params, max_cols);
    RunResult res;
    if (e == GXY_OK) e = run_units(s->ctx, W, plan, tsegs, qsegs, pat, s->params, false, res);
    cleanup();
    if (e != GXY_OK) return e;
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->st.reruns += res.stats.reruns;
        s->st.busy_ms += res.stats.device_ms;
    }
    for (size_t i = 0; i < res.hsps.size(); i++) {
        const auto& o = unit_owner[res.unit[i]];
        (o.second ? batch[o.first]->minus : batch[o.first]->plus).push_back(res.hsps[i]);
    }
    return GXY_OK;
}

void dispatcher(gxy_server* s) {
    cudaSetDevice(s->ctx->device);
    gxy_status err;
    Worker* W = checkout(s->ctx, &err);
    if (!W) {
        std::lock_guard<std::mutex> g(s->mu);
        for (Request* q : s->pending) {
            q->status = err;
            q->done = true;
            q->done_at = Clock::now();
        }
        s->pending.clear();
        s->started++;
        s->cv_done.notify_all();
        return;
    }
    const uint32_t strands = s->opts.both_strands ? 2 : 1;
    if (s->opts.warm_bases) {
        // The raw-hit estimate run_units makes for a query of warm_bases on
        // the largest table (windows x variants x mean bucket, 1.5x margin).
        const Pattern& pat = s->tables[0]->pat;
        const uint32_t w = pat.weight;
        const double n_var = 1.0 + (s->params.transitions >= 1 ? w : 0) +
                             (s->params.transitions >= 2 ? w * (w - 1) / 2.0 : 0.0);
        double avg = 0.0;
        for (const gxy_table* t : s->tables)
            if (t->num_words) avg = std::max(avg, (double)t->npos / (double)t->num_words);
        const double est = (double)(1 << 20) + 1.5 * (double)s->opts.warm_bases * n_var * avg * strands;
        reserve_worker(s->ctx, W, (uint64_t)est, (uint64_t)(est / kHitsPerCandidate), s->opts.max_batch_units);
    }
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->started++;
    }
    s->cv_done.notify_all();
    for (;;) {
        std::vector<Request*> batch;
        bool batch_big = false;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_work.wait(lk, [&] { return s->stop || !s->pending.empty(); });
            if (s->stop && s->pending.empty()) break;
            // Free memory now: what was free at creation, less the pool's
            // growth since, less the estimates of the requests in flight
            // (their buffers may not be allocated yet).
            uint64_t reserved = 0;
            if (s->pool) cudaMemPoolGetAttribute(s->pool, cudaMemPoolAttrReservedMemCurrent, &reserved);
            const uint64_t grown = (reserved > s->pool_at_create ? reserved - s->pool_at_create : 0) + s->bytes_in_use;
            size_t free_b = s->free_at_create > grown ? s->free_at_create - grown : 0;
            uint64_t batch_units = 0, batch_bases = 0;
            // Arrival order, except that a big request waits in place (and
            // the smaller ones behind it go ahead) while the big slots are
            // taken; a big request always runs in a batch of its own.  A
            // batch holds requests of one table only: the table's bucket
            // bounds then stay in L2 for the whole launch.
            for (auto it = s->pending.begin(); it != s->pending.end();) {
                Request* q = *it;
                const bool big = q->len >= s->opts.big_bases;
                if ((big && (!batch.empty() || s->big_in_flight >= s->opts.max_big_inflight)) ||
                    (!batch.empty() && q->table != batch[0]->table)) {
                    ++it;
                    continue;
                }
                const bool fits_mem = s->bytes_in_use + q->bytes <= s->opts.max_device_bytes &&
                                      q->bytes + (64ull << 20) <= free_b;
                const bool fits_units = s->units_in_flight + strands <= s->opts.max_units;
                // The per-batch limits bound what joins a batch, never its first request.
                const bool fits_batch = batch.empty() ||
                                        (batch_units + strands <= s->opts.max_batch_units &&
                                         batch_bases + (uint64_t)q->len * strands <= s->opts.max_batch_bases);
                // A request that could never fit alone is still run alone.
                const bool alone = batch.empty() && s->units_in_flight == 0;
                if (!(fits_mem && fits_units && fits_batch) && !alone) break;
                it = s->pending.erase(it);
                batch.push_back(q);
                s->bytes_in_use += q->bytes;
                s->units_in_flight += strands;
                batch_units += strands;
                batch_bases += (uint64_t)q->len * strands;
                if (free_b > q->bytes) free_b -= q->bytes;
                if (big) {
                    batch_big = true;
                    s->big_in_flight++;
                    break;
                }
            }
            if (batch.empty()) {
                // Budget taken by batches in flight: wait for one to finish.
                s->cv_done.wait_for(lk, std::chrono::milliseconds(2));
                continue;
            }
            s->st.batches++;
            s->st.max_inflight_units = std::max<uint64_t>(s->st.max_inflight_units, s->units_in_flight);
            s->st.bytes_in_use = s->bytes_in_use;
        }
        std::vector<gxy_status> status(batch.size(), run_batch(s, W, batch));
        if (status[0] != GXY_OK && batch.size() > 1) {
            // One request's failure (an allocation, an input outside the
            // exact envelope) must not fail its batch-mates: rerun the
            // requests one at a time, each with its own status.
            {
                std::lock_guard<std::mutex> g(s->mu);
                s->st.isolated++;
            }
            for (size_t i = 0; i < batch.size(); i++) {
                std::vector<Request*> one{batch[i]};
                batch[i]->plus.clear();
                batch[i]->minus.clear();
                status[i] = run_batch(s, W, one);
            }
        }
        {
            std::lock_guard<std::mutex> g(s->mu);
            const auto now = Clock::now();
            if (batch_big) s->big_in_flight--;
            for (size_t i = 0; i < batch.size(); i++) {
                Request* q = batch[i];
                q->status = q->canceled ? GXY_ECANCELED : status[i];
                if (q->status != GXY_OK) {
                    q->plus.clear();
                    q->minus.clear();
                    if (q->canceled) s->st.canceled++;
                    else s->st.failed++;
                }
                q->done = true;
                q->done_at = now;
                q->codes.clear();
                q->codes.shrink_to_fit();
                q->valid.clear();
                q->valid.shrink_to_fit();
                q->mask.clear();
                q->mask.shrink_to_fit();
                s->bytes_in_use -= q->bytes;
                s->units_in_flight -= strands;
                s->st.completed++;
            }
            s->st.bytes_in_use = s->bytes_in_use;
        }
        s->cv_done.notify_all();
        s->cv_work.notify_all();
    }
    checkin(s->ctx, W);
}

// Re-reads the device's free memory at most every kMemRefreshMs, and only
// while the server is idle (no request queued or in flight): cudaMemGetInfo
// can take tens of milliseconds on a busy device and holds up the other
// threads' CUDA calls meanwhile, so it never runs under a batch.  The
// admission estimate is re-based on what it returns.
void memory_monitor(gxy_server* s) {
    cudaSetDevice(s->ctx->device);
    std::unique_lock<std::mutex> lk(s->mu);
    while (!s->stop) {
        s->cv_stop.wait_for(lk, std::chrono::milliseconds(kMemRefreshMs), [&] { return s->stop; });
        if (s->stop) break;
        if (s->units_in_flight || !s->pending.empty()) continue;
        lk.unlock();
        size_t free_b = 0, total_b = 0;
        uint64_t reserved = 0;
        const bool ok = cudaMemGetInfo(&free_b, &total_b) == cudaSuccess;
        if (ok && s->pool) cudaMemPoolGetAttribute(s->pool, cudaMemPoolAttrReservedMemCurrent, &reserved);
        cudaGetLastError();
        lk.lock();
        if (ok) {
            // Free memory now already excludes the pool's current reservation.
            s->free_at_create = free_b;
            s->pool_at_create = reserved;
            s->st.mem_refreshes++;
        }
    }
}

gxy_status copy_out(const std::vector<gxy_hsp>& v, gxy_hsp_buf* out) {
    if (!out) return GXY_OK;
    out->len = v.size();
    out->cap = v.size();
    out->hsps = static_cast<gxy_hsp*>(malloc(std::max<size_t>(v.size(), 1) * sizeof(gxy_hsp)));
    if (!out->hsps) return GXY_ENOMEM;
    if (!v.empty()) memcpy(out->hsps, v.data(), v.size() * sizeof(gxy_hsp));
    return GXY_OK;
}

}  // namespace

extern "C" {

gxy_status gxy_server_create(gxy_ctx* ctx, uint32_t n_tables, const gxy_table* const* tables,
                             const gxy_search_params* params, const gxy_server_opts* opts, gxy_server** out) {
    if (!ctx || !n_tables || !tables || !params || !out) return GXY_EINVAL;
    for (uint32_t i = 0; i < n_tables; i++) {
        if (!tables[i]) return GXY_EINVAL;
        if (tables[i]->pat.len != tables[0]->pat.len || tables[i]->pat.care_mask != tables[0]->pat.care_mask) {
            set_error("all resident tables of a server must share one seed pattern");
            return GXY_EINVAL;
        }
    }
    if (params->step < 1) {
        set_error("step must be >= 1");
        return GXY_EINVAL;
    }
    gxy_server* s = new gxy_server();
    s->ctx = ctx;
    {
        cudaSetDevice(ctx->device);
        size_t total_b = 0;
        if (cudaMemGetInfo(&s->free_at_create, &total_b) != cudaSuccess) s->free_at_create = SIZE_MAX;
        if (cudaDeviceGetDefaultMemPool(&s->pool, ctx->device) != cudaSuccess) s->pool = nullptr;
        if (s->pool) cudaMemPoolGetAttribute(s->pool, cudaMemPoolAttrReservedMemCurrent, &s->pool_at_create);
        cudaGetLastError();
    }
    s->tables.assign(tables, tables + n_tables);
    s->params = *params;
    gxy_server_opts o = opts ? *opts : gxy_server_opts{};
    if (!o.max_device_bytes) o.max_device_bytes = 16ull << 30;
    if (!o.max_units) o.max_units = 8192;
    if (!o.max_streams) o.max_streams = 2;
    if (!o.max_batch_units) o.max_batch_units = 1024;
    if (!o.max_batch_bases) o.max_batch_bases = 16ull << 20;
    // Batches no larger than the warmed buffers: one that outgrew them would
    // reallocate gigabytes while requests wait.
    if (o.warm_bases) o.max_batch_bases = std::min<uint64_t>(o.max_batch_bases, o.warm_bases * (o.both_strands ? 2 : 1));
    if (!o.big_bases) o.big_bases = 1ull << 20;
    if (!o.max_big_inflight) o.max_big_inflight = 1;
    s->opts = o;
    for (uint32_t i = 0; i < o.max_streams; i++) s->threads.emplace_back(dispatcher, s);
    s->monitor = std::thread(memory_monitor, s);
    if (o.warm_bases) {
        // Return once every dispatcher holds its warmed buffers.
        std::unique_lock<std::mutex> lk(s->mu);
        s->cv_done.wait(lk, [&] { return s->started >= o.max_streams; });
    }
    *out = s;
    return GXY_OK;
}

gxy_status gxy_server_submit(gxy_server* s, uint32_t table, const gxy_packed_seq* query, uint64_t* request_id) {
    if (!s || !query || !request_id || table >= s->tables.size()) return GXY_EINVAL;
    if (query->len && (!query->codes || !query->valid || !query->mask)) return GXY_EINVAL;
    if (query->len >= (1ull << 32)) return GXY_EUNSUPPORTED;
    Request* q = new Request();
    q->table = table;
    q->len = query->len;
    q->codes.assign(query->codes, query->codes + (query->len + 3) / 4);
    q->valid.assign(query->valid, query->valid + (query->len + 7) / 8);
    q->mask.assign(query->mask, query->mask + (query->len + 7) / 8);
    // Device bytes while in flight: the query and its reverse complement
    // (0.5 B/bp each with pads) plus a per-base share of the raw-hit and
    // candidate scratch.
    q->bytes = (uint64_t)q->len * 24 + (1u << 20);
    q->submitted = Clock::now();
    {
        std::lock_guard<std::mutex> g(s->mu);
        if (s->stop) {
            delete q;
            return GXY_EINVAL;
        }
        q->id = s->next_id++;
        auto f = s->future_faults.find(q->id);
        if (f != s->future_faults.end()) {
            q->fault = f->second;
            s->future_faults.erase(f);
        }
        s->requests[q->id] = q;
        s->pending.push_back(q);
        s->st.submitted++;
        *request_id = q->id;
    }
    s->cv_work.notify_one();
    return GXY_OK;
}

gxy_status gxy_server_wait(gxy_server* s, uint64_t request_id, uint32_t timeout_ms, gxy_hsp_buf* plus,
                           gxy_hsp_buf* minus, double* latency_ms) {
    if (!s) return GXY_EINVAL;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->requests.find(request_id);
    if (it == s->requests.end()) {
        set_error("unknown request id");
        return GXY_EINVAL;
    }
    Request* q = it->second;
    if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] { return q->done; })) {
        set_error("request still running after the timeout");
        return GXY_ETIMEDOUT;
    }
    s->requests.erase(it);
    lk.unlock();
    gxy_status e = q->status;
    if (e == GXY_OK) e = copy_out(q->plus, plus);
    if (e == GXY_OK) e = copy_out(q->minus, minus);
    if (latency_ms) latency_ms[0] = std::chrono::duration<double, std::milli>(q->done_at - q->submitted).count();
    delete q;
    return e;
}

gxy_status gxy_server_get_stats(gxy_server* s, gxy_server_stats* st) {
    if (!s || !st) return GXY_EINVAL;
    std::lock_guard<std::mutex> g(s->mu);
    *st = s->st;
    return GXY_OK;
}

gxy_status gxy_server_cancel(gxy_server* s, uint64_t request_id) {
    if (!s) return GXY_EINVAL;
    std::lock_guard<std::mutex> g(s->mu);
    auto it = s->requests.find(request_id);
    if (it == s->requests.end()) {
        set_error("unknown request id");
        return GXY_EINVAL;
    }
    Request* q = it->second;
    if (q->done) return GXY_OK;
    q->canceled = true;
    auto p = std::find(s->pending.begin(), s->pending.end(), q);
    if (p != s->pending.end()) {
        // Still queued: it never reaches the device.
        s->pending.erase(p);
        q->status = GXY_ECANCELED;
        q->done = true;
        q->done_at = Clock::now();
        q->codes.clear();
        q->valid.clear();
        q->mask.clear();
        s->st.canceled++;
        s->st.completed++;
        s->cv_done.notify_all();
    }
    return GXY_OK;
}

gxy_status gxy_server_inject_fault(gxy_server* s, uint64_t request_id, gxy_status status) {
    if (!s) return GXY_EINVAL;
    std::lock_guard<std::mutex> g(s->mu);
    auto it = s->requests.find(request_id);
    if (it == s->requests.end()) {
        if (request_id >= s->next_id) {
            // Ids are handed out in submission order: the fault waits for it.
            s->future_faults[request_id] = status;
            return GXY_OK;
        }
        set_error("unknown request id");
        return GXY_EINVAL;
    }
    it->second->fault = status;
    return GXY_OK;
}

gxy_status gxy_server_destroy(gxy_server* s) {
    if (!s) return GXY_OK;
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    s->cv_stop.notify_all();
    if (s->monitor.joinable()) s->monitor.join();
    for (auto& t : s->threads) t.join();
    for (auto& kv : s->requests) delete kv.second;
    delete s;
    return GXY_OK;
}

}  // extern "C"
