// gxy_engine.cu -- the host engine: device sequences, workers, and the
// screen -> sort -> walk -> compaction pipeline over a list of units.
#include "gxy_engine.cuh"

#include <algorithm>
#include <cmath>
#include <atomic>
#include <cstdlib>
#include <cstring>

namespace gxy {

static thread_local std::string g_err;
static std::atomic<uint64_t> g_launches{0};
void count_launch(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
uint64_t launches() { return g_launches.load(std::memory_order_relaxed); }
void set_error(const std::string& msg) { g_err = msg; }
const char* last_error() { return g_err.c_str(); }

#define API_TRY_ENGINE(expr)          \
    do {                              \
        gxy_status s_ = (expr);       \
        if (s_ != GXY_OK) return s_;  \
    } while (0)

cudaError_t DevBuf::ensure(size_t need) {
    if (need <= bytes && p) return cudaSuccess;
    if (p) cudaFreeAsync(p, st);
    p = nullptr;
    bytes = 0;
    size_t b = need < 256 ? 256 : need;
    cudaError_t e = cudaMallocAsync(&p, b, st);
    if (e == cudaSuccess) bytes = b;
    return e;
}
void DevBuf::release() {
    if (p) cudaFreeAsync(p, st);
    p = nullptr;
    bytes = 0;
}

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

cudaError_t dev_alloc(void** p, size_t bytes, cudaStream_t st) {
    return cudaMallocAsync(p, bytes ? bytes : 256, st);
}

void dev_free(void* p) {
    if (!p) return;
    // Pool memory goes back after every stream that may still use it is done.
    cudaDeviceSynchronize();
    cudaFreeAsync(p, 0);
    cudaStreamSynchronize(0);
}

gxy_status dseq_alloc(gxy_ctx* ctx, uint64_t len, gxy_dseq** out, cudaStream_t st) {
    gxy_dseq* d = new gxy_dseq();
    d->ctx = ctx;
    d->device = ctx->device;
    d->len = len;
    uint64_t nw = (kPad + len + kTailPad + 31) / 32;
    nw = (nw + 3) & ~3ull;   // each array a multiple of 16 bytes
    d->nwords = nw;
    const size_t cb = align256(nw * 8), vb = align256(nw * 4);
    d->bytes = cb + 2 * vb;
    cudaError_t e = dev_alloc(&d->alloc, d->bytes, st);
    if (e != cudaSuccess) {
        delete d;
        set_error(std::string("cudaMallocAsync(sequence): ") + cudaGetErrorString(e));
        return GXY_ENOMEM;
    }
    d->st = st;
    d->codes = static_cast<uint64_t*>(d->alloc);
    d->valid = reinterpret_cast<uint32_t*>(static_cast<char*>(d->alloc) + cb);
    d->mask = reinterpret_cast<uint32_t*>(static_cast<char*>(d->alloc) + cb + vb);
    e = cudaMemsetAsync(d->alloc, 0, d->bytes, st);
    if (e != cudaSuccess) {
        dev_free(d->alloc);
        delete d;
        set_error(std::string("cudaMemsetAsync(sequence): ") + cudaGetErrorString(e));
        return GXY_ECUDA;
    }
    *out = d;
    return GXY_OK;
}

void dseq_destroy_async(gxy_dseq* s, cudaStream_t st) {
    if (!s) return;
    if (s->alloc) cudaFreeAsync(s->alloc, st);
    delete s;
}

void dseq_destroy(gxy_dseq* s) {
    if (!s) return;
    dev_free(s->alloc);
    delete s;
}

gxy_status dseq_fill_host(gxy_dseq* d, const gxy_packed_seq* h, cudaStream_t st) {
    const uint64_t n = h->len;
    if (!n) return GXY_OK;
    GXY_CK(cudaMemcpyAsync(reinterpret_cast<char*>(d->codes) + kPad / 4, h->codes, (n + 3) / 4,
                           cudaMemcpyHostToDevice, st));
    GXY_CK(cudaMemcpyAsync(reinterpret_cast<char*>(d->valid) + kPad / 8, h->valid, (n + 7) / 8,
                           cudaMemcpyHostToDevice, st));
    GXY_CK(cudaMemcpyAsync(reinterpret_cast<char*>(d->mask) + kPad / 8, h->mask, (n + 7) / 8,
                           cudaMemcpyHostToDevice, st));
    return GXY_OK;
}

SeqView view_of(const gxy_dseq* s, uint64_t lo, uint64_t hi) {
    SeqView v;
    v.codes = s->codes;
    v.valid = s->valid;
    v.mask = s->mask;
    v.base = kPad + lo;
    v.len = (uint32_t)(hi - lo);
    v.key_base = 0;
    return v;
}

SeqView table_view(const gxy_table* t) {
    SeqView v = view_of(t->seq, t->lo, t->hi);
    if (t->mem && t->mem->ilv) {
        v.ilv = t->mem->ilv;
        v.ilv_first = t->mem->ilv_first;
    }
    return v;
}

Worker* checkout(gxy_ctx* ctx, gxy_status* err) {
    {
        std::lock_guard<std::mutex> g(ctx->mu);
        if (!ctx->free_workers.empty()) {
            // Prefer the primary worker so single-threaded callers share one stream.
            auto it = ctx->free_workers.begin();
            for (auto j = ctx->free_workers.begin(); j != ctx->free_workers.end(); ++j)
                if (*j == ctx->all_workers[0]) it = j;
            Worker* w = *it;
            ctx->free_workers.erase(it);
            *err = GXY_OK;
            return w;
        }
    }
    Worker* w = new Worker();
    cudaError_t e = cudaStreamCreateWithFlags(&w->st, cudaStreamNonBlocking);
    for (DevBuf* b : {&w->tk0, &w->tv0, &w->tk1, &w->tv1, &w->prim_sums, &w->prim_hist, &w->counters, &w->d_units,
                      &w->d_tsegs, &w->d_qsegs, &w->ck0, &w->ck1, &w->cv0, &w->cv1, &w->cands, &w->flags,
                      &w->offsets, &w->ohsp, &w->rhsp, &w->runit, &w->rhsp2, &w->runit2, &w->perm, &w->perm2,
                      &w->hits, &w->surv, &w->redo, &w->rk0, &w->rk1, &w->rv0, &w->rv1, &w->tocc,
                      &w->gpool, &w->gruns, &w->gaux, &w->gscr})
        b->st = w->st;
    for (int i = 0; i < 5 && e == cudaSuccess; i++) e = cudaEventCreate(&w->ev[i]);
    w->ps.grid = ctx->sm_count * 2;
    w->ps.sort_grid_max = ctx->sm_count * 8;
    if (e == cudaSuccess)
        e = w->prim_sums.ensure(((size_t)std::max(w->ps.grid, w->ps.sort_grid_max) + 1) * sizeof(uint32_t));
    if (e == cudaSuccess)
        e = w->prim_hist.ensure(((size_t)kRadixMax * std::max(w->ps.grid, w->ps.sort_grid_max) + 1) *
                                sizeof(uint32_t));
    if (e == cudaSuccess) e = w->counters.ensure(kCounterWords * 4);
    if (e == cudaSuccess) e = cudaMallocHost(&w->h_pinned, 1 << 16);
    if (e != cudaSuccess) {
        set_error(std::string("worker setup: ") + cudaGetErrorString(e));
        *err = e == cudaErrorMemoryAllocation ? GXY_ENOMEM : GXY_ECUDA;
        return nullptr;
    }
    w->h_pinned_bytes = 1 << 16;
    w->ps.block_sums = w->prim_sums.as<uint32_t>();
    w->ps.hist = w->prim_hist.as<uint32_t>();
    {
        std::lock_guard<std::mutex> g(ctx->mu);
        ctx->all_workers.push_back(w);
    }
    *err = GXY_OK;
    return w;
}

void checkin(gxy_ctx* ctx, Worker* w) {
    std::lock_guard<std::mutex> g(ctx->mu);
    ctx->free_workers.push_back(w);
}

// SeedPattern::parse (src/seeds.rs:38-51) with the engine's limits.
gxy_status parse_pattern(const char* s, Pattern& pat) {
    if (!s) {
        set_error("pattern is null");
        return GXY_EINVAL;
    }
    memset(&pat, 0, sizeof(pat));
    uint32_t len = 0, w = 0;
    for (const char* c = s; *c; c++) {
        if (*c != '0' && *c != '1') {
            set_error(std::string("seed pattern character '") + *c + "' is not '0' or '1'");
            return GXY_EINVAL;
        }
        if (len >= 32) {
            set_error("seed pattern exceeds the 32-position limit (src/seeds.rs:28-32)");
            return GXY_EINVAL;
        }
        if (*c == '1') {
            if (w >= (uint32_t)kMaxWeight) {
                set_error("seed weight > 15 needs more than 2^30 buckets; unsupported");
                return GXY_EUNSUPPORTED;
            }
            pat.care[w++] = (uint8_t)len;
            pat.care_mask |= 1u << len;
        }
        len++;
    }
    if (len == 0) {
        set_error("seed pattern is empty");
        return GXY_EINVAL;
    }
    pat.len = len;
    pat.weight = w;
    return GXY_OK;
}

gxy_status check_params(const gxy_search_params* p, uint64_t max_cols) {
    if (!p) {
        set_error("params is null");
        return GXY_EINVAL;
    }
    if (p->step < 1) {
        set_error("step must be >= 1 (src/pos_table.rs:36)");
        return GXY_EINVAL;
    }
    int64_t m = p->ambig < 0 ? -(int64_t)p->ambig : p->ambig;
    for (int i = 0; i < 16; i++) {
        const int64_t a = p->sub[i] < 0 ? -(int64_t)p->sub[i] : p->sub[i];
        m = std::max(m, a);
    }
    // Every partial sum is bounded by m * columns; the x-drop gap by
    // |xdrop| + 33 m.  Within this envelope i32 adds never saturate, so the
    // device's plain adds equal the reference's saturating ones.
    const int64_t lim = 0x7fffffffLL;
    const int64_t xd = p->xdrop < 0 ? -(int64_t)p->xdrop : p->xdrop;
    if (m * (int64_t)(max_cols + 64) >= lim || xd + 33 * m >= lim) {
        set_error("scores x sequence length can overflow i32; outside the exact envelope");
        return GXY_EUNSUPPORTED;
    }
    return GXY_OK;
}

static int bits_for(uint64_t x) {
    int b = 0;
    while (b < 64 && (1ull << b) <= x) b++;
    return b;   // smallest b with x < 2^b
}

static void build_variants(const Pattern& pat, uint32_t transitions, uint32_t* vx, uint32_t& nv) {
    // src/seed_search.rs:63, :303-316.
    const uint32_t w = pat.weight;
    uint32_t shifts[16];
    for (uint32_t i = 0; i < w; i++) shifts[i] = 2 * (w - 1 - i);
    nv = 0;
    vx[nv++] = 0;
    if (transitions >= 1)
        for (uint32_t i = 0; i < w; i++) vx[nv++] = 2u << shifts[i];
    if (transitions >= 2)
        for (uint32_t i = 0; i < w; i++)
            for (uint32_t j = i + 1; j < w; j++) vx[nv++] = (2u << shifts[i]) ^ (2u << shifts[j]);
}

gxy_status reserve_worker(gxy_ctx* ctx, Worker* W, uint64_t est_hits, uint64_t candidates, uint32_t max_units) {
    const uint64_t max_hits = std::max<uint32_t>(4096, ctx->tuning.max_hits_per_pass);
    const uint64_t hits = std::min(est_hits, max_hits);
    // The filter's survivors, sized as run_units sizes them.
    const uint64_t want_s = std::min<uint64_t>(max_hits, (1 << 20) + (uint64_t)(est_hits / kRawPerSurvivorSlot));
    if (want_s > W->surv_cap) {
        W->surv.release();
        W->surv_cap = want_s;
    }
    GXY_CK(W->surv.ensure((size_t)W->surv_cap * sizeof(Hit)));
    GXY_CK(W->redo.ensure((size_t)2 * kRedoCap * 4));
    const size_t mu = std::max<uint32_t>(max_units, 1);
    GXY_CK(W->d_units.ensure(mu * sizeof(UnitDev)));
    GXY_CK(W->d_tsegs.ensure(mu * sizeof(SeqView)));
    GXY_CK(W->d_qsegs.ensure(mu * sizeof(SeqView)));
    candidates = std::min<uint64_t>(candidates, kMaxPresizedCandidates);
    if (hits > W->hit_cap) {
        W->hits.release();
        W->hit_cap = hits;
    }
    if (candidates > W->cand_cap) W->cand_cap = (uint32_t)candidates;
    const size_t cap = W->cand_cap;
    GXY_CK(W->hits.ensure((size_t)W->hit_cap * sizeof(Hit)));
    DevBuf* by8[] = {&W->ck0, &W->ck1};
    for (DevBuf* b : by8) GXY_CK(b->ensure(cap * 8));
    DevBuf* by4[] = {&W->cv0, &W->cv1, &W->runit, &W->runit2, &W->perm, &W->perm2};
    for (DevBuf* b : by4) GXY_CK(b->ensure(cap * 4));
    GXY_CK(W->cands.ensure(cap * sizeof(Cand)));
    GXY_CK(W->flags.ensure(cap));
    GXY_CK(W->offsets.ensure(cap * 4 + 4));
    DevBuf* byh[] = {&W->ohsp, &W->rhsp, &W->rhsp2};
    for (DevBuf* b : byh) GXY_CK(b->ensure(cap * sizeof(Hsp)));
    // Pinned result staging for a tenth of the candidates as HSPs with units.
    const size_t want = std::max<size_t>(1 << 20, cap / 10 * (sizeof(Hsp) + 4));
    if (want > W->h_res_bytes) {
        if (W->h_res) GXY_CK(cudaFreeHost(W->h_res));
        W->h_res = nullptr;
        W->h_res_bytes = 0;
        GXY_CK(cudaMallocHost(&W->h_res, want));
        W->h_res_bytes = want;
    }
    GXY_CK(cudaStreamSynchronize(W->st));
    return GXY_OK;
}

// Captures what `issue` launches on the worker's stream into a CUDA graph and
// launches it.  The instantiated graph stays with the worker: a later call
// with the same shape (the same kernels in the same order; launch arguments
// may differ) updates it in place instead of instantiating anew.
template <typename F>
static gxy_status run_graph(Worker* W, F&& issue) {
    cudaStream_t st = W->st;
    GXY_CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    const gxy_status is = issue();
    cudaGraph_t g = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(st, &g);
    if (is != GXY_OK || ce != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        if (is != GXY_OK) return is;
        set_error(std::string("cudaStreamEndCapture: ") + cudaGetErrorString(ce));
        return GXY_ECUDA;
    }
    bool updated = false;
    if (W->gexec) {
        cudaGraphExecUpdateResultInfo info;
        updated = cudaGraphExecUpdate(W->gexec, g, &info) == cudaSuccess;
        if (!updated) {
            cudaGetLastError();
            cudaGraphExecDestroy(W->gexec);
            W->gexec = nullptr;
        }
    }
    cudaError_t e = cudaSuccess;
    if (!updated) e = cudaGraphInstantiate(&W->gexec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        W->gexec = nullptr;
        set_error(std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
        return GXY_ECUDA;
    }
    W->graph_updates += updated ? 1 : 0;
    GXY_CK(cudaGraphLaunch(W->gexec, st));
    return GXY_OK;
}

gxy_status run_units(gxy_ctx* ctx, Worker* W, const std::vector<UnitPlan>& units, std::vector<SeqView>& tsegs,
                     std::vector<SeqView>& qsegs, const Pattern& pat, const gxy_search_params& p, bool use_graph,
                     RunResult& out) {
    cudaStream_t st = W->st;
    out.hsps.clear();
    out.unit.clear();
    out.records.clear();
    out.stats = gxy_stats{};
    const uint32_t nu = (uint32_t)units.size();
    // Key axes: every target and query segment gets a private key range.
    uint64_t tk = 0, qk = 0;
    for (auto& s : tsegs) {
        s.key_base = (uint32_t)tk;
        tk += s.len;
    }
    for (auto& s : qsegs) {
        s.key_base = (uint32_t)qk;
        qk += s.len;
    }
    if (tk + qk >= (1ull << 32)) {
        set_error("batch too large: total target + query length must be < 2^32");
        return GXY_EUNSUPPORTED;
    }
    std::vector<UnitDev> ud(nu);
    uint64_t tiles = 0;
    for (uint32_t i = 0; i < nu; i++) {
        const UnitPlan& u = units[i];
        ud[i].tseg = u.tseg;
        ud[i].qseg = u.qseg;
        ud[i].starts = u.starts;
        ud[i].positions = u.positions;
        ud[i].occ = u.occ;
        ud[i].nwin = u.nwin;
        ud[i].tile_base = (uint32_t)tiles;
        ud[i].primary_lo = u.primary_lo;
        ud[i].primary_hi = u.primary_hi;
        tiles += (u.nwin + 31) / 32;
    }
    if (tiles >= (1ull << 32)) {
        set_error("too many query windows");
        return GXY_EUNSUPPORTED;
    }
    if (nu == 0 || tiles == 0) return GXY_OK;

    GXY_CK(W->d_units.ensure(nu * sizeof(UnitDev)));
    GXY_CK(W->d_tsegs.ensure(tsegs.size() * sizeof(SeqView)));
    GXY_CK(W->d_qsegs.ensure(qsegs.size() * sizeof(SeqView)));
    const bool records = out.places != nullptr;
    if (records) GXY_CK(W->d_place.ensure(nu * sizeof(Place)));
    {
        // Descriptors go through the pinned staging when they fit (the
        // worker's stream is idle here: every call ends synchronized).
        const size_t bu = nu * sizeof(UnitDev), bt = tsegs.size() * sizeof(SeqView),
                     bq = qsegs.size() * sizeof(SeqView), bp = records ? nu * sizeof(Place) : 0;
        const size_t off = 32768;   // the counters come back into [0, kCounterWords * 4)
        if (off + bu + bt + bq + bp <= W->h_pinned_bytes) {
            unsigned char* h = static_cast<unsigned char*>(W->h_pinned) + off;
            memcpy(h, ud.data(), bu);
            memcpy(h + bu, tsegs.data(), bt);
            memcpy(h + bu + bt, qsegs.data(), bq);
            if (bp) memcpy(h + bu + bt + bq, out.places, bp);
            GXY_CK(cudaMemcpyAsync(W->d_units.p, h, bu, cudaMemcpyHostToDevice, st));
            GXY_CK(cudaMemcpyAsync(W->d_tsegs.p, h + bu, bt, cudaMemcpyHostToDevice, st));
            GXY_CK(cudaMemcpyAsync(W->d_qsegs.p, h + bu + bt, bq, cudaMemcpyHostToDevice, st));
            if (bp) GXY_CK(cudaMemcpyAsync(W->d_place.p, h + bu + bt + bq, bp, cudaMemcpyHostToDevice, st));
        } else {
            GXY_CK(cudaMemcpyAsync(W->d_units.p, ud.data(), bu, cudaMemcpyHostToDevice, st));
            GXY_CK(cudaMemcpyAsync(W->d_tsegs.p, tsegs.data(), bt, cudaMemcpyHostToDevice, st));
            GXY_CK(cudaMemcpyAsync(W->d_qsegs.p, qsegs.data(), bq, cudaMemcpyHostToDevice, st));
            if (bp) GXY_CK(cudaMemcpyAsync(W->d_place.p, out.places, bp, cudaMemcpyHostToDevice, st));
            GXY_CK(cudaStreamSynchronize(st));   // the host vectors die with this call
        }
    }
    // Record key widths: group, global t, q, span (span <= min(target, query)).
    int rb_g = 0, rb_t = 0, rb_q = 0, rb_l = 0;
    if (records) {
        uint64_t mg = 0, mt = 0, mq = 0, ml = 0;
        for (uint32_t i = 0; i < nu; i++) {
            const uint64_t tl = tsegs[units[i].tseg].len, ql = qsegs[units[i].qseg].len;
            mg = std::max<uint64_t>(mg, out.places[i].group);
            mt = std::max<uint64_t>(mt, out.places[i].t_offset + tl);
            mq = std::max<uint64_t>(mq, ql);
            ml = std::max<uint64_t>(ml, std::min(tl, ql));
        }
        rb_g = bits_for(mg);
        rb_t = bits_for(mt ? mt - 1 : 0);
        rb_q = bits_for(mq ? mq - 1 : 0);
        rb_l = bits_for(ml);
    }

    ScreenArgs sa;
    memset(&sa, 0, sizeof(sa));
    sa.units = W->d_units.as<UnitDev>();
    sa.tsegs = W->d_tsegs.as<SeqView>();
    sa.qsegs = W->d_qsegs.as<SeqView>();
    sa.n_units = nu;
    sa.tile_lo = 0;
    sa.tile_hi = (uint32_t)tiles;
    sa.pat = pat;
    sa.step = p.step;
    build_variants(pat, p.transitions, sa.var_xor, sa.n_var);
    memcpy(sa.sc.sub, p.sub, sizeof(p.sub));
    sa.sc.ambig = p.ambig;
    sa.sc.xdrop = p.xdrop;
    sa.sc.hspthresh = p.hspthresh;
    sa.cap = std::max<uint32_t>(32, ctx->tuning.screen_cap);
    sa.qkey_total = (uint32_t)qk;
    // The upper-bound filter runs between enumeration and the exact screen
    // when the scores admit class bounds (every matrix with a class whose
    // scores are all <= 0); otherwise the exact screen takes every raw hit.
    sa.f_cap = std::max<uint32_t>(32, ctx->tuning.filter_cap);
    sa.f_claim = ctx->tuning.filter_claim > 1 ? ctx->tuning.filter_claim : 0u;
    const bool use_filter = filter_bounds(sa);

    RadixPass passes[16];
    const int npass = plan_radix(0, bits_for(tk ? tk - 1 : 0), 32, bits_for(tk + qk), passes, 16);

    uint32_t* cnt = W->counters.as<uint32_t>();
    unsigned long long* st64 = reinterpret_cast<unsigned long long*>(cnt + kCStats);
    unsigned long long* hitc = reinterpret_cast<unsigned long long*>(cnt + kCHits);
    unsigned long long* survc = reinterpret_cast<unsigned long long*>(cnt + kCSurv);
    if (ctx->tuning.initial_candidates) W->cand_cap = ctx->tuning.initial_candidates;
    if (W->cand_cap == 0) W->cand_cap = 2u << 20;
    if (W->hit_cap == 0) W->hit_cap = 32ull << 20;
    const uint64_t kMaxHitCap = std::max<uint32_t>(4096, ctx->tuning.max_hits_per_pass);
    if (W->hit_cap > kMaxHitCap) {
        W->hits.release();
        W->hit_cap = kMaxHitCap;
    }
    // Size the raw-hit buffer from the expected hits (windows x variants x
    // mean bucket, with margin); a launch with more raw hits than the buffer
    // holds runs as several passes, each taking tiles until the buffer is
    // full and handing the tile that did not fit to the next pass, all on
    // the device.
    double est = 1 << 20;
    for (const UnitPlan& u : units) est += 1.5 * (double)u.nwin * sa.n_var * u.avg_bucket;
    {
        if (use_filter) {
            const uint64_t want_s = (uint64_t)std::min<double>((double)kMaxHitCap, (1 << 20) + est / kRawPerSurvivorSlot);
            if (want_s > W->surv_cap) {
                W->surv.release();
                W->surv_cap = want_s;
            }
        }
        // Candidates from the same estimate (a few percent of the raw hits
        // pass the screen): an overflow would rerun the whole launch.
        const uint64_t want_cand = std::min<uint64_t>((uint64_t)(est / kHitsPerCandidate), kMaxPresizedCandidates);
        if (want_cand > W->cand_cap) W->cand_cap = (uint32_t)want_cand;
        const uint64_t want_hits = std::min<uint64_t>(kMaxHitCap, (uint64_t)est);
        if (want_hits > W->hit_cap) {
            W->hits.release();
            W->hit_cap = want_hits;
        }
    }
    const int blocks_screen = ctx->sm_count * (int)std::max<uint32_t>(1, ctx->tuning.screen_blocks_per_sm);
    const int blocks_misc = ctx->sm_count * 4;
    const int walk_warps = ctx->tuning.walk_warps == 4 ? 4 : 8;
    GXY_CK(W->redo.ensure((size_t)2 * kRedoCap * 4));

    // One pass: start it (k_pass_reset), enumerate into the hit buffer, filter
    // and screen.  With timing (a one-pass launch outside a graph) the kernels
    // are bracketed by events 0 / 4 / 3 / 1.
    auto pass = [&](bool timing) {
        launch_pass_reset(cnt, use_filter ? W->surv_cap : ~0ull, st);
        if (timing) cudaEventRecord(W->ev[0], st);
        launch_enumerate(sa, ctx->sm_count, st);
        if (timing) cudaEventRecord(W->ev[4], st);
        if (use_filter) {
            // Raw hits -> the bounded filter -> survivors -> the exact screen.
            ScreenArgs sv = sa;
            sv.hits = W->surv.as<Hit>();
            sv.hit_cap = W->surv_cap;
            sv.hit_count = survc;
            FilterIO io{sa.hits, hitc, sa.hit_cap, cnt + kCFiltNext};
            launch_filter_hits(sv, io, ctx->sm_count, st);
            if (timing) cudaEventRecord(W->ev[3], st);
            launch_screen(sv, (int)ctx->tuning.screen_warps, blocks_screen, st);
        } else {
            if (timing) cudaEventRecord(W->ev[3], st);
            launch_screen(sa, (int)ctx->tuning.screen_warps, blocks_screen, st);
        }
        if (timing) cudaEventRecord(W->ev[1], st);
    };

    // After the passes: sort the candidates by (diagonal, t), walk the
    // diagonals, compact, group by unit, order each run, and (with places)
    // make the driver's records; then the counters come back to the host.
    Hsp* fin = nullptr;
    uint32_t* fin_unit = nullptr;
    uint32_t cap = W->cand_cap;
    auto epilogue = [&]() -> gxy_status {
        const int which = radix_sort_u64(W->ck0.as<uint64_t>(), W->cv0.as<uint32_t>(), W->ck1.as<uint64_t>(),
                                             W->cv1.as<uint32_t>(), cnt + kCCand, 0, cap, passes, npass, W->ps, st);
            const uint64_t* skeys = which ? W->ck1.as<uint64_t>() : W->ck0.as<uint64_t>();
            const uint32_t* sidx = which ? W->cv1.as<uint32_t>() : W->cv0.as<uint32_t>();
            GXY_CK(cudaMemsetAsync(W->flags.p, 0, cap, st));
            WalkArgs wa;
            memset(&wa, 0, sizeof(wa));
            wa.keys = skeys;
            wa.idx = sidx;
            wa.cands = W->cands.as<Cand>();
            wa.n_dev = cnt + kCCand;
            wa.n_cap = cap;
            wa.units = sa.units;
            wa.tsegs = sa.tsegs;
            wa.qsegs = sa.qsegs;
            wa.seed_len = pat.len;
            wa.sc = sa.sc;
            wa.has_entropy = p.has_entropy;
            wa.entropy_thr = p.entropy_thr;
            wa.out_flag = W->flags.as<uint8_t>();
            wa.out_hsp = W->ohsp.as<Hsp>();
            wa.chunk_next = cnt + kCWalk;
            wa.n_units = nu;
            GXY_CK(cudaMemsetAsync(cnt + kCWalk, 0, 4, st));
            launch_walk(wa, walk_warps, blocks_misc, st);
            scan_u8(W->flags.as<uint8_t>(), W->offsets.as<uint32_t>(), cnt + kCCand, 0, cap, false, cnt + kCHsps, W->ps,
                    st);
            launch_compact(W->flags.as<uint8_t>(), W->offsets.as<uint32_t>(), W->ohsp.as<Hsp>(), sidx,
                           W->cands.as<Cand>(), cnt + kCCand, cap, W->rhsp.as<Hsp>(), W->runit.as<uint32_t>(), blocks_misc, st);
            fin = W->rhsp.as<Hsp>();
            fin_unit = W->runit.as<uint32_t>();
            if (nu > 1) {
                // Group by unit, keeping each unit's (diagonal, t) order: stable sort.
                RadixPass up[4];
                const int nup = plan_radix(0, bits_for(nu - 1), 0, 0, up, 4);
                launch_iota(W->perm.as<uint32_t>(), cnt + kCHsps, cap, blocks_misc, st);
                GXY_CK(cudaMemcpyAsync(W->runit2.p, W->runit.p, (size_t)cap * 4, cudaMemcpyDeviceToDevice, st));
                const int w2 = radix_sort_u32(W->runit2.as<uint32_t>(), W->perm.as<uint32_t>(), W->offsets.as<uint32_t>(),
                                              W->perm2.as<uint32_t>(), cnt + kCHsps, 0, cap, up, nup, W->ps, st);
                const uint32_t* perm = w2 ? W->perm2.as<uint32_t>() : W->perm.as<uint32_t>();
                launch_gather_hsp(W->rhsp.as<Hsp>(), W->runit.as<uint32_t>(), perm, cnt + kCHsps, cap, W->rhsp2.as<Hsp>(),
                                  W->runit2.as<uint32_t>(), blocks_misc, st);
                fin = W->rhsp2.as<Hsp>();
                fin_unit = W->runit2.as<uint32_t>();
            }
            launch_fixup(fin, fin_unit, cnt + kCHsps, cap, W->flags.as<uint8_t>(), blocks_misc, st);
            if (records) {
                // Driver records (src/driver.rs:371-391): stable LSD sort by
                // (group, global t, q, span) over the unit-major HSP order, then
                // drop repeats of the same four fields, keeping the first.  One
                // sort of a packed key when the fields fit 64 bits, else (q, span)
                // first and (group, t) second.
                const Place* pl = W->d_place.as<Place>();
                RadixPass rp[16];
                const uint32_t* perm;
                if (rb_g + rb_t + rb_q + rb_l <= 64) {
                    const int sh_q = rb_l, sh_t = rb_l + rb_q, sh_g = rb_l + rb_q + rb_t;
                    launch_record_keys(fin, fin_unit, pl, nullptr, cnt + kCHsps, cap, 0, sh_g, sh_t, sh_q,
                                       W->rk0.as<uint64_t>(), W->rv0.as<uint32_t>(), blocks_misc, st);
                    const int np = plan_radix(0, rb_l + rb_q + rb_t + rb_g, 0, 0, rp, 16);
                    const int w = radix_sort_u64(W->rk0.as<uint64_t>(), W->rv0.as<uint32_t>(), W->rk1.as<uint64_t>(),
                                                 W->rv1.as<uint32_t>(), cnt + kCHsps, 0, cap, rp, np, W->ps, st);
                    perm = w ? W->rv1.as<uint32_t>() : W->rv0.as<uint32_t>();
                } else {
                    launch_record_keys(fin, fin_unit, pl, nullptr, cnt + kCHsps, cap, 1, 0, 0, 0, W->rk0.as<uint64_t>(),
                                       W->rv0.as<uint32_t>(), blocks_misc, st);
                    int np = plan_radix(0, rb_l, 32, rb_q, rp, 16);
                    int w = radix_sort_u64(W->rk0.as<uint64_t>(), W->rv0.as<uint32_t>(), W->rk1.as<uint64_t>(),
                                           W->rv1.as<uint32_t>(), cnt + kCHsps, 0, cap, rp, np, W->ps, st);
                    const uint32_t* p1 = w ? W->rv1.as<uint32_t>() : W->rv0.as<uint32_t>();
                    uint64_t* k2 = w ? W->rk0.as<uint64_t>() : W->rk1.as<uint64_t>();
                    uint32_t* v2 = w ? W->rv0.as<uint32_t>() : W->rv1.as<uint32_t>();
                    uint64_t* k3 = w ? W->rk1.as<uint64_t>() : W->rk0.as<uint64_t>();
                    uint32_t* v3 = w ? W->rv1.as<uint32_t>() : W->rv0.as<uint32_t>();
                    launch_record_keys(fin, fin_unit, pl, p1, cnt + kCHsps, cap, 2, 0, 0, 0, k2, v2, blocks_misc, st);
                    np = plan_radix(0, rb_t, 32, rb_g, rp, 16);
                    w = radix_sort_u64(k2, v2, k3, v3, cnt + kCHsps, 0, cap, rp, np, W->ps, st);
                    perm = w ? v3 : v2;
                }
                launch_record_heads(fin, fin_unit, pl, perm, cnt + kCHsps, cap, W->flags.as<uint8_t>(), blocks_misc, st);
                scan_u8(W->flags.as<uint8_t>(), W->offsets.as<uint32_t>(), cnt + kCHsps, 0, cap, false, cnt + kCRecs,
                        W->ps, st);
                launch_record_emit(fin, fin_unit, pl, perm, W->flags.as<uint8_t>(), W->offsets.as<uint32_t>(),
                                   cnt + kCHsps, cap, W->rrec.as<Record>(), blocks_misc, st);
            }
            GXY_CK(cudaMemcpyAsync(W->h_pinned, W->counters.p, kCounterWords * 4, cudaMemcpyDeviceToHost, st));
        return GXY_OK;
    };

    // Passes in the first round: the estimate's share of the buffer, with
    // room to spare (a pass with nothing left to do returns at once).
    const uint64_t est_hits = (uint64_t)est;
    const uint64_t first_round = std::min<uint64_t>(
        256, std::max<uint64_t>(1, (est_hits + W->hit_cap - 1) / std::max<uint64_t>(1, W->hit_cap)));
    uint32_t reruns = 0;   // launches repeated after a buffer had to grow
    const uint64_t graph_updates0 = W->graph_updates;
    uint32_t rounds = 0;
    for (int attempt = 0; attempt < 16; attempt++) {
        cap = W->cand_cap;
        GXY_CK(W->hits.ensure((size_t)W->hit_cap * sizeof(Hit)));
        if (use_filter) GXY_CK(W->surv.ensure((size_t)W->surv_cap * sizeof(Hit)));
        GXY_CK(W->ck0.ensure((size_t)cap * 8));
        GXY_CK(W->ck1.ensure((size_t)cap * 8));
        GXY_CK(W->cv0.ensure((size_t)cap * 4));
        GXY_CK(W->cv1.ensure((size_t)cap * 4));
        GXY_CK(W->cands.ensure((size_t)cap * sizeof(Cand)));
        GXY_CK(W->flags.ensure((size_t)cap));
        GXY_CK(W->offsets.ensure((size_t)cap * 4 + 4));
        GXY_CK(W->ohsp.ensure((size_t)cap * sizeof(Hsp)));
        GXY_CK(W->rhsp.ensure((size_t)cap * sizeof(Hsp)));
        GXY_CK(W->runit.ensure((size_t)cap * 4));
        GXY_CK(W->rhsp2.ensure((size_t)cap * sizeof(Hsp)));
        GXY_CK(W->runit2.ensure((size_t)cap * 4));
        GXY_CK(W->perm.ensure((size_t)cap * 4));
        GXY_CK(W->perm2.ensure((size_t)cap * 4));
        if (records) {
            GXY_CK(W->rrec.ensure((size_t)cap * sizeof(Record)));
            GXY_CK(W->rk0.ensure((size_t)cap * 8));
            GXY_CK(W->rk1.ensure((size_t)cap * 8));
            GXY_CK(W->rv0.ensure((size_t)cap * 4));
            GXY_CK(W->rv1.ensure((size_t)cap * 4));
        }
        sa.tile_counter = cnt + kCTile;
        sa.cand_count = cnt + kCCand;
        sa.hit_next = cnt + kCHitNext;
        sa.hit_count = hitc;
        sa.hits = W->hits.as<Hit>();
        sa.hit_cap = W->hit_cap;
        sa.stats = st64;
        sa.cand_keys = W->ck0.as<uint64_t>();
        sa.cand_vals = W->cv0.as<uint32_t>();
        sa.cands = W->cands.as<Cand>();
        sa.cand_cap = cap;
        sa.ctl = cnt;
        sa.redo = W->redo.as<uint32_t>();

        // Round one: counters cleared, the passes, the epilogue and the
        // counters' copy back -- one CUDA graph (kept across calls and
        // updated in place) when use_graph, else plain launches.
        const uint32_t n_round = (uint32_t)first_round;
        const bool timing = !use_graph && n_round == 1;
        GXY_CK(cudaMemsetAsync(W->counters.p, 0, kCounterWords * 4, st));
        if (use_graph) {
            GXY_CK(cudaEventRecord(W->ev[0], st));
            API_TRY_ENGINE(run_graph(W, [&]() -> gxy_status {
                for (uint32_t i = 0; i < n_round; i++) pass(false);
                return epilogue();
            }));
        } else {
            if (!timing) GXY_CK(cudaEventRecord(W->ev[0], st));
            for (uint32_t i = 0; i < n_round; i++) pass(timing);
            API_TRY_ENGINE(epilogue());
        }
        GXY_CK(cudaEventRecord(W->ev[2], st));
        GXY_CK(cudaGetLastError());
        GXY_CK(cudaStreamSynchronize(st));
        rounds = 1;
        const uint32_t* hc = static_cast<const uint32_t*>(W->h_pinned);
        // Further rounds while tiles remain (the estimate was short): more
        // passes, then the epilogue again over all candidates so far.
        bool multi = n_round > 1;
        uint64_t last_tile = ~0ull, last_redo = ~0ull;
        for (int round = 0;; round++) {
            if (round > 4096) {
                set_error("the passes made no progress");
                return GXY_ECUDA;
            }
            const uint32_t np = hc[kCPass];
            const uint64_t tile_at = hc[kCTile], redo_left = hc[kCRedoN + (np & 1u)];
            if (hc[kCRedoOver]) {
                set_error("more tiles than the hit buffer's passes can carry over");
                return GXY_ENOMEM;
            }
            if (tile_at < tiles || redo_left) {
                if (tile_at == last_tile && redo_left == last_redo) {
                    const unsigned long long mf = *reinterpret_cast<const unsigned long long*>(hc + kCMaxFail);
                    if (mf > W->hit_cap) {
                        set_error("one tile of 32 query windows has more raw hits than the hit buffer holds");
                        return GXY_ENOMEM;
                    }
                }
                last_tile = tile_at;
                last_redo = redo_left;
                multi = true;
                const uint64_t more = std::min<uint64_t>(
                    256, (uint64_t)((double)(tiles - std::min<uint64_t>(tile_at, tiles)) / tiles * first_round) + 2);
                for (uint64_t i = 0; i < more; i++) pass(false);
                API_TRY_ENGINE(epilogue());
                rounds++;
                GXY_CK(cudaEventRecord(W->ev[2], st));
                GXY_CK(cudaGetLastError());
                GXY_CK(cudaStreamSynchronize(st));
                continue;
            }
            break;
        }
        const unsigned long long* hs = reinterpret_cast<const unsigned long long*>(hc + kCStats);
        const unsigned long long nhits_last = *reinterpret_cast<const unsigned long long*>(hc + kCHits);
        const unsigned long long nsurv_last = *reinterpret_cast<const unsigned long long*>(hc + kCSurv);
        const uint32_t ncand = hc[kCCand];
        if (use_filter && (hc[kCSurvOver] || nsurv_last > W->surv_cap)) {
            // A pass had more survivors than the survivor buffer holds: grow
            // it to the raw-hit buffer's size (survivors <= raw hits).
            W->surv.release();
            W->surv_cap = std::max<uint64_t>(W->surv_cap * 2, std::min<uint64_t>(W->hit_cap, W->surv_cap * 8));
            reruns++;
            continue;
        }
        if (ncand > cap) {
            // Candidate buffer overflowed: grow and rerun (results so far are void).
            uint64_t nc = (uint64_t)ncand + ncand / 4 + 1024;
            if (nc >= (1ull << 31)) {
                set_error("candidate count exceeds 2^31");
                return GXY_EUNSUPPORTED;
            }
            W->cand_cap = (uint32_t)nc;
            reruns++;
            continue;
        }
        const uint32_t work_passes = hc[kCWorkPasses] + (nhits_last ? 1u : 0u);
        out.stats.windows = hs[0];
        out.stats.raw_hits = hs[1];
        out.stats.columns = hs[2];
        out.stats.filter_columns = hs[3];
        out.stats.candidates = ncand;
        float ms = 0.f, ms_enum = 0.f, ms_filter = 0.f, ms_screen = 0.f;
        GXY_CK(cudaEventElapsedTime(&ms, W->ev[0], W->ev[2]));
        if (timing && !multi) {
            GXY_CK(cudaEventElapsedTime(&ms_enum, W->ev[0], W->ev[4]));
            GXY_CK(cudaEventElapsedTime(&ms_filter, W->ev[4], W->ev[3]));
            GXY_CK(cudaEventElapsedTime(&ms_screen, W->ev[3], W->ev[1]));
        }
        out.stats.device_ms = ms;
        out.stats.enum_ms = ms_enum;
        out.stats.filter_ms = ms_filter;
        out.stats.screen_ms = ms_screen;
        out.stats.passes = std::max<uint32_t>(1, work_passes);
        out.stats.reruns = reruns;
        out.stats.rounds = rounds;
        out.stats.graph_updates = (uint32_t)(W->graph_updates - graph_updates0);
        out.stats.survivors = use_filter ? hs[4] + nsurv_last : hs[1];
        const uint32_t nh = hc[kCHsps];
        out.stats.hsps = nh;
        if (records) {
            const uint32_t nr = hc[kCRecs];
            out.records.resize(nr);
            if (nr) {
                const size_t rb = (size_t)nr * sizeof(Record);
                if (rb > W->h_res_bytes) {
                    if (W->h_res) GXY_CK(cudaFreeHost(W->h_res));
                    W->h_res = nullptr;
                    W->h_res_bytes = 0;
                    const size_t want = std::max<size_t>(1 << 20, rb + rb / 2);
                    GXY_CK(cudaMallocHost(&W->h_res, want));
                    W->h_res_bytes = want;
                }
                GXY_CK(cudaMemcpyAsync(W->h_res, W->rrec.p, rb, cudaMemcpyDeviceToHost, st));
                GXY_CK(cudaStreamSynchronize(st));
                memcpy(out.records.data(), W->h_res, rb);
            }
            return GXY_OK;
        }
        // Results come back through the worker's pinned staging.
        const size_t hb = (size_t)nh * sizeof(Hsp), ub = nu > 1 ? (size_t)nh * 4 : 0;
        if (hb + ub > W->h_res_bytes) {
            if (W->h_res) GXY_CK(cudaFreeHost(W->h_res));
            W->h_res = nullptr;
            W->h_res_bytes = 0;
            const size_t want = std::max<size_t>(1 << 20, (hb + ub) + (hb + ub) / 2);
            GXY_CK(cudaMallocHost(&W->h_res, want));
            W->h_res_bytes = want;
        }
        unsigned char* hr = static_cast<unsigned char*>(W->h_res);
        if (nh) {
            GXY_CK(cudaMemcpyAsync(hr, fin, hb, cudaMemcpyDeviceToHost, st));
            if (ub) GXY_CK(cudaMemcpyAsync(hr + hb, fin_unit, ub, cudaMemcpyDeviceToHost, st));
            GXY_CK(cudaStreamSynchronize(st));
        }
        static_assert(sizeof(Hsp) == sizeof(gxy_hsp), "device and ABI HSP layouts differ");
        const gxy_hsp* hh = reinterpret_cast<const gxy_hsp*>(hr);
        if (out.want_view && nu == 1) {
            out.view = hh;
            out.n_view = nh;
            return GXY_OK;
        }
        out.hsps.assign(hh, hh + nh);
        if (ub) {
            const uint32_t* uu = reinterpret_cast<const uint32_t*>(hr + hb);
            out.unit.assign(uu, uu + nh);
        } else {
            out.unit.assign(nh, 0u);
        }
        return GXY_OK;
    }
    set_error("candidate buffer did not converge");
    return GXY_ENOMEM;
}

}  // namespace gxy
