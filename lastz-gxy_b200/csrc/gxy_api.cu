// gxy_api.cu -- the extern "C" boundary declared in include/gxy_seed.h.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "gxy_engine.cuh"

using namespace gxy;

namespace gxy {
const char* last_error();
uint64_t launches();
}

#define API_CK(call)                                                                         \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess) {                                                             \
            set_error(std::string(#call) + ": " + cudaGetErrorString(e_));                    \
            return e_ == cudaErrorMemoryAllocation ? GXY_ENOMEM : GXY_ECUDA;                 \
        }                                                                                    \
    } while (0)

#define API_TRY(expr)                      \
    do {                                   \
        gxy_status s_ = (expr);            \
        if (s_ != GXY_OK) return s_;       \
    } while (0)

namespace {

// RAII checkout of a worker.
struct WorkerLease {
    gxy_ctx* ctx;
    Worker* w;
    gxy_status err;
    explicit WorkerLease(gxy_ctx* c) : ctx(c), w(nullptr), err(GXY_OK) { w = checkout(c, &err); }
    ~WorkerLease() {
        if (w) checkin(ctx, w);
    }
};

gxy_status set_device(gxy_ctx* ctx) {
    API_CK(cudaSetDevice(ctx->device));
    return GXY_OK;
}

bool same_host_seq(const gxy_table* t, const gxy_packed_seq* s) {
    return s->codes == t->hc && s->valid == t->hv && s->mask == t->hm && s->len == t->hlen;
}

// prune_hot_words (src/pos_table.rs:113-136): counts of kept buckets ->
// exclusive scan -> copy the kept buckets in word order.
gxy_status prune_table(gxy_table* t, uint32_t limit, Worker* W) {
    cudaStream_t st = W->st;
    const uint64_t nw = t->num_words;
    uint32_t* new_starts = nullptr;
    uint32_t* newpos = nullptr;
    cudaError_t e = dev_alloc((void**)&new_starts, (nw + 1) * 4, st);
    if (e != cudaSuccess) {
        set_error("table prune allocation");
        return GXY_ENOMEM;
    }
    launch_prune_counts(t->starts, nw, limit, new_starts, st);
    scan_u32(new_starts, new_starts, nullptr, nw, nw, true, nullptr, W->ps, st);
    uint32_t total2 = 0;
    e = cudaMemcpyAsync(&total2, new_starts + nw, 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = dev_alloc((void**)&newpos, (size_t)std::max<uint32_t>(total2, 1) * 4, st);
    if (e == cudaSuccess) {
        launch_prune_copy(t->positions, t->starts, nw, new_starts, limit, newpos, st);
        e = cudaStreamSynchronize(st);
    }
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) {
        dev_free(new_starts);
        dev_free(newpos);
        set_error(std::string("table prune: ") + cudaGetErrorString(e));
        return GXY_ECUDA;
    }
    if (t->own_arrays) {
        dev_free(t->starts);
        dev_free(t->positions);
    }
    t->starts = new_starts;
    t->positions = newpos;
    t->pos_base = 0;
    t->own_arrays = true;
    t->npos = total2;
    // Pruned buckets are empty now: their occupancy bits go.
    launch_occupancy(t->starts, nw, t->occ, st);
    e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error(std::string("table prune: ") + cudaGetErrorString(e));
        return GXY_ECUDA;
    }
    return GXY_OK;
}

}  // namespace

TableMem::~TableMem() {
    cudaSetDevice(device);
    dev_free(starts);
    dev_free(positions);
    dev_free(occ);
    dev_free(ilv);
}

namespace {

// PosTable::build for n views [lo[v], hi[v]) of seq, as one sort; out[v] is
// view v's table.  The tables share one TableMem.
gxy_status build_tables(gxy_ctx* ctx, const gxy_dseq* seq, uint32_t n, const uint64_t* lo, const uint64_t* hi,
                        const Pattern& pat, uint32_t step, uint32_t mwc, gxy_table** out) {
    WorkerLease L(ctx);
    if (!L.w) return L.err;
    Worker* W = L.w;
    cudaStream_t st = W->st;
    const uint64_t nw = 1ull << (2 * pat.weight);
    const uint64_t G = (uint64_t)n * nw;   // buckets of all views
    uint64_t total = 0;
    for (uint32_t v = 0; v < n; v++) total += n_windows(hi[v] - lo[v], pat.len, step);
    auto mem = std::make_shared<TableMem>();
    mem->device = ctx->device;
    // Counts -> scan -> fill -> in-bucket sorts (src/pos_table.rs:42-75),
    // with the occupancy bitmap the searches test before they read a
    // bucket's bounds.
    cudaError_t e = dev_alloc((void**)&mem->starts, (size_t)(G + 1) * 4, st);
    if (e == cudaSuccess) e = dev_alloc((void**)&mem->positions, (size_t)std::max<uint64_t>(total, 1) * 4, st);
    if (e == cudaSuccess) e = dev_alloc((void**)&mem->occ, (size_t)((G + 31) / 32) * 4, st);
    if (e != cudaSuccess) {
        set_error(std::string("table allocation: ") + cudaGetErrorString(e));
        return GXY_ENOMEM;
    }
    // The interleaved copy of the sequence words the views cover (with two
    // words of margin each side: the filter's windows reach 32 positions
    // left of a view and one word past its end).
    {
        uint64_t lo_min = UINT64_MAX, hi_max = 0;
        for (uint32_t v = 0; v < n; v++) {
            lo_min = std::min(lo_min, lo[v]);
            hi_max = std::max(hi_max, hi[v]);
        }
        const uint64_t w0 = (kPad + lo_min) / 32, w1 = (kPad + hi_max) / 32;
        mem->ilv_first = w0 >= 2 ? w0 - 2 : 0;
        const uint64_t last = std::min<uint64_t>(seq->nwords - 1, w1 + 2);
        e = dev_alloc((void**)&mem->ilv, (size_t)(last + 1 - mem->ilv_first) * 16, st);
        if (e != cudaSuccess) {
            set_error(std::string("table allocation: ") + cudaGetErrorString(e));
            return GXY_ENOMEM;
        }
        launch_interleave(seq->codes, seq->valid, seq->mask, mem->ilv_first, last + 1 - mem->ilv_first, mem->ilv, st);
    }
    std::vector<uint32_t> first((size_t)n + 1);
    API_TRY(atomic_build_views(seq, n, lo, hi, pat, step, mem->starts, mem->positions, mem->occ, first.data(), W));
    std::vector<gxy_table*> made;
    auto fail = [&](gxy_status s) {
        for (gxy_table* t : made) {
            if (t->own_arrays) {
                dev_free(t->starts);
                dev_free(t->positions);
            }
            delete t;
        }
        return s;
    };
    for (uint32_t v = 0; v < n; v++) {
        gxy_table* t = new gxy_table();
        made.push_back(t);
        t->ctx = ctx;
        t->device = ctx->device;
        t->seq = seq;
        t->lo = lo[v];
        t->hi = hi[v];
        t->num_words = nw;
        t->pat = pat;
        t->step = step;
        t->mem = mem;
        t->starts = mem->starts + (size_t)v * nw;
        t->positions = mem->positions;
        t->pos_base = first[v];
        t->occ = mem->occ + (size_t)v * nw / 32;
        t->npos = first[v + 1] - first[v];
        if (mwc > 0) {
            const gxy_status ps = prune_table(t, mwc, W);
            if (ps != GXY_OK) return fail(ps);
        }
    }
    e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error(std::string("table build: ") + cudaGetErrorString(e));
        return fail(GXY_ECUDA);
    }
    for (uint32_t v = 0; v < n; v++) out[v] = made[v];
    return GXY_OK;
}

gxy_status build_table(gxy_ctx* ctx, const gxy_dseq* seq, uint64_t lo, uint64_t hi, const Pattern& pat,
                       uint32_t step, uint32_t mwc, gxy_table** out) {
    return build_tables(ctx, seq, 1, &lo, &hi, pat, step, mwc, out);
}


gxy_status deliver(const gxy_hsp* v, uint64_t n, gxy_hsp_buf* out) {
    if (!out) return GXY_OK;
    if (out->hsps == nullptr) {
        out->hsps = static_cast<gxy_hsp*>(malloc(std::max<uint64_t>(n, 1) * sizeof(gxy_hsp)));
        if (!out->hsps) {
            set_error("host allocation of the HSP buffer");
            return GXY_ENOMEM;
        }
        out->cap = n;
    } else if (out->cap < n) {
        out->len = n;
        set_error("caller HSP buffer too small");
        return GXY_EOVERFLOW;
    }
    if (n) memcpy(out->hsps, v, n * sizeof(gxy_hsp));
    out->len = n;
    return GXY_OK;
}

gxy_status search_impl(gxy_ctx* ctx, Worker* W, const gxy_table* table, const SeqView& T, const SeqView& Q,
                       const gxy_search_params* p, gxy_hsp_buf* out, gxy_stats* stats) {
    API_TRY(check_params(p, std::min<uint64_t>(T.len, Q.len)));
    std::vector<SeqView> tsegs{T}, qsegs{Q};
    std::vector<UnitPlan> units(1);
    units[0].tseg = 0;
    units[0].qseg = 0;
    units[0].starts = table->starts;
    units[0].positions = table->positions;
    units[0].occ = table->occ;
    units[0].nwin = n_windows(Q.len, table->pat.len, p->step);
    units[0].primary_lo = units[0].primary_hi = 0;
    units[0].avg_bucket = table->num_words ? (double)table->npos / (double)table->num_words : 0.0;
    RunResult r;
    r.want_view = true;
    API_TRY(run_units(ctx, W, units, tsegs, qsegs, table->pat, *p, false, r));
    if (stats) *stats = r.stats;
    return deliver(r.view, r.n_view, out);
}

}  // namespace

extern "C" {

const char* gxy_status_string(gxy_status s) {
    switch (s) {
        case GXY_OK: return "ok";
        case GXY_EINVAL: return "invalid argument";
        case GXY_ENOMEM: return "out of memory";
        case GXY_EUNSUPPORTED: return "unsupported";
        case GXY_ETIMEDOUT: return "timed out";
        case GXY_ECUDA: return "CUDA error";
        case GXY_ENOTREADY: return "not ready";
        case GXY_EOVERFLOW: return "buffer too small";
        case GXY_ECANCELED: return "cancelled";
    }
    return "unknown status";
}

const char* gxy_last_error(void) { return last_error(); }
uint32_t gxy_abi_version(void) { return 3; }
uint64_t gxy_kernel_launches(void) { return launches(); }

gxy_status gxy_ctx_create(int device, gxy_ctx** out) {
    if (!out) return GXY_EINVAL;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        set_error(std::string("no CUDA device: ") + cudaGetErrorString(e));
        return GXY_ECUDA;
    }
    if (device < 0 || device >= n) {
        set_error("device index out of range");
        return GXY_EINVAL;
    }
    API_CK(cudaSetDevice(device));
    cudaDeviceProp prop;
    API_CK(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10) {
        set_error(std::string("this library is built for sm_100a; device is ") + prop.name);
        return GXY_EUNSUPPORTED;
    }
    // Keep freed pool memory reserved so repeated allocations stay cheap.
    cudaMemPool_t pool;
    API_CK(cudaDeviceGetDefaultMemPool(&pool, device));
    uint64_t thr = ~0ull;
    API_CK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
    prims_init();
    filter_init();
    table_init();
    gxy_ctx* c = new gxy_ctx();
    c->device = device;
    c->sm_count = prop.multiProcessorCount;
    for (int i = 0; i < 16; i++) API_CK(cudaEventCreate(&c->marks[i]));
    gxy_status err;
    Worker* w = checkout(c, &err);   // the primary worker
    if (!w) {
        delete c;
        return err;
    }
    checkin(c, w);
    *out = c;
    return GXY_OK;
}

gxy_status gxy_ctx_destroy(gxy_ctx* ctx) {
    if (!ctx) return GXY_OK;
    cudaSetDevice(ctx->device);
    for (Worker* w : ctx->all_workers) {
        cudaStreamSynchronize(w->st);
        DevBuf* bufs[] = {&w->prim_sums, &w->prim_hist, &w->counters, &w->d_units, &w->d_tsegs, &w->d_qsegs,
                          &w->ck0, &w->ck1, &w->cv0, &w->cv1, &w->cands, &w->flags, &w->offsets, &w->ohsp,
                          &w->rhsp, &w->runit, &w->rhsp2, &w->runit2, &w->perm, &w->perm2, &w->hits,
                          &w->d_place, &w->rrec, &w->surv, &w->redo, &w->rk0, &w->rk1, &w->rv0, &w->rv1};
        for (DevBuf* b : bufs) b->release();
        if (w->gexec) cudaGraphExecDestroy(w->gexec);
        dseq_destroy(w->qstage);
        dseq_destroy(w->tstage);
        for (gxy_dseq* d : w->rc_tmp) dseq_destroy(d);
        DevBuf* tb[] = {&w->tk0, &w->tv0, &w->tk1, &w->tv1, &w->tocc, &w->gpool, &w->gruns, &w->gaux, &w->gscr};
        for (DevBuf* b : tb) b->release();
        for (int i = 0; i < 5; i++)
            if (w->ev[i]) cudaEventDestroy(w->ev[i]);
        if (w->h_pinned) cudaFreeHost(w->h_pinned);
        if (w->h_res) cudaFreeHost(w->h_res);
        cudaStreamDestroy(w->st);
        delete w;
    }
    for (int i = 0; i < 16; i++)
        if (ctx->marks[i]) cudaEventDestroy(ctx->marks[i]);
    delete ctx;
    return GXY_OK;
}

gxy_status gxy_ctx_mark(gxy_ctx* ctx, uint32_t slot) {
    if (!ctx || slot >= 16 || ctx->all_workers.empty()) return GXY_EINVAL;
    API_TRY(set_device(ctx));
    API_CK(cudaEventRecord(ctx->marks[slot], ctx->all_workers[0]->st));
    return GXY_OK;
}

gxy_status gxy_ctx_elapsed_ms(gxy_ctx* ctx, uint32_t a, uint32_t b, double* ms) {
    if (!ctx || a >= 16 || b >= 16 || !ms) return GXY_EINVAL;
    API_TRY(set_device(ctx));
    API_CK(cudaEventSynchronize(ctx->marks[b]));
    float f = 0.f;
    API_CK(cudaEventElapsedTime(&f, ctx->marks[a], ctx->marks[b]));
    *ms = f;
    return GXY_OK;
}

gxy_status gxy_ctx_set_tuning(gxy_ctx* ctx, const gxy_tuning* t) {
    if (!ctx || !t) return GXY_EINVAL;
    std::lock_guard<std::mutex> g(ctx->mu);
    if (t->screen_warps) {
        if (t->screen_warps != 4 && t->screen_warps != 8 && t->screen_warps != 16) {
            set_error("screen_warps must be 4, 8 or 16");
            return GXY_EINVAL;
        }
        ctx->tuning.screen_warps = t->screen_warps;
    }
    if (t->screen_cap) ctx->tuning.screen_cap = std::max<uint32_t>(32, t->screen_cap);
    if (t->screen_blocks_per_sm) ctx->tuning.screen_blocks_per_sm = std::min<uint32_t>(t->screen_blocks_per_sm, 16);
    if (t->walk_warps) ctx->tuning.walk_warps = t->walk_warps == 4 ? 4 : 8;
    if (t->max_hits_per_pass) ctx->tuning.max_hits_per_pass = std::max<uint32_t>(4096, t->max_hits_per_pass);
    if (t->initial_candidates) ctx->tuning.initial_candidates = std::max<uint32_t>(1024, t->initial_candidates);
    if (t->filter_cap) ctx->tuning.filter_cap = std::min<uint32_t>(256, std::max<uint32_t>(32, t->filter_cap & ~31u));
    if (t->filter_claim)
        ctx->tuning.filter_claim = t->filter_claim == 1 ? 1u : std::min<uint32_t>(4096, std::max<uint32_t>(32, t->filter_claim));
    if (t->gapped_pool_blocks) ctx->tuning.gapped_pool_blocks = t->gapped_pool_blocks == 0xffffffffu ? 0u : t->gapped_pool_blocks;
    if (t->gapped_cells) {
        if (t->gapped_cells != 4 && t->gapped_cells != 8) {
            set_error("gapped_cells must be 4 or 8");
            return GXY_EINVAL;
        }
        ctx->tuning.gapped_cells = t->gapped_cells;
    }
    return GXY_OK;
}

gxy_status gxy_ctx_get_tuning(gxy_ctx* ctx, gxy_tuning* t) {
    if (!ctx || !t) return GXY_EINVAL;
    std::lock_guard<std::mutex> g(ctx->mu);
    *t = ctx->tuning;
    return GXY_OK;
}

gxy_status gxy_dseq_upload(gxy_ctx* ctx, const gxy_packed_seq* host, gxy_dseq** out) {
    if (!ctx || !host || !out || (host->len && (!host->codes || !host->valid || !host->mask))) return GXY_EINVAL;
    if (host->len >= (1ull << 32)) {
        set_error("sequences are limited to u32 positions (src/pos_table.rs:56)");
        return GXY_EUNSUPPORTED;
    }
    API_TRY(set_device(ctx));
    WorkerLease L(ctx);
    if (!L.w) return L.err;
    gxy_dseq* d = nullptr;
    API_TRY(dseq_alloc(ctx, host->len, &d, L.w->st));
    gxy_status s = dseq_fill_host(d, host, L.w->st);
    if (s == GXY_OK && cudaStreamSynchronize(L.w->st) != cudaSuccess) s = GXY_ECUDA;
    if (s != GXY_OK) {
        dseq_destroy(d);
        return s;
    }
    *out = d;
    return GXY_OK;
}

gxy_status gxy_dseq_from_ascii(gxy_ctx* ctx, const uint8_t* ascii, uint64_t n, gxy_dseq** out) {
    if (!ctx || (!ascii && n) || !out) return GXY_EINVAL;
    if (n >= (1ull << 32)) return GXY_EUNSUPPORTED;
    API_TRY(set_device(ctx));
    WorkerLease L(ctx);
    if (!L.w) return L.err;
    gxy_dseq* d = nullptr;
    API_TRY(dseq_alloc(ctx, n, &d, L.w->st));
    void* dbuf = nullptr;
    cudaError_t e = cudaSuccess;
    if (n) {
        e = cudaMalloc(&dbuf, n);
        if (e == cudaSuccess) e = cudaMemcpyAsync(dbuf, ascii, n, cudaMemcpyHostToDevice, L.w->st);
        if (e == cudaSuccess) launch_pack_ascii(static_cast<uint8_t*>(dbuf), n, d->codes, d->valid, d->mask, L.w->st);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(L.w->st);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (dbuf) cudaFree(dbuf);
    if (e != cudaSuccess) {
        dseq_destroy(d);
        set_error(std::string("pack: ") + cudaGetErrorString(e));
        return GXY_ECUDA;
    }
    *out = d;
    return GXY_OK;
}

gxy_status gxy_dseq_reverse_complement(gxy_ctx* ctx, const gxy_dseq* in, gxy_dseq** out) {
    if (!ctx || !in || !out) return GXY_EINVAL;
    API_TRY(set_device(ctx));
    WorkerLease L(ctx);
    if (!L.w) return L.err;
    gxy_dseq* d = nullptr;
    API_TRY(dseq_alloc(ctx, in->len, &d, L.w->st));
    launch_reverse_complement(in->codes, in->valid, in->mask, in->len, d->codes, d->valid, d->mask, L.w->st);
    cudaError_t e = cudaStreamSynchronize(L.w->st);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) {
        dseq_destroy(d);
        set_error(std::string("reverse complement: ") + cudaGetErrorString(e));
        return GXY_ECUDA;
    }
    *out = d;
    return GXY_OK;
}

gxy_status gxy_dseq_download(const gxy_dseq* s, uint8_t* codes, uint8_t* valid, uint8_t* mask) {
    if (!s) return GXY_EINVAL;
    API_TRY(set_device(s->ctx));
    const uint64_t n = s->len;
    if (!n) return GXY_OK;
    if (codes) API_CK(cudaMemcpy(codes, reinterpret_cast<const char*>(s->codes) + kPad / 4, (n + 3) / 4,
                                 cudaMemcpyDeviceToHost));
    if (valid) API_CK(cudaMemcpy(valid, reinterpret_cast<const char*>(s->valid) + kPad / 8, (n + 7) / 8,
                                 cudaMemcpyDeviceToHost));
    if (mask) API_CK(cudaMemcpy(mask, reinterpret_cast<const char*>(s->mask) + kPad / 8, (n + 7) / 8,
                                cudaMemcpyDeviceToHost));
    return GXY_OK;
}

uint64_t gxy_dseq_len(const gxy_dseq* s) { return s ? s->len : 0; }

gxy_status gxy_dseq_free(gxy_dseq* s) {
    if (!s) return GXY_OK;
    cudaSetDevice(s->device);
    dseq_destroy(s);
    return GXY_OK;
}

gxy_status gxy_table_build(gxy_ctx* ctx, const gxy_packed_seq* target, const char* pattern01, uint32_t step,
                           uint32_t max_word_count, gxy_table** out) {
    if (!ctx || !target || !out) return GXY_EINVAL;
    if (step < 1) {
        set_error("step must be >= 1 (src/pos_table.rs:36)");
        return GXY_EINVAL;
    }
    Pattern pat;
    API_TRY(parse_pattern(pattern01, pat));
    gxy_dseq* d = nullptr;
    API_TRY(gxy_dseq_upload(ctx, target, &d));
    gxy_table* t = nullptr;
    gxy_status s = build_table(ctx, d, 0, d->len, pat, step, max_word_count, &t);
    if (s != GXY_OK) {
        dseq_destroy(d);
        return s;
    }
    t->owned = d;
    t->hc = target->codes;
    t->hv = target->valid;
    t->hm = target->mask;
    t->hlen = target->len;
    *out = t;
    return GXY_OK;
}

gxy_status gxy_table_build_view(gxy_ctx* ctx, const gxy_dseq* target, uint64_t lo, uint64_t hi,
                                const char* pattern01, uint32_t step, uint32_t max_word_count, gxy_table** out) {
    if (!ctx || !target || !out || lo > hi || hi > target->len) return GXY_EINVAL;
    if (step < 1) {
        set_error("step must be >= 1 (src/pos_table.rs:36)");
        return GXY_EINVAL;
    }
    Pattern pat;
    API_TRY(parse_pattern(pattern01, pat));
    API_TRY(set_device(ctx));
    return build_table(ctx, target, lo, hi, pat, step, max_word_count, out);
}

gxy_status gxy_table_build_views(gxy_ctx* ctx, const gxy_dseq* target, uint32_t n, const uint64_t* lo,
                                 const uint64_t* hi, const char* pattern01, uint32_t step, uint32_t max_word_count,
                                 gxy_table** out) {
    if (!ctx || !target || !out || (n && (!lo || !hi))) return GXY_EINVAL;
    for (uint32_t v = 0; v < n; v++)
        if (lo[v] > hi[v] || hi[v] > target->len) {
            set_error("view outside the sequence");
            return GXY_EINVAL;
        }
    if (step < 1) {
        set_error("step must be >= 1 (src/pos_table.rs:36)");
        return GXY_EINVAL;
    }
    if (n == 0) return GXY_OK;
    Pattern pat;
    API_TRY(parse_pattern(pattern01, pat));
    API_TRY(set_device(ctx));
    if (pat.weight >= 3 && (uint64_t)n << (2 * pat.weight) < (1ull << 32))
        return build_tables(ctx, target, n, lo, hi, pat, step, max_word_count, out);
    // Views of under 32 buckets, or more buckets than 32-bit starts can
    // index: one build per view.
    for (uint32_t v = 0; v < n; v++) {
        const gxy_status s = build_tables(ctx, target, 1, lo + v, hi + v, pat, step, max_word_count, out + v);
        if (s != GXY_OK) {
            for (uint32_t u = 0; u < v; u++) {
                gxy_table_free(out[u]);
                out[u] = nullptr;
            }
            return s;
        }
    }
    return GXY_OK;
}

gxy_status gxy_table_prune_hot_words(gxy_table* t, uint32_t limit) {
    if (!t) return GXY_EINVAL;
    API_TRY(set_device(t->ctx));
    WorkerLease L(t->ctx);
    if (!L.w) return L.err;
    return prune_table(t, limit, L.w);
}

gxy_status gxy_table_info(const gxy_table* t, uint64_t* num_words, uint64_t* n_positions, uint32_t* pattern_len,
                          uint32_t* weight) {
    if (!t) return GXY_EINVAL;
    if (num_words) *num_words = t->num_words;
    if (n_positions) *n_positions = t->npos;
    if (pattern_len) *pattern_len = t->pat.len;
    if (weight) *weight = t->pat.weight;
    return GXY_OK;
}

gxy_status gxy_table_download(const gxy_table* t, uint32_t* starts, uint32_t* positions) {
    if (!t) return GXY_EINVAL;
    API_TRY(set_device(t->ctx));
    if (starts) {
        API_CK(cudaMemcpy(starts, t->starts, (t->num_words + 1) * 4, cudaMemcpyDeviceToHost));
        // The table's own indices: from its first position on.
        if (t->pos_base)
            for (uint64_t w = 0; w <= t->num_words; w++) starts[w] -= t->pos_base;
    }
    if (positions && t->npos)
        API_CK(cudaMemcpy(positions, t->positions + t->pos_base, t->npos * 4, cudaMemcpyDeviceToHost));
    return GXY_OK;
}

gxy_status gxy_table_free(gxy_table* t) {
    if (!t) return GXY_OK;
    cudaSetDevice(t->device);
    if (t->own_arrays) {
        dev_free(t->starts);
        dev_free(t->positions);
    }
    t->mem.reset();
    dseq_destroy(t->owned);
    delete t;
    return GXY_OK;
}

gxy_status gxy_search(gxy_ctx* ctx, const gxy_table* table, const gxy_packed_seq* target,
                      const gxy_packed_seq* query, const gxy_search_params* params, gxy_hsp_buf* out,
                      gxy_stats* stats) {
    if (!ctx || !table || !target || !query || !params) return GXY_EINVAL;
    if (query->len && (!query->codes || !query->valid || !query->mask)) return GXY_EINVAL;
    if (query->len >= (1ull << 32)) return GXY_EUNSUPPORTED;
    API_TRY(set_device(ctx));
    WorkerLease L(ctx);
    if (!L.w) return L.err;
    Worker* W = L.w;
    SeqView T = table_view(table);
    if (!same_host_seq(table, target)) {
        if (target->len != table->hi - table->lo) {
            set_error("target length differs from the sequence the table was built on");
            return GXY_EINVAL;
        }
        if (!W->tstage || W->tstage->len < target->len) {
            dseq_destroy(W->tstage);
            W->tstage = nullptr;
            API_TRY(dseq_alloc(ctx, target->len, &W->tstage, W->st));
        }
        API_TRY(dseq_fill_host(W->tstage, target, W->st));
        T = view_of(W->tstage, 0, target->len);
    }
    if (!W->qstage || W->qstage->len < query->len || W->qstage->len > 2 * query->len + (1u << 20)) {
        dseq_destroy(W->qstage);
        W->qstage = nullptr;
        API_TRY(dseq_alloc(ctx, query->len, &W->qstage, W->st));
    }
    API_TRY(dseq_fill_host(W->qstage, query, W->st));
    const SeqView Q = view_of(W->qstage, 0, query->len);
    return search_impl(ctx, W, table, T, Q, params, out, stats);
}

gxy_status gxy_search_dseq(gxy_ctx* ctx, const gxy_table* table, const gxy_dseq* query,
                           const gxy_search_params* params, gxy_hsp_buf* out, gxy_stats* stats) {
    if (!ctx || !table || !query || !params) return GXY_EINVAL;
    API_TRY(set_device(ctx));
    WorkerLease L(ctx);
    if (!L.w) return L.err;
    const SeqView T = table_view(table);
    const SeqView Q = view_of(query, 0, query->len);
    return search_impl(ctx, L.w, table, T, Q, params, out, stats);
}

void gxy_hsp_buf_free(gxy_hsp_buf* buf) {
    if (!buf) return;
    free(buf->hsps);
    buf->hsps = nullptr;
    buf->len = buf->cap = 0;
}

// The shared body of gxy_batch_search and gxy_batch_records: validates the
// units, reverse-complements each query once per strand that needs it and
// runs the engine (n_units > 0).
static gxy_status batch_run(gxy_ctx* ctx, uint32_t n_tables, const gxy_table* const* tables, uint32_t n_queries,
                            const gxy_dseq* const* queries, uint32_t n_units, const gxy_unit* units,
                            const gxy_search_params* params, const gxy_batch_opts* opts, RunResult& r) {
    const Pattern& pat = tables[units[0].table]->pat;
    uint64_t max_cols = 0;
    for (uint32_t i = 0; i < n_units; i++) {
        const gxy_unit& u = units[i];
        if (u.table >= n_tables || u.query >= n_queries || u.strand > 1) {
            set_error("unit references a missing table or query, or a strand other than 0/1");
            return GXY_EINVAL;
        }
        const gxy_table* t = tables[u.table];
        if (t->pat.len != pat.len || t->pat.care_mask != pat.care_mask) {
            set_error("all tables of a batch must share one seed pattern");
            return GXY_EINVAL;
        }
        max_cols = std::max<uint64_t>(max_cols, std::min<uint64_t>(t->hi - t->lo, queries[u.query]->len));
    }
    API_TRY(check_params(params, max_cols));
    WorkerLease L(ctx);
    if (!L.w) return L.err;
    Worker* W = L.w;
    // Reverse complements once per query that needs one.
    for (gxy_dseq* d : W->rc_tmp) dseq_destroy(d);
    W->rc_tmp.clear();
    std::vector<int> qseg_of(2 * (size_t)n_queries, -1);
    std::vector<int> tseg_of(n_tables, -1);
    std::vector<SeqView> tsegs, qsegs;
    std::vector<UnitPlan> plan(n_units);
    for (uint32_t i = 0; i < n_units; i++) {
        const gxy_unit& u = units[i];
        const gxy_table* t = tables[u.table];
        if (tseg_of[u.table] < 0) {
            tseg_of[u.table] = (int)tsegs.size();
            tsegs.push_back(table_view(t));
        }
        const size_t qi = 2 * (size_t)u.query + u.strand;
        if (qseg_of[qi] < 0) {
            const gxy_dseq* q = queries[u.query];
            if (u.strand == 1) {
                gxy_dseq* rc = nullptr;
                API_TRY(dseq_alloc(ctx, q->len, &rc, W->st));
                launch_reverse_complement(q->codes, q->valid, q->mask, q->len, rc->codes, rc->valid, rc->mask, W->st);
                W->rc_tmp.push_back(rc);
                q = rc;
            }
            qseg_of[qi] = (int)qsegs.size();
            qsegs.push_back(view_of(q, 0, q->len));
        }
        plan[i].tseg = (uint32_t)tseg_of[u.table];
        plan[i].qseg = (uint32_t)qseg_of[qi];
        plan[i].starts = t->starts;
        plan[i].positions = t->positions;
        plan[i].occ = t->occ;
        plan[i].nwin = n_windows(queries[u.query]->len, pat.len, params->step);
        plan[i].primary_lo = u.primary_lo;
        plan[i].primary_hi = u.primary_hi;
        plan[i].avg_bucket = t->num_words ? (double)t->npos / (double)t->num_words : 0.0;
    }
    return run_units(ctx, W, plan, tsegs, qsegs, pat, *params, opts && opts->use_graph, r);
}

gxy_status gxy_batch_search(gxy_ctx* ctx, uint32_t n_tables, const gxy_table* const* tables, uint32_t n_queries,
                            const gxy_dseq* const* queries, uint32_t n_units, const gxy_unit* units,
                            const gxy_search_params* params, const gxy_batch_opts* opts, gxy_batch_result* out,
                            gxy_stats* stats) {
    if (!ctx || (!tables && n_tables) || (!queries && n_queries) || (!units && n_units) || !params || !out)
        return GXY_EINVAL;
    API_TRY(set_device(ctx));
    memset(out, 0, sizeof(*out));
    if (n_units == 0) {
        out->unit_offsets = static_cast<uint64_t*>(calloc(1, sizeof(uint64_t)));
        return GXY_OK;
    }
    RunResult r;
    API_TRY(batch_run(ctx, n_tables, tables, n_queries, queries, n_units, units, params, opts, r));
    if (stats) *stats = r.stats;
    const uint64_t n = r.hsps.size();
    out->hsps = static_cast<gxy_hsp*>(malloc(std::max<uint64_t>(n, 1) * sizeof(gxy_hsp)));
    out->unit_offsets = static_cast<uint64_t*>(calloc((size_t)n_units + 1, sizeof(uint64_t)));
    if (!out->hsps || !out->unit_offsets) {
        gxy_batch_result_free(out);
        set_error("host allocation of the batch result");
        return GXY_ENOMEM;
    }
    if (n) memcpy(out->hsps, r.hsps.data(), n * sizeof(gxy_hsp));
    for (uint64_t i = 0; i < n; i++) out->unit_offsets[r.unit[i] + 1]++;
    for (uint32_t u = 0; u < n_units; u++) out->unit_offsets[u + 1] += out->unit_offsets[u];
    out->n_hsps = n;
    out->n_units = n_units;
    return GXY_OK;
}

void gxy_batch_result_free(gxy_batch_result* r) {
    if (!r) return;
    free(r->hsps);
    free(r->unit_offsets);
    memset(r, 0, sizeof(*r));
}

gxy_status gxy_batch_records(gxy_ctx* ctx, uint32_t n_tables, const gxy_table* const* tables, uint32_t n_queries,
                             const gxy_dseq* const* queries, uint32_t n_units, const gxy_unit* units,
                             const gxy_unit_place* places, const gxy_search_params* params,
                             const gxy_batch_opts* opts, gxy_record_result* out, gxy_stats* stats) {
    if (!ctx || (!tables && n_tables) || (!queries && n_queries) || (!units && n_units) || (!places && n_units) ||
        !params || !out)
        return GXY_EINVAL;
    API_TRY(set_device(ctx));
    memset(out, 0, sizeof(*out));
    uint32_t n_groups = 0;
    for (uint32_t i = 0; i < n_units; i++) {
        if (units[i].table >= n_tables) {
            set_error("unit references a missing table");
            return GXY_EINVAL;
        }
        const gxy_table* t = tables[units[i].table];
        // build_ungapped_record adds the chunk start in u32 (src/driver.rs:459).
        if ((uint64_t)places[i].t_offset + (t->hi - t->lo) > (1ull << 32)) {
            set_error("t_offset + target length exceeds 2^32");
            return GXY_EINVAL;
        }
        if (places[i].group == UINT32_MAX) {
            set_error("group index 2^32 - 1 is reserved");
            return GXY_EINVAL;
        }
        n_groups = std::max(n_groups, places[i].group + 1);
    }
    out->group_offsets = static_cast<uint64_t*>(calloc((size_t)n_groups + 1, sizeof(uint64_t)));
    if (!out->group_offsets) {
        set_error("host allocation of the record result");
        return GXY_ENOMEM;
    }
    out->n_groups = n_groups;
    if (n_units == 0) return GXY_OK;
    static_assert(sizeof(Place) == sizeof(gxy_unit_place), "device and ABI place layouts differ");
    static_assert(sizeof(Record) == sizeof(gxy_record), "device and ABI record layouts differ");
    RunResult r;
    r.places = reinterpret_cast<const Place*>(places);
    gxy_status e = batch_run(ctx, n_tables, tables, n_queries, queries, n_units, units, params, opts, r);
    if (e != GXY_OK) {
        gxy_record_result_free(out);
        return e;
    }
    if (stats) *stats = r.stats;
    const uint64_t n = r.records.size();
    out->records = static_cast<gxy_record*>(malloc(std::max<uint64_t>(n, 1) * sizeof(gxy_record)));
    if (!out->records) {
        gxy_record_result_free(out);
        set_error("host allocation of the record result");
        return GXY_ENOMEM;
    }
    if (n) memcpy(out->records, r.records.data(), n * sizeof(gxy_record));
    for (uint64_t i = 0; i < n; i++) out->group_offsets[out->records[i].group + 1]++;
    for (uint32_t g = 0; g < n_groups; g++) out->group_offsets[g + 1] += out->group_offsets[g];
    out->n_records = n;
    out->n_groups = n_groups;
    return GXY_OK;
}

void gxy_record_result_free(gxy_record_result* r) {
    if (!r) return;
    free(r->records);
    free(r->group_offsets);
    memset(r, 0, sizeof(*r));
}

gxy_status gxy_chunk_plan(uint64_t target_len, uint32_t primary_bp, uint32_t halo_bp, uint64_t* quads, uint64_t cap,
                          uint64_t* n) {
    if (!n) return GXY_EINVAL;
    // chunk_target, src/driver.rs:156-194 (u32 arithmetic as the reference).
    const uint32_t t_len = (uint32_t)target_len;
    uint64_t k = 0;
    auto put = [&](uint64_t a, uint64_t b, uint64_t c, uint64_t d) {
        if (quads && k < cap) {
            quads[4 * k + 0] = a;
            quads[4 * k + 1] = b;
            quads[4 * k + 2] = c;
            quads[4 * k + 3] = d;
        }
        k++;
    };
    if (primary_bp == 0 || (uint64_t)t_len <= (uint64_t)primary_bp + halo_bp) {
        put(0, t_len, 0, t_len);
    } else {
        uint32_t ps = 0;
        while (ps < t_len) {
            const uint32_t pe = (uint32_t)std::min<uint64_t>((uint64_t)ps + primary_bp, t_len);
            const uint32_t lo = ps > halo_bp ? ps - halo_bp : 0;
            const uint32_t hi = (uint32_t)std::min<uint64_t>((uint64_t)pe + halo_bp, t_len);
            put(lo, hi, ps - lo, pe - lo);
            if (pe == t_len) break;
            ps = pe;
        }
    }
    *n = k;
    return (quads && k > cap) ? GXY_EOVERFLOW : GXY_OK;
}

gxy_status gxy_extend_hits(gxy_ctx* ctx, const gxy_dseq* target, const gxy_dseq* query,
                           const gxy_search_params* params, uint64_t n, const uint32_t* t_pos, const uint32_t* q_pos,
                           uint32_t seed_len, uint32_t mode, gxy_hsp* out, uint8_t* ok) {
    if (!ctx || !target || !query || !params || (n && (!t_pos || !q_pos || !out || !ok)) || seed_len > 32)
        return GXY_EINVAL;
    API_TRY(check_params(params, std::min<uint64_t>(target->len, query->len)));
    API_TRY(set_device(ctx));
    if (!n) return GXY_OK;
    WorkerLease L(ctx);
    if (!L.w) return L.err;
    cudaStream_t st = L.w->st;
    DevBuf bt, bq, bo, bk;
    cudaError_t e = bt.ensure(n * 4);
    if (e == cudaSuccess) e = bq.ensure(n * 4);
    if (e == cudaSuccess) e = bo.ensure(n * sizeof(Hsp));
    if (e == cudaSuccess) e = bk.ensure(n);
    if (e == cudaSuccess) e = cudaMemcpyAsync(bt.p, t_pos, n * 4, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(bq.p, q_pos, n * 4, cudaMemcpyHostToDevice, st);
    Score sc;
    memcpy(sc.sub, params->sub, sizeof(sc.sub));
    sc.ambig = params->ambig;
    sc.xdrop = params->xdrop;
    sc.hspthresh = params->hspthresh;
    if (e == cudaSuccess)
        launch_extend_hits(view_of(target, 0, target->len), view_of(query, 0, query->len), sc, bt.as<uint32_t>(),
                           bq.as<uint32_t>(), n, seed_len, mode, bo.as<Hsp>(), bk.as<uint8_t>(), st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, bo.p, n * sizeof(Hsp), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ok, bk.p, n, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = cudaGetLastError();
    bt.release(); bq.release(); bo.release(); bk.release();
    if (e != cudaSuccess) {
        set_error(std::string("extend_hits: ") + cudaGetErrorString(e));
        return GXY_ECUDA;
    }
    return GXY_OK;
}

}  // extern "C"
