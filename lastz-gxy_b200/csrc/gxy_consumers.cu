// gxy_consumers.cu -- the two direct consumers of the HSP list:
//  - choose_anchor (src/anchor.rs:25-69): one warp per HSP on the device.
//  - best_chain (src/chain.rs:19-69): the same chain, found in O(n log n)
//    on the host instead of the reference's O(n^2) scan.
#include <algorithm>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "gxy_engine.cuh"

using namespace gxy;

namespace {

// ---------------------------------------------------------------------------
// choose_anchor: column scores along the HSP's diagonal, the w-column window
// with the highest sum (the first one on ties: the reference updates on `>`),
// anchor = window start + w / 2.  One warp per HSP: window sums are
// P[s + w] - P[s] over prefix sums P, so the warp walks the starts 32 at a
// time with two running prefix scans, one at the window's start and one at
// its end, and keeps the best (sum, start).
// ---------------------------------------------------------------------------
__device__ __forceinline__ int32_t anchor_col(const SeqView& T, const SeqView& Q, uint32_t t, uint32_t q,
                                              const int32_t* lut, int32_t ambig) {
    const uint64_t tg = T.base + t, qg = Q.base + q;
    const uint32_t tc = (uint32_t)(__ldg(T.codes + (tg >> 5)) >> (2 * (tg & 31))) & 3u;
    const uint32_t qc = (uint32_t)(__ldg(Q.codes + (qg >> 5)) >> (2 * (qg & 31))) & 3u;
    const bool v = ((__ldg(T.valid + (tg >> 5)) >> (tg & 31)) & 1u) && ((__ldg(Q.valid + (qg >> 5)) >> (qg & 31)) & 1u);
    return v ? lut[(tc << 2) | qc] : ambig;
}

// Inclusive warp scan; every lane gets its prefix, lane 31 the chunk total.
__device__ __forceinline__ int32_t warp_incl(int32_t x) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int32_t y = __shfl_up_sync(kFull, x, o);
        if (lane >= o) x += y;
    }
    return x;
}

__global__ void k_anchors(SeqView T, SeqView Q, Score sc, const gxy_hsp* hsps, uint64_t n, uint32_t window,
                          uint32_t* out_t, uint32_t* out_q) {
    __shared__ int32_t s_lut[16];
    if (threadIdx.x < 16) s_lut[threadIdx.x] = sc.sub[threadIdx.x];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const uint64_t nw = (uint64_t)gridDim.x * (blockDim.x >> 5);
    for (uint64_t h = blockIdx.x * (uint64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); h < n; h += nw) {
        const gxy_hsp H = hsps[h];
        const uint32_t len = H.length;
        const uint32_t w = window < 1 ? 1 : (window > len ? len : window);
        // P[w] = sum of the first w columns.
        int32_t pw = 0;
        for (uint32_t c = 0; c < w; c += 32) {
            const uint32_t k = c + lane;
            int32_t x = k < w ? anchor_col(T, Q, H.t_start + k, H.q_start + k, s_lut, sc.ambig) : 0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(kFull, x, o);
            pw += x;
        }
        // Starts 0 .. len - w, 32 at a time.
        int32_t ca = 0, cb = pw;   // P[c] and P[c + w]
        int32_t best = INT32_MIN;
        uint32_t best_start = 0;
        const uint32_t nstart = len - w + 1;
        for (uint32_t c = 0; c < nstart; c += 32) {
            const uint32_t s = c + lane;
            const bool on = s < nstart;
            // Column s leaves the window and column s + w enters it.
            const int32_t xa = on ? anchor_col(T, Q, H.t_start + s, H.q_start + s, s_lut, sc.ambig) : 0;
            const int32_t xb = (on && s + w < len)
                                   ? anchor_col(T, Q, H.t_start + s + w, H.q_start + s + w, s_lut, sc.ambig)
                                   : 0;
            const int32_t ia = warp_incl(xa), ib = warp_incl(xb);
            // Window at start s: P[s + w] - P[s] = (cb + ib - xb) - (ca + ia - xa).
            const int32_t win = (cb + ib - xb) - (ca + ia - xa);
            int32_t v = on ? win : INT32_MIN;
            uint32_t at = s;
            // Warp max; on equal sums the smaller start wins.
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const int32_t v2 = __shfl_xor_sync(kFull, v, o);
                const uint32_t a2 = __shfl_xor_sync(kFull, at, o);
                if (v2 > v || (v2 == v && a2 < at)) {
                    v = v2;
                    at = a2;
                }
            }
            if (v > best) {
                best = v;
                best_start = at;
            }
            ca += __shfl_sync(kFull, ia, 31);
            cb += __shfl_sync(kFull, ib, 31);
        }
        if (lane == 0) {
            const uint32_t mid = best_start + w / 2;
            out_t[h] = H.t_start + mid;
            out_q[h] = H.q_start + mid;
        }
    }
}

struct WorkerLease {
    gxy_ctx* ctx;
    Worker* w;
    gxy_status err;
    explicit WorkerLease(gxy_ctx* c) : ctx(c), w(nullptr), err(GXY_OK) { w = checkout(c, &err); }
    ~WorkerLease() {
        if (w) checkin(ctx, w);
    }
};

}  // namespace

extern "C" {

gxy_status gxy_choose_anchors(gxy_ctx* ctx, const gxy_dseq* target, const gxy_dseq* query,
                              const gxy_search_params* params, const gxy_hsp* hsps, uint64_t n, uint32_t window,
                              uint32_t* t_pos, uint32_t* q_pos) {
    if (!ctx || !target || !query || !params || (n && (!hsps || !t_pos || !q_pos))) return GXY_EINVAL;
    for (uint64_t i = 0; i < n; i++) {
        const gxy_hsp& h = hsps[i];
        if (h.length == 0) {
            set_error("empty HSP cannot be anchored (src/anchor.rs:32)");
            return GXY_EINVAL;
        }
        if ((uint64_t)h.t_start + h.length > target->len || (uint64_t)h.q_start + h.length > query->len) {
            set_error("HSP extends past its sequence");
            return GXY_EINVAL;
        }
    }
    if (n == 0) return GXY_OK;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return GXY_ECUDA;
    WorkerLease L(ctx);
    if (!L.w) return L.err;
    cudaStream_t st = L.w->st;
    gxy_hsp* dh = nullptr;
    uint32_t* dt = nullptr;
    cudaError_t e = cudaMallocAsync((void**)&dh, n * sizeof(gxy_hsp), st);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&dt, n * 8, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dh, hsps, n * sizeof(gxy_hsp), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        Score sc;
        memcpy(sc.sub, params->sub, sizeof(sc.sub));
        sc.ambig = params->ambig;
        sc.xdrop = params->xdrop;
        sc.hspthresh = params->hspthresh;
        const uint64_t blocks = std::min<uint64_t>((n + 7) / 8, (uint64_t)ctx->sm_count * 16);
        count_launch();
        k_anchors<<<(unsigned)blocks, 256, 0, st>>>(view_of(target, 0, target->len), view_of(query, 0, query->len),
                                                      sc, dh, n, window, dt, dt + n);
        e = cudaMemcpyAsync(t_pos, dt, n * 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(q_pos, dt + n, n * 4, cudaMemcpyDeviceToHost, st);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = cudaGetLastError();
    cudaFreeAsync(dh, st);
    cudaFreeAsync(dt, st);
    cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        set_error(std::string("choose_anchors: ") + cudaGetErrorString(e));
        return GXY_ECUDA;
    }
    return GXY_OK;
}

// best_chain (src/chain.rs:19-69).  The reference sorts by (t_start, q_start)
// (stable), and for HSP i takes best[i] = score_i + best[j] of the first j
// (in sorted order) with the largest best[j] > 0 among those that end
// before i on both axes (t_end_j <= t_start_i, q_end_j <= q_start_i); the
// chain ends at the first i with the largest best.  Any such j has
// t_start_j < t_end_j <= t_start_i, so it precedes i in the sorted order,
// and the predecessors of i are exactly the HSPs whose t_end has been
// reached when i's t_start is: a sweep in t order that activates HSPs by
// t_end and asks a prefix-maximum tree over q_end for (best, first index)
// finds the same chain in O(n log n).
gxy_status gxy_best_chain(const gxy_hsp* hsps, uint64_t n, gxy_hsp* out, uint64_t* out_n) {
    if ((n && (!hsps || !out)) || !out_n) return GXY_EINVAL;
    *out_n = 0;
    if (n == 0) return GXY_OK;
    for (uint64_t i = 0; i < n; i++)
        if (hsps[i].length == 0) {
            // Every predecessor must then start strictly before its successor,
            // which the sweep relies on; search() never returns empty HSPs.
            set_error("empty HSP in best_chain input");
            return GXY_EINVAL;
        }
    std::vector<uint64_t> ord(n);
    std::iota(ord.begin(), ord.end(), 0);
    std::stable_sort(ord.begin(), ord.end(), [&](uint64_t a, uint64_t b) {
        return hsps[a].t_start != hsps[b].t_start ? hsps[a].t_start < hsps[b].t_start
                                                  : hsps[a].q_start < hsps[b].q_start;
    });
    std::vector<gxy_hsp> s(n);
    for (uint64_t i = 0; i < n; i++) s[i] = hsps[ord[i]];
    // q_end coordinates, compressed.
    std::vector<uint64_t> qe(n);
    for (uint64_t i = 0; i < n; i++) qe[i] = (uint64_t)s[i].q_start + s[i].length;
    std::vector<uint64_t> qs = qe;
    std::sort(qs.begin(), qs.end());
    qs.erase(std::unique(qs.begin(), qs.end()), qs.end());
    const size_t m = qs.size();
    // Fenwick tree of (best, -index) maxima over q_end ranks.
    struct Key {
        int64_t best;
        int64_t idx;   // sorted position; smaller wins ties
    };
    auto better = [](const Key& a, const Key& b) { return a.best > b.best || (a.best == b.best && a.idx < b.idx); };
    const Key none{INT64_MIN, INT64_MAX};
    std::vector<Key> fen(m + 1, none);
    auto update = [&](size_t r, Key k) {
        for (size_t x = r + 1; x <= m; x += x & (~x + 1))
            if (better(k, fen[x])) fen[x] = k;
    };
    auto query = [&](size_t r_incl) {   // best over ranks [0, r_incl]
        Key k = none;
        for (size_t x = r_incl + 1; x > 0; x -= x & (~x + 1))
            if (better(fen[x], k)) k = fen[x];
        return k;
    };
    // Activation order: by t_end.
    std::vector<uint64_t> by_end(n);
    std::iota(by_end.begin(), by_end.end(), 0);
    std::sort(by_end.begin(), by_end.end(), [&](uint64_t a, uint64_t b) {
        return (uint64_t)s[a].t_start + s[a].length < (uint64_t)s[b].t_start + s[b].length;
    });
    std::vector<int64_t> best(n);
    std::vector<int64_t> parent(n, -1);
    uint64_t act = 0;
    for (uint64_t i = 0; i < n; i++) {
        while (act < n && (uint64_t)s[by_end[act]].t_start + s[by_end[act]].length <= s[i].t_start) {
            const uint64_t j = by_end[act++];
            const size_t r = std::lower_bound(qs.begin(), qs.end(), qe[j]) - qs.begin();
            update(r, Key{best[j], (int64_t)j});
        }
        int64_t prev = 0, pidx = -1;
        // Predecessors need q_end <= q_start_i.
        const size_t cnt = std::upper_bound(qs.begin(), qs.end(), (uint64_t)s[i].q_start) - qs.begin();
        if (cnt) {
            const Key k = query(cnt - 1);
            if (k.idx != INT64_MAX && k.best > 0) {
                prev = k.best;
                pidx = k.idx;
            }
        }
        best[i] = prev + s[i].score;
        parent[i] = pidx;
    }
    uint64_t end = 0;
    for (uint64_t i = 1; i < n; i++)
        if (best[i] > best[end]) end = i;
    std::vector<gxy_hsp> chain;
    for (int64_t c = (int64_t)end; c >= 0; c = parent[c]) chain.push_back(s[c]);
    std::reverse(chain.begin(), chain.end());
    memcpy(out, chain.data(), chain.size() * sizeof(gxy_hsp));
    *out_n = chain.size();
    return GXY_OK;
}

}  // extern "C"
