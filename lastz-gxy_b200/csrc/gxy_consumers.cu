// gxy_consumers.cu -- the two direct consumers of the HSP list:
//  - choose_anchor (src/anchor.rs:25-69): one warp per HSP on the device.
//  - best_chain (src/chain.rs:19-69): for many groups of HSPs at once on the
//    device (gxy_best_chain_groups: one block per group runs the
//    reference's O(n^2) scan with its threads over the predecessors), and
//    for one group on the host in O(n log n) (gxy_best_chain).
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

// ---------------------------------------------------------------------------
// best_chain (src/chain.rs:19-69) for many groups on the device.  The HSPs
// come sorted by (group, t_start, q_start) -- stably, as the reference's
// sort_by_key -- as structure-of-arrays.  One block per group walks i in
// that order; its threads scan the predecessors j < i (t_end_j <= t_start_i,
// q_end_j <= q_start_i, best_j > 0) and a block reduction keeps the largest
// best, the smallest j on ties: the reference's first j with the largest
// best (its update is a strict `>`).  Groups of at most kChainSmem HSPs keep
// their ends and bests in shared memory.
// ---------------------------------------------------------------------------
constexpr uint32_t kChainThreads = 256;
constexpr uint32_t kChainSmem = 4096;

struct ChainSoA {
    const uint32_t* ts;
    const uint32_t* te;   // t_start + length
    const uint32_t* qs;
    const uint32_t* qe;   // q_start + length
    const int32_t* score;
};

// (best, index) with the larger best first, the smaller index on ties.
__device__ __forceinline__ bool chain_better(int64_t b, int64_t i, int64_t b2, int64_t i2) {
    return b > b2 || (b == b2 && i < i2);
}

__device__ __forceinline__ void chain_reduce(int64_t& b, int64_t& i, int64_t* sb, int64_t* si) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const int64_t ob = __shfl_xor_sync(kFull, b, o), oi = __shfl_xor_sync(kFull, i, o);
        if (chain_better(ob, oi, b, i)) {
            b = ob;
            i = oi;
        }
    }
    if (lane == 0) {
        sb[w] = b;
        si[w] = i;
    }
    __syncthreads();
    if (w == 0) {
        b = lane < (int)(kChainThreads / 32) ? sb[lane] : INT64_MIN;
        i = lane < (int)(kChainThreads / 32) ? si[lane] : INT64_MAX;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const int64_t ob = __shfl_xor_sync(kFull, b, o), oi = __shfl_xor_sync(kFull, i, o);
            if (chain_better(ob, oi, b, i)) {
                b = ob;
                i = oi;
            }
        }
        if (lane == 0) {
            sb[0] = b;
            si[0] = i;
        }
    }
    __syncthreads();
    b = sb[0];
    i = si[0];
    __syncthreads();
}

template <bool kSmem>
__global__ __launch_bounds__(kChainThreads) void k_chain_groups(ChainSoA h, const uint64_t* goff, uint32_t n_groups,
                                                                int64_t* best_g, int32_t* parent, uint32_t* end_out) {
    __shared__ int64_t sb[kChainThreads / 32], si[kChainThreads / 32];
    extern __shared__ __align__(16) unsigned char chain_smem[];
    for (uint32_t g = blockIdx.x; g < n_groups; g += gridDim.x) {
        const uint64_t lo = goff[g];
        const uint32_t m = (uint32_t)(goff[g + 1] - lo);
        if (kSmem != (m <= kChainSmem)) continue;   // the other instantiation takes it
        if (m == 0) continue;
        const uint32_t* te = h.te + lo;
        const uint32_t* qe = h.qe + lo;
        int64_t* best = best_g + lo;
        if (kSmem) {
            // ends and bests of the group staged in shared memory
            int64_t* s_best = reinterpret_cast<int64_t*>(chain_smem);
            uint32_t* s_te = reinterpret_cast<uint32_t*>(s_best + kChainSmem);
            uint32_t* s_qe = s_te + kChainSmem;
            for (uint32_t j = threadIdx.x; j < m; j += kChainThreads) {
                s_te[j] = te[j];
                s_qe[j] = qe[j];
            }
            __syncthreads();
            te = s_te;
            qe = s_qe;
            best = s_best;
        }
        for (uint32_t i = 0; i < m; i++) {
            const uint32_t tsi = h.ts[lo + i], qsi = h.qs[lo + i];
            int64_t bb = 0, bj = INT64_MAX;   // best_prev_score starts at 0 (src/chain.rs:37)
            for (uint32_t j = threadIdx.x; j < i; j += kChainThreads) {
                if (te[j] <= tsi && qe[j] <= qsi) {
                    const int64_t bjv = best[j];
                    if (bjv > bb || (bjv == bb && bjv > 0 && (int64_t)j < bj)) {
                        bb = bjv;
                        bj = j;
                    }
                }
            }
            chain_reduce(bb, bj, sb, si);
            if (threadIdx.x == 0) {
                const bool found = bj != INT64_MAX && bb > 0;
                best[i] = (found ? bb : 0) + h.score[lo + i];
                parent[lo + i] = found ? (int32_t)bj : -1;
            }
            __syncthreads();
        }
        // The chain ends at the first HSP with the largest best.
        int64_t eb = INT64_MIN, ei = INT64_MAX;
        for (uint32_t i = threadIdx.x; i < m; i += kChainThreads)
            if (chain_better(best[i], i, eb, ei)) {
                eb = best[i];
                ei = i;
            }
        chain_reduce(eb, ei, sb, si);
        if (threadIdx.x == 0) end_out[g] = (uint32_t)ei;
        if (kSmem) {
            for (uint32_t j = threadIdx.x; j < m; j += kChainThreads) best_g[lo + j] = best[j];
        }
        __syncthreads();
    }
}

// Walks each group's parents from its end: the chain's length, then its
// HSPs (sorted positions) into out_idx[lo .. lo + len) in t_start order.
__global__ void k_chain_trace(const uint64_t* goff, uint32_t n_groups, const int32_t* parent, const uint32_t* end,
                              uint32_t* out_idx, uint64_t* len_out) {
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < n_groups; g += gridDim.x * blockDim.x) {
        const uint64_t lo = goff[g];
        const uint32_t m = (uint32_t)(goff[g + 1] - lo);
        if (m == 0) {
            len_out[g] = 0;
            continue;
        }
        uint32_t len = 0;
        for (int32_t c = (int32_t)end[g]; c >= 0; c = parent[lo + c]) len++;
        uint32_t k = len;
        for (int32_t c = (int32_t)end[g]; c >= 0; c = parent[lo + c]) out_idx[lo + --k] = (uint32_t)c;
        len_out[g] = len;
    }
}

__global__ void k_chain_group_ids(const uint64_t* goff, uint32_t n_groups, uint32_t* gid) {
    for (uint32_t g = blockIdx.x; g < n_groups; g += gridDim.x)
        for (uint64_t i = goff[g] + threadIdx.x; i < goff[g + 1]; i += blockDim.x) gid[i] = g;
}

// key[i] = field f of hsp[perm[i]] (perm null: i): 0 q_start, 1 t_start, 2 group.
__global__ void k_chain_keys(const gxy_hsp* hsp, const uint32_t* gid, const uint32_t* perm, uint64_t n, int f,
                             uint32_t* key, uint32_t* val) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t j = perm ? perm[i] : (uint32_t)i;
        key[i] = f == 0 ? hsp[j].q_start : (f == 1 ? hsp[j].t_start : gid[j]);
        val[i] = j;
    }
}

__global__ void k_chain_soa(const gxy_hsp* hsp, const uint32_t* perm, uint64_t n, uint32_t* ts, uint32_t* te,
                            uint32_t* qs, uint32_t* qe, int32_t* sc) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const gxy_hsp x = hsp[perm[i]];
        ts[i] = x.t_start;
        te[i] = x.t_start + x.length;
        qs[i] = x.q_start;
        qe[i] = x.q_start + x.length;
        sc[i] = x.score;
    }
}

__global__ void k_chain_gather(const gxy_hsp* hsp, const uint32_t* perm, const uint32_t* idx, const uint64_t* goff,
                               const uint64_t* len, uint32_t n_groups, gxy_hsp* out) {
    for (uint32_t g = blockIdx.x; g < n_groups; g += gridDim.x) {
        const uint64_t lo = goff[g];
        for (uint64_t k = threadIdx.x; k < len[g]; k += blockDim.x) out[lo + k] = hsp[perm[lo + idx[lo + k]]];
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

// best_chain for n_groups groups on the device: group g is
// hsps[group_offsets[g] .. group_offsets[g + 1]); its chain goes to
// out[group_offsets[g] ..] in t_start order and its length to chain_len[g].
gxy_status gxy_best_chain_groups(gxy_ctx* ctx, const gxy_hsp* hsps, const uint64_t* group_offsets, uint32_t n_groups,
                                 gxy_hsp* out, uint64_t* chain_len) {
    if (!ctx || !group_offsets || (n_groups && !chain_len)) return GXY_EINVAL;
    const uint64_t n = n_groups ? group_offsets[n_groups] : 0;
    for (uint32_t g = 0; g < n_groups; g++)
        if (group_offsets[g + 1] < group_offsets[g]) {
            set_error("group offsets must not decrease");
            return GXY_EINVAL;
        }
    if (n && (!hsps || !out)) return GXY_EINVAL;
    if (group_offsets[0] != 0) {
        set_error("group_offsets[0] must be 0");
        return GXY_EINVAL;
    }
    if (n >= (1ull << 31)) {
        set_error("more than 2^31 HSPs");
        return GXY_EUNSUPPORTED;
    }
    if (n_groups == 0) return GXY_OK;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return GXY_ECUDA;
    WorkerLease L(ctx);
    if (!L.w) return L.err;
    Worker* W = L.w;
    cudaStream_t st = W->st;
    const size_t nn = std::max<uint64_t>(n, 1);
    // One allocation: HSPs, offsets, group ids, two key/value ping-pongs,
    // the structure of arrays, bests, parents, ends, trace and lengths.
    const size_t off_hsp = 0, off_goff = off_hsp + nn * 16, off_gid = off_goff + ((size_t)n_groups + 1) * 8,
                 off_k0 = off_gid + nn * 4, off_v0 = off_k0 + nn * 4, off_k1 = off_v0 + nn * 4, off_v1 = off_k1 + nn * 4,
                 off_ts = off_v1 + nn * 4, off_te = off_ts + nn * 4, off_qs = off_te + nn * 4, off_qe = off_qs + nn * 4,
                 off_sc = off_qe + nn * 4, off_best = (off_sc + nn * 4 + 7) & ~(size_t)7, off_par = off_best + nn * 8,
                 off_end = off_par + nn * 4, off_idx = off_end + (size_t)n_groups * 4,
                 off_len = (off_idx + nn * 4 + 7) & ~(size_t)7, off_out = off_len + (size_t)n_groups * 8,
                 total = off_out + nn * 16;
    unsigned char* base = nullptr;
    cudaError_t e = cudaMallocAsync((void**)&base, total, st);
    if (e != cudaSuccess) {
        set_error(std::string("best_chain_groups allocation: ") + cudaGetErrorString(e));
        return GXY_ENOMEM;
    }
    gxy_hsp* dh = reinterpret_cast<gxy_hsp*>(base + off_hsp);
    uint64_t* dg = reinterpret_cast<uint64_t*>(base + off_goff);
    uint32_t* gid = reinterpret_cast<uint32_t*>(base + off_gid);
    uint32_t *k0 = reinterpret_cast<uint32_t*>(base + off_k0), *v0 = reinterpret_cast<uint32_t*>(base + off_v0);
    uint32_t *k1 = reinterpret_cast<uint32_t*>(base + off_k1), *v1 = reinterpret_cast<uint32_t*>(base + off_v1);
    ChainSoA soa;
    uint32_t* ts = reinterpret_cast<uint32_t*>(base + off_ts);
    uint32_t* te = reinterpret_cast<uint32_t*>(base + off_te);
    uint32_t* qs = reinterpret_cast<uint32_t*>(base + off_qs);
    uint32_t* qe = reinterpret_cast<uint32_t*>(base + off_qe);
    int32_t* sc = reinterpret_cast<int32_t*>(base + off_sc);
    soa.ts = ts;
    soa.te = te;
    soa.qs = qs;
    soa.qe = qe;
    soa.score = sc;
    int64_t* best = reinterpret_cast<int64_t*>(base + off_best);
    int32_t* parent = reinterpret_cast<int32_t*>(base + off_par);
    uint32_t* endi = reinterpret_cast<uint32_t*>(base + off_end);
    uint32_t* idx = reinterpret_cast<uint32_t*>(base + off_idx);
    uint64_t* len = reinterpret_cast<uint64_t*>(base + off_len);
    gxy_hsp* dout = reinterpret_cast<gxy_hsp*>(base + off_out);
    if (n) e = cudaMemcpyAsync(dh, hsps, n * 16, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && n) e = cudaMemsetAsync(dout, 0, n * 16, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dg, group_offsets, ((size_t)n_groups + 1) * 8, cudaMemcpyHostToDevice, st);
    const int gb = (int)std::min<uint64_t>(std::max<uint64_t>(1, (n + 255) / 256), (uint64_t)ctx->sm_count * 8);
    const int grp_blocks = (int)std::min<uint32_t>(n_groups, (uint32_t)ctx->sm_count * 16);
    if (e == cudaSuccess && n) {
        // Stable sort by (group, t_start, q_start): least significant field first.
        count_launch(1);
        k_chain_group_ids<<<grp_blocks, 256, 0, st>>>(dg, n_groups, gid);
        const uint32_t* perm = nullptr;
        for (int f = 0; f < 3; f++) {
            RadixPass rp[8];
            int bits = 32;
            if (f == 2) {
                bits = 1;
                while (bits < 32 && (1ull << bits) < n_groups) bits++;
            }
            const int np = plan_radix(0, bits, 0, 0, rp, 8);
            count_launch(1);
            k_chain_keys<<<gb, 256, 0, st>>>(dh, gid, perm, n, f, k0, v0);
            const int which = radix_sort_u32(k0, v0, k1, v1, nullptr, n, n, rp, np, W->ps, st);
            if (which) {
                e = cudaMemcpyAsync(v0, v1, n * 4, cudaMemcpyDeviceToDevice, st);
                if (e != cudaSuccess) break;
            }
            perm = v0;
        }
        count_launch(1);
        k_chain_soa<<<gb, 256, 0, st>>>(dh, v0, n, ts, te, qs, qe, sc);
        const size_t smem = kChainSmem * (8 + 4 + 4);
        if (e == cudaSuccess) e = cudaFuncSetAttribute(k_chain_groups<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                       (int)smem);
        count_launch(3);
        k_chain_groups<true><<<grp_blocks, kChainThreads, smem, st>>>(soa, dg, n_groups, best, parent, endi);
        k_chain_groups<false><<<grp_blocks, kChainThreads, 0, st>>>(soa, dg, n_groups, best, parent, endi);
        k_chain_trace<<<(n_groups + 127) / 128, 128, 0, st>>>(dg, n_groups, parent, endi, idx, len);
        count_launch(1);
        k_chain_gather<<<grp_blocks, 128, 0, st>>>(dh, v0, idx, dg, len, n_groups, dout);
        if (e == cudaSuccess) e = cudaMemcpyAsync(out, dout, n * 16, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(chain_len, len, (size_t)n_groups * 8, cudaMemcpyDeviceToHost, st);
    } else if (e == cudaSuccess) {
        for (uint32_t g = 0; g < n_groups; g++) chain_len[g] = 0;
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = cudaGetLastError();
    cudaFreeAsync(base, st);
    cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        set_error(std::string("best_chain_groups: ") + cudaGetErrorString(e));
        return GXY_ECUDA;
    }
    return GXY_OK;
}

}  // extern "C"
