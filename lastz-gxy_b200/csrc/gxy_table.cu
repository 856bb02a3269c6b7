// gxy_table.cu -- PosTable::build (src/pos_table.rs:35-83) on the device, for
// one view of a sequence or for many views at once (the driver's chunk
// tables, src/driver.rs:156-210).
//
// The reference counts every seedable window's word, scans the counts into
// bucket starts and scatters the positions in ascending order through
// per-word cursors (src/pos_table.rs:42-75): a stable counting sort of the
// windows by word.  Here the same order comes from a stable LSD radix sort of
// (view, word, position) triples by (view, word), 8 bits a pass:
//
//  1. the first pass computes each window's word from the sequence as it
//     histograms and scatters (no key array is read), drops the unseedable
//     windows, and counts the kept ones on the device;
//  2. the remaining passes sort the kept triples, and the last one writes the
//     positions straight into the tables' positions array (view after view);
//  3. k_tbl_first finds where each view's run begins in the sorted keys, and
//     k_tbl_starts walks the sorted keys once: where the word changes from a
//     to b inside a view, that view's buckets a+1 .. b start at this index
//     (less the view's first index), which fills every view's `starts` and
//     occupancy bitmap without atomics on 4^w counters; runs of empty buckets
//     longer than kInlineGap go to k_tbl_gaps, a block each.
//
// Positions inside a bucket come out ascending -- the reference's order --
// because every pass is stable and the windows enter in position order.
#include "gxy_engine.cuh"
#include "gxy_kernels.cuh"
#include "gxy_radix.cuh"

#include <vector>

namespace gxy {

namespace {

// The seedable windows of n views of one sequence, step apart: item i is
// window i - woff[v] of the view v with woff[v] <= i < woff[v + 1], at
// view-local position (i - woff[v]) * step; its key is (v << wbits) | word
// (SeedExtractor::word_at, src/seeds.rs:133-147), its value the position.
struct ViewsSrc {
    const uint64_t* codes;
    const uint32_t* valid;
    const uint32_t* mask;
    const uint64_t* vbase;   // per view: its first position in the sequence arrays
    const uint32_t* vlen;    // per view: its length
    const uint64_t* woff;    // n_views + 1 window offsets
    Pattern pat;
    uint32_t step;
    uint32_t n_views;
    uint32_t wbits;
    __device__ __forceinline__ uint32_t view_at(uint64_t i) const {
        uint32_t lo = 0, hi = n_views;   // the last v with woff[v] <= i
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (woff[mid] <= i) lo = mid;
            else hi = mid;
        }
        return lo;
    }
    __device__ __forceinline__ bool load(uint64_t i, uint32_t& k, uint32_t& p) const {
        const uint32_t v = view_at(i);
        const SeqView sv{codes, valid, mask, vbase[v], vlen[v], 0u};
        p = (uint32_t)(i - woff[v]) * step;
        uint32_t w;
        if (!word_at(sv, pat, p, w)) return false;
        k = (v << wbits) | w;
        return true;
    }
    __device__ __forceinline__ bool key(uint64_t i, uint32_t& k) const {
        uint32_t p;
        return load(i, k, p);
    }
};

constexpr uint32_t kInlineGap = 64;   // empty-bucket runs up to this long are filled inline

struct StartsArgs {
    const uint32_t* keys;   // sorted (view, word) keys
    const uint32_t* n_dev;  // kept windows
    uint64_t n_cap;
    uint64_t nw;            // buckets per view
    uint32_t wbits;
    uint32_t n_views;
    uint32_t* first;        // n_views + 1: index of each view's first key (n at the end)
    uint32_t* starts;       // n_views x (nw + 1)
    uint32_t* occ;          // n_views x occ_words
    uint64_t occ_words;
    uint4* gaps;            // (view, first bucket, last bucket, value)
    uint32_t* n_gaps;
};

// first[v] for the views whose run begins at index i (empty views included).
__global__ void k_tbl_first(StartsArgs a) {
    const uint64_t n = min((uint64_t)*a.n_dev, a.n_cap);
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i <= n; i += (uint64_t)gridDim.x * blockDim.x) {
        const int64_t vp = i ? (int64_t)(a.keys[i - 1] >> a.wbits) : -1;
        const int64_t vc = i < n ? (int64_t)(a.keys[i] >> a.wbits) : (int64_t)a.n_views;
        for (int64_t v = vp + 1; v <= vc; v++) a.first[v] = (uint32_t)i;
    }
}

__device__ __forceinline__ void fill_run(const StartsArgs& a, uint32_t v, uint64_t lo, uint64_t hi, uint32_t val) {
    if (hi < lo) return;
    if (hi - lo < kInlineGap) {
        uint32_t* s = a.starts + (uint64_t)v * (a.nw + 1);
        for (uint64_t w = lo; w <= hi; w++) s[w] = val;
    } else {
        // Runs this long are disjoint within a view: at most (nw + 1) / kInlineGap + 1 per view.
        const uint32_t g = atomicAdd(a.n_gaps, 1u);
        a.gaps[g] = make_uint4(v, (uint32_t)lo, (uint32_t)hi, val);
    }
}

// For i in [0, n]: inside one view, the buckets after the previous key's word
// up to this key's word start at i - first[view]; at a view change the old
// view's remaining buckets start at its size, the views in between are empty
// and the new view's buckets up to this word start at 0.
__global__ void k_tbl_starts(StartsArgs a) {
    const uint64_t n = min((uint64_t)*a.n_dev, a.n_cap);
    const uint32_t wmask = (uint32_t)(a.nw - 1);
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i <= n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t kc = i < n ? a.keys[i] : 0u;
        const int64_t vp = i ? (int64_t)(a.keys[i - 1] >> a.wbits) : -1;
        const int64_t vc = i < n ? (int64_t)(kc >> a.wbits) : (int64_t)a.n_views;
        const uint64_t wp = i ? (uint64_t)(a.keys[i - 1] & wmask) : 0;
        const uint64_t wc = kc & wmask;
        if (i < n && (i == 0 || a.keys[i - 1] != kc))
            atomicOr(&a.occ[(uint64_t)vc * a.occ_words + (wc >> 5)], 1u << (wc & 31u));
        if (vp == vc) {
            fill_run(a, (uint32_t)vc, wp + 1, wc, (uint32_t)(i - a.first[vc]));
            continue;
        }
        if (vp >= 0) fill_run(a, (uint32_t)vp, wp + 1, a.nw, (uint32_t)(i - a.first[vp]));
        for (int64_t v = vp + 1; v < vc; v++) fill_run(a, (uint32_t)v, 0, a.nw, 0u);
        if (vc < (int64_t)a.n_views) fill_run(a, (uint32_t)vc, 0, wc, 0u);
    }
}

__global__ void k_tbl_gaps(const uint4* __restrict__ gaps, const uint32_t* n_gaps, uint32_t* __restrict__ starts,
                           uint64_t nw) {
    const uint32_t ng = *n_gaps;
    for (uint32_t g = blockIdx.x; g < ng; g += gridDim.x) {
        const uint4 e = gaps[g];
        uint32_t* s = starts + (uint64_t)e.x * (nw + 1);
        for (uint64_t w = (uint64_t)e.y + threadIdx.x; w <= e.z; w += blockDim.x) s[w] = e.w;
    }
}

}  // namespace

void table_init() {
    cudaFuncSetAttribute(k_radix_scatter<uint32_t, ViewsSrc>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sizeof(SortSmem<uint32_t>));
}

int table_view_bits(uint32_t n_views) {
    int b = 0;
    while ((1ull << b) < n_views) b++;
    return b;
}

gxy_status sort_build_views(const gxy_dseq* seq, uint32_t n_views, const uint64_t* lo, const uint64_t* hi,
                            const Pattern& pat, uint32_t step, uint32_t* starts, uint32_t* positions, uint32_t* occ,
                            uint32_t* first_host, Worker* W) {
    cudaStream_t st = W->st;
    const uint64_t nw = 1ull << (2 * pat.weight);
    const uint64_t occ_words = (nw + 31) / 32;
    const uint32_t wbits = 2 * pat.weight;
    const int vbits = table_view_bits(n_views);
    if (n_views == 0 || wbits + vbits > 32) {
        set_error("views x words must fit a 32-bit key");
        return GXY_EUNSUPPORTED;
    }
    // The view table, one upload: vbase[n] and woff[n + 1] as u64, vlen[n] as u32.
    std::vector<uint64_t> meta((size_t)n_views * 3 + 1);
    uint64_t total = 0;
    for (uint32_t v = 0; v < n_views; v++) {
        meta[v] = kPad + lo[v];
        meta[n_views + v] = total;
        total += n_windows(hi[v] - lo[v], pat.len, step);
    }
    meta[2 * (size_t)n_views] = total;
    uint32_t* vlen_h = reinterpret_cast<uint32_t*>(meta.data() + 2 * (size_t)n_views + 1);
    for (uint32_t v = 0; v < n_views; v++) vlen_h[v] = (uint32_t)(hi[v] - lo[v]);
    if (total >= (1ull << 32)) {
        set_error("more than 2^32 windows in one table build");
        return GXY_EUNSUPPORTED;
    }
    const uint64_t cap = std::max<uint64_t>(total, 1);
    const uint64_t n_gap_cap = (uint64_t)n_views * ((nw + 1) / kInlineGap + 2);
    GXY_CK(W->tk0.ensure(cap * 4));
    GXY_CK(W->tk1.ensure(cap * 4));
    GXY_CK(W->tv0.ensure(std::max<uint64_t>(cap * 4, n_gap_cap * 16)));
    // tv1: the counters (kept windows, empty-bucket runs), first[n_views + 1]
    // and the view table.
    const size_t off_first = 64, off_meta = (off_first + ((size_t)n_views + 1) * 4 + 15) & ~(size_t)15;
    GXY_CK(W->tv1.ensure(off_meta + meta.size() * 8));
    unsigned char* t1 = static_cast<unsigned char*>(W->tv1.p);
    uint32_t* cnt = reinterpret_cast<uint32_t*>(t1);
    uint32_t* first = reinterpret_cast<uint32_t*>(t1 + off_first);
    const uint64_t* dmeta = reinterpret_cast<const uint64_t*>(t1 + off_meta);
    GXY_CK(cudaMemcpyAsync(t1 + off_meta, meta.data(), meta.size() * 8, cudaMemcpyHostToDevice, st));
    GXY_CK(cudaMemsetAsync(cnt, 0, 8, st));
    GXY_CK(cudaMemsetAsync(occ, 0, (size_t)n_views * occ_words * 4, st));
    RadixPass rp[8];
    const int np = plan_radix(0, (int)wbits + vbits, 0, 0, rp, 8);
    // Pass 0 writes (A), pass p >= 1 alternates; the last pass's values land
    // in `positions`.
    const bool last_in_a = ((np - 1) & 1) == 0;
    uint32_t* ka = W->tk0.as<uint32_t>();
    uint32_t* kb = W->tk1.as<uint32_t>();
    uint32_t* va = last_in_a ? positions : W->tv0.as<uint32_t>();
    uint32_t* vb = last_in_a ? W->tv0.as<uint32_t>() : positions;
    if (total) {
        const ViewsSrc src{seq->codes,
                           seq->valid,
                           seq->mask,
                           dmeta,
                           reinterpret_cast<const uint32_t*>(dmeta + 2 * (size_t)n_views + 1),
                           dmeta + n_views,
                           pat,
                           step,
                           n_views,
                           wbits};
        const uint64_t want = (cap + 2 * (uint64_t)kSortTile - 1) / (2 * (uint64_t)kSortTile);
        const int grid = (int)std::max<uint64_t>(1, std::min<uint64_t>(want, (uint64_t)W->ps.sort_grid_max));
        count_launch(3);
        k_radix_hist<uint32_t><<<grid, kSortThreads, 0, st>>>(src, nullptr, total, cap, rp[0].shift, rp[0].bits,
                                                              W->ps.hist);
        k_radix_digit_scan<<<1 << rp[0].bits, 256, 0, st>>>(W->ps.hist, grid, W->ps.block_sums);
        k_radix_scatter<uint32_t><<<grid, kSortThreads, sizeof(SortSmem<uint32_t>), st>>>(
            src, ka, va, nullptr, total, cap, rp[0].shift, rp[0].bits, W->ps.hist, W->ps.block_sums, cnt);
        if (np > 1) radix_sort_u32(ka, va, kb, vb, cnt, 0, cap, rp + 1, np - 1, W->ps, st);
    }
    StartsArgs a;
    a.keys = last_in_a ? ka : kb;
    a.n_dev = cnt;
    a.n_cap = cap;
    a.nw = nw;
    a.wbits = wbits;
    a.n_views = n_views;
    a.first = first;
    a.starts = starts;
    a.occ = occ;
    a.occ_words = occ_words;
    // tv0 held the values of an earlier pass, done with by now: it takes the
    // empty-bucket runs.
    a.gaps = reinterpret_cast<uint4*>(W->tv0.p);
    a.n_gaps = cnt + 1;
    const int blocks = (int)std::min<uint64_t>((cap + 255) / 256 + 1, (uint64_t)W->ps.sort_grid_max * 2);
    count_launch(3);
    k_tbl_first<<<blocks, 256, 0, st>>>(a);
    k_tbl_starts<<<blocks, 256, 0, st>>>(a);
    k_tbl_gaps<<<W->ps.sort_grid_max, 256, 0, st>>>(a.gaps, a.n_gaps, starts, nw);
    GXY_CK(cudaGetLastError());
    if (first_host) {
        GXY_CK(cudaMemcpyAsync(first_host, first, ((size_t)n_views + 1) * 4, cudaMemcpyDeviceToHost, st));
        GXY_CK(cudaStreamSynchronize(st));
    }
    return GXY_OK;
}

}  // namespace gxy
