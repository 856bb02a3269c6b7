// gxy_filter.cu -- seed-hit enumeration fused with an upper-bound x-drop
// filter, for sm_100a.
//
// search() (src/seed_search.rs:92-116) extends every admitted seed hit, but
// only a hit whose HSP reaches hspthresh changes the output: the diagonal
// filter records cover for passing HSPs only (src/seed_search.rs:113).  So a
// hit that provably cannot reach hspthresh can be dropped before anything
// else looks at it.  This kernel proves it cheaply, without writing the raw
// hits to HBM:
//
//  - Enumeration, as in k_enumerate: one warp per tile of 32 query windows;
//    each lane forms its window's seed word and transition variants
//    (src/seed_search.rs:76-90) and reads the bounds of each variant's bucket
//    (src/pos_table.rs:102-108).  A bucket is looked up in `starts` only when
//    the table's occupancy bitmap says it is non-empty (about two thirds of
//    the variant words of a 10 Mbp target are empty buckets).  The hits go
//    into a per-warp queue in shared memory.
//  - Filter: one lane per queued hit runs extend_one_side
//    (src/hsp.rs:160-195) on both sides with every column score replaced by
//    an upper bound -- the largest score of the column's class
//    x = t_code ^ q_code (match, the two transversion classes, transition);
//    invalid columns take a class whose bound is >= the ambiguous score.
//    With scores raised, every running sum and best is raised and the drop
//    best - run can only shrink, so the bounded side breaks no earlier and
//    its best is an upper bound of the exact best.  The break is tested
//    every 32 columns only, which again can only raise the best.  Four
//    columns are scored per step through a 256-entry table of (sum, maximum
//    prefix) indexed by the four columns' classes.  A hit survives when the
//    bounded seed footprint + both sides' bests reach hspthresh, or when a
//    side is still running after f_cap columns.
//  - Survivors go to the hit array, where the exact screen (k_screen) takes
//    them: about 2-5 % of the raw hits on chromosome-scale inputs.
//
// The dropped hits are exactly hits whose exact score is below hspthresh, so
// the pipeline's output does not change.
#include "gxy_kernels.cuh"

#include <algorithm>
#include <atomic>

namespace gxy {

namespace {

constexpr int kQCap = 512;                      // queued hits per warp
constexpr int kLutBytes = 256 * 32 * 8;         // (sum, max prefix) x 32 lane copies
constexpr int kFilterWarps = 16;                // warps per block (one block per SM)

// Columns whose bit in `keep` is clear take the classes of `pat`.
__device__ __forceinline__ uint64_t fold_cols(uint64_t x, uint32_t keep, uint64_t pat) {
    const uint64_t m = spread_bits_to_pairs(keep);
    return (x & m) | (pat & ~m);
}

struct FSide {
    int32_t run;
    int32_t best;
};

// Four columns (byte g of w, column k at bits 2k..2k+1): the table entry of
// the byte gives their bounded sum and the maximum of their four prefix sums.
// The entry of byte b for lane l sits at b * 256 + l * 8, so the 16 lanes of
// each half-warp read distinct banks; one byte permute forms that address.
__device__ __forceinline__ void f_group(FSide& S, uint32_t w, uint32_t lane8, int g, const unsigned char* lut) {
    const uint32_t ad = __byte_perm(w, lane8, 0x5504u | ((uint32_t)g << 4));
    const int2 e = *reinterpret_cast<const int2*>(lut + ad);
    S.best = max(S.best, S.run + e.y);
    S.run += e.x;
}

// 32 columns of two independent sides, interleaved so that the two serial
// chains issue side by side.
__device__ __forceinline__ void f_scan2(FSide& A, uint64_t xa, FSide& B, uint64_t xb, uint32_t lane8,
                                        const unsigned char* lut) {
    const uint32_t a0 = (uint32_t)xa, a1 = (uint32_t)(xa >> 32);
    const uint32_t b0 = (uint32_t)xb, b1 = (uint32_t)(xb >> 32);
#pragma unroll
    for (int g = 0; g < 4; g++) {
        f_group(A, a0, lane8, g, lut);
        f_group(B, b0, lane8, g, lut);
    }
#pragma unroll
    for (int g = 0; g < 4; g++) {
        f_group(A, a1, lane8, g, lut);
        f_group(B, b1, lane8, g, lut);
    }
}

template <uint32_t kRegVar, int NW>
__global__ __launch_bounds__(NW * 32, 1) void k_seed_filter(const __grid_constant__ ScreenArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    unsigned char* lut = smem;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint2* queue = reinterpret_cast<uint2*>(smem + kLutBytes) + wid * kQCap;
    for (uint32_t i = threadIdx.x; i < 256u * 32u; i += blockDim.x) {
        const uint32_t b = i >> 5;
        int32_t p = 0, mp = INT32_MIN;
#pragma unroll
        for (int c = 0; c < 4; c++) {
            p += a.fub[(b >> (2 * c)) & 3u];
            mp = max(mp, p);
        }
        reinterpret_cast<int2*>(lut)[i] = make_int2(p, mp);
    }
    __syncthreads();

    const uint32_t lane8 = (uint32_t)lane * 8u, lt = lanemask_lt();
    const uint32_t L = a.pat.len;
    const int32_t X = a.sc.xdrop, thresh = a.sc.hspthresh;
    const int32_t need = thresh - a.f_seed_max;   // both sides' bests below this: no seed can lift the hit
    const int32_t ub0 = a.fub[0];
    const uint32_t ntile = a.tile_hi - a.tile_lo;
    unsigned long long n_windows = 0, n_raw = 0, n_cols = 0;
    uint32_t qn = 0, qunit = 0xffffffffu;         // queue fill and the unit of the queued hits
    SeqView T{}, Q{};

    // Runs the bounded x-drop over queue[0, qn) and empties the queue.
    auto flush = [&]() {
        __syncwarp();
        uint32_t head = 0;
        bool busy = false, ralive = false, lalive = false;
        uint32_t ht = 0, hq = 0, rext = 0, lext = 0, rrem = 0, lrem = 0;
        int32_t rrun = 0, rbest = 0, lrun = 0, lbest = 0;
        for (;;) {
            const uint32_t im = __ballot_sync(kFull, !busy);
            if (!busy) {
                const uint32_t i = head + __popc(im & lt);
                if (i < qn) {
                    const uint2 e = queue[i];
                    ht = e.x;
                    hq = e.y;
                    busy = true;
                    rrem = min(T.len - ht - L, Q.len - hq - L);
                    lrem = min(ht, hq);
                    rrun = rbest = lrun = lbest = 0;
                    rext = lext = 0;
                    ralive = rrem > 0;
                    lalive = lrem > 0;
                }
            }
            head = min(qn, head + (uint32_t)__popc(im));
            if (!__any_sync(kFull, busy)) break;

            // The next chunk of each running side: right chunks read upwards
            // from the column after the last one scanned, left chunks are the
            // 32 positions below it, reversed (column 0 next to the seed).
            const uint32_t nr = ralive ? min(32u, rrem) : 0u, nl = lalive ? min(32u, lrem) : 0u;
            uint64_t xr = 0, xl = 0;
            uint32_t vr = kFull, vl = kFull;
            if (nr) {
                const uint64_t tg = T.base + ht + L + rext, qg = Q.base + hq + L + rext;
                xr = load_codes32(T.codes, tg) ^ load_codes32(Q.codes, qg);
                vr = load_bits32(T.valid, tg) & load_bits32(Q.valid, qg);
            }
            if (nl) {
                const uint64_t tg = T.base + ht - lext - 32, qg = Q.base + hq - lext - 32;
                xl = rev_pairs64(load_codes32(T.codes, tg) ^ load_codes32(Q.codes, qg));
                vl = __brev(load_bits32(T.valid, tg) & load_bits32(Q.valid, qg));
            }
            const bool slow = (nr && (nr < 32 || vr != kFull)) || (nl && (nl < 32 || vl != kFull));
            if (__any_sync(kFull, slow)) {
                // Invalid columns take the invalid class; columns past the
                // side's end take the lowest class (bound <= 0), so they raise
                // no prefix maximum.
                const uint32_t er = nr >= 32 ? kFull : ((1u << nr) - 1u);
                const uint32_t el = nl >= 32 ? kFull : ((1u << nl) - 1u);
                xr = fold_cols(fold_cols(xr, vr, a.f_inv), er, a.f_end);
                xl = fold_cols(fold_cols(xl, vl, a.f_inv), el, a.f_end);
            }
            FSide R{rrun, rbest}, Lf{lrun, lbest};
            f_scan2(R, xr, Lf, xl, lane8, lut);
            n_cols += nr + nl;
            if (nr) {
                rrun = R.run;
                rbest = R.best;
                rext += nr;
                rrem -= nr;
                ralive = rrem > 0 && rbest - rrun <= X;
            }
            if (nl) {
                lrun = Lf.run;
                lbest = Lf.best;
                lext += nl;
                lrem -= nl;
                lalive = lrem > 0 && lbest - lrun <= X;
            }
            const bool capped = busy && ((ralive && rext >= a.f_cap) || (lalive && lext >= a.f_cap));
            const bool done = busy && (capped || (!ralive && !lalive));
            bool surv = done && (capped || rbest + lbest >= need);
            if (__any_sync(kFull, surv && !capped)) {
                if (surv && !capped) {
                    // The seed footprint's bound: all L columns (src/hsp.rs:119-123).
                    const uint64_t tg = T.base + ht, qg = Q.base + hq;
                    const uint64_t x = fold_cols(load_codes32(T.codes, tg) ^ load_codes32(Q.codes, qg),
                                                 load_bits32(T.valid, tg) & load_bits32(Q.valid, qg), a.f_inv);
                    int32_t sd = 0;
#pragma unroll
                    for (int g = 0; g < 8; g++) {
                        if (4u * g >= L) break;
                        const uint32_t w = g < 4 ? (uint32_t)x : (uint32_t)(x >> 32);
                        const uint32_t r = min(4u, L - 4u * g);
                        uint32_t byte = (w >> (8 * (g & 3))) & 0xFFu;
                        if (r < 4) byte &= (1u << (2 * r)) - 1u;   // columns past L: class 0, taken off below
                        const int2 e = *reinterpret_cast<const int2*>(lut + (byte << 8) + lane8);
                        sd += e.x - (int32_t)(4u - r) * ub0;
                    }
                    surv = sd + rbest + lbest >= thresh;
                }
            }
            const uint32_t sm = __ballot_sync(kFull, surv);
            if (sm) {
                unsigned long long base = 0;
                if (lane == 0) base = atomicAdd(a.hit_count, (unsigned long long)__popc(sm));
                base = __shfl_sync(kFull, base, 0);
                if (surv) {
                    const unsigned long long slot = base + __popc(sm & lt);
                    if (slot < a.hit_cap) {
                        Hit h;
                        h.t = ht;
                        h.q = hq;
                        h.unit = qunit;
                        a.hits[slot] = h;
                    }
                }
            }
            if (done) busy = false;
        }
        qn = 0;
        __syncwarp();
    };

    // Tiles are claimed two at a time, the next claim made while the current
    // tiles are processed (as in k_enumerate).
    constexpr uint32_t kClaim = 2;
    uint32_t next = 0;
    if (lane == 0) next = atomicAdd(a.tile_counter, kClaim);
    for (;;) {
        const uint32_t batch = __shfl_sync(kFull, next, 0);
        if (batch >= ntile) break;
        if (lane == 0) next = atomicAdd(a.tile_counter, kClaim);
        const uint32_t batch_end = min(ntile, batch + kClaim);
        for (uint32_t tl = batch; tl < batch_end; tl++) {
            const uint32_t tile = tl + a.tile_lo;
            uint32_t lo = 0, hi = a.n_units;
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) >> 1;
                if (a.units[mid].tile_base <= tile) lo = mid;
                else hi = mid;
            }
            const uint32_t u = lo;
            const UnitDev U = a.units[u];
            const uint32_t k = (tile - U.tile_base) * 32 + lane;
            const uint32_t q = k * a.step;
            uint32_t word = 0;
            bool wv = false;
            if (k < U.nwin) wv = word_at(a.qsegs[U.qseg], a.pat, q, word);
            n_windows += wv ? 1 : 0;
            // Bucket bounds of every variant: the occupancy bit first, the
            // `starts` pair only for non-empty buckets.
            uint32_t rb[kRegVar], rc[kRegVar], ob[kRegVar];
#pragma unroll
            for (uint32_t v = 0; v < kRegVar; v++) {
                ob[v] = 0;
                if (wv && v < a.n_var) ob[v] = __ldg(U.occ + ((word ^ a.var_xor[v]) >> 5));
            }
            uint32_t tot = 0;
#pragma unroll
            for (uint32_t v = 0; v < kRegVar; v++) {
                rb[v] = 0;
                rc[v] = 0;
                const uint32_t vw = word ^ a.var_xor[v];
                if (wv && v < a.n_var && ((ob[v] >> (vw & 31u)) & 1u)) {
                    rb[v] = __ldg(U.starts + vw);
                    rc[v] = __ldg(U.starts + vw + 1) - rb[v];
                    tot += rc[v];
                }
            }
            if (wv) {
                for (uint32_t v = kRegVar; v < a.n_var; v++) {
                    const uint32_t vw = word ^ a.var_xor[v];
                    if ((__ldg(U.occ + (vw >> 5)) >> (vw & 31u)) & 1u)
                        tot += __ldg(U.starts + vw + 1) - __ldg(U.starts + vw);
                }
            }
            uint32_t incl = tot;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(kFull, incl, o);
                if (lane >= o) incl += y;
            }
            const uint32_t wtot = __shfl_sync(kFull, incl, 31);
            if (wtot == 0) continue;
            n_raw += lane == 0 ? wtot : 0;
            if (u != qunit) {
                if (qn) flush();
                qunit = u;
                T = a.tsegs[U.tseg];
                Q = a.qsegs[U.qseg];
            }
            // Queue the tile's hits [0, wtot) (this lane's are [off, off + tot)),
            // in rounds when they do not fit.
            const uint32_t off = incl - tot;
            for (uint32_t r0 = 0; r0 < wtot;) {
                if (qn >= (uint32_t)kQCap) flush();
                const uint32_t r1 = min(wtot, r0 + ((uint32_t)kQCap - qn));
                uint2* dst = queue + qn;   // hit index j goes to dst[j - r0]
                uint32_t o = off;
#pragma unroll
                for (uint32_t v = 0; v < kRegVar; v++) {
                    const uint32_t b = rb[v], c = rc[v];
                    if (c && c <= 16) {
                        const uint32_t j0 = max(o, r0), j1 = min(o + c, r1);
                        for (uint32_t j = j0; j < j1; j++) dst[j - r0] = make_uint2(__ldg(U.positions + b + (j - o)), q);
                    }
                    uint32_t bm = __ballot_sync(kFull, c > 16 && o < r1 && o + c > r0);
                    while (bm) {
                        const int src = __ffs(bm) - 1;
                        bm &= bm - 1;
                        const uint32_t bb = __shfl_sync(kFull, b, src), cc = __shfl_sync(kFull, c, src);
                        const uint32_t oo = __shfl_sync(kFull, o, src), qq = __shfl_sync(kFull, q, src);
                        const uint32_t j0 = max(oo, r0), j1 = min(oo + cc, r1);
                        for (uint32_t j = j0 + lane; j < j1; j += 32)
                            dst[j - r0] = make_uint2(__ldg(U.positions + bb + (j - oo)), qq);
                    }
                    o += c;
                }
                for (uint32_t v = kRegVar; v < a.n_var; v++) {
                    uint32_t b = 0, c = 0;
                    if (wv) {
                        const uint32_t vw = word ^ a.var_xor[v];
                        if ((__ldg(U.occ + (vw >> 5)) >> (vw & 31u)) & 1u) {
                            b = __ldg(U.starts + vw);
                            c = __ldg(U.starts + vw + 1) - b;
                        }
                    }
                    if (c && c <= 16) {
                        const uint32_t j0 = max(o, r0), j1 = min(o + c, r1);
                        for (uint32_t j = j0; j < j1; j++) dst[j - r0] = make_uint2(__ldg(U.positions + b + (j - o)), q);
                    }
                    uint32_t bm = __ballot_sync(kFull, c > 16 && o < r1 && o + c > r0);
                    while (bm) {
                        const int src = __ffs(bm) - 1;
                        bm &= bm - 1;
                        const uint32_t bb = __shfl_sync(kFull, b, src), cc = __shfl_sync(kFull, c, src);
                        const uint32_t oo = __shfl_sync(kFull, o, src), qq = __shfl_sync(kFull, q, src);
                        const uint32_t j0 = max(oo, r0), j1 = min(oo + cc, r1);
                        for (uint32_t j = j0 + lane; j < j1; j += 32)
                            dst[j - r0] = make_uint2(__ldg(U.positions + bb + (j - oo)), qq);
                    }
                    o += c;
                }
                qn += r1 - r0;
                r0 = r1;
            }
            if (qn >= a.f_flush) flush();
        }
    }
    if (qn) flush();
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) n_windows += __shfl_xor_sync(kFull, n_windows, o);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) n_cols += __shfl_xor_sync(kFull, n_cols, o);
    if (lane == 0) {
        atomicAdd(&a.stats[0], n_windows);
        atomicAdd(&a.stats[1], n_raw);
        atomicAdd(&a.stats[3], n_cols);
    }
}

__global__ void k_occupancy(const uint32_t* __restrict__ starts, uint64_t nw, uint32_t* __restrict__ occ) {
    const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
    const uint64_t w0 = (uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const uint32_t lane = threadIdx.x & 31;
    for (uint64_t base = w0 * 32; base < nw; base += warps * 32) {
        const uint64_t w = base + lane;
        const bool set = w < nw && __ldg(starts + w + 1) > __ldg(starts + w);
        const uint32_t m = __ballot_sync(kFull, set);
        if (lane == 0) occ[base >> 5] = m;
    }
}

// Dynamic shared memory of k_seed_filter: the table and the warps' queues.
constexpr size_t kFilterSmem = (size_t)kLutBytes + (size_t)kFilterWarps * kQCap * sizeof(uint2);

template <uint32_t kRegVar>
void launch_filter_t(const ScreenArgs& a, int sm_count, cudaStream_t st) {
    // The attribute is set once per device (it belongs to the device's context).
    static std::atomic<uint64_t> ready{0};
    int dev = 0;
    cudaGetDevice(&dev);
    const uint64_t bit = 1ull << (dev & 63);
    if (!(ready.load(std::memory_order_acquire) & bit)) {
        cudaFuncSetAttribute(k_seed_filter<kRegVar, kFilterWarps>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kFilterSmem);
        ready.fetch_or(bit, std::memory_order_acq_rel);
    }
    k_seed_filter<kRegVar, kFilterWarps><<<sm_count, kFilterWarps * 32, kFilterSmem, st>>>(a);
}

}  // namespace

bool filter_bounds(ScreenArgs& a) {
    // Per class x = t ^ q: the largest score among the four (t, q) pairs of
    // that class.  sub is indexed (t << 2) | q (src/scoring.rs:32-40).
    int32_t ub[4];
    for (int x = 0; x < 4; x++) {
        int32_t m = INT32_MIN;
        for (int t = 0; t < 4; t++) m = std::max(m, a.sc.sub[(t << 2) | (t ^ x)]);
        ub[x] = m;
    }
    // Invalid columns score `ambig`: they take the class with the smallest
    // bound that is still >= ambig.  Past-the-end columns take the lowest
    // class, whose bound must be <= 0 (else a bounded side would never
    // break and the filter keeps nothing).
    int inv = -1, end = 0;
    for (int x = 0; x < 4; x++) {
        if (ub[x] >= a.sc.ambig && (inv < 0 || ub[x] < ub[inv])) inv = x;
        if (ub[x] < ub[end]) end = x;
    }
    if (inv < 0 || ub[end] > 0) return false;
    int64_t top = ub[0];
    for (int x = 1; x < 4; x++) top = std::max<int64_t>(top, ub[x]);
    // The bounded sums stay in i32: 4-column sums and prefixes are small,
    // and a side's run over f_cap columns is within the exact envelope the
    // host already checked for the scores' magnitude.
    for (int x = 0; x < 4; x++) a.fub[x] = ub[x];
    auto repeat = [](int x) {
        uint64_t p = 0;
        for (int k = 0; k < 32; k++) p |= (uint64_t)x << (2 * k);
        return p;
    };
    a.f_inv = repeat(inv);
    a.f_end = repeat(end);
    a.f_seed_max = (int32_t)(top * (int64_t)a.pat.len);
    return true;
}

void launch_seed_filter(const ScreenArgs& a, int sm_count, int /*warps_per_block*/, cudaStream_t st) {
    count_launch();
    if (a.n_var == 1) launch_filter_t<1>(a, sm_count, st);
    else if (a.n_var == 13) launch_filter_t<13>(a, sm_count, st);
    else launch_filter_t<16>(a, sm_count, st);
}

void launch_occupancy(const uint32_t* starts, uint64_t num_words, uint32_t* occ, cudaStream_t st) {
    const uint64_t words = (num_words + 31) / 32;
    const int blocks = (int)std::min<uint64_t>((words + 7) / 8, 148 * 16);
    count_launch();
    k_occupancy<<<std::max(blocks, 1), 256, 0, st>>>(starts, num_words, occ);
}

}  // namespace gxy
