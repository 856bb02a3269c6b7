// gxy_filter.cu -- the upper-bound x-drop filter between seed-hit
// enumeration and the exact screen, for sm_100a.
//
// search() (src/seed_search.rs:92-116) extends every admitted seed hit, but
// only a hit whose HSP reaches hspthresh changes the output: the diagonal
// filter records cover for passing HSPs only (src/seed_search.rs:113).  So a
// hit that provably cannot reach hspthresh can be dropped before the exact
// screen looks at it.  k_filter_hits proves it cheaply, one lane per raw hit
// of the hit array that k_enumerate wrote:
//
//  - it runs extend_one_side (src/hsp.rs:160-195) on both sides with every
//    column score replaced by an upper bound -- the largest score of the
//    column's class x = t_code ^ q_code (match, transition, and the two
//    transversion classes); invalid columns take a class whose bound is
//    >= the ambiguous score.  With scores raised, every running sum and best
//    is raised and the drop best - run can only shrink, so a bounded side
//    breaks no earlier and its best is an upper bound of the exact best.  The
//    break is tested every 32 columns only, which again can only raise the
//    best;
//  - four columns are scored per step through a 256-entry table of
//    (sum, maximum prefix) indexed by the four columns' classes: one byte
//    permute, one shared-memory load and three integer operations per four
//    columns, against five operations per column in the exact screen;
//  - a hit survives when the bounded seed footprint + both sides' bests reach
//    hspthresh, or when a side is still running after f_cap columns;
//  - target windows come from the table's interleaved copy of its target
//    (two 16-byte loads per 32-position window): the lanes' target positions
//    are random, and these gathers are what bounds the kernel, while a warp's
//    query positions come from one tile of windows.
//
// Survivors (about 1 % of the raw hits on chromosome-scale inputs) go to a
// second hit array, where the exact screen (k_screen) takes them.  The
// dropped hits are exactly hits whose exact score is below hspthresh, so the
// pipeline's output does not change.
#include "gxy_kernels.cuh"

#include <algorithm>

namespace gxy {

namespace {

constexpr int kLutBytes = 256 * 32 * 8;         // (sum, max prefix) x 32 lane copies
constexpr int kFilterWarps = 16;                // warps per block, two blocks per SM

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

__device__ __forceinline__ void lut_fill(unsigned char* lut, const int32_t* fub) {
    for (uint32_t i = threadIdx.x; i < 256u * 32u; i += blockDim.x) {
        const uint32_t b = i >> 5;
        int32_t p = 0, mp = INT32_MIN;
#pragma unroll
        for (int c = 0; c < 4; c++) {
            p += fub[(b >> (2 * c)) & 3u];
            mp = max(mp, p);
        }
        reinterpret_cast<int2*>(lut)[i] = make_int2(p, mp);
    }
}

// The seed footprint's bound: all L columns at (t, q) (src/hsp.rs:119-123).
__device__ __forceinline__ int32_t seed_bound(const SeqView& T, const SeqView& Q, uint32_t t, uint32_t q,
                                              uint32_t L, uint64_t f_inv, int32_t ub0, uint32_t lane8,
                                              const unsigned char* lut) {
    const uint64_t tg = T.base + t, qg = Q.base + q;
    uint64_t tc;
    uint32_t tv;
    load_window32(T, tg, tc, tv);
    const uint64_t x = fold_cols(tc ^ load_codes32(Q.codes, qg), tv & load_bits32(Q.valid, qg), f_inv);
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
    return sd;
}

// The bounded x-drop over the raw-hit array written by k_enumerate: one lane
// per hit, hits claimed by the warp in chunks from a global cursor and dealt
// to its idle lanes (as in k_screen).  A side still running after a chunk
// continues while the idle lanes take new hits.  Survivors go to a.hits.
template <int NW>
__global__ __launch_bounds__(NW * 32, 2) void k_filter_hits(const __grid_constant__ ScreenArgs a,
                                                             const __grid_constant__ FilterIO io) {
    extern __shared__ __align__(16) unsigned char smem[];
    unsigned char* lut = smem;
    lut_fill(lut, a.fub);
    __syncthreads();
    // Past the buffer's end the pass did not write (those tiles went to the
    // next pass).
    const uint32_t n_hits = (uint32_t)min(*io.raw_count, (unsigned long long)io.raw_cap);
    const int lane = threadIdx.x & 31;
    const uint32_t lane8 = (uint32_t)lane * 8u, lt = lanemask_lt();
    const uint32_t L = a.pat.len;
    const int32_t X = a.sc.xdrop, thresh = a.sc.hspthresh;
    const int32_t need = thresh - a.f_seed_max;
    const int32_t ub0 = a.fub[0];
    const uint32_t n_warps = gridDim.x * NW;
    const uint32_t chunk = a.f_claim ? a.f_claim : max(32u, min(512u, n_hits / max(1u, n_warps * 8u)));
    uint32_t wcur = 0, wend = 0;
    bool exhausted = false;
    unsigned long long n_cols = 0;

    bool busy = false, ralive = false, lalive = false;
    uint32_t ht = 0, hq = 0, hu = 0xffffffffu, cur_unit = 0xffffffffu;
    uint32_t rext = 0, lext = 0, rrem = 0, lrem = 0;
    int32_t rrun = 0, rbest = 0, lrun = 0, lbest = 0;
    SeqView T{}, Q{};
    for (;;) {
        const uint32_t im = __ballot_sync(kFull, !busy);
        const uint32_t need_n = __popc(im);
        const uint32_t avail = wend - wcur;
        uint32_t nb = 0, ncount = 0;
        if (need_n > avail && !exhausted) {
            if (lane == 0) nb = atomicAdd(io.cursor, chunk);
            nb = __shfl_sync(kFull, nb, 0);
            ncount = nb < n_hits ? min(chunk, n_hits - nb) : 0u;
            if (nb + chunk >= n_hits) exhausted = true;
        }
        if (!busy) {
            const uint32_t rk = __popc(im & lt);
            uint32_t hidx = 0xffffffffu;
            if (rk < avail) hidx = wcur + rk;
            else if (rk - avail < ncount) hidx = nb + (rk - avail);
            if (hidx != 0xffffffffu) {
                const Hit h = io.raw[hidx];
                ht = h.t;
                hq = h.q;
                hu = h.unit;
                if (hu != kNoUnit && hu != cur_unit) {
                    cur_unit = hu;
                    const UnitDev U = a.units[hu];
                    T = a.tsegs[U.tseg];
                    Q = a.qsegs[U.qseg];
                }
                busy = hu != kNoUnit;   // else an unused slot of a failed reservation
                if (busy) {
                    rrem = min(T.len - ht - L, Q.len - hq - L);
                    lrem = min(ht, hq);
                    rrun = rbest = lrun = lbest = 0;
                    rext = lext = 0;
                    ralive = rrem > 0;
                    lalive = lrem > 0;
                }
            }
        }
        {
            const uint32_t from_old = min(need_n, avail);
            if (ncount) {
                wcur = nb + min(need_n - from_old, ncount);
                wend = nb + ncount;
            } else {
                wcur += from_old;
            }
        }
        if (!__any_sync(kFull, busy)) {
            if (exhausted && wcur == wend) break;
            continue;
        }
        const uint32_t nr = ralive ? min(32u, rrem) : 0u, nl = lalive ? min(32u, lrem) : 0u;
        uint64_t xr = 0, xl = 0;
        uint32_t vr = kFull, vl = kFull;
        if (nr) {
            const uint64_t tg = T.base + ht + L + rext, qg = Q.base + hq + L + rext;
            uint64_t tc;
            uint32_t tv;
            load_window32(T, tg, tc, tv);
            xr = tc ^ load_codes32(Q.codes, qg);
            vr = tv & load_bits32(Q.valid, qg);
        }
        if (nl) {
            const uint64_t tg = T.base + ht - lext - 32, qg = Q.base + hq - lext - 32;
            uint64_t tc;
            uint32_t tv;
            load_window32(T, tg, tc, tv);
            xl = rev_pairs64(tc ^ load_codes32(Q.codes, qg));
            vl = __brev(tv & load_bits32(Q.valid, qg));
        }
        const bool slow = (nr && (nr < 32 || vr != kFull)) || (nl && (nl < 32 || vl != kFull));
        if (__any_sync(kFull, slow)) {
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
            if (surv && !capped) surv = seed_bound(T, Q, ht, hq, L, a.f_inv, ub0, lane8, lut) + rbest + lbest >= thresh;
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
                    h.unit = hu;
                    a.hits[slot] = h;
                }
            }
        }
        if (done) {
            busy = false;
            ralive = lalive = false;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) n_cols += __shfl_xor_sync(kFull, n_cols, o);
    if (lane == 0) atomicAdd(&a.stats[3], n_cols);
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

void filter_init() {
    cudaFuncSetAttribute(k_filter_hits<kFilterWarps>, cudaFuncAttributeMaxDynamicSharedMemorySize, kLutBytes);
}

void launch_filter_hits(const ScreenArgs& a, const FilterIO& io, int sm_count, cudaStream_t st) {
    count_launch();
    k_filter_hits<kFilterWarps><<<sm_count * 2, kFilterWarps * 32, kLutBytes, st>>>(a, io);
}

void launch_occupancy(const uint32_t* starts, uint64_t num_words, uint32_t* occ, cudaStream_t st) {
    const uint64_t words = (num_words + 31) / 32;
    const int blocks = (int)std::min<uint64_t>((words + 7) / 8, 148 * 16);
    count_launch();
    k_occupancy<<<std::max(blocks, 1), 256, 0, st>>>(starts, num_words, occ);
}

}  // namespace gxy
