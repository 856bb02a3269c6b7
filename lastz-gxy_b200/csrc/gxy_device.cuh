// gxy_device.cuh -- device data layout and the x-drop extenders.
//
// Sequences live in HBM in the reference's PackedSeq bit layout
// (src/sequences.rs:53-66) behind a 64-position leading pad, read as
// little-endian words: a u64 of `codes` holds 32 positions (2 bits each,
// position 32*i+k at bits 2k), a u32 of `valid`/`mask` holds 32 positions.
// Global position gp = kPad + local position, so a 32-position load at any
// gp >= 0 is in bounds; the tail carries kTailPad positions of zeros.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace gxy {

constexpr uint32_t kPad = 64;         // leading pad (positions)
constexpr uint32_t kTailPad = 1536;   // trailing pad (positions); covers one warp stage
constexpr int kMaxWeight = 15;        // 4^15 buckets; starts[] is u32 x (2^30 + 1)
constexpr int kMaxVariants = 1 + 15 + 105;
constexpr uint32_t kFull = 0xffffffffu;

// Process-wide count of kernels this library launched (gxy_kernel_launches).
void count_launch(uint64_t n = 1);

// One sequence segment as the kernels see it.  `base` is the global position
// of local position 0 (a chunk view of a target starts at kPad + chunk_lo);
// `key_base` places the segment on a private axis of the candidate sort key
// so that units never share a (target, query) coordinate pair.
struct SeqView {
    const uint64_t* codes;
    const uint32_t* valid;
    const uint32_t* mask;
    uint64_t base;
    uint32_t len;
    uint32_t key_base;
    // Optional interleaved copy (a table's target): the 32-position word i's
    // codes, valid and mask bits as one 16-byte record ilv[i - ilv_first], so
    // that a random 32-position window takes two loads instead of four.
    const uint4* ilv = nullptr;
    uint64_t ilv_first = 0;
};

// Codes and valid bits of the 32 positions from global position gp, from the
// interleaved copy when the view has one.
__device__ __forceinline__ void load_window32(const SeqView& S, uint64_t gp, uint64_t& codes, uint32_t& valid) {
    const uint64_t i = gp >> 5;
    const uint32_t s = (uint32_t)(gp & 31);
    if (S.ilv) {
        const uint4 a = __ldg(S.ilv + (i - S.ilv_first));
        const uint4 b = __ldg(S.ilv + (i + 1 - S.ilv_first));
        const uint64_t lo = ((uint64_t)a.y << 32) | a.x, hi = ((uint64_t)b.y << 32) | b.x;
        codes = s ? ((lo >> (2 * s)) | (hi << (64 - 2 * s))) : lo;
        valid = __funnelshift_r(a.z, b.z, s);
    } else {
        const uint64_t lo = __ldg(S.codes + i), hi = __ldg(S.codes + i + 1);
        codes = s ? ((lo >> (2 * s)) | (hi << (64 - 2 * s))) : lo;
        valid = __funnelshift_r(__ldg(S.valid + i), __ldg(S.valid + i + 1), s);
    }
}

// One reference search() call: a (target segment, query segment) pair with
// the target's position table (src/seed_search.rs:45-51).
struct UnitDev {
    uint32_t tseg;
    uint32_t qseg;
    const uint32_t* starts;
    const uint32_t* positions;
    const uint32_t* occ;  // bucket occupancy bitmap (bit w & 31 of occ[w >> 5])
    uint32_t nwin;        // query windows 0, step, ... <= len - L
    uint32_t tile_base;   // first screen tile of this unit
    uint32_t primary_lo;  // driver primary-region filter, src/driver.rs:250-256
    uint32_t primary_hi;  // (lo == hi disables it)
};

// A hit that survived the screen: it either reaches hspthresh within the
// column cap (its extension result is exact and stored), or it is still
// extending at the cap (kCandLong) and is re-extended in full by the walk.
struct Cand {
    uint32_t unit;
    uint32_t t;
    uint32_t q;
    uint32_t flags;
    uint32_t lext;
    uint32_t rext;
    int32_t score;
    uint32_t pad_;
};
constexpr uint32_t kCandLong = 1u;

// Output record, layout-identical to gxy_hsp / the reference's Hsp.
struct Hsp {
    uint32_t t_start;
    uint32_t q_start;
    uint32_t length;
    int32_t score;
};

// Scoring parameters the extenders read (src/scoring.rs:32-40, src/hsp.rs:46-49).
struct Score {
    int32_t sub[16];
    int32_t ambig;
    int32_t xdrop;
    int32_t hspthresh;
};

__device__ __forceinline__ uint64_t load_codes32(const uint64_t* __restrict__ codes, uint64_t gp) {
    const uint64_t i = gp >> 5;
    const uint32_t s = (uint32_t)(gp & 31) * 2;
    const uint64_t lo = __ldg(codes + i);
    const uint64_t hi = __ldg(codes + i + 1);
    return s ? ((lo >> s) | (hi << (64 - s))) : lo;
}

__device__ __forceinline__ uint32_t load_bits32(const uint32_t* __restrict__ bits, uint64_t gp) {
    const uint64_t i = gp >> 5;
    const uint32_t s = (uint32_t)(gp & 31);
    return __funnelshift_r(__ldg(bits + i), __ldg(bits + i + 1), s);
}

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Each set bit of x becomes a set 2-bit pair (bit k -> bits 2k, 2k+1).
__device__ __forceinline__ uint64_t spread_bits_to_pairs(uint32_t x) {
    uint64_t v = x;
    v = (v | (v << 16)) & 0x0000FFFF0000FFFFull;
    v = (v | (v << 8)) & 0x00FF00FF00FF00FFull;
    v = (v | (v << 4)) & 0x0F0F0F0F0F0F0F0Full;
    v = (v | (v << 2)) & 0x3333333333333333ull;
    v = (v | (v << 1)) & 0x5555555555555555ull;
    return v * 3;   // each set bit -> a set 2-bit pair
}

// Reverses the order of the 32 two-bit codes of a word (a left-side chunk
// read upwards becomes column 0 = the position next to the seed).
__device__ __forceinline__ uint64_t rev_pairs64(uint64_t c) {
    c = __brevll(c);
    return ((c >> 1) & 0x5555555555555555ull) | ((c & 0x5555555555555555ull) << 1);
}

// Column score (src/hsp.rs:198-211): ambig when either base is invalid.
__device__ __forceinline__ int32_t col_score(uint64_t tc, uint64_t qc, uint32_t vv, int sh,
                                             const int32_t* lut, int32_t ambig) {
    const uint32_t idx = (((uint32_t)(tc >> (2 * sh)) & 3u) << 2) | ((uint32_t)(qc >> (2 * sh)) & 3u);
    return ((vv >> sh) & 1u) ? lut[idx] : ambig;
}

// One side of extend_one_side (src/hsp.rs:160-195), one lane, 32 columns per
// pair of loads.  t0/q0 are the local positions of the first column; forward
// walks up, backward walks down.  Returns true when the side ended (x-drop
// break or sequence bound) within `cap` columns, false when it is still
// running after `cap` columns (the caller then defers the hit to the walk).
// The arithmetic is plain i32: the host admits a search only when no partial
// sum can leave i32, so the reference's saturating adds never saturate.
template <bool kForward>
__device__ __forceinline__ bool side_lane(const SeqView& T, const SeqView& Q, uint32_t t0,
                                          uint32_t q0, uint32_t maxext, uint32_t cap,
                                          int32_t xdrop, const int32_t* lut, int32_t ambig,
                                          int32_t& best_out, uint32_t& bext_out) {
    int32_t run = 0, best = 0;
    uint32_t bext = 0, ext = 0;
    while (ext < maxext) {
        const uint64_t tg = kForward ? T.base + t0 + ext : T.base + t0 - ext - 31;
        const uint64_t qg = kForward ? Q.base + q0 + ext : Q.base + q0 - ext - 31;
        const uint64_t tc = load_codes32(T.codes, tg);
        const uint64_t qc = load_codes32(Q.codes, qg);
        const uint32_t vv = load_bits32(T.valid, tg) & load_bits32(Q.valid, qg);
        const uint32_t n = min(32u, maxext - ext);
#pragma unroll
        for (int i = 0; i < 32; i++) {
            if ((uint32_t)i >= n) break;
            const int sh = kForward ? i : 31 - i;
            run += col_score(tc, qc, vv, sh, lut, ambig);
            if (run > best) {
                best = run;
                bext = ext + i + 1;
            } else if (best - run > xdrop) {
                best_out = best;
                bext_out = bext;
                return true;
            }
        }
        ext += n;
        if (ext >= cap && ext < maxext) {
            best_out = best;
            bext_out = bext;
            return false;
        }
    }
    best_out = best;
    bext_out = bext;
    return true;
}

struct LaneExt {
    int32_t score;
    uint32_t lext;
    uint32_t rext;
    bool done;   // both sides ended within the cap: the result is exact
};

// extend_hit_scalar (src/hsp.rs:98-148) for one lane with a column cap per
// side.  Requires t + L <= T.len and q + L <= Q.len (the caller checks).
__device__ __forceinline__ LaneExt extend_lane(const SeqView& T, const SeqView& Q, uint32_t t,
                                               uint32_t q, uint32_t L, uint32_t cap,
                                               int32_t xdrop, const int32_t* lut, int32_t ambig) {
    LaneExt r;
    // Seed footprint: all L columns, care and don't-care (src/hsp.rs:119-123).
    const uint64_t tc = load_codes32(T.codes, T.base + t);
    const uint64_t qc = load_codes32(Q.codes, Q.base + q);
    const uint32_t vv = load_bits32(T.valid, T.base + t) & load_bits32(Q.valid, Q.base + q);
    int32_t seed = 0;
#pragma unroll
    for (int k = 0; k < 32; k++) {
        if ((uint32_t)k >= L) break;
        seed += col_score(tc, qc, vv, k, lut, ambig);
    }
    int32_t rb, lb = 0;
    uint32_t re, le = 0;
    const uint32_t rmax = min(T.len - t - L, Q.len - q - L);
    r.done = side_lane<true>(T, Q, t + L, q + L, rmax, cap, xdrop, lut, ambig, rb, re);
    if (r.done) {
        const uint32_t lmax = min(t, q);
        if (lmax) r.done = side_lane<false>(T, Q, t - 1, q - 1, lmax, cap, xdrop, lut, ambig, lb, le);
    }
    r.score = seed + lb + rb;
    r.lext = le;
    r.rext = re;
    return r;
}

// ---------------------------------------------------------------------------
// Warp-cooperative x-drop: one warp per hit, 64 columns per step (two per
// lane), the x-drop cut found with shuffle scans.  Column k of a step breaks the reference's
// loop iff run_k <= PM_{k-1} and PM_{k-1} - run_k > xdrop, where
// PM_{k-1} = max(best, run_0..run_{k-1}); the best extent is the first column
// whose running score equals the step's maximum (the reference updates only
// on a strict increase).  Sequence bytes are staged through shared memory in
// 16-byte vector loads: kStageSpan positions per refill.
// ---------------------------------------------------------------------------
constexpr uint32_t kStageCols = 1024;
constexpr uint32_t kStageSpan = kStageCols + 128;          // positions staged per refill
struct WarpStage {
    uint64_t tcodes[kStageSpan / 32];
    uint64_t qcodes[kStageSpan / 32];
    uint32_t tvalid[kStageSpan / 32];
    uint32_t qvalid[kStageSpan / 32];
};

// Copies positions [a, a + kStageSpan) (a a multiple of 128) of one sequence
// into the stage with 16-byte loads: codes 288 bytes, valid 144 bytes.
__device__ __forceinline__ void stage_fill(const uint64_t* codes, const uint32_t* valid, uint64_t a,
                                           uint64_t* scodes, uint32_t* svalid, int lane) {
    const uint4* c4 = reinterpret_cast<const uint4*>(codes + (a >> 5));
    const uint4* v4 = reinterpret_cast<const uint4*>(valid + (a >> 5));
    constexpr int kC4 = kStageSpan / 32 * 8 / 16;   // 18
    constexpr int kV4 = kStageSpan / 32 * 4 / 16;   // 9
    if (lane < kC4) reinterpret_cast<uint4*>(scodes)[lane] = __ldg(c4 + lane);
    if (lane < kV4) reinterpret_cast<uint4*>(svalid)[lane] = __ldg(v4 + lane);
}

__device__ __forceinline__ uint64_t stage_codes32(const uint64_t* s, uint32_t off) {
    const uint32_t i = off >> 5, sh = (off & 31) * 2;
    const uint64_t lo = s[i], hi = s[i + 1];
    return sh ? ((lo >> sh) | (hi << (64 - sh))) : lo;
}
__device__ __forceinline__ uint32_t stage_bits32(const uint32_t* s, uint32_t off) {
    return __funnelshift_r(s[off >> 5], s[(off >> 5) + 1], off & 31);
}

template <bool kForward>
__device__ void side_warp(const SeqView& T, const SeqView& Q, uint32_t t0, uint32_t q0,
                          uint32_t maxext, int32_t xdrop, const int32_t* lut, int32_t ambig,
                          WarpStage* st, int32_t& best_out, uint32_t& bext_out) {
    // 64 columns per step: lane l scores columns 2l and 2l+1.  A refill
    // stages 1,152 positions, enough for 15 steps (960 columns) with every
    // lane's 32-position funnel read inside the stage.
    constexpr uint32_t kSteps = 960;
    const int lane = threadIdx.x & 31;
    int32_t run = 0, best = 0;
    uint32_t bext = 0, ext = 0;
    uint64_t ta = 0, qa = 0;   // staged windows' first global positions
    uint32_t staged = 0;       // columns left in the current stage
    const uint32_t c0 = 2u * (uint32_t)lane, c1 = c0 + 1;
    while (ext < maxext) {
        // The step's 64 positions: [tg, tg + 64).
        const uint64_t tg = kForward ? T.base + t0 + ext : T.base + t0 - ext - 63;
        const uint64_t qg = kForward ? Q.base + q0 + ext : Q.base + q0 - ext - 63;
        if (staged < 64) {
            __syncwarp();
            if (kForward) {
                ta = tg & ~127ull;
                qa = qg & ~127ull;
            } else {
                const uint64_t tl = tg + 63 >= kSteps ? tg + 63 - (kSteps - 1) : 0;
                const uint64_t ql = qg + 63 >= kSteps ? qg + 63 - (kSteps - 1) : 0;
                ta = tl & ~127ull;
                qa = ql & ~127ull;
            }
            stage_fill(T.codes, T.valid, ta, st->tcodes, st->tvalid, lane);
            stage_fill(Q.codes, Q.valid, qa, st->qcodes, st->qvalid, lane);
            __syncwarp();
            staged = kSteps;
        }
        // This lane's two columns sit at window offsets c0, c1 (forward) or
        // 63 - c0, 63 - c1 (backward): one funnel read from the lower one.
        const uint32_t lo = kForward ? c0 : 62u - c0;
        const uint32_t to = (uint32_t)(tg - ta) + lo, qo = (uint32_t)(qg - qa) + lo;
        const uint64_t tc = stage_codes32(st->tcodes, to);
        const uint64_t qc = stage_codes32(st->qcodes, qo);
        const uint32_t vv = stage_bits32(st->tvalid, to) & stage_bits32(st->qvalid, qo);
        const uint32_t n = min(64u, maxext - ext);
        const bool a0 = c0 < n, a1 = c1 < n;
        const int32_t x0 = a0 ? col_score(tc, qc, vv, kForward ? 0 : 1, lut, ambig) : 0;
        const int32_t x1 = a1 ? col_score(tc, qc, vv, kForward ? 1 : 0, lut, ambig) : 0;
        int32_t x = x0 + x1;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int32_t y = __shfl_up_sync(kFull, x, o);
            if (lane >= o) x += y;
        }
        const int32_t r1 = run + x;      // running score after column c1
        const int32_t r0 = r1 - x1;      // after column c0
        int32_t m = a0 ? (a1 ? max(r0, r1) : r0) : INT32_MIN;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int32_t y = __shfl_up_sync(kFull, m, o);
            if (lane >= o) m = max(m, y);
        }
        int32_t pm = __shfl_up_sync(kFull, m, 1);
        if (lane == 0) pm = INT32_MIN;
        pm = max(pm, best);              // prefix maximum before column c0
        const bool brk0 = a0 && r0 <= pm && (pm - r0 > xdrop);
        const int32_t pm1 = max(pm, r0); // before column c1
        const bool brk1 = a1 && r1 <= pm1 && (pm1 - r1 > xdrop);
        const uint32_t bm = __ballot_sync(kFull, brk0 || brk1);
        uint32_t nproc = n;              // columns before the break column
        if (bm) {
            const int bl = __ffs(bm) - 1;
            const bool b0 = __shfl_sync(kFull, brk0, bl);
            nproc = 2u * (uint32_t)bl + (b0 ? 0u : 1u);
        }
        int32_t c = INT32_MIN;
        if (c0 < nproc) c = r0;
        if (c1 < nproc) c = max(c, r1);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) c = max(c, __shfl_xor_sync(kFull, c, o));
        if (c > best) {
            // The first column that reaches the step's maximum.
            const bool e0 = c0 < nproc && r0 == c;
            const bool e1 = c1 < nproc && r1 == c;
            const uint32_t eq = __ballot_sync(kFull, e0 || e1);
            const int el = __ffs(eq) - 1;
            const bool f0 = __shfl_sync(kFull, e0, el);
            bext = ext + 2u * (uint32_t)el + (f0 ? 1u : 2u);
            best = c;
        }
        if (bm) break;
        run = __shfl_sync(kFull, r1, 31);
        ext += n;
        staged -= 64;
    }
    best_out = best;
    bext_out = bext;
}

// extend_hit_scalar (src/hsp.rs:98-148) with one warp; every lane returns the
// same result.
__device__ __forceinline__ LaneExt extend_warp(const SeqView& T, const SeqView& Q, uint32_t t,
                                               uint32_t q, uint32_t L, int32_t xdrop,
                                               const int32_t* lut, int32_t ambig, WarpStage* st) {
    const int lane = threadIdx.x & 31;
    LaneExt r;
    const uint64_t tc = load_codes32(T.codes, T.base + t);
    const uint64_t qc = load_codes32(Q.codes, Q.base + q);
    const uint32_t vv = load_bits32(T.valid, T.base + t) & load_bits32(Q.valid, Q.base + q);
    int32_t s = ((uint32_t)lane < L) ? col_score(tc, qc, vv, lane, lut, ambig) : 0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kFull, s, o);
    int32_t rb, lb = 0;
    uint32_t re, le = 0;
    const uint32_t rmax = min(T.len - t - L, Q.len - q - L);
    side_warp<true>(T, Q, t + L, q + L, rmax, xdrop, lut, ambig, st, rb, re);
    const uint32_t lmax = min(t, q);
    if (lmax) side_warp<false>(T, Q, t - 1, q - 1, lmax, xdrop, lut, ambig, st, lb, le);
    r.score = s + lb + rb;
    r.lext = le;
    r.rext = re;
    r.done = true;
    return r;
}

}  // namespace gxy
