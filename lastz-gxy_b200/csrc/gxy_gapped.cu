// gxy_gapped.cu -- gapped extension (src/gapped_extend.rs:78-460) on the device.
//
// extend() runs a banded 3-state affine x-drop DP (Gotoh M/X/Y) to the right
// of an anchor and, on reversed inputs, to its left, then traces the best
// cell back into a run-length edit script.  The DP is row by row: row i's
// band is [lo - R, hi + R] around the previous row's surviving cells, capped
// at band_width = min(4R + 4, m + 1) cells; after a row, the cells whose best
// state is more than y_drop below the best score so far are killed.  These
// rules (the band, the row-major first maximum, the kill) decide the result,
// so the device keeps the row order.  One block of W warps runs one side of
// one anchor, S = 4 (or 8) cells of a row a thread, W = band_width / (32 S)
// rounded up (10 for HOXD70's defaults at S = 4):
//
//  - Thread k owns cells [S k, S k + S) of the row.  X and M of a cell need the
//    previous row only, so a thread forms them for its cells first (phase A).
//  - Y is a max-plus recurrence along the row, Y[j] = max(M[j-1] - (O+E),
//    Y[j-1] - E).  Each thread reduces its cells to one affine-max function
//    x -> max(a, x - S E); a warp shuffle scan composes them, and each warp
//    folds in the warps before it through shared memory, giving every thread
//    the exact Y entering its cells (phase B then runs the recurrence from
//    there; the entering Y's source is M exactly when the M term reaches it).
//    The arithmetic is the reference's i32 arithmetic: max-plus composition
//    is exact.
//  - The row lives in shared memory (best state H = max(M, X, Y) with its
//    argmax, and the next row's X = max(M - (O+E), X - E) with its source),
//    stored transposed (cell p at (p mod S) * threads + p / S), so both the
//    current row's writes and the next row's reads, at any shift of the
//    band, hit distinct banks.  A cell killed by the x-drop rule is not
//    rewritten: the next row compares its H with the row's threshold and
//    reads NEG_INF in its place, as the reference's cleared cell reads.
//  - The three back-pointers of a cell (4 bits; S / 8 words per thread and row)
//    go to global memory, rows in pool blocks of kRows kept by the CUDA block
//    across its tasks (a chain it grows from a shared pool as its longest side
//    needs).  After the last row, the block stages one pool block at a time
//    in shared memory and thread 0 walks it from the best cell to (0, 0),
//    writing the runs.  Sides whose rows did not fit the pool run again
//    with exactly sized storage.
//
// A last kernel joins the two sides per anchor: total = anchor column + left
// best + right best (saturating), the left runs in walk order, the anchor's
// Match merged with its neighbours, the right runs reversed
// (src/gapped_extend.rs:99-131, src/edit_script.rs:63-92).
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "gxy_engine.cuh"

using namespace gxy;

namespace {

constexpr int32_t kNegInf = INT32_MIN / 4;   // NEG_INF (src/gapped_extend.rs:44)
constexpr int32_t kLow = INT32_MIN / 2;      // "no contribution" in the row scan: below every DP value
constexpr int kMaxCells = 2048;               // band_width at most (cells of a row per block)
constexpr int kRows = 32;                     // DP rows per traceback block
constexpr int kHdr = 4;                       // block header words: previous block, next block, first row, -
constexpr uint32_t kNone = 0xffffffffu;

// Side flags.
constexpr uint32_t kFlagPool = 1;    // the traceback pool ran out: rerun with a larger one
constexpr uint32_t kFlagRuns = 2;    // the run buffer ran out: the first pass reruns with a larger one
constexpr uint32_t kFlagState = 4;   // inconsistent back-pointers (a bug; reported as an error)
constexpr uint32_t kFlagScratch = 8; // more runs than the block's scratch holds: the second pass
constexpr uint32_t kScratchWords = 16384;   // first pass: run scratch per CUDA block (64 KB)
constexpr uint32_t kSideRuns2 = 1u << 8;   // the side's runs are in the second run buffer

// Counters (u64): task cursor, pool blocks claimed, run words reserved, rows,
// cells, flags, the most rows of one side.
enum { kCtrTask = 0, kCtrBlocks, kCtrRuns, kCtrRows, kCtrCells, kCtrFlags, kCtrMaxRows, kCtrWords = 8 };

struct GapSide {
    int32_t score;
    uint32_t t_span;
    uint32_t q_span;
    uint32_t n_runs;
    uint64_t run_off;
    uint32_t flags;   // kFlag* | kSideRuns2
    uint32_t rows;    // DP rows computed
};

struct GapArgs {
    SeqView T, Q;
    const uint32_t* t_pos;
    const uint32_t* q_pos;
    uint32_t n_anchors;
    int32_t sub[16];
    int32_t ambig;
    int32_t goe;      // gap_open + gap_extend
    int32_t ge;       // gap_extend
    int32_t ydrop;
    int64_t radius;   // band radius; < 0: m + 1 (gap_extend <= 0)
    uint32_t* pool;
    uint64_t pool_blocks;
    uint32_t block_words;
    uint32_t* runs;       // where this pass's tracebacks write
    uint64_t runs_cap;
    const uint32_t* runs2;   // the second pass's runs (for the join)
    unsigned long long* ctr;
    GapSide* sides;   // [2a] left, [2a + 1] right
    // Second pass: only the listed sides, side list[k] with its rows in the
    // pool blocks base[k], base[k] + 1, ... (no chains); runs go to the second
    // run buffer.  list == nullptr: every side, blocks in per-warp chains.
    const uint32_t* list;
    const uint64_t* base;
    uint64_t n_list;
    // First pass: each CUDA block walks its sides' tracebacks into its own
    // scratch of scratch_words words, then copies the runs out to a range of
    // exactly their number.  The grid has at most scratch_blocks blocks.
    uint32_t* scratch;
    uint32_t scratch_words;
    uint32_t scratch_blocks;
};

__device__ __forceinline__ int32_t sat_sub32(int32_t a, int32_t b) {
    const int64_t r = (int64_t)a - b;
    return r > INT32_MAX ? INT32_MAX : (r < INT32_MIN ? INT32_MIN : (int32_t)r);
}
__device__ __forceinline__ int32_t sat_add32(int32_t a, int32_t b) {
    const int64_t r = (int64_t)a + b;
    return r > INT32_MAX ? INT32_MAX : (r < INT32_MIN ? INT32_MIN : (int32_t)r);
}

// Swaps the two bits of every 2-bit field (undoes __brevll's swap inside a code).
__device__ __forceinline__ uint64_t swap_pairs(uint64_t x) {
    return ((x >> 1) & 0x5555555555555555ull) | ((x & 0x5555555555555555ull) << 1);
}

__device__ __forceinline__ uint32_t code_at(const SeqView& S, uint64_t gp) {
    return (uint32_t)(__ldg(S.codes + (gp >> 5)) >> (2 * (gp & 31))) & 3u;
}
__device__ __forceinline__ uint32_t valid_at(const SeqView& S, uint64_t gp) {
    return (__ldg(S.valid + (gp >> 5)) >> (gp & 31)) & 1u;
}

// (value, cell, state) with the larger value first, the smaller cell on ties:
// the reference's strict `>` over a row-major scan keeps the first maximum.
__device__ __forceinline__ void best_reduce(int32_t& v, int32_t& pc, uint32_t& st) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const int32_t v2 = __shfl_xor_sync(kFull, v, o);
        const int32_t p2 = __shfl_xor_sync(kFull, pc, o);
        const uint32_t s2 = __shfl_xor_sync(kFull, st, o);
        if (v2 > v || (v2 == v && p2 < pc)) {
            v = v2;
            pc = p2;
            st = s2;
        }
    }
}

// One side of one anchor per block of W warps, tasks claimed from a cursor.
// Thread k of the block owns cells [S k, S k + S) of the row (band_width <= 32 W S).
template <int W, int S>
__global__ void __launch_bounds__(W * 32) k_gapped_sides(GapArgs a) {
    static_assert(S == 4 || S == 8, "cells per thread");
    constexpr int NT = W * 32;             // threads per block
    constexpr int kRowWords = NT * S / 8;  // back-pointer words of a row (4 bits a cell)
    extern __shared__ int32_t g_sm[];
    int32_t* sH = g_sm;                       // the row: best state H
    int32_t* sNX = sH + NT * S;               // the next row's X
    uint8_t* sST = reinterpret_cast<uint8_t*>(sNX + NT * S);   // H's state | next X's source << 2
    // One pool block staged for the traceback (after the row buffer).
    uint32_t* sBlk = reinterpret_cast<uint32_t*>(sST + ((NT * S + 15) & ~15));
    __shared__ int32_t s_wA[W];               // each warp's composed row function
    __shared__ int32_t s_wM[W];               // M of each warp's last cell
    __shared__ int32_t s_bv[W], s_bp[W], s_first[W], s_last[W];
    __shared__ uint32_t s_bs[W];
    __shared__ unsigned long long s_task;
    __shared__ uint32_t s_blk, s_head;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int32_t goe = a.goe, ge = a.ge;
    // X of a cell whose upper neighbour is dead or outside the band.
    const int32_t nx_dead = max(kNegInf - goe, kNegInf - ge);
    const uint32_t nx_dead_from = (kNegInf - goe >= kNegInf - ge) ? 0u : 1u;
    const uint64_t ntasks = a.list ? a.n_list : 2ull * a.n_anchors;
    const int32_t lane_shift = S * ge;        // Y decays by this over one thread's cells
    // This block's chain of traceback blocks (kept across tasks; thread 0's).
    uint32_t chain_head = kNone, chain_len = 0;
    for (;;) {
        if (tid == 0) s_task = atomicAdd(a.ctr + kCtrTask, 1ull);
        __syncthreads();
        unsigned long long task = s_task;
        __syncthreads();
        if (task >= ntasks) break;
        const uint64_t fixed_base = a.list ? a.base[task] : 0;
        if (a.list) task = a.list[task];
        const uint32_t an = (uint32_t)(task >> 1);
        const bool right = task & 1;
        const int64_t dir = right ? 1 : -1;
        const uint32_t t0 = a.t_pos[an], q0 = a.q_pos[an];
        const int64_t n = right ? (int64_t)a.T.len - t0 - 1 : (int64_t)t0;
        const int64_t m = right ? (int64_t)a.Q.len - q0 - 1 : (int64_t)q0;
        GapSide res{};
        if (n == 0 || m == 0) {
            if (tid == 0) a.sides[task] = res;
            continue;
        }
        const int64_t R = a.radius >= 0 ? a.radius : m + 1;
        const int64_t bw = min(4 * R + 4, m + 1);
        int64_t lo = 0, hi = 0;        // surviving cells of the previous row
        int64_t pjl = 0;               // previous row's band start
        int32_t pw = 0;                // previous row's band width
        int32_t thr_prev = 0;          // previous row's kill threshold
        int32_t best = 0;
        int64_t bi = 0, bj = 0;
        uint32_t bst = 0;
        uint32_t flags = 0;
        uint32_t cur_blk = kNone;      // thread 0: the chain block holding the current row
        uint32_t blk_index = 0;
        if (a.list) chain_len = 0;
        bool store = true;
        uint64_t rows = 0, cells = 0;
        const int cbase = tid * S;
        for (int64_t i = 0; i <= n; i++) {
            const int64_t jl = lo > R ? lo - R : 0;
            int64_t jh = min(hi + R, m);
            jh = min(jh, jl + bw - 1);
            const int32_t width = (int32_t)(jh - jl + 1);
            if (width > NT * S) {   // cannot happen: the host sizes W from band_width
                flags |= kFlagState;
                break;
            }
            rows++;
            cells += (uint64_t)width;
            // Thread 0 takes the traceback block of this row (every kRows rows).
            if (tid == 0 && store && (i % kRows) == 0) {
                uint32_t nb = kNone;
                if (a.list) {   // second pass: this side's blocks are consecutive
                    nb = (uint32_t)(fixed_base + (uint64_t)(i / kRows));
                    uint32_t* hdr = a.pool + (uint64_t)nb * a.block_words;
                    hdr[0] = i == 0 ? kNone : nb - 1;
                    hdr[1] = nb + 1;
                    if (i == 0) chain_head = nb;
                } else if (blk_index < chain_len) {
                    nb = cur_blk == kNone ? chain_head : a.pool[(uint64_t)cur_blk * a.block_words + 1];
                } else {
                    const unsigned long long b = atomicAdd(a.ctr + kCtrBlocks, 1ull);
                    if (b < a.pool_blocks) {
                        nb = (uint32_t)b;
                        uint32_t* hdr = a.pool + (uint64_t)nb * a.block_words;
                        hdr[0] = cur_blk;   // previous block in the chain
                        hdr[1] = kNone;     // next
                        if (cur_blk == kNone) {
                            chain_head = nb;
                        } else {
                            a.pool[(uint64_t)cur_blk * a.block_words + 1] = nb;
                        }
                        chain_len++;
                    }
                }
                if (nb != kNone) {
                    a.pool[(uint64_t)nb * a.block_words + 2] = (uint32_t)i;
                    cur_blk = nb;
                    blk_index++;
                }
                s_blk = nb;
            }
            // Scores of the row's target base against query codes 0..3.
            int32_t s0 = a.ambig, s1 = a.ambig, s2 = a.ambig, s3 = a.ambig;
            if (i >= 1) {
                const uint64_t tg = a.T.base + (uint64_t)((int64_t)t0 + dir * i);
                if (valid_at(a.T, tg)) {
                    const uint32_t tc = code_at(a.T, tg);
                    s0 = a.sub[tc * 4 + 0];
                    s1 = a.sub[tc * 4 + 1];
                    s2 = a.sub[tc * 4 + 2];
                    s3 = a.sub[tc * 4 + 3];
                }
            }
            const int32_t con = min(max(width - cbase, 0), S);
            // The thread's query bases, cell c at offset c (2 bits each) and its valid bit.
            uint64_t qc64 = 0;
            uint32_t qv = 0;
            if (con > 0 && i >= 1) {
                if (right) {
                    load_window32(a.Q, a.Q.base + (uint64_t)((int64_t)q0 + jl + cbase), qc64, qv);
                } else {
                    uint64_t c0;
                    uint32_t v0;
                    load_window32(a.Q, (uint64_t)((int64_t)a.Q.base + (int64_t)q0 - jl - cbase - 31), c0, v0);
                    qc64 = swap_pairs(__brevll(c0));
                    qv = __brev(v0);
                }
            }
            const bool col0 = (jl == 0) && tid == 0;   // this thread's cell 0 is column 0
            const int32_t d = (int32_t)(jl - pjl);      // previous-frame index of this row's cell 0
            // ---- phase A: X and M of the thread's cells from the previous row.
            int32_t Mr[S], Xr[S];
            uint32_t tb = 0;
            int32_t hm1 = kNegInf;   // H of the previous row's cell left of the current one (killed: NEG_INF)
            uint32_t sm1 = 0;
            if (i >= 1) {
                const int32_t p = d + cbase - 1;
                if (p >= 0 && p < pw) {
                    const int ad = (p & (S - 1)) * NT + p / S;
                    const int32_t h = sH[ad];
                    if (h >= thr_prev) {
                        hm1 = h;
                        sm1 = sST[ad] & 3u;
                    }
                }
            }
            int32_t yl = kLow;   // Y of the thread's cells without what enters from the left
#pragma unroll
            for (int c = 0; c < S; c++) {
                const bool on = c < con;
                const int32_t p = d + cbase + c;
                int32_t hp = kNegInf, nxp = nx_dead;
                uint32_t stp = 0, nxf = nx_dead_from;
                if (i >= 1 && on && p >= 0 && p < pw) {
                    const int ad = (p & (S - 1)) * NT + p / S;
                    const int32_t h = sH[ad];
                    if (h >= thr_prev) {
                        const uint32_t st = sST[ad];
                        hp = h;
                        nxp = sNX[ad];
                        stp = st & 3u;
                        nxf = (st >> 2) & 1u;
                    }
                }
                int32_t M, X;
                uint32_t mf = 0, xf = 0;
                if (i == 0) {
                    X = kNegInf;
                    M = (c == 0 && col0) ? 0 : kNegInf;
                } else {
                    X = nxp;
                    xf = nxf;
                    if (c == 0 && col0) {
                        M = kNegInf;
                    } else {
                        const uint32_t qc = (uint32_t)(qc64 >> (2 * c)) & 3u;
                        const bool qvb = (qv >> c) & 1u;
                        const int32_t s =
                            qvb ? ((qc & 2) ? ((qc & 1) ? s3 : s2) : ((qc & 1) ? s1 : s0)) : a.ambig;
                        M = hm1 + s;
                        mf = sm1;
                    }
                }
                if (!on) {
                    M = kNegInf;
                    X = kNegInf;
                }
                Mr[c] = M;
                Xr[c] = X;
                tb |= (mf | (xf << 2)) << (4 * c);
                hm1 = hp;
                sm1 = stp;
                if (c + 1 < S) yl = max(max(M - goe, yl - ge), kLow);
            }
            // What the thread passes on: Y entering the cell after its last.
            int32_t A = max(max(Mr[S - 1] - goe, yl - ge), kLow);
            // ---- the row scan: compose x -> max(a_k, x - S*E) over the threads.
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int32_t Ap = __shfl_up_sync(kFull, A, o);
                if (lane >= o) A = max(A, max(Ap - o * lane_shift, kLow));
            }
            if (lane == 31) {
                s_wA[wid] = A;
                s_wM[wid] = Mr[S - 1];
            }
            __syncthreads();   // every thread's reads of the previous row are done
            // Y of the row's first cell: NEG_INF when it is column 0 (no Y
            // there), else what NEG_INF neighbours give; then across the
            // warps before this one.
            int32_t Tw = jl == 0 ? kNegInf : max(kNegInf - goe, kNegInf - ge);
            for (int v = 0; v < wid; v++) Tw = max(s_wA[v], max(Tw - 32 * lane_shift, kLow));
            const int32_t tout = max(A, max(Tw - (lane + 1) * lane_shift, kLow));
            int32_t tin = __shfl_up_sync(kFull, tout, 1);
            int32_t mleft = __shfl_up_sync(kFull, Mr[S - 1], 1);
            if (lane == 0) {
                tin = Tw;
                mleft = wid == 0 ? kNegInf : s_wM[wid - 1];
            }
            const uint32_t blk = store ? s_blk : kNone;
            // ---- phase B: Y, the cell's best state, the next row's X, the best.
            int32_t lbest = INT32_MIN, lpc = INT32_MAX;
            uint32_t lst = 0;
            int32_t yleft = 0;
#pragma unroll
            for (int c = 0; c < S; c++) {
                const bool on = c < con;
                int32_t Y;
                uint32_t yf = 0;
                if (c == 0 && col0) {
                    Y = kNegInf;
                } else if (c == 0) {
                    // Y = max(M_left - (O+E), Y_left - E), formed by the scan;
                    // its source is M exactly when the M term reaches it.
                    Y = tin;
                    yf = (tin == mleft - goe) ? 0u : 1u;
                } else {
                    const int32_t fm = mleft - goe, fy = yleft - ge;
                    Y = fm >= fy ? fm : fy;
                    yf = fm >= fy ? 0u : 1u;
                }
                const int32_t M = Mr[c], X = Xr[c];
                mleft = M;
                yleft = Y;
                const uint32_t hs = (M >= X && M >= Y) ? 0u : (X >= Y ? 1u : 2u);
                const int32_t H = hs == 0 ? M : (hs == 1 ? X : Y);
                const int32_t fm = M - goe, fx = X - ge;
                const int32_t NX = fm >= fx ? fm : fx;
                const uint32_t nxf = fm >= fx ? 0u : 1u;
                if (on) {
                    const int ad = c * NT + tid;
                    sH[ad] = H;
                    sNX[ad] = NX;
                    sST[ad] = (uint8_t)(hs | (nxf << 2));
                    if (H > lbest) {
                        lbest = H;
                        lpc = cbase + c;
                        lst = hs;
                    }
                }
                tb |= (yf << 3) << (4 * c);
                Xr[c] = on ? H : kLow;   // H from here on
            }
            // ---- back-pointers of the row: one word (8 cells) per thread.
            if (blk != kNone) {
                uint32_t* bp = a.pool + (uint64_t)blk * a.block_words;
                const int r = (int)(i % kRows);
                if (tid == 0) bp[kHdr + r] = (uint32_t)jl;
                if (con > 0) {
                    if (S == 8) {
                        bp[kHdr + kRows + (uint64_t)r * kRowWords + tid] = tb;
                    } else {
                        reinterpret_cast<uint16_t*>(bp + kHdr + kRows + (uint64_t)r * kRowWords)[tid] = (uint16_t)tb;
                    }
                }
            } else if (store) {
                store = false;
                flags |= kFlagPool;   // the DP goes on: score, best cell and rows stay exact
            }
            // ---- the row's best, the threshold and the surviving cells.
            best_reduce(lbest, lpc, lst);
            if (lane == 0) {
                s_bv[wid] = lbest;
                s_bp[wid] = lpc;
                s_bs[wid] = lst;
            }
            // The threshold needs the row's best: the surviving cells are
            // found against the best of the rows so far and this row's best.
            __syncthreads();
            int32_t rv = s_bv[0], rp = s_bp[0];
            uint32_t rs = s_bs[0];
            for (int v = 1; v < W; v++) {
                if (s_bv[v] > rv) {   // warps in cell order: the first maximum stays on ties
                    rv = s_bv[v];
                    rp = s_bp[v];
                    rs = s_bs[v];
                }
            }
            if (rv > best) {
                best = rv;
                bi = i;
                bj = jl + rp;
                bst = rs;
            }
            const int32_t thr = sat_sub32(best, a.ydrop);
            int32_t first = INT32_MAX, last = -1;
#pragma unroll
            for (int c = 0; c < S; c++) {
                if (Xr[c] >= thr) {
                    first = min(first, cbase + c);
                    last = cbase + c;
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                first = min(first, __shfl_xor_sync(kFull, first, o));
                last = max(last, __shfl_xor_sync(kFull, last, o));
            }
            if (lane == 0) {
                s_first[wid] = first;
                s_last[wid] = last;
            }
            __syncthreads();
            first = s_first[0];
            last = s_last[0];
            for (int v = 1; v < W; v++) {
                first = min(first, s_first[v]);
                last = max(last, s_last[v]);
            }
            if (last < 0) break;   // the whole row is dead
            lo = jl + first;
            hi = jl + last;
            pjl = jl;
            pw = width;
            thr_prev = thr;
        }
        res.score = best;
        res.t_span = (uint32_t)bi;
        res.q_span = (uint32_t)bj;
        if (!store) flags |= kFlagPool;
        if (tid == 0) s_head = chain_head;
        __syncthreads();   // back-pointer rows written by every thread are visible to every thread
        // ---- traceback from the best cell (src/gapped_extend.rs:404-437),
        // runs written in walk order (tip to root).  The block stages one pool
        // block (32 rows) at a time in shared memory; thread 0 walks it.
        // The first pass walks into the block's scratch and reserves exactly
        // the runs written; the second pass reserves best_i + best_j words (the
        // longest possible script) and writes in place.
        int64_t ti = bi, tj = bj;
        uint32_t st = bst, op = 3, cnt = 0, nr = 0;
        uint64_t off = 0, cap = 0, step = 0;
        bool walk = false;
        uint32_t* wr = nullptr;   // where the walk writes its runs
        uint64_t wcap = 0;        // and how many it may write there
        if (tid == 0) {
            if (!(flags & (kFlagPool | kFlagState))) {
                cap = (uint64_t)(bi + bj);
                if (a.list) {
                    if (cap) off = atomicAdd(a.ctr + kCtrRuns, (unsigned long long)cap);
                    flags |= kSideRuns2;
                    if (off + cap > a.runs_cap) {
                        flags |= kFlagRuns;
                    } else {
                        walk = true;
                        wr = a.runs + off;
                        wcap = cap;
                        res.run_off = off;
                    }
                } else {
                    walk = true;
                    wr = a.scratch + (uint64_t)blockIdx.x * a.scratch_words;
                    wcap = a.scratch_words;
                }
            }
            // The block of row bi: the chain's blocks hold rows in order.
            uint32_t blk = s_head;
            if (walk)
                for (int64_t k = 0; k < bi / kRows; k++) blk = a.pool[(uint64_t)blk * a.block_words + 1];
            s_blk = walk && (ti > 0 || tj > 0) ? blk : kNone;
        }
        __syncthreads();
        for (;;) {
            const uint32_t blk = s_blk;
            if (blk == kNone) break;
            const uint32_t* src = a.pool + (uint64_t)blk * a.block_words;
            for (uint32_t k = tid; k < a.block_words; k += NT) sBlk[k] = src[k];
            __syncthreads();
            if (tid == 0) {
                const int64_t first_row = sBlk[2];
                uint32_t next = kNone;
                while (ti > 0 || tj > 0) {
                    if (step++ >= cap) {   // every step lowers ti + tj
                        flags |= kFlagState;
                        break;
                    }
                    if (ti < first_row) {   // rows before this block: stage the previous one
                        step--;
                        next = sBlk[0];
                        if (next == kNone) flags |= kFlagState;
                        break;
                    }
                    const int r = (int)(ti - first_row);
                    const int64_t p = tj - (int64_t)sBlk[kHdr + r];
                    if (p < 0 || p >= NT * S) {
                        flags |= kFlagState;
                        break;
                    }
                    const uint32_t nib = (sBlk[kHdr + kRows + r * kRowWords + (int)(p >> 3)] >> (4 * (p & 7))) & 15u;
                    uint32_t eop;
                    if (st == 0) {   // M: both advance
                        if (ti == 0 || tj == 0) {
                            flags |= kFlagState;
                            break;
                        }
                        eop = 0;
                        st = nib & 3u;
                        ti--;
                        tj--;
                    } else if (st == 1) {   // X: gap in the query (DeleteQuery)
                        if (ti == 0) {
                            flags |= kFlagState;
                            break;
                        }
                        eop = 2;
                        st = ((nib >> 2) & 1u) ? 1u : 0u;
                        ti--;
                    } else {   // Y: gap in the target (InsertQuery)
                        if (tj == 0) {
                            flags |= kFlagState;
                            break;
                        }
                        eop = 1;
                        st = ((nib >> 3) & 1u) ? 2u : 0u;
                        tj--;
                    }
                    if (eop == op) {
                        cnt++;
                    } else {
                        if (cnt) {
                            if (nr >= wcap) {   // more runs than the scratch holds: the second pass
                                flags |= kFlagScratch;
                                break;
                            }
                            wr[nr++] = (cnt << 2) | op;
                        }
                        op = eop;
                        cnt = 1;
                    }
                }
                s_blk = (flags & (kFlagState | kFlagScratch)) ? kNone : next;
            }
            __syncthreads();
        }
        if (tid == 0) {
            if (walk && !(flags & (kFlagState | kFlagScratch))) {
                if (ti > 0 || tj > 0) flags |= kFlagState;
                if (cnt) {
                    if (nr >= wcap) flags |= kFlagScratch;
                    else wr[nr++] = (cnt << 2) | op;
                }
                res.n_runs = nr;
            }
            // First pass: the runs' range in the run buffer, exactly nr words.
            s_task = ~0ull;   // no copy
            if (!a.list && walk && !(flags & (kFlagState | kFlagScratch))) {
                if (nr) off = atomicAdd(a.ctr + kCtrRuns, (unsigned long long)nr);
                if (off + nr > a.runs_cap) {
                    flags |= kFlagRuns;
                } else {
                    res.run_off = off;
                    s_task = ((unsigned long long)nr << 40) | off;
                }
            }
        }
        __syncthreads();
        {
            const unsigned long long cp = s_task;
            if (cp != ~0ull) {
                const uint32_t n_cp = (uint32_t)(cp >> 40);
                const uint64_t o_cp = cp & ((1ull << 40) - 1);
                const uint32_t* sc = a.scratch + (uint64_t)blockIdx.x * a.scratch_words;
                for (uint32_t k = tid; k < n_cp; k += NT) a.runs[o_cp + k] = sc[k];
            }
        }
        if (tid == 0) {
            res.flags = flags;
            res.rows = (uint32_t)rows;
            a.sides[task] = res;
            atomicAdd(a.ctr + kCtrRows, (unsigned long long)rows);
            atomicAdd(a.ctr + kCtrCells, (unsigned long long)cells);
            atomicMax(a.ctr + kCtrMaxRows, (unsigned long long)rows);
            if (flags) atomicOr(a.ctr + kCtrFlags, (unsigned long long)flags);
        }
        __syncthreads();
    }
}

__device__ __forceinline__ const uint32_t* side_runs(const GapArgs& a, const GapSide& s) {
    return ((s.flags & kSideRuns2) ? a.runs2 : a.runs) + s.run_off;
}

// Per anchor: the total, pass or fail, the joined run count.
__global__ void k_gapped_join(GapArgs a, int32_t threshold, gxy_gapped_aln* out, uint32_t* counts) {
    const uint32_t an = blockIdx.x * blockDim.x + threadIdx.x;
    if (an >= a.n_anchors) return;
    const GapSide L = a.sides[2 * an], R = a.sides[2 * an + 1];
    const uint32_t t0 = a.t_pos[an], q0 = a.q_pos[an];
    const uint64_t tg = a.T.base + t0, qg = a.Q.base + q0;
    const int32_t col = (valid_at(a.T, tg) && valid_at(a.Q, qg)) ? a.sub[code_at(a.T, tg) * 4 + code_at(a.Q, qg)]
                                                                  : a.ambig;
    const int32_t total = sat_add32(sat_add32(col, L.score), R.score);
    gxy_gapped_aln o{};
    o.score = total;
    uint32_t cnt = 0;
    if (total >= threshold) {
        o.passed = 1;
        o.t_start = t0 - L.t_span;
        o.q_start = q0 - L.q_span;
        o.t_len = L.t_span + 1 + R.t_span;
        o.q_len = L.q_span + 1 + R.q_span;
        const uint32_t* lr = side_runs(a, L), * rr = side_runs(a, R);
        const uint32_t lm = L.n_runs && (lr[L.n_runs - 1] & 3u) == 0;
        const uint32_t rm = R.n_runs && (rr[R.n_runs - 1] & 3u) == 0;
        cnt = L.n_runs + R.n_runs + 1 - lm - rm;
    }
    o.script_len = cnt;
    out[an] = o;
    counts[an] = cnt;
}

// Per anchor (one warp): the joined runs at offs[an].
__global__ void k_gapped_emit(GapArgs a, const gxy_gapped_aln* alns, const uint32_t* offs, uint32_t* out) {
    const int lane = threadIdx.x & 31;
    const uint64_t nw = (uint64_t)gridDim.x * (blockDim.x >> 5);
    for (uint64_t an = blockIdx.x * (uint64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); an < a.n_anchors; an += nw) {
        if (!alns[an].passed) continue;
        const GapSide L = a.sides[2 * an], R = a.sides[2 * an + 1];
        const uint32_t* lr = side_runs(a, L);
        const uint32_t* rr = side_runs(a, R);
        const uint32_t lm = L.n_runs && (lr[L.n_runs - 1] & 3u) == 0;
        const uint32_t rm = R.n_runs && (rr[R.n_runs - 1] & 3u) == 0;
        const uint32_t nl = L.n_runs - lm, nr = R.n_runs - rm;
        uint32_t* o = out + offs[an];
        for (uint32_t k = lane; k < nl; k += 32) o[k] = lr[k];
        if (lane == 0) {
            const uint32_t mid = 1 + (lm ? lr[L.n_runs - 1] >> 2 : 0) + (rm ? rr[R.n_runs - 1] >> 2 : 0);
            o[nl] = mid << 2;
        }
        for (uint32_t k = lane; k < nr; k += 32) o[nl + 1 + k] = rr[nr - 1 - k];
    }
}

// Dynamic shared memory of k_gapped_sides<W, S>: the row (9 bytes a cell)
// and one staged pool block.
size_t sides_smem(int W, int S, uint32_t block_words) {
    const size_t cells = (size_t)W * 32 * S;
    return cells * 8 + ((cells + 15) & ~(size_t)15) + (size_t)block_words * 4;
}

template <int W, int S>
cudaError_t launch_sides(const GapArgs& a, int sm_count, cudaStream_t st) {
    const size_t smem = sides_smem(W, S, a.block_words);
    cudaError_t e = cudaFuncSetAttribute(k_gapped_sides<W, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_gapped_sides<W, S>, W * 32, smem);
    if (e != cudaSuccess) return e;
    int blocks = sm_count * std::max(per_sm, 1);
    if (!a.list) blocks = std::min<int>(blocks, (int)a.scratch_blocks);   // one run scratch a block
    count_launch();
    k_gapped_sides<W, S><<<blocks, W * 32, smem, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_sides_for(int W, int S, const GapArgs& a, int sm_count, cudaStream_t st) {
    if (S == 8) {
        switch (W) {
            case 1: return launch_sides<1, 8>(a, sm_count, st);
            case 2: return launch_sides<2, 8>(a, sm_count, st);
            case 3: return launch_sides<3, 8>(a, sm_count, st);
            case 4: return launch_sides<4, 8>(a, sm_count, st);
            case 5: return launch_sides<5, 8>(a, sm_count, st);
            case 6: return launch_sides<6, 8>(a, sm_count, st);
            case 7: return launch_sides<7, 8>(a, sm_count, st);
            default: return launch_sides<8, 8>(a, sm_count, st);
        }
    }
    switch (W) {
        case 1: return launch_sides<1, 4>(a, sm_count, st);
        case 2: return launch_sides<2, 4>(a, sm_count, st);
        case 3: return launch_sides<3, 4>(a, sm_count, st);
        case 4: return launch_sides<4, 4>(a, sm_count, st);
        case 5: return launch_sides<5, 4>(a, sm_count, st);
        case 6: return launch_sides<6, 4>(a, sm_count, st);
        case 7: return launch_sides<7, 4>(a, sm_count, st);
        case 8: return launch_sides<8, 4>(a, sm_count, st);
        case 9: return launch_sides<9, 4>(a, sm_count, st);
        case 10: return launch_sides<10, 4>(a, sm_count, st);
        case 11: return launch_sides<11, 4>(a, sm_count, st);
        case 12: return launch_sides<12, 4>(a, sm_count, st);
        case 13: return launch_sides<13, 4>(a, sm_count, st);
        case 14: return launch_sides<14, 4>(a, sm_count, st);
        case 15: return launch_sides<15, 4>(a, sm_count, st);
        default: return launch_sides<16, 4>(a, sm_count, st);
    }
}

// Blocks the persistent launch runs at most (the first pass's pool is sized per block).
int max_blocks(int W, int S, uint32_t block_words, int sm_count) {
    const size_t smem = sides_smem(W, S, block_words);
    int per_sm = (int)std::min<size_t>((size_t)(228 * 1024) / (smem + 1024), (size_t)(64 / W));
    return sm_count * std::max(per_sm, 1);
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

gxy_status fail(gxy_status s, const std::string& m) {
    set_error(m);
    return s;
}

}  // namespace

extern "C" {

gxy_status gxy_gapped_extend(gxy_ctx* ctx, const gxy_dseq* target, uint64_t t_lo, uint64_t t_hi,
                             const gxy_dseq* query, const gxy_search_params* params, const gxy_gapped_params* gp,
                             const uint32_t* t_pos, const uint32_t* q_pos, uint64_t n, gxy_gapped_result* out,
                             gxy_gapped_stats* stats) {
    if (!ctx || !target || !query || !params || !gp || !out || (n && (!t_pos || !q_pos)))
        return fail(GXY_EINVAL, "null argument");
    memset(out, 0, sizeof(*out));
    if (stats) memset(stats, 0, sizeof(*stats));
    if (t_lo == 0 && t_hi == 0) t_hi = target->len;
    if (t_lo > t_hi || t_hi > target->len) return fail(GXY_EINVAL, "target view outside the target");
    const uint64_t lt = t_hi - t_lo, lq = query->len;
    if (lt >= (1ull << 32) || lq >= (1ull << 32)) return fail(GXY_EUNSUPPORTED, "sequences of 2^32 bases or more");
    if (n >= (1ull << 31)) return fail(GXY_EUNSUPPORTED, "2^31 anchors or more");
    for (uint64_t k = 0; k < n; k++)
        if (t_pos[k] >= lt || q_pos[k] >= lq) return fail(GXY_EINVAL, "anchor outside its sequence");
    // The exact envelope: every DP value formed stays far from i32 limits, and
    // values formed from NEG_INF stay below every threshold.
    int64_t smax = std::abs((int64_t)params->ambig);
    for (int k = 0; k < 16; k++) smax = std::max<int64_t>(smax, std::abs((int64_t)params->sub[k]));
    if (smax > (1 << 16)) return fail(GXY_EUNSUPPORTED, "substitution scores beyond +-65536");
    if (gp->gap_open < 0 || gp->gap_open > (1 << 20) || gp->gap_extend < 0 || gp->gap_extend > (1 << 16))
        return fail(GXY_EUNSUPPORTED, "gap costs outside [0, 2^20] (open) / [0, 2^16] (extend)");
    if (gp->y_drop < 0 || gp->y_drop > (1 << 27)) return fail(GXY_EUNSUPPORTED, "y_drop outside [0, 2^27]");
    // A cell's score is at most the largest positive column score times the
    // columns of the shorter sequence.
    int64_t spos = std::max<int64_t>(0, params->ambig);
    for (int k = 0; k < 16; k++) spos = std::max<int64_t>(spos, params->sub[k]);
    if ((double)spos * (double)(std::min(lt, lq) + 2) >= 2147483648.0 - 1048576.0)
        return fail(GXY_EUNSUPPORTED, "scores could exceed 2^31 - 2^20 on sequences this long");
    const int32_t goe = gp->gap_open + gp->gap_extend, ge = gp->gap_extend;
    int64_t radius = -1;
    if (ge > 0) {
        const int64_t r = ((int64_t)gp->y_drop - goe) / ge;   // truncates toward zero, as Rust's i32 `/`
        radius = std::max<int64_t>(r, 0) + 2;
    }
    // Band width bound over all sides: min(4R + 4, m + 1) with m < lq.
    const int64_t bw_max = radius >= 0 ? std::min<int64_t>(4 * radius + 4, (int64_t)lq) : (int64_t)lq;
    int Sc = 4;   // 4 cells a thread: 3.1-3.4 us a row at W = 10 against 3.85 us with 8 at W = 5
    {
        std::lock_guard<std::mutex> g(ctx->mu);
        if (ctx->tuning.gapped_cells == 8) Sc = 8;
    }
    const int Wd = (int)std::max<int64_t>(1, (bw_max + 32 * Sc - 1) / (32 * Sc));
    if (bw_max > kMaxCells)
        return fail(GXY_EUNSUPPORTED, "band wider than 2048 cells (y_drop / gap_extend too large for the device DP)");
    out->n_alns = n;
    out->alns = n ? (gxy_gapped_aln*)calloc(n, sizeof(gxy_gapped_aln)) : nullptr;
    if (n && !out->alns) return fail(GXY_ENOMEM, "host allocation");
    if (n == 0) return GXY_OK;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(GXY_ECUDA, "cudaSetDevice");
    WorkerLease Lw(ctx);
    if (!Lw.w) {
        gxy_gapped_result_free(out);
        return Lw.err;
    }
    Worker* W = Lw.w;
    cudaStream_t st = W->st;
    // Per-anchor arrays: anchors (2 x u32), sides (2 x 32 B), joined records,
    // run counts and offsets (+1), counters.
    const size_t off_t = 0, off_q = off_t + n * 4, off_side = (off_q + n * 4 + 255) & ~(size_t)255,
                 off_aln = off_side + 2 * n * sizeof(GapSide), off_cnt = off_aln + n * sizeof(gxy_gapped_aln),
                 off_offs = off_cnt + n * 4, off_ctr = (off_offs + (n + 1) * 4 + 255) & ~(size_t)255,
                 aux_bytes = off_ctr + kCtrWords * 8;
    cudaError_t e = W->gaux.ensure(aux_bytes);
    if (e != cudaSuccess) {
        gxy_gapped_result_free(out);
        return fail(GXY_ENOMEM, std::string("gapped buffers: ") + cudaGetErrorString(e));
    }
    unsigned char* aux = W->gaux.as<unsigned char>();
    GapArgs A{};
    A.T = view_of(target, t_lo, t_hi);
    A.Q = view_of(query, 0, lq);
    A.t_pos = reinterpret_cast<uint32_t*>(aux + off_t);
    A.q_pos = reinterpret_cast<uint32_t*>(aux + off_q);
    A.n_anchors = (uint32_t)n;
    memcpy(A.sub, params->sub, sizeof(A.sub));
    A.ambig = params->ambig;
    A.goe = goe;
    A.ge = ge;
    A.ydrop = gp->y_drop;
    A.radius = radius;
    A.ctr = reinterpret_cast<unsigned long long*>(aux + off_ctr);
    A.sides = reinterpret_cast<GapSide*>(aux + off_side);
    gxy_gapped_aln* d_aln = reinterpret_cast<gxy_gapped_aln*>(aux + off_aln);
    uint32_t* d_cnt = reinterpret_cast<uint32_t*>(aux + off_cnt);
    uint32_t* d_offs = reinterpret_cast<uint32_t*>(aux + off_offs);
    e = cudaMemcpyAsync(aux + off_t, t_pos, n * 4, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(aux + off_q, q_pos, n * 4, cudaMemcpyHostToDevice, st);
    // Pass 1: every side, back-pointers in per-block chains of pool blocks.
    // The pool is sized for 64 pool blocks per CUDA block and grows toward what earlier
    // calls needed, within a quarter of the free device memory.
    A.block_words = (uint32_t)(kHdr + kRows + kRows * 32 * Wd * Sc / 8);
    const uint64_t block_bytes = (uint64_t)A.block_words * 4;
    const int blocks_max = max_blocks(Wd, Sc, A.block_words, ctx->sm_count);
    size_t free_b = 0, total_b = 0;
    uint32_t pool_limit = 0;
    {
        std::lock_guard<std::mutex> g(ctx->mu);
        pool_limit = ctx->tuning.gapped_pool_blocks;
    }
    uint64_t want_pool = std::max<uint64_t>((uint64_t)blocks_max * 64 * block_bytes, W->gpool_want);
    if (want_pool > W->gpool.bytes) {   // growing: at most a quarter of the free memory
        if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) free_b = 0;
        const uint64_t pool_cap = std::max<uint64_t>((uint64_t)blocks_max * 4 * block_bytes, free_b / 4);
        want_pool = std::max<uint64_t>(std::min(want_pool, pool_cap), W->gpool.bytes);
    } else {
        want_pool = W->gpool.bytes;
    }
    // Runs: a first-pass side reserves exactly the runs it wrote (the second
    // pass reserves best_i + best_j words in a buffer of its own).
    uint64_t want_runs = std::max<uint64_t>(std::max<uint64_t>(n * 512, std::min<uint64_t>(n * 4096, 1ull << 28)),
                                            W->gruns.bytes / 4);
    cudaEvent_t e0 = W->ev[0], e1 = W->ev[2];
    unsigned long long ctr[kCtrWords] = {};
    uint32_t reruns = 0;
    A.list = nullptr;
    A.base = nullptr;
    A.n_list = 0;
    A.runs2 = nullptr;
    // First pass: a run scratch per resident CUDA block.
    A.scratch_words = kScratchWords;
    A.scratch_blocks = (uint32_t)blocks_max;
    if (e == cudaSuccess) e = W->gscr.ensure((size_t)blocks_max * kScratchWords * 4);
    A.scratch = W->gscr.as<uint32_t>();
    for (int attempt = 0; e == cudaSuccess; attempt++) {
        e = W->gpool.ensure(want_pool);
        if (e == cudaSuccess) e = W->gruns.ensure(want_runs * 4);
        if (e != cudaSuccess) break;
        A.pool = W->gpool.as<uint32_t>();
        A.pool_blocks = W->gpool.bytes / block_bytes;
        if (pool_limit) A.pool_blocks = std::min<uint64_t>(A.pool_blocks, pool_limit);
        A.runs = W->gruns.as<uint32_t>();
        A.runs_cap = W->gruns.bytes / 4;
        e = cudaMemsetAsync(A.ctr, 0, kCtrWords * 8, st);
        if (e == cudaSuccess) e = cudaEventRecord(e0, st);
        if (e == cudaSuccess) e = launch_sides_for(Wd, Sc, A, ctx->sm_count, st);
        if (e == cudaSuccess) e = cudaEventRecord(e1, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(ctr, A.ctr, sizeof(ctr), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) break;
        // Only a short run buffer reruns the whole pass (the pool's shortfall
        // goes to pass 2): grow it to what the sides reserved.
        if (!(ctr[kCtrFlags] & kFlagRuns) || attempt >= 2) break;
        want_runs = std::max<uint64_t>(want_runs * 2, ctr[kCtrRuns] * 5 / 4 + 1024);
        reruns++;
    }
    float ms = 0.f;
    if (e == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
    if (e == cudaSuccess && (ctr[kCtrFlags] & kFlagState)) {
        gxy_gapped_result_free(out);
        return fail(GXY_ECUDA, "gapped extension: inconsistent traceback state");
    }
    // Pass 2: the sides pass 1 could not store, each with exactly the blocks
    // its rows need (pass 1 counted them), in groups that fit half the free
    // memory; their runs go to a second buffer of exactly their reservations.
    uint32_t* d_pool2 = nullptr;
    uint32_t* d_runs2 = nullptr;
    void* d_list = nullptr;
    uint64_t pass2_sides = 0, pass2_cells = 0;
    if (e == cudaSuccess && (ctr[kCtrFlags] & (kFlagPool | kFlagRuns | kFlagScratch))) {
        std::vector<GapSide> sides(2 * n);
        e = cudaMemcpyAsync(sides.data(), A.sides, 2 * n * sizeof(GapSide), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        std::vector<uint32_t> list;
        std::vector<uint64_t> need;
        uint64_t runs2 = 0, max_need = 0, tot_need = 0;
        for (uint64_t k = 0; e == cudaSuccess && k < 2 * n; k++) {
            if (!(sides[k].flags & (kFlagPool | kFlagRuns | kFlagScratch))) continue;
            list.push_back((uint32_t)k);
            const uint64_t nb = ((uint64_t)sides[k].rows + kRows - 1) / kRows;
            need.push_back(nb);
            max_need = std::max(max_need, nb);
            tot_need += nb;
            runs2 += (uint64_t)sides[k].t_span + sides[k].q_span;
        }
        pass2_sides = list.size();
        if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) free_b = 0;
        const uint64_t budget = std::max<uint64_t>(max_need, free_b / 2 / block_bytes);
        const uint64_t group_blocks = std::min<uint64_t>(budget, tot_need);
        if (e == cudaSuccess) e = cudaMallocAsync((void**)&d_runs2, std::max<uint64_t>(runs2, 1) * 4, st);
        if (e == cudaSuccess) e = cudaMallocAsync((void**)&d_pool2, group_blocks * block_bytes, st);
        if (e == cudaSuccess) e = cudaMallocAsync(&d_list, list.size() * 16, st);
        // Later calls start with a pass-1 pool closer to this need.
        W->gpool_want = (A.pool_blocks + tot_need) * block_bytes;
        GapArgs B = A;
        B.pool = d_pool2;
        B.runs = d_runs2;
        B.runs_cap = std::max<uint64_t>(runs2, 1);
        uint32_t* dl = reinterpret_cast<uint32_t*>(d_list);
        uint64_t* dbase = reinterpret_cast<uint64_t*>(reinterpret_cast<unsigned char*>(d_list) + list.size() * 8);
        std::vector<uint64_t> base(list.size());
        std::vector<uint32_t> lst(list.begin(), list.end());
        uint64_t k0 = 0;
        unsigned long long c2[kCtrWords] = {};
        bool first_group = true;
        while (e == cudaSuccess && k0 < list.size()) {
            uint64_t k1 = k0, used = 0;
            while (k1 < list.size() && used + need[k1] <= group_blocks) {
                base[k1] = used;
                used += need[k1];
                k1++;
            }
            B.list = dl + k0;
            B.base = dbase + k0;
            B.n_list = k1 - k0;
            B.pool_blocks = group_blocks;
            e = cudaMemcpyAsync(dl + k0, lst.data() + k0, (k1 - k0) * 4, cudaMemcpyHostToDevice, st);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(dbase + k0, base.data() + k0, (k1 - k0) * 8, cudaMemcpyHostToDevice, st);
            // The task cursor restarts; the run counter keeps counting across groups.
            if (e == cudaSuccess) e = cudaMemsetAsync(B.ctr + kCtrTask, 0, 8, st);
            if (e == cudaSuccess && first_group) e = cudaMemsetAsync(B.ctr + kCtrRuns, 0, 8, st);
            // Rows and cells count this group's sides only.
            if (e == cudaSuccess) e = cudaMemsetAsync(B.ctr + kCtrRows, 0, 16, st);
            if (e == cudaSuccess) e = cudaMemsetAsync(B.ctr + kCtrFlags, 0, 8, st);
            if (e == cudaSuccess) e = cudaEventRecord(e0, st);
            if (e == cudaSuccess) e = launch_sides_for(Wd, Sc, B, ctx->sm_count, st);
            if (e == cudaSuccess) e = cudaEventRecord(e1, st);
            if (e == cudaSuccess) e = cudaMemcpyAsync(c2, B.ctr, sizeof(c2), cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e == cudaSuccess && (c2[kCtrFlags] & (kFlagPool | kFlagRuns | kFlagState))) {
                cudaFreeAsync(d_pool2, st);
                cudaFreeAsync(d_runs2, st);
                cudaFreeAsync(d_list, st);
                cudaStreamSynchronize(st);
                gxy_gapped_result_free(out);
                return fail(GXY_ECUDA, "gapped extension: the exactly sized second pass fell short");
            }
            float gms = 0.f;
            if (e == cudaSuccess) cudaEventElapsedTime(&gms, e0, e1);
            ms += gms;
            pass2_cells += c2[kCtrCells];
            first_group = false;
            k0 = k1;
        }
        A.runs2 = d_runs2;
    }
    uint32_t total_runs = 0;
    if (e == cudaSuccess) {
        count_launch();
        k_gapped_join<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(A, gp->gapped_threshold, d_aln, d_cnt);
        scan_u32(d_cnt, d_offs, nullptr, n, n, true, nullptr, W->ps, st);
        e = cudaMemcpyAsync(&total_runs, d_offs + n, 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(out->alns, d_aln, n * sizeof(gxy_gapped_aln), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
    uint32_t* d_final = nullptr;
    if (e == cudaSuccess && total_runs) {
        out->runs = (uint32_t*)malloc((size_t)total_runs * 4);
        if (!out->runs) {
            gxy_gapped_result_free(out);
            return fail(GXY_ENOMEM, "host allocation");
        }
        e = cudaMallocAsync((void**)&d_final, (size_t)total_runs * 4, st);
        if (e == cudaSuccess) {
            const uint64_t blocks = std::min<uint64_t>((n + 7) / 8, (uint64_t)ctx->sm_count * 16);
            count_launch();
            k_gapped_emit<<<(unsigned)blocks, 256, 0, st>>>(A, d_aln, d_offs, d_final);
            e = cudaMemcpyAsync(out->runs, d_final, (size_t)total_runs * 4, cudaMemcpyDeviceToHost, st);
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (d_final) cudaFreeAsync(d_final, st);
    }
    if (d_pool2) cudaFreeAsync(d_pool2, st);
    if (d_runs2) cudaFreeAsync(d_runs2, st);
    if (d_list) cudaFreeAsync(d_list, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) {
        gxy_gapped_result_free(out);
        return fail(e == cudaErrorMemoryAllocation ? GXY_ENOMEM : GXY_ECUDA,
                    std::string("gapped extension: ") + cudaGetErrorString(e));
    }
    out->n_runs = total_runs;
    // Offsets of the passing anchors' scripts: the scan's output, on the host.
    uint64_t acc = 0;
    for (uint64_t k = 0; k < n; k++) {
        out->alns[k].script_off = acc;
        acc += out->alns[k].script_len;
    }
    if (stats) {
        stats->rows = ctr[kCtrRows];
        stats->cells = ctr[kCtrCells];
        stats->device_ms = ms;
        stats->reruns = reruns;
        stats->second_pass_sides = pass2_sides;
        stats->second_pass_cells = pass2_cells;
        stats->warps_per_side = (uint32_t)Wd;
        stats->cells_per_thread = (uint32_t)Sc;
        stats->max_side_rows = ctr[kCtrMaxRows];
    }
    return GXY_OK;
}

void gxy_gapped_result_free(gxy_gapped_result* r) {
    if (!r) return;
    free(r->alns);
    free(r->runs);
    r->alns = nullptr;
    r->runs = nullptr;
    r->n_alns = r->n_runs = 0;
}

}  // extern "C"
