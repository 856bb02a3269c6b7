// gxy_kernels.cu -- the seed->HSP kernels for sm_100a.
//
// Work is integer and byte work bounded by HBM/L2, so there are no tensor
// cores here.  Shapes: grids are persistent (a multiple of the SM count) or
// grid-stride; every sequence access goes through the padded layout of
// gxy_device.cuh.
#include "gxy_kernels.cuh"

namespace gxy {

__host__ __device__ __forceinline__ uint64_t umin64(uint64_t a, uint64_t b) { return a < b ? a : b; }

// ---------------------------------------------------------------------------
// Packing
// ---------------------------------------------------------------------------

// encode_base (src/dna.rs:12-20) on one byte: code, valid, soft-masked.
__device__ __forceinline__ void encode(uint8_t b, uint32_t& code, uint32_t& valid, uint32_t& masked) {
    const uint8_t u = b & 0xDF;   // ASCII upper case
    code = 0;
    valid = 1;
    if (u == 'A') code = 0;
    else if (u == 'C') code = 1;
    else if (u == 'G') code = 2;
    else if (u == 'T' || u == 'U') code = 3;
    else valid = 0;
    masked = valid && (b >= 'a' && b <= 'z');
}

// One thread per 32 positions: reads 32 ASCII bytes (two 16-byte loads when
// aligned), writes one u64 of codes and one u32 each of valid and mask.
__global__ void k_pack_ascii(const uint8_t* __restrict__ ascii, uint64_t n, uint64_t* codes, uint32_t* valid,
                             uint32_t* mask) {
    const uint64_t nw = (n + 31) / 32;
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < nw; w += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t p0 = w * 32;
        uint64_t c = 0;
        uint32_t v = 0, m = 0;
#pragma unroll 8
        for (int k = 0; k < 32; k++) {
            const uint64_t p = p0 + k;
            if (p >= n) break;
            uint32_t code, val, msk;
            encode(ascii[p], code, val, msk);
            c |= (uint64_t)code << (2 * k);
            v |= val << k;
            m |= msk << k;
        }
        // Local position p lives at global kPad + p; kPad is a multiple of 32.
        codes[kPad / 32 + w] = c;
        valid[kPad / 32 + w] = v;
        mask[kPad / 32 + w] = m;
    }
}

void launch_pack_ascii(const uint8_t* ascii, uint64_t n, uint64_t* codes, uint32_t* valid, uint32_t* mask,
                       cudaStream_t st) {
    const uint64_t nw = (n + 31) / 32;
    if (!nw) return;
    const int blocks = (int)umin64((nw + 255) / 256, 148 * 16);
    count_launch();
    k_pack_ascii<<<blocks, 256, 0, st>>>(ascii, n, codes, valid, mask);
}

// Reverse complement: output position o takes input position n-1-o; a valid
// base becomes its complement (3 - c), an invalid one code 0 and unmasked,
// and the mask bit moves with the base (src/sequences.rs:303-318).  One thread
// per 32 output positions; the 32 input positions are one unaligned load.

__global__ void k_reverse_complement(const uint64_t* __restrict__ ic, const uint32_t* __restrict__ iv,
                                     const uint32_t* __restrict__ im, uint64_t n, uint64_t* oc, uint32_t* ov,
                                     uint32_t* om) {
    const uint64_t nw = (n + 31) / 32;
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < nw; w += (uint64_t)gridDim.x * blockDim.x) {
        // Output positions [32w, 32w+32) <- input positions n-1-32w down to n-32-32w.
        // Load the 32 input positions ending at n-1-32w: start gp = kPad + n - 32 - 32w
        // (never below 32 because kPad = 64).
        const uint64_t gp = kPad + n - 32 - 32 * w;
        uint64_t c = load_codes32(ic, gp);
        uint32_t v = load_bits32(iv, gp);
        uint32_t m = load_bits32(im, gp);
        // Input lane j (position gp + j) maps to output lane 31 - j.
        v = __brev(v);
        m = __brev(m) & v;
        c = __brevll(c);
        // __brevll reverses bits; swap the two bits of each pair back.
        c = ((c >> 1) & 0x5555555555555555ull) | ((c & 0x5555555555555555ull) << 1);
        c = (~c) & spread_bits_to_pairs(v);
        const uint32_t nvalid = (uint32_t)umin64(32, n - 32 * w);
        if (nvalid < 32) {
            const uint32_t keep = (1u << nvalid) - 1;
            v &= keep;
            m &= keep;
            c &= spread_bits_to_pairs(keep);
        }
        oc[kPad / 32 + w] = c;
        ov[kPad / 32 + w] = v;
        om[kPad / 32 + w] = m;
    }
}

void launch_reverse_complement(const uint64_t* icodes, const uint32_t* ivalid, const uint32_t* imask, uint64_t n,
                               uint64_t* ocodes, uint32_t* ovalid, uint32_t* omask, cudaStream_t st) {
    const uint64_t nw = (n + 31) / 32;
    if (!nw) return;
    const int blocks = (int)umin64((nw + 255) / 256, 148 * 16);
    count_launch();
    k_reverse_complement<<<blocks, 256, 0, st>>>(icodes, ivalid, imask, n, ocodes, ovalid, omask);
}

// ---------------------------------------------------------------------------
// Seed words and the table build
// ---------------------------------------------------------------------------

__global__ void k_seed_words(SeqView view, Pattern pat, uint32_t step, uint32_t nwin, uint32_t sentinel,
                             uint32_t* keys, uint32_t* vals, uint32_t* counts) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nwin; k += gridDim.x * blockDim.x) {
        const uint32_t p = k * step;
        uint32_t w;
        if (word_at(view, pat, p, w)) {
            keys[k] = w;
            atomicAdd(&counts[w], 1u);
        } else {
            keys[k] = sentinel;
        }
        vals[k] = p;
    }
}

void launch_seed_words(SeqView view, Pattern pat, uint32_t step, uint32_t nwin, uint32_t sentinel, uint32_t* keys,
                       uint32_t* vals, uint32_t* counts, cudaStream_t st) {
    if (!nwin) return;
    const int blocks = (int)umin64((nwin + 255) / 256, 148 * 16);
    count_launch();
    k_seed_words<<<blocks, 256, 0, st>>>(view, pat, step, nwin, sentinel, keys, vals, counts);
}


__global__ void k_prune_counts(const uint32_t* starts, uint64_t nw, uint32_t limit, uint32_t* counts2) {
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < nw; w += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t c = starts[w + 1] - starts[w];
        counts2[w] = c <= limit ? c : 0u;
    }
}

void launch_prune_counts(const uint32_t* starts, uint64_t num_words, uint32_t limit, uint32_t* counts2,
                         cudaStream_t st) {
    count_launch();
    k_prune_counts<<<148 * 8, 256, 0, st>>>(starts, num_words, limit, counts2);
}

__global__ void k_prune_copy(const uint32_t* pos, const uint32_t* starts, uint64_t nw, const uint32_t* new_starts,
                             uint32_t limit, uint32_t* new_pos) {
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < nw; w += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t s = starts[w], e = starts[w + 1];
        if (e - s > limit) continue;
        const uint32_t o = new_starts[w];
        for (uint32_t i = s; i < e; i++) new_pos[o + (i - s)] = pos[i];
    }
}

void launch_prune_copy(const uint32_t* positions, const uint32_t* starts, uint64_t num_words,
                       const uint32_t* new_starts, uint32_t limit, uint32_t* new_positions, cudaStream_t st) {
    count_launch();
    k_prune_copy<<<148 * 8, 256, 0, st>>>(positions, starts, num_words, new_starts, limit, new_positions);
}

// ---------------------------------------------------------------------------
// Scan helpers of the exact lane-per-hit screens below (k_screen_wide and
// the packed k_screen).  The screens read hits from a global array written
// either by k_enumerate (every raw hit) or by k_seed_filter in gxy_filter.cu
// (only the hits whose upper-bound x-drop might reach hspthresh).
// ---------------------------------------------------------------------------

// 32 positions starting at offset o of a 4-word window (o <= 96).
__device__ __forceinline__ uint64_t win_codes(const uint64_t (&w)[4], uint32_t o) {
    const uint32_t i = o >> 5, s = (o & 31) * 2;
    const uint64_t lo = i == 0 ? w[0] : (i == 1 ? w[1] : w[2]);
    const uint64_t hi = i == 0 ? w[1] : (i == 1 ? w[2] : w[3]);
    return s ? ((lo >> s) | (hi << (64 - s))) : lo;
}
__device__ __forceinline__ uint32_t win_bits(const uint32_t (&w)[4], uint32_t o) {
    const uint32_t i = o >> 5;
    const uint32_t lo = i == 0 ? w[0] : (i == 1 ? w[1] : w[2]);
    const uint32_t hi = i == 0 ? w[1] : (i == 1 ? w[2] : w[3]);
    return __funnelshift_r(lo, hi, o & 31);
}

// Spreads the 2-bit codes of 16 columns (32 bits) into 16 nibbles (64 bits).
__device__ __forceinline__ uint64_t spread16(uint32_t x) {
    uint64_t v = x;
    v = (v | (v << 16)) & 0x0000FFFF0000FFFFull;
    v = (v | (v << 8)) & 0x00FF00FF00FF00FFull;
    v = (v | (v << 4)) & 0x0F0F0F0F0F0F0F0Full;
    v = (v | (v << 2)) & 0x3333333333333333ull;
    return v;
}

// The x-drop scan of extend_one_side (src/hsp.rs:179-193) over up to 32
// columns whose codes and validity are in registers (column k at bits 2k /
// bit k).  Continues a side from (run, best, bext) after ext0 columns; n = 0
// is a no-op.  Sets ended when the x-drop break fired; used = columns consumed.
template <bool kCheckValid>
__device__ __forceinline__ void scan32(uint64_t tc, uint64_t qc, uint32_t vv, uint32_t n, int32_t xd,
                                       const int32_t* lut, int32_t ambig, uint32_t ext0, int32_t& run,
                                       int32_t& best, uint32_t& bext, bool& ended, uint32_t& used) {
    // idx_k = (t_k << 2) | q_k as nibble k of nib[k / 16].
    const uint64_t nib0 = (spread16((uint32_t)tc) << 2) | spread16((uint32_t)qc);
    const uint64_t nib1 = (spread16((uint32_t)(tc >> 32)) << 2) | spread16((uint32_t)(qc >> 32));
    int32_t r = run, b = best;
    uint32_t be = bext, lim = n, brk = n;
#pragma unroll
    for (int g = 0; g < 4; g++) {
        if (!__any_sync(kFull, (uint32_t)(g * 8) < lim)) break;
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const int k = g * 8 + i;
            if ((uint32_t)k < lim) {
                const uint32_t idx = (uint32_t)(((k < 16 ? nib0 : nib1) >> (4 * (k & 15))) & 15u);
                int32_t sc = lut[idx];
                if (kCheckValid) sc = ((vv >> k) & 1u) ? sc : ambig;
                r += sc;
                if (r > b) {
                    b = r;
                    be = ext0 + k + 1;
                } else if (b - r > xd) {
                    brk = k;
                    lim = 0;
                }
            }
        }
    }
    ended = brk < n;
    used = ended ? brk + 1 : n;
    run = r;
    best = b;
    bext = be;
}

// One side's scan state for the interleaved scans below.
struct SideScan {
    uint64_t nib0, nib1;   // (t << 2 | q) nibbles of columns 0-15 and 16-31
    uint32_t vv;           // column validity
    uint32_t lim;          // columns still to scan (0 once the side broke)
    uint32_t brk;          // break column, or n when the side did not break
    uint32_t ext0;         // columns of this side already scanned
    int32_t r, b;          // running score, best
    uint32_t be;           // best extent
};

__device__ __forceinline__ void side_init(SideScan& S, uint64_t tc, uint64_t qc, uint32_t vv, uint32_t n,
                                          uint32_t ext0, int32_t run, int32_t best, uint32_t bext) {
    S.nib0 = (spread16((uint32_t)tc) << 2) | spread16((uint32_t)qc);
    S.nib1 = (spread16((uint32_t)(tc >> 32)) << 2) | spread16((uint32_t)(qc >> 32));
    S.vv = vv;
    S.lim = n;
    S.brk = n;
    S.ext0 = ext0;
    S.r = run;
    S.b = best;
    S.be = bext;
}

template <bool kCheckValid, int k>
__device__ __forceinline__ void side_step(SideScan& S, int32_t xd, const int32_t* lut, int32_t ambig) {
    if ((uint32_t)k < S.lim) {
        const uint32_t idx = (uint32_t)(((k < 16 ? S.nib0 : S.nib1) >> (4 * (k & 15))) & 15u);
        int32_t sc = lut[idx];
        if (kCheckValid) sc = ((S.vv >> k) & 1u) ? sc : ambig;
        S.r += sc;
        if (S.r > S.b) {
            S.b = S.r;
            S.be = S.ext0 + k + 1;
        } else if (S.b - S.r > xd) {
            S.brk = k;
            S.lim = 0;
        }
    }
}

// Two independent sides scanned column by column in lockstep: the x-drop
// recurrence of each side is a serial chain, and interleaving two chains
// lets the scheduler issue from both.
template <bool kCheckValid>
__device__ __forceinline__ void scan_pair(SideScan& A, SideScan& B, int32_t xd, const int32_t* lut,
                                          int32_t ambig) {
#define GXY_STEP8(g)                                                             \
    side_step<kCheckValid, g * 8 + 0>(A, xd, lut, ambig);                        \
    side_step<kCheckValid, g * 8 + 0>(B, xd, lut, ambig);                        \
    side_step<kCheckValid, g * 8 + 1>(A, xd, lut, ambig);                        \
    side_step<kCheckValid, g * 8 + 1>(B, xd, lut, ambig);                        \
    side_step<kCheckValid, g * 8 + 2>(A, xd, lut, ambig);                        \
    side_step<kCheckValid, g * 8 + 2>(B, xd, lut, ambig);                        \
    side_step<kCheckValid, g * 8 + 3>(A, xd, lut, ambig);                        \
    side_step<kCheckValid, g * 8 + 3>(B, xd, lut, ambig);                        \
    side_step<kCheckValid, g * 8 + 4>(A, xd, lut, ambig);                        \
    side_step<kCheckValid, g * 8 + 4>(B, xd, lut, ambig);                        \
    side_step<kCheckValid, g * 8 + 5>(A, xd, lut, ambig);                        \
    side_step<kCheckValid, g * 8 + 5>(B, xd, lut, ambig);                        \
    side_step<kCheckValid, g * 8 + 6>(A, xd, lut, ambig);                        \
    side_step<kCheckValid, g * 8 + 6>(B, xd, lut, ambig);                        \
    side_step<kCheckValid, g * 8 + 7>(A, xd, lut, ambig);                        \
    side_step<kCheckValid, g * 8 + 7>(B, xd, lut, ambig);
    if (!__any_sync(kFull, A.lim > 0 || B.lim > 0)) return;
    GXY_STEP8(0)
    if (!__any_sync(kFull, A.lim > 8 || B.lim > 8)) return;
    GXY_STEP8(1)
    if (!__any_sync(kFull, A.lim > 16 || B.lim > 16)) return;
    GXY_STEP8(2)
    if (!__any_sync(kFull, A.lim > 24 || B.lim > 24)) return;
    GXY_STEP8(3)
#undef GXY_STEP8
}

__device__ __forceinline__ void scan_pair_any(SideScan& A, SideScan& B, uint32_t na, uint32_t nb, int32_t xd,
                                              const int32_t* lut, int32_t ambig) {
    const uint32_t need_a = na >= 32 ? 0xffffffffu : ((1u << na) - 1u);
    const uint32_t need_b = nb >= 32 ? 0xffffffffu : ((1u << nb) - 1u);
    if (__any_sync(kFull, (A.vv & need_a) != need_a || (B.vv & need_b) != need_b))
        scan_pair<true>(A, B, xd, lut, ambig);
    else
        scan_pair<false>(A, B, xd, lut, ambig);
}

// ---------------------------------------------------------------------------
// Enumeration: one warp per tile of 32 consecutive query windows of one unit.
// Each lane forms its window's seed word and transition variants
// (src/seed_search.rs:76-90); the warp reserves room for all hits of the
// tile with one atomic and writes (t, q, unit) for every position of every
// variant's bucket (src/pos_table.rs:102-108).  Large buckets are copied by
// the whole warp.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void store_hit(Hit* p, uint32_t t, uint32_t q, uint32_t u) {
    p->t = t;
    p->q = q;
    p->unit = u;
}
__device__ __forceinline__ Hit load_hit(const Hit* p) { return *p; }

// kRegVar: variants whose bucket bounds stay in registers between the two
// passes (the rest are re-read): 1 without transitions, 13 for weight 12 with
// one transition, else 16.
template <uint32_t kRegVar>
__global__ __launch_bounds__(256, 4) void k_enumerate(const __grid_constant__ ScreenArgs a) {
    const int lane = threadIdx.x & 31;
    const uint32_t ntile = a.tile_hi - a.tile_lo;
    unsigned long long n_windows = 0, n_raw = 0;
    uint32_t* const ctl = a.ctl;
    unsigned long long* const max_fail = reinterpret_cast<unsigned long long*>(ctl + kCMaxFail);
    // This pass takes the tiles the previous pass could not fit first (its
    // redo list), then fresh tiles until the hit buffer is full.
    const uint32_t pass = ctl[kCPass];
    const uint32_t* redo_in = a.redo + ((pass - 1) & 1u) * kRedoCap;
    uint32_t* redo_out = a.redo + (pass & 1u) * kRedoCap;
    const uint32_t n_redo = ctl[kCRedoN + ((pass - 1) & 1u)];
    uint32_t* const n_redo_out = ctl + kCRedoN + (pass & 1u);
    // A tile that did not fit this pass goes to the next pass's list.
    auto defer = [&](uint32_t tl, unsigned long long wtot) {
        atomicExch(ctl + kCStop, 1u);
        const uint32_t i = atomicAdd(n_redo_out, 1u);
        if (i < kRedoCap) redo_out[i] = tl;
        else atomicExch(ctl + kCRedoOver, 1u);
        atomicMax(max_fail, wtot);
    };
    bool redo_done = false;
    // Fresh tiles are claimed kClaim at a time, and the next claim is made
    // while the current tiles are processed: one atomic per kClaim tiles
    // (all warps hit that counter), its round trip off the critical path.
    // (Measured on the 10 Mbp plain launch: 2 beats 4 by 2 % and 8 is slower.)
    constexpr uint32_t kClaim = 2;
    uint32_t next = 0xffffffffu;   // a claimed batch not yet started (warp-uniform)
    for (;;) {
      uint32_t batch, batch_end;
      if (!redo_done) {
          uint32_t i = 0;
          if (lane == 0) i = atomicAdd(ctl + kCRedoTake, 1u);
          i = __shfl_sync(kFull, i, 0);
          if (i < n_redo) {
              batch = redo_in[i];
              batch_end = batch + 1;
          } else {
              redo_done = true;
              continue;
          }
      } else {
          if (next == 0xffffffffu) {
              // Stop claiming once the buffer is full; the tiles not claimed
              // yet wait for the next pass behind the tile cursor.
              if (*reinterpret_cast<volatile uint32_t*>(ctl + kCStop)) break;
              uint32_t c = 0;
              if (lane == 0) c = atomicAdd(a.tile_counter, kClaim);
              next = __shfl_sync(kFull, c, 0);
          }
          batch = next;
          if (batch >= ntile) break;
          next = 0xffffffffu;
          if (!*reinterpret_cast<volatile uint32_t*>(ctl + kCStop)) {
              uint32_t c = 0;
              if (lane == 0) c = atomicAdd(a.tile_counter, kClaim);
              next = __shfl_sync(kFull, c, 0);
          }
          batch_end = min(ntile, batch + kClaim);
      }
      for (uint32_t tl = batch; tl < batch_end; tl++) {
        uint32_t tile = tl + a.tile_lo;
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
        // Pass 1: this lane's hit count over all variants.  The bucket
        // bounds of the first kRegVar variants stay in registers for pass 2.
        uint32_t rb[kRegVar], rc[kRegVar];
        uint32_t tot = 0;
        // The occupancy bit first: `starts` is read for non-empty buckets
        // only (about two thirds of the variant words of a 10 Mbp target
        // fall in empty buckets, and the 2 MB bitmap stays in L2).
        uint32_t ob[kRegVar];
#pragma unroll
        for (uint32_t v = 0; v < kRegVar; v++)
            ob[v] = (wv && v < a.n_var) ? __ldg(U.occ + ((word ^ a.var_xor[v]) >> 5)) : 0u;
#pragma unroll
        for (uint32_t v = 0; v < kRegVar; v++) {
            rb[v] = 0;
            rc[v] = 0;
            const uint32_t vw = word ^ a.var_xor[v];
            if ((ob[v] >> (vw & 31u)) & 1u) {
                rb[v] = __ldg(U.starts + vw);
                rc[v] = __ldg(U.starts + vw + 1) - rb[v];
                tot += rc[v];
            }
        }
        if (wv) {
            for (uint32_t v = kRegVar; v < a.n_var; v++) {
                const uint32_t vw = word ^ a.var_xor[v];
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
        if (wtot == 0) {
            n_windows += wv ? 1 : 0;
            continue;
        }
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(a.hit_count, (unsigned long long)wtot);
        // Pass 2: write this lane's hits into its slots [dst, dst + tot).
        // Their order within the slots is free (candidates are sorted by a
        // unique (diagonal, t) key later), so the first position of every
        // small bucket is loaded at once, before the rest; the first batch of
        // those loads is in flight while the reservation comes back.
        uint32_t first[8];
#pragma unroll
        for (uint32_t i = 0; i < 8; i++)
            if (i < kRegVar) first[i] = (rc[i] != 0 && rc[i] <= 16) ? __ldg(U.positions + rb[i]) : 0u;
        base = __shfl_sync(kFull, base, 0);
        if (base + wtot > a.hit_cap) {
            // The buffer is full: this tile goes to the next pass, and the
            // part of its reservation inside the buffer is marked unused.
            if (lane == 0) defer(tl, wtot);
            for (uint64_t j = base + lane; j < min((unsigned long long)a.hit_cap, base + wtot); j += 32)
                a.hits[j].unit = kNoUnit;
            continue;
        }
        n_windows += wv ? 1 : 0;
        n_raw += lane == 0 ? wtot : 0;
        uint64_t dst = base + (incl - tot);
#pragma unroll
        for (uint32_t v0 = 0; v0 < kRegVar; v0 += 8) {
            if (v0) {
#pragma unroll
                for (uint32_t i = 0; i < 8; i++)
                    if (v0 + i < kRegVar)
                        first[i] = (rc[v0 + i] != 0 && rc[v0 + i] <= 16) ? __ldg(U.positions + rb[v0 + i]) : 0u;
            }
#pragma unroll
            for (uint32_t i = 0; i < 8; i++)
                if (v0 + i < kRegVar && rc[v0 + i] != 0 && rc[v0 + i] <= 16)
                    store_hit(a.hits + dst++, first[i], q, u);
        }
        for (uint32_t v = 0; v < a.n_var; v++) {
            uint32_t b = 0, c = 0;
            if (v < kRegVar) {
#pragma unroll
                for (uint32_t x = 0; x < kRegVar; x++)
                    if (x == v) {
                        b = rb[x];
                        c = rc[x];
                    }
            } else if (wv) {
                const uint32_t vw = word ^ a.var_xor[v];
                b = __ldg(U.starts + vw);
                c = __ldg(U.starts + vw + 1) - b;
            }
            const bool big = c > 16;
            // Small buckets of the first kRegVar variants wrote their first position above.
            const uint32_t j0 = (v < kRegVar && !big) ? 1u : 0u;
            if (!big) {
                for (uint32_t j = j0; j < c; j++) store_hit(a.hits + dst++, __ldg(U.positions + b + j), q, u);
            }
            uint32_t bm = __ballot_sync(kFull, big);
            while (bm) {
                const int src = __ffs(bm) - 1;
                bm &= bm - 1;
                const uint32_t bb = __shfl_sync(kFull, b, src), cc = __shfl_sync(kFull, c, src);
                const uint32_t qq = __shfl_sync(kFull, q, src);
                const uint64_t dd = __shfl_sync(kFull, dst, src);
                for (uint32_t j = lane; j < cc; j += 32) store_hit(a.hits + dd + j, __ldg(U.positions + bb + j), qq, u);
            }
            if (big) dst += c;
        }
      }
    }
    // A batch claimed ahead but not started: the next pass takes it.
    if (next != 0xffffffffu && lane == 0)
        for (uint32_t tl = next; tl < min(ntile, next + kClaim); tl++) defer(tl, 0);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) n_windows += __shfl_xor_sync(kFull, n_windows, o);
    if (lane == 0) {
        atomicAdd(&a.stats[0], n_windows);
        atomicAdd(&a.stats[1], n_raw);
    }
}

__global__ void k_pass_reset(uint32_t* ctl, uint64_t surv_cap) {
    if (threadIdx.x != 0) return;
    unsigned long long* hits = reinterpret_cast<unsigned long long*>(ctl + kCHits);
    unsigned long long* surv = reinterpret_cast<unsigned long long*>(ctl + kCSurv);
    if (*surv > surv_cap) ctl[kCSurvOver] = 1u;   // the previous pass lost survivors
    if (*hits) ctl[kCWorkPasses]++;
    reinterpret_cast<unsigned long long*>(ctl + kCStats)[4] += *surv;   // survivors of the launch
    const uint32_t p = ctl[kCPass] + 1;
    ctl[kCPass] = p;
    ctl[kCRedoN + (p & 1u)] = 0;
    ctl[kCRedoTake] = 0;
    ctl[kCStop] = 0;
    ctl[kCHitNext] = 0;
    ctl[kCFiltNext] = 0;
    *hits = 0;
    *surv = 0;
}

void launch_pass_reset(uint32_t* ctl, uint64_t surv_cap, cudaStream_t st) {
    count_launch();
    k_pass_reset<<<1, 32, 0, st>>>(ctl, surv_cap);
}

void launch_enumerate(const ScreenArgs& a, int sm_count, cudaStream_t st) {
    count_launch();
    if (a.n_var == 1) k_enumerate<1><<<sm_count * 8, 256, 0, st>>>(a);
    else if (a.n_var == 13) k_enumerate<13><<<sm_count * 8, 256, 0, st>>>(a);
    else k_enumerate<16><<<sm_count * 8, 256, 0, st>>>(a);
}

// ---------------------------------------------------------------------------
// Screen: capped lane-per-hit x-drop over the enumerated hits.
//
// Each idle lane takes the next hit from the pass's hit array and loads one
// 128-position window of the target and of the query around it; from those
// registers it scores the seed footprint and the first 32 columns of both
// sides of extend_hit (src/hsp.rs:98-195) -- the sides are independent and
// are scanned in lockstep.  A side still running after 32 columns continues
// one chunk per iteration with fresh loads while the other lanes take new
// hits.  A hit is extended up to `cap` columns per side:
//  - ended below hspthresh: dropped.  Such a hit can never change the output:
//    search() only records diagonal cover for a hit whose HSP passes
//    (src/seed_search.rs:95-114), so whether it was admitted is irrelevant.
//  - ended at or above hspthresh, or still running at the cap: kept as a
//    candidate for the walk, which applies the diagonal rule in order.
// ---------------------------------------------------------------------------
template <int WARPS, int MINB>
__global__ __launch_bounds__(WARPS * 32, MINB) void k_screen_wide(const __grid_constant__ ScreenArgs a) {
    __shared__ int32_t s_lut[16];
    if (threadIdx.x < 16) s_lut[threadIdx.x] = a.sc.sub[threadIdx.x];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const uint32_t lt = lanemask_lt();
    const uint32_t L = a.pat.len;
    const int32_t ambig = a.sc.ambig, xdrop = a.sc.xdrop, thresh = a.sc.hspthresh;
    // Past the buffer's end the pass did not write (those tiles went to the
    // next pass).
    const uint32_t n_hits = (uint32_t)min(*a.hit_count, (unsigned long long)a.hit_cap);
    unsigned long long n_cols = 0;
    bool exhausted = false;

    bool busy = false, rdone = true, ldone = true;
    uint32_t ht = 0, hq = 0, hu = 0xffffffffu;
    int32_t seed = 0;
    int32_t rrun = 0, rbest = 0, lrun = 0, lbest = 0;
    uint32_t rbext = 0, lbext = 0, rext = 0, lext = 0, rrem = 0, lrem = 0;
    SeqView T{}, Q{};
    uint32_t cur_unit = 0xffffffffu;

    for (;;) {
        // ---------------- assign ----------------
        const uint32_t im = __ballot_sync(kFull, !busy);
        uint32_t base = 0, take = 0;
        if (!exhausted && im) {
            if (lane == 0) base = atomicAdd(a.hit_next, (uint32_t)__popc(im));
            base = __shfl_sync(kFull, base, 0);
            take = base < n_hits ? min((uint32_t)__popc(im), n_hits - base) : 0u;
            if (base + (uint32_t)__popc(im) >= n_hits) exhausted = true;
        }
        bool fresh = false;
        if (!busy) {
            const uint32_t rk = __popc(im & lt);
            if (rk < take) {
                const Hit h = load_hit(a.hits + base + rk);
                ht = h.t;
                hq = h.q;
                hu = h.unit;
                if (hu != kNoUnit && hu != cur_unit) {
                    cur_unit = hu;
                    const UnitDev U = a.units[hu];
                    T = a.tsegs[U.tseg];
                    Q = a.qsegs[U.qseg];
                }
                fresh = hu != kNoUnit;   // an unused slot of a failed reservation
                busy = fresh;
            }
        }
        if (!__any_sync(kFull, busy)) {
            if (exhausted) break;
            continue;
        }

        // ---------------- chunk data ----------------
        // Scan A: a fresh hit's first right chunk, or a continuing side's next chunk.
        // Scan B: a fresh hit's first left chunk.
        uint64_t atc = 0, aqc = 0, btc = 0, bqc = 0;
        uint32_t avv = 0, bvv = 0, an = 0, bn = 0;
        const bool a_right = fresh || !rdone;   // which side scan A advances
        if (fresh) {
            const uint64_t tb = T.base + ht, qb = Q.base + hq;
            const uint64_t tw = (tb - 32) & ~31ull, qw = (qb - 32) & ~31ull;
            uint64_t twc[4], qwc[4];
            uint32_t twv[4], qwv[4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                twc[j] = __ldg(T.codes + (tw >> 5) + j);
                qwc[j] = __ldg(Q.codes + (qw >> 5) + j);
                twv[j] = __ldg(T.valid + (tw >> 5) + j);
                qwv[j] = __ldg(Q.valid + (qw >> 5) + j);
            }
            const uint32_t ot = (uint32_t)(tb - tw), oq = (uint32_t)(qb - qw);   // both in [32, 63]
            // Seed footprint: all L columns (src/hsp.rs:119-123).
            {
                const uint64_t tc = win_codes(twc, ot), qc = win_codes(qwc, oq);
                const uint32_t vv = win_bits(twv, ot) & win_bits(qwv, oq);
                int32_t sd = 0;
#pragma unroll
                for (int k = 0; k < 32; k++) {
                    if ((uint32_t)k >= L) break;
                    sd += col_score(tc, qc, vv, k, s_lut, ambig);
                }
                seed = sd;
            }
            rrem = min(T.len - ht - L, Q.len - hq - L);
            lrem = min(ht, hq);
            rrun = rbest = lrun = lbest = 0;
            rbext = lbext = rext = lext = 0;
            rdone = rrem == 0;
            ldone = lrem == 0;
            an = min(32u, rrem);
            atc = win_codes(twc, ot + L);
            aqc = win_codes(qwc, oq + L);
            avv = win_bits(twv, ot + L) & win_bits(qwv, oq + L);
            bn = min(32u, lrem);
            btc = rev_pairs64(win_codes(twc, ot - 32));
            bqc = rev_pairs64(win_codes(qwc, oq - 32));
            bvv = __brev(win_bits(twv, ot - 32) & win_bits(qwv, oq - 32));
        } else if (busy) {
            if (!rdone) {
                const uint64_t tg = T.base + ht + L + rext, qg = Q.base + hq + L + rext;
                atc = load_codes32(T.codes, tg);
                aqc = load_codes32(Q.codes, qg);
                avv = load_bits32(T.valid, tg) & load_bits32(Q.valid, qg);
                an = min(32u, rrem);
            } else {
                // Left side continues below position ht - 1 - lext.
                const uint64_t tg = T.base + ht - lext - 32, qg = Q.base + hq - lext - 32;
                atc = rev_pairs64(load_codes32(T.codes, tg));
                aqc = rev_pairs64(load_codes32(Q.codes, qg));
                avv = __brev(load_bits32(T.valid, tg) & load_bits32(Q.valid, qg));
                an = min(32u, lrem);
            }
        }

        // ---------------- scans ----------------
        {
            if (!busy) an = 0;
            if (!fresh) bn = 0;
            SideScan A, B;
            side_init(A, atc, aqc, avv, an, a_right ? rext : lext, a_right ? rrun : lrun, a_right ? rbest : lbest,
                      a_right ? rbext : lbext);
            side_init(B, btc, bqc, bvv, bn, 0, lrun, lbest, lbext);
            scan_pair_any(A, B, an, bn, xdrop, s_lut, ambig);
            const bool aend = A.brk < an, bend = B.brk < bn;
            const uint32_t aused = aend ? A.brk + 1 : an, bused = bend ? B.brk + 1 : bn;
            n_cols += aused + bused;
            if (busy) {
                if (a_right) {
                    rrun = A.r; rbest = A.b; rbext = A.be; rext += aused; rrem -= aused;
                    rdone = rdone || aend || rrem == 0;
                } else {
                    lrun = A.r; lbest = A.b; lbext = A.be; lext += aused; lrem -= aused;
                    ldone = ldone || aend || lrem == 0;
                }
            }
            if (fresh) {
                lrun = B.r; lbest = B.b; lbext = B.be; lext += bused; lrem -= bused;
                ldone = ldone || bend || lrem == 0;
            }
        }

        // ---------------- bookkeeping ----------------
        bool finish = false, cand = false, is_long = false;
        int32_t score = 0;
        if (busy) {
            if (rdone && ldone) {
                finish = true;
                score = seed + rbest + lbest;
                cand = score >= thresh;
            } else if ((!rdone && rext >= a.cap) || (!ldone && lext >= a.cap)) {
                finish = true;      // still extending at the cap: defer to the walk
                cand = true;
                is_long = true;
            }
        }
        const uint32_t m = __ballot_sync(kFull, finish && cand);
        if (m) {
            uint32_t slot0 = 0;
            if (lane == 0) slot0 = atomicAdd(a.cand_count, (uint32_t)__popc(m));
            slot0 = __shfl_sync(kFull, slot0, 0);
            if (finish && cand) {
                const uint32_t slot = slot0 + __popc(m & lt);
                if (slot < a.cand_cap) {
                    const uint32_t tk = T.key_base + ht, qk = Q.key_base + hq;
                    a.cand_keys[slot] = ((uint64_t)(tk - qk + a.qkey_total) << 32) | tk;
                    a.cand_vals[slot] = slot;
                    Cand c;
                    c.unit = hu; c.t = ht; c.q = hq;
                    c.flags = is_long ? kCandLong : 0u;
                    c.lext = lbext; c.rext = rbext; c.score = score; c.pad_ = 0;
                    a.cands[slot] = c;
                }
            }
        }
        if (finish) busy = false;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) n_cols += __shfl_xor_sync(kFull, n_cols, o);
    if (lane == 0) atomicAdd(&a.stats[2], n_cols);
}

// ---------------------------------------------------------------------------
// Screen, packed form.  The same lane-per-hit screen as k_screen_wide, with
// the x-drop state of a side packed into two integers:
//     P = 256 * run  + (255 - columns scanned)
//     B = 256 * best + (255 - best extent)
// One column of extend_one_side (src/hsp.rs:179-193) is then
//     P += 256 * score - 1;  B = max(B, P);  break when B - P >= 256 (xdrop + 1)
// and this is exact:
//  - run > best: P exceeds B by at least 1, so B takes P -- best and its
//    extent move together, as in the reference.
//  - run <= best: P < B (a later column has a smaller low byte), so B keeps the
//    first extent that reached the best, as the reference's strict `>` does.
//  - then B - P = 256 (best - run) + d with 1 <= d <= 255, and
//    B - P >= 256 (xdrop + 1)  <=>  best - run > xdrop.
// It needs at most 255 columns per side in the screen (cap <= 192), xdrop in
// [0, 2^22] and |scores| <= 16383, so that no packed value leaves i32; the
// host uses k_screen_wide outside that envelope.
// ---------------------------------------------------------------------------
struct PkSide {
    uint64_t e, o;         // nibble j of e: column 2j, of o: column 2j+1; nibble = q << 2 | t
    uint32_t vv;           // column validity
    uint32_t n;            // columns present in this chunk
    int32_t p, b;          // packed run and best
};

// A side with no columns starts dead (b - p = T) so that no column moves it.
__device__ __forceinline__ void pk_init(PkSide& S, uint64_t tc, uint64_t qc, uint32_t vv, uint32_t n, int32_t p,
                                        int32_t b, int32_t T) {
    constexpr uint64_t m = 0x3333333333333333ull;
    S.e = (tc & m) | ((qc << 2) & ~m);
    S.o = ((tc >> 2) & m) | (qc & ~m);
    S.vv = vv;
    S.n = n;
    S.b = b;
    S.p = n ? p : b - T;
}

// Column k of a side, branch-free.  A side is alive while b - p < T; once the
// x-drop break fires its later columns add 0, so p and b (and b - p >= T)
// stay as the break left them.  kSlow: the chunk may hold invalid bases
// (scored `ambig`) or end before column 32 (absent columns add 0 and keep
// the side alive).  plut is indexed by (q << 2) | t.
template <bool kSlow, int k>
__device__ __forceinline__ void pk_step(PkSide& S, int32_t T, const int32_t* plut, int32_t pamb) {
    const uint32_t idx = (uint32_t)(((k & 1) ? S.o : S.e) >> (4 * (k >> 1))) & 15u;
    int32_t s = plut[idx];
    bool go = S.b - S.p < T;
    if (kSlow) {
        s = ((S.vv >> k) & 1u) ? s : pamb;
        go = go && (uint32_t)k < S.n;
    }
    s = go ? s : 0;
    S.p += s;
    S.b = max(S.b, S.p);
}

// Column k of a side that cannot break yet (no x-drop test).
template <int k>
__device__ __forceinline__ void pk_step_free(PkSide& S, const int32_t* plut) {
    const uint32_t idx = (uint32_t)(((k & 1) ? S.o : S.e) >> (4 * (k >> 1))) & 15u;
    S.p += plut[idx];
    S.b = max(S.b, S.p);
}

// The fast path with side B fresh: its first kFree columns cannot reach the
// x-drop (each column lowers p by at most 256 * |min score| + 1), so they skip
// the test.  A dead B (no columns) is updated too, but its result is unused.
template <int kFree>
__device__ __forceinline__ void pk_scan_pair_bfresh(PkSide& A, PkSide& B, int32_t T, const int32_t* plut,
                                                    int32_t pamb) {
#define GXY_PKF(k)                                                         \
    pk_step<false, k>(A, T, plut, pamb);                                   \
    if (k < kFree) pk_step_free<k>(B, plut); else pk_step<false, k>(B, T, plut, pamb);
    GXY_PKF(0) GXY_PKF(1) GXY_PKF(2) GXY_PKF(3) GXY_PKF(4) GXY_PKF(5) GXY_PKF(6) GXY_PKF(7)
    GXY_PKF(8) GXY_PKF(9) GXY_PKF(10) GXY_PKF(11) GXY_PKF(12) GXY_PKF(13) GXY_PKF(14) GXY_PKF(15)
    GXY_PKF(16) GXY_PKF(17) GXY_PKF(18) GXY_PKF(19) GXY_PKF(20) GXY_PKF(21) GXY_PKF(22) GXY_PKF(23)
    GXY_PKF(24) GXY_PKF(25) GXY_PKF(26) GXY_PKF(27) GXY_PKF(28) GXY_PKF(29) GXY_PKF(30) GXY_PKF(31)
#undef GXY_PKF
}

// Both sides column by column in lockstep: two independent serial chains.
template <bool kSlow>
__device__ __forceinline__ void pk_scan_pair(PkSide& A, PkSide& B, int32_t T, const int32_t* plut, int32_t pamb) {
#define GXY_PK4(g)                                                         \
    pk_step<kSlow, g * 4 + 0>(A, T, plut, pamb);                           \
    pk_step<kSlow, g * 4 + 0>(B, T, plut, pamb);                           \
    pk_step<kSlow, g * 4 + 1>(A, T, plut, pamb);                           \
    pk_step<kSlow, g * 4 + 1>(B, T, plut, pamb);                           \
    pk_step<kSlow, g * 4 + 2>(A, T, plut, pamb);                           \
    pk_step<kSlow, g * 4 + 2>(B, T, plut, pamb);                           \
    pk_step<kSlow, g * 4 + 3>(A, T, plut, pamb);                           \
    pk_step<kSlow, g * 4 + 3>(B, T, plut, pamb);
    GXY_PK4(0) GXY_PK4(1) GXY_PK4(2) GXY_PK4(3) GXY_PK4(4) GXY_PK4(5) GXY_PK4(6) GXY_PK4(7)
#undef GXY_PK4
}

__device__ __forceinline__ int32_t pk_run(int32_t p) { return p >> 8; }            // arithmetic shift
__device__ __forceinline__ uint32_t pk_ext(int32_t p) { return 255u - ((uint32_t)p & 255u); }
constexpr int32_t kPkStart = 255;   // run 0, no columns

// 64 bits from the 128-bit pair (hi:lo) starting at bit s (0 <= s < 64).
__device__ __forceinline__ uint64_t funnel64(uint64_t lo, uint64_t hi, uint32_t s) {
    return s ? ((lo >> s) | (hi << (64 - s))) : lo;
}

// Seed footprint score, all L columns at t / q (src/hsp.rs:119-123): three
// columns per table read, the rest singly, invalid columns re-scored ambig.
__device__ __forceinline__ int32_t seed_score(const SeqView& T, const SeqView& Q, uint32_t t, uint32_t q,
                                              uint32_t L, uint32_t seed_mask, const int32_t* s_tri,
                                              const int32_t* s_lut, int32_t ambig) {
    const uint64_t tc = load_codes32(T.codes, T.base + t), qc = load_codes32(Q.codes, Q.base + q);
    const uint32_t vv = load_bits32(T.valid, T.base + t) & load_bits32(Q.valid, Q.base + q);
    int32_t sd = 0;
#pragma unroll
    for (int k = 0; k + 3 <= 32; k += 3) {
        if ((uint32_t)k + 3 > L) break;
        sd += s_tri[((((uint32_t)(tc >> (2 * k))) & 63u) << 6) | ((uint32_t)(qc >> (2 * k)) & 63u)];
    }
    for (uint32_t k = L - L % 3; k < L; k++)
        sd += s_lut[((((uint32_t)(tc >> (2 * k))) & 3u) << 2) | ((uint32_t)(qc >> (2 * k)) & 3u)];
    uint32_t bad = ~vv & seed_mask;
    while (bad) {
        const uint32_t k = __ffs(bad) - 1;
        bad &= bad - 1;
        sd += ambig - s_lut[((((uint32_t)(tc >> (2 * k))) & 3u) << 2) | ((uint32_t)(qc >> (2 * k)) & 3u)];
    }
    return sd;
}

template <int WARPS, int MINB>
__global__ __launch_bounds__(WARPS * 32, MINB) void k_screen(const __grid_constant__ ScreenArgs a) {
    __shared__ int32_t s_lut[16];     // raw column scores, index (t << 2) | q
    __shared__ int32_t s_plut[16];    // 256 * score - 1, index (q << 2) | t
    __shared__ int32_t s_tri[4096];   // sum of three columns' scores, index (t3 << 6) | q3
    for (uint32_t i = threadIdx.x; i < 4096; i += blockDim.x) {
        int32_t v = 0;
#pragma unroll
        for (int c = 0; c < 3; c++) v += a.sc.sub[(((i >> (6 + 2 * c)) & 3u) << 2) | ((i >> (2 * c)) & 3u)];
        s_tri[i] = v;
    }
    if (threadIdx.x < 16) {
        s_lut[threadIdx.x] = a.sc.sub[threadIdx.x];
        s_plut[threadIdx.x] = a.sc.sub[((threadIdx.x & 3u) << 2) | (threadIdx.x >> 2)] * 256 - 1;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const uint32_t lt = lanemask_lt();
    const uint32_t L = a.pat.len;
    const int32_t ambig = a.sc.ambig, thresh = a.sc.hspthresh;
    const int32_t pamb = ambig * 256 - 1;
    const int32_t T = (a.sc.xdrop + 1) * 256;
    // Columns a fresh side scans before its first possible break.
    int32_t worst = a.sc.ambig;
    for (int i = 0; i < 16; i++) worst = min(worst, a.sc.sub[i]);
    const int32_t per_col = worst < 0 ? 256 * (-worst) + 1 : 1;
    const int free_cols = (int)min(8, (T - 1) / per_col);
    const uint32_t seed_mask = L >= 32 ? 0xffffffffu : ((1u << L) - 1u);
    // No seed footprint scores above this: a hit whose two sides' bests stay
    // below thresh - seed_ub can never pass, whatever its seed scores.
    int32_t top = ambig;
    for (int i = 0; i < 16; i++) top = max(top, a.sc.sub[i]);
    const int32_t seed_ub = top * (int32_t)L;
    // Past the buffer's end the pass did not write (those hits went to the
    // next pass, or were lost with a survivor overflow, which reruns the launch).
    const uint32_t n_hits = (uint32_t)min(*a.hit_count, (unsigned long long)a.hit_cap);
    // Each warp claims hits in chunks (one atomic per chunk) and deals them
    // to its idle lanes; chunks shrink for small launches so that every warp
    // still gets work.
    const uint32_t n_warps = gridDim.x * WARPS;
    const uint32_t chunk = max(32u, min(256u, n_hits / max(1u, n_warps * 8u)));
    uint32_t wcur = 0, wend = 0;   // this warp's claimed, not yet dealt hits
    uint32_t n_cols = 0;
    unsigned long long n_cols_all = 0;
    bool exhausted = false;

    bool busy = false, rdone = true, ldone = true;
    uint32_t ht = 0, hq = 0, hu = 0xffffffffu;
    int32_t rp = kPkStart, rb = kPkStart, lp = kPkStart, lb = kPkStart;
    uint32_t rrem = 0, lrem = 0;
    SeqView T_{}, Q_{};
    uint32_t cur_unit = 0xffffffffu;

    for (;;) {
        // ---------------- assign ----------------
        const uint32_t im = __ballot_sync(kFull, !busy);
        const uint32_t need = __popc(im);
        const uint32_t avail = wend - wcur;
        uint32_t nb = 0, ncount = 0;
        if (need > avail && !exhausted) {
            if (lane == 0) nb = atomicAdd(a.hit_next, chunk);
            nb = __shfl_sync(kFull, nb, 0);
            ncount = nb < n_hits ? min(chunk, n_hits - nb) : 0u;
            if (nb + chunk >= n_hits) exhausted = true;
        }
        bool fresh = false;
        if (!busy) {
            const uint32_t rk = __popc(im & lt);
            uint32_t hidx = 0xffffffffu;
            if (rk < avail) hidx = wcur + rk;
            else if (rk - avail < ncount) hidx = nb + (rk - avail);
            if (hidx != 0xffffffffu) {
                const Hit h = load_hit(a.hits + hidx);
                ht = h.t;
                hq = h.q;
                hu = h.unit;
                if (hu != kNoUnit && hu != cur_unit) {
                    cur_unit = hu;
                    const UnitDev U = a.units[hu];
                    T_ = a.tsegs[U.tseg];
                    Q_ = a.qsegs[U.qseg];
                }
                fresh = hu != kNoUnit;   // an unused slot of a failed reservation
                busy = fresh;
            }
        }
        {
            const uint32_t from_old = min(need, avail);
            if (ncount) {
                wcur = nb + min(need - from_old, ncount);
                wend = nb + ncount;
            } else {
                wcur += from_old;
            }
        }
        if (!__any_sync(kFull, busy)) {
            if (exhausted && wcur == wend) break;
            continue;
        }

        // ---------------- chunk data ----------------
        // Side A: the next chunk of the side this hit is on (a fresh hit's
        // first right chunk); side B: a fresh hit's first left chunk.  Right
        // chunks read forward from the column after the last one scanned,
        // left chunks the 32 positions below it, reversed.
        uint64_t atc = 0, aqc = 0, btc = 0, bqc = 0;
        uint32_t avv = 0, bvv = 0, an = 0, bn = 0;
        const bool a_right = fresh || !rdone;
        if (fresh) {
            rrem = min(T_.len - ht - L, Q_.len - hq - L);
            lrem = min(ht, hq);
            rp = rb = lp = lb = kPkStart;
            rdone = rrem == 0;
            ldone = lrem == 0;
        }
        if (busy) {
            const uint32_t ext = pk_ext(a_right ? rp : lp);
            const uint64_t ta = a_right ? T_.base + ht + L + ext : T_.base + ht - ext - 32;
            const uint64_t qa = a_right ? Q_.base + hq + L + ext : Q_.base + hq - ext - 32;
            atc = load_codes32(T_.codes, ta);
            aqc = load_codes32(Q_.codes, qa);
            avv = load_bits32(T_.valid, ta) & load_bits32(Q_.valid, qa);
            if (!a_right) {
                atc = rev_pairs64(atc);
                aqc = rev_pairs64(aqc);
                avv = __brev(avv);
            }
            an = min(32u, a_right ? rrem : lrem);
        }
        if (fresh) {
            const uint64_t tb = T_.base + ht - 32, qb = Q_.base + hq - 32;
            btc = rev_pairs64(load_codes32(T_.codes, tb));
            bqc = rev_pairs64(load_codes32(Q_.codes, qb));
            bvv = __brev(load_bits32(T_.valid, tb) & load_bits32(Q_.valid, qb));
            bn = min(32u, lrem);
        }

        // ---------------- scans ----------------
        {
            PkSide A, B;
            const int32_t a0 = a_right ? rp : lp;
            pk_init(A, atc, aqc, avv, an, a0, a_right ? rb : lb, T);
            pk_init(B, btc, bqc, bvv, bn, lp, lb, T);
            const bool slow = (an != 0 && (an < 32 || avv != 0xffffffffu)) ||
                              (bn != 0 && (bn < 32 || bvv != 0xffffffffu));
            if (__any_sync(kFull, slow)) pk_scan_pair<true>(A, B, T, s_plut, pamb);
            else if (free_cols >= 7) pk_scan_pair_bfresh<7>(A, B, T, s_plut, pamb);
            else pk_scan_pair<false>(A, B, T, s_plut, pamb);
            if (an) {
                const uint32_t used = ((uint32_t)a0 & 255u) - ((uint32_t)A.p & 255u);
                const bool end = A.b - A.p >= T;
                n_cols += used;
                if (a_right) {
                    rp = A.p; rb = A.b; rrem -= used;
                    rdone = end || rrem == 0;
                } else {
                    lp = A.p; lb = A.b; lrem -= used;
                    ldone = end || lrem == 0;
                }
            }
            if (bn) {
                const uint32_t used = ((uint32_t)lp & 255u) - ((uint32_t)B.p & 255u);
                const bool end = B.b - B.p >= T;
                n_cols += used;
                lp = B.p; lb = B.b; lrem -= used;
                ldone = end || lrem == 0;
            }
        }
        if (n_cols >= (1u << 30)) {
            n_cols_all += n_cols;
            n_cols = 0;
        }

        // ---------------- bookkeeping ----------------
        bool finish = false, cand = false, is_long = false;
        int32_t score = 0;
        if (busy) {
            if (rdone && ldone) {
                finish = true;
                score = pk_run(rb) + pk_run(lb);
                cand = score >= thresh - seed_ub;   // else the seed cannot lift it to thresh
            } else if ((!rdone && pk_ext(rp) >= a.cap) || (!ldone && pk_ext(lp) >= a.cap)) {
                finish = true;      // still extending at the cap: defer to the walk
                cand = true;
                is_long = true;
            }
        }
        if (__any_sync(kFull, finish && cand && !is_long)) {
            if (finish && cand && !is_long) {
                score += seed_score(T_, Q_, ht, hq, L, seed_mask, s_tri, s_lut, ambig);
                cand = score >= thresh;
            }
        }
        const uint32_t m = __ballot_sync(kFull, finish && cand);
        if (m) {
            uint32_t slot0 = 0;
            if (lane == 0) slot0 = atomicAdd(a.cand_count, (uint32_t)__popc(m));
            slot0 = __shfl_sync(kFull, slot0, 0);
            if (finish && cand) {
                const uint32_t slot = slot0 + __popc(m & lt);
                if (slot < a.cand_cap) {
                    const uint32_t tk = T_.key_base + ht, qk = Q_.key_base + hq;
                    a.cand_keys[slot] = ((uint64_t)(tk - qk + a.qkey_total) << 32) | tk;
                    a.cand_vals[slot] = slot;
                    Cand c;
                    c.unit = hu; c.t = ht; c.q = hq;
                    c.flags = is_long ? kCandLong : 0u;
                    c.lext = pk_ext(lb); c.rext = pk_ext(rb); c.score = is_long ? 0 : score; c.pad_ = 0;
                    a.cands[slot] = c;
                }
            }
        }
        if (finish) busy = false;
    }
    n_cols_all += n_cols;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) n_cols_all += __shfl_xor_sync(kFull, n_cols_all, o);
    if (lane == 0) atomicAdd(&a.stats[2], n_cols_all);
}

// The packed screen's envelope (see above).
static bool packed_ok(const ScreenArgs& a) {
    int64_t m = a.sc.ambig < 0 ? -(int64_t)a.sc.ambig : a.sc.ambig;
    for (int i = 0; i < 16; i++) m = std::max<int64_t>(m, a.sc.sub[i] < 0 ? -(int64_t)a.sc.sub[i] : a.sc.sub[i]);
    return a.cap <= 192 && m <= 16383 && a.sc.xdrop >= 0 && a.sc.xdrop <= (1 << 22);
}

void launch_screen(const ScreenArgs& a, int warps, int blocks, cudaStream_t st) {
    // blocks = SMs x blocks-per-SM; for 8-warp blocks the register budget
    // follows the requested blocks per SM (2: 128, 3: 85, 4: 64 registers).
    const int per_sm = blocks / 148 > 0 ? blocks / 148 : 1;
    count_launch();
    if (packed_ok(a)) {
        switch (warps) {
            case 4: k_screen<4, 4><<<blocks, 128, 0, st>>>(a); break;
            case 16: k_screen<16, 1><<<blocks, 512, 0, st>>>(a); break;
            default:
                if (per_sm >= 4) k_screen<8, 4><<<blocks, 256, 0, st>>>(a);
                else if (per_sm == 3) k_screen<8, 3><<<blocks, 256, 0, st>>>(a);
                else k_screen<8, 2><<<blocks, 256, 0, st>>>(a);
                break;
        }
        return;
    }
    switch (warps) {
        case 4: k_screen_wide<4, 4><<<blocks, 128, 0, st>>>(a); break;
        case 16: k_screen_wide<16, 1><<<blocks, 512, 0, st>>>(a); break;
        default:
            if (per_sm >= 4) k_screen_wide<8, 4><<<blocks, 256, 0, st>>>(a);
            else if (per_sm == 3) k_screen_wide<8, 3><<<blocks, 256, 0, st>>>(a);
            else k_screen_wide<8, 2><<<blocks, 256, 0, st>>>(a);
            break;
    }
}

// ---------------------------------------------------------------------------
// Walk: diagonal suppression over the sorted candidates.
//
// Along one diagonal the reference visits hits in ascending t (query windows
// ascend, and one window meets a diagonal once).  A hit is admitted iff
// t >= cover, cover being the t_end of the last HSP emitted on the diagonal
// (src/diag_hash.rs:34-53); only a passing HSP moves cover.  The walk replays
// exactly that over the candidates of one (unit, diagonal) segment, which
// are the only hits that can pass.  Deferred (long) candidates are extended
// in full here with the warp x-drop when they are admitted.
// ---------------------------------------------------------------------------
// Entropy gate (src/entropy.rs:27-67) over target [ts, te), one warp, f64.
__device__ bool entropy_gate_warp(const SeqView& T, uint32_t ts, uint32_t te, int32_t score, int32_t thr) {
    const int lane = threadIdx.x & 31;
    const uint32_t e = min(te, T.len);
    uint32_t cnt[4] = {0, 0, 0, 0};
    for (uint32_t p = ts + 32 * lane; p < e; p += 32 * 32) {
        const uint64_t c = load_codes32(T.codes, T.base + p);
        uint32_t v = load_bits32(T.valid, T.base + p);
        const uint32_t nn = min(32u, e - p);
        if (nn < 32) v &= (1u << nn) - 1;
        // Split codes into low/high bit planes and count each code.
        uint32_t lo = 0, hi = 0;
#pragma unroll
        for (int k = 0; k < 32; k++) {
            lo |= (uint32_t)((c >> (2 * k)) & 1u) << k;
            hi |= (uint32_t)((c >> (2 * k + 1)) & 1u) << k;
        }
        cnt[0] += __popc(v & ~hi & ~lo);
        cnt[1] += __popc(v & ~hi & lo);
        cnt[2] += __popc(v & hi & ~lo);
        cnt[3] += __popc(v & hi & lo);
    }
#pragma unroll
    for (int k = 0; k < 4; k++)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) cnt[k] += __shfl_xor_sync(kFull, cnt[k], o);
    const uint32_t total = cnt[0] + cnt[1] + cnt[2] + cnt[3];
    double h = 0.0;
    if (total) {
        const double tt = (double)total;
        for (int k = 0; k < 4; k++) {
            if (cnt[k] == 0) continue;
            const double p = (double)cnt[k] / tt;
            h -= p * log2(p);
        }
    }
    const double scaled = (double)score * (h / 2.0);
    return scaled >= (double)thr;
}

template <int WARPS>
__global__ __launch_bounds__(WARPS * 32) void k_walk(const __grid_constant__ WalkArgs a) {
    __shared__ int32_t s_lut[16];
    __shared__ WarpStage s_stage[WARPS];
    if (threadIdx.x < 16) s_lut[threadIdx.x] = a.sc.sub[threadIdx.x];
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t n = min(*a.n_dev, a.n_cap);
    const uint32_t L = a.seed_len;
    // Chunks of 32 sorted positions are claimed dynamically: a segment with
    // long candidates (full re-extension) can take far longer than the rest.
    for (;;) {
        uint32_t r = 0;
        if (lane == 0) r = atomicAdd(a.chunk_next, 1u);
        r = __shfl_sync(kFull, r, 0);
        if ((uint64_t)r * 32 >= n) break;
        const uint32_t i = r * 32 + lane;
        bool head = false;
        uint32_t key_hi = 0;
        if (i < n) {
            key_hi = (uint32_t)(a.keys[i] >> 32);
            head = (i == 0) || (key_hi != (uint32_t)(a.keys[i - 1] >> 32));
        }
        // A diagonal segment of one candidate needs no walk: nothing can
        // cover it, so it is kept when it passes.  Its own lane settles it
        // when its extension is already exact (not a long candidate, and no
        // entropy gate, which takes the whole warp).
        bool alone = false;
        if (head && !a.has_entropy) {
            const bool tail = (i + 1 >= n) || (key_hi != (uint32_t)(a.keys[i + 1] >> 32));
            if (tail) {
                const Cand c = a.cands[a.idx[i]];
                if (!(c.flags & kCandLong)) {
                    alone = true;
                    if (c.score >= a.sc.hspthresh) {
                        const UnitDev U = a.units[c.unit];
                        const uint32_t ts = c.t - c.lext, len = a.seed_len + c.lext + c.rext;
                        Hsp o;
                        o.t_start = ts; o.q_start = c.q - c.lext; o.length = len; o.score = c.score;
                        a.out_hsp[i] = o;
                        a.out_flag[i] = (U.primary_hi <= U.primary_lo || (ts >= U.primary_lo && ts < U.primary_hi))
                                            ? 1 : 0;
                    }
                }
            }
        }
        uint32_t hb = __ballot_sync(kFull, head && !alone);
        while (hb) {
            const uint32_t h = r * 32 + (uint32_t)(__ffs(hb) - 1);
            hb &= hb - 1;
            const uint32_t segkey = (uint32_t)(a.keys[h] >> 32);
            // A segment (one diagonal key) can hold the candidates of several
            // units that share a target segment, interleaved in t.  Each unit
            // is walked by its own pass with its own cover: first the unit of
            // the segment's first candidate (u0), then the other units in
            // ascending order -- those above u0, then those below it.  Each
            // pass finds the next unit as the smallest one above the current
            // one (and below `ceil`); a segment of one unit takes one pass.
            const uint32_t u0 = a.cands[a.idx[h]].unit;
            uint32_t cur_unit = u0, ceil = 0xffffffffu, below = 0xffffffffu;
            for (;;) {
            uint32_t j = h;
            uint32_t cover = 0;
            uint32_t next = 0xffffffffu;
            for (;;) {
                const uint32_t jj = j + lane;
                const bool inseg = jj < n && (uint32_t)(a.keys[jj] >> 32) == segkey;
                Cand c;
                c.unit = 0xffffffffu; c.t = 0;
                if (inseg) c = a.cands[a.idx[jj]];
                const bool elig = inseg && c.unit == cur_unit && c.t >= cover;
                const uint32_t be = __ballot_sync(kFull, !inseg);
                const uint32_t bc = __ballot_sync(kFull, elig);
                const uint32_t stop = be ? (uint32_t)(__ffs(be) - 1) : 32u;
                const uint32_t first = bc ? (uint32_t)(__ffs(bc) - 1) : 32u;
                // Other units among the positions this step passes over.
                if (a.n_units > 1) {
                    const uint32_t upto = min(first, stop);
                    const bool seen = (uint32_t)lane <= upto && inseg;
                    next = min(next, __reduce_min_sync(kFull, (seen && c.unit > cur_unit && c.unit < ceil)
                                                                  ? c.unit : 0xffffffffu));
                    below = min(below, __reduce_min_sync(kFull, (seen && c.unit < u0) ? c.unit : 0xffffffffu));
                }
                if (first < stop) {
                    const uint32_t unit = cur_unit;
                    const uint32_t t = __shfl_sync(kFull, c.t, first);
                    const uint32_t q = __shfl_sync(kFull, c.q, first);
                    const uint32_t flags = __shfl_sync(kFull, c.flags, first);
                    int32_t score = __shfl_sync(kFull, c.score, first);
                    uint32_t lext = __shfl_sync(kFull, c.lext, first);
                    uint32_t rext = __shfl_sync(kFull, c.rext, first);
                    const UnitDev U = a.units[unit];
                    const SeqView T = a.tsegs[U.tseg];
                    if (flags & kCandLong) {
                        const SeqView Q = a.qsegs[U.qseg];
                        const LaneExt r = extend_warp(T, Q, t, q, L, a.sc.xdrop, s_lut, a.sc.ambig, &s_stage[w]);
                        score = r.score;
                        lext = r.lext;
                        rext = r.rext;
                    }
                    bool pass = score >= a.sc.hspthresh;
                    const uint32_t ts = t - lext, len = L + lext + rext;
                    if (pass && a.has_entropy) pass = entropy_gate_warp(T, ts, ts + len, score, a.entropy_thr);
                    if (pass) {
                        cover = ts + len;   // mark_covered(t_end) (src/diag_hash.rs:43-53)
                        if (lane == 0) {
                            const bool keep = U.primary_hi <= U.primary_lo ||
                                              (ts >= U.primary_lo && ts < U.primary_hi);
                            const uint32_t pos = j + first;
                            Hsp o;
                            o.t_start = ts; o.q_start = q - lext; o.length = len; o.score = score;
                            a.out_hsp[pos] = o;
                            a.out_flag[pos] = keep ? 1 : 0;
                        }
                    }
                    j = j + first + 1;
                    continue;
                }
                if (stop < 32) break;
                j += 32;
            }
            if (next != 0xffffffffu) {
                cur_unit = next;                      // the next unit above
            } else if (ceil == 0xffffffffu && below != 0xffffffffu) {
                cur_unit = below;                     // then the units below u0, ascending
                ceil = u0;
            } else {
                break;
            }
            }
        }
    }
}

void launch_walk(const WalkArgs& a, int warps, int blocks, cudaStream_t st) {
    switch (warps) {
        case 4: count_launch(); k_walk<4><<<blocks, 128, 0, st>>>(a); break;
        default: count_launch(); k_walk<8><<<blocks, 256, 0, st>>>(a); break;
    }
}

__global__ void k_compact(const uint8_t* flag, const uint32_t* off, const Hsp* hsp, const uint32_t* idx,
                          const Cand* cands, const uint32_t* n_dev, uint32_t n_cap, Hsp* out, uint32_t* out_unit) {
    const uint32_t n = min(*n_dev, n_cap);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (!flag[i]) continue;
        const uint32_t o = off[i];
        out[o] = hsp[i];
        out_unit[o] = cands[idx[i]].unit;
    }
}

void launch_compact(const uint8_t* flag, const uint32_t* offsets, const Hsp* hsp, const uint32_t* idx,
                    const Cand* cands, const uint32_t* n_dev, uint32_t n_cap, Hsp* out, uint32_t* out_unit,
                    int blocks, cudaStream_t st) {
    count_launch();
    k_compact<<<blocks, 256, 0, st>>>(flag, offsets, hsp, idx, cands, n_dev, n_cap, out, out_unit);
}

__device__ __forceinline__ int64_t diag_of(const Hsp& h) { return (int64_t)h.t_start - (int64_t)h.q_start; }
__device__ __forceinline__ bool hsp_less(const Hsp& x, const Hsp& y) {
    if (x.t_start != y.t_start) return x.t_start < y.t_start;
    if (x.length != y.length) return x.length < y.length;
    return x.score < y.score;
}

// Each (unit, diagonal) run arrives in hit order; the canonical order within
// a run is (t_start, length, score).  Run heads are marked first (from the
// unmodified array), then one thread per run insertion-sorts it; runs are
// short and almost always already ordered.
__global__ void k_mark_runs(const Hsp* hsp, const uint32_t* unit, const uint32_t* n_dev, uint32_t n_cap,
                            uint8_t* head) {
    const uint32_t n = min(*n_dev, n_cap);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        head[i] = (i == 0 || unit[i - 1] != unit[i] || diag_of(hsp[i - 1]) != diag_of(hsp[i])) ? 1 : 0;
}

__global__ void k_fixup(Hsp* hsp, const uint8_t* head, const uint32_t* n_dev, uint32_t n_cap) {
    const uint32_t n = min(*n_dev, n_cap);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (!head[i]) continue;
        uint32_t e = i + 1;
        bool sorted = true;
        while (e < n && !head[e]) {
            if (hsp_less(hsp[e], hsp[e - 1])) sorted = false;
            e++;
        }
        if (sorted) continue;
        for (uint32_t x = i + 1; x < e; x++) {
            const Hsp key = hsp[x];
            uint32_t y = x;
            while (y > i && hsp_less(key, hsp[y - 1])) {
                hsp[y] = hsp[y - 1];
                y--;
            }
            hsp[y] = key;
        }
    }
}

void launch_fixup(Hsp* hsp, const uint32_t* unit, const uint32_t* n_dev, uint32_t n_cap, uint8_t* head_scratch,
                  int blocks, cudaStream_t st) {
    count_launch();
    k_mark_runs<<<blocks, 256, 0, st>>>(hsp, unit, n_dev, n_cap, head_scratch);
    count_launch();
    k_fixup<<<blocks, 256, 0, st>>>(hsp, head_scratch, n_dev, n_cap);
}

__global__ void k_gather_hsp(const Hsp* in, const uint32_t* in_unit, const uint32_t* perm, const uint32_t* n_dev,
                             uint32_t n_cap, Hsp* out, uint32_t* out_unit) {
    const uint32_t n = min(*n_dev, n_cap);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t p = perm[i];
        out[i] = in[p];
        out_unit[i] = in_unit[p];
    }
}

void launch_gather_hsp(const Hsp* in, const uint32_t* in_unit, const uint32_t* perm, const uint32_t* n_dev,
                       uint32_t n_cap, Hsp* out, uint32_t* out_unit, int blocks, cudaStream_t st) {
    count_launch();
    k_gather_hsp<<<blocks, 256, 0, st>>>(in, in_unit, perm, n_dev, n_cap, out, out_unit);
}

__global__ void k_iota(uint32_t* v, const uint32_t* n_dev, uint32_t n_cap) {
    const uint32_t n = min(*n_dev, n_cap);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[i] = i;
}

void launch_iota(uint32_t* v, const uint32_t* n_dev, uint32_t n_cap, int blocks, cudaStream_t st) {
    count_launch();
    k_iota<<<blocks, 256, 0, st>>>(v, n_dev, n_cap);
}

// ---------------------------------------------------------------------------
// Driver records: global coordinates, per-group order and dedup
// (build_ungapped_record src/driver.rs:437-468; sort and dedup_by :371-391).
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t shl64(uint64_t x, int s) { return s >= 64 ? 0ull : x << s; }

__global__ void k_record_keys(const Hsp* hsp, const uint32_t* unit, const Place* place, const uint32_t* perm,
                              const uint32_t* n_dev, uint32_t n_cap, int mode, int sh_g, int sh_t, int sh_q,
                              uint64_t* key, uint32_t* val) {
    const uint32_t n = min(*n_dev, n_cap);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t p = perm ? perm[i] : i;
        const Hsp h = hsp[p];
        const Place pl = place[unit[p]];
        const uint32_t t = h.t_start + pl.t_offset;
        uint64_t k;
        if (mode == 0)
            k = shl64(pl.group, sh_g) | shl64(t, sh_t) | shl64(h.q_start, sh_q) | h.length;
        else if (mode == 1)
            k = ((uint64_t)h.q_start << 32) | h.length;
        else
            k = ((uint64_t)pl.group << 32) | t;
        key[i] = k;
        val[i] = p;
    }
}

void launch_record_keys(const Hsp* hsp, const uint32_t* unit, const Place* place, const uint32_t* perm,
                        const uint32_t* n_dev, uint32_t n_cap, int mode, int sh_g, int sh_t, int sh_q, uint64_t* key,
                        uint32_t* val, int blocks, cudaStream_t st) {
    count_launch();
    k_record_keys<<<blocks, 256, 0, st>>>(hsp, unit, place, perm, n_dev, n_cap, mode, sh_g, sh_t, sh_q, key, val);
}

__device__ __forceinline__ Record make_record(const Hsp* hsp, const uint32_t* unit, const Place* place,
                                              uint32_t p) {
    const Hsp h = hsp[p];
    const uint32_t u = unit[p];
    const Place pl = place[u];
    Record r;
    r.group = pl.group;
    r.t_start = h.t_start + pl.t_offset;
    r.q_start = h.q_start;
    r.span = h.length;
    r.score = h.score;
    r.unit = u;
    return r;
}

__global__ void k_record_heads(const Hsp* hsp, const uint32_t* unit, const Place* place, const uint32_t* perm,
                               const uint32_t* n_dev, uint32_t n_cap, uint8_t* flag) {
    const uint32_t n = min(*n_dev, n_cap);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint8_t head = 1;
        if (i > 0) {
            const Record a = make_record(hsp, unit, place, perm[i - 1]);
            const Record b = make_record(hsp, unit, place, perm[i]);
            head = (a.group != b.group || a.t_start != b.t_start || a.q_start != b.q_start || a.span != b.span);
        }
        flag[i] = head;
    }
}

void launch_record_heads(const Hsp* hsp, const uint32_t* unit, const Place* place, const uint32_t* perm,
                         const uint32_t* n_dev, uint32_t n_cap, uint8_t* flag, int blocks, cudaStream_t st) {
    count_launch();
    k_record_heads<<<blocks, 256, 0, st>>>(hsp, unit, place, perm, n_dev, n_cap, flag);
}

__global__ void k_record_emit(const Hsp* hsp, const uint32_t* unit, const Place* place, const uint32_t* perm,
                              const uint8_t* flag, const uint32_t* offsets, const uint32_t* n_dev, uint32_t n_cap,
                              Record* out) {
    const uint32_t n = min(*n_dev, n_cap);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (flag[i]) out[offsets[i]] = make_record(hsp, unit, place, perm[i]);
}

void launch_record_emit(const Hsp* hsp, const uint32_t* unit, const Place* place, const uint32_t* perm,
                        const uint8_t* flag, const uint32_t* offsets, const uint32_t* n_dev, uint32_t n_cap,
                        Record* out, int blocks, cudaStream_t st) {
    count_launch();
    k_record_emit<<<blocks, 256, 0, st>>>(hsp, unit, place, perm, flag, offsets, n_dev, n_cap, out);
}

// ---------------------------------------------------------------------------
// x-drop of given hits (extend_hit, src/hsp.rs:66-148): mode 0 one lane per
// hit (uncapped), mode 1 one warp per hit.
// ---------------------------------------------------------------------------
__global__ void k_extend_lane(SeqView T, SeqView Q, Score sc, const uint32_t* tp, const uint32_t* qp, uint64_t n,
                              uint32_t L, Hsp* out, uint8_t* ok) {
    __shared__ int32_t s_lut[16];
    if (threadIdx.x < 16) s_lut[threadIdx.x] = sc.sub[threadIdx.x];
    __syncthreads();
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t t = tp[i], q = qp[i];
        if ((uint64_t)t + L > T.len || (uint64_t)q + L > Q.len) {   // src/hsp.rs:113-115
            ok[i] = 0;
            continue;
        }
        const LaneExt r = extend_lane(T, Q, t, q, L, 0xffffffffu, sc.xdrop, s_lut, sc.ambig);
        const bool pass = r.score >= sc.hspthresh;
        ok[i] = pass ? 1 : 0;
        Hsp o;
        o.t_start = t - r.lext; o.q_start = q - r.lext; o.length = L + r.lext + r.rext; o.score = r.score;
        out[i] = o;
    }
}

__global__ void k_extend_warp(SeqView T, SeqView Q, Score sc, const uint32_t* tp, const uint32_t* qp, uint64_t n,
                              uint32_t L, Hsp* out, uint8_t* ok) {
    __shared__ int32_t s_lut[16];
    __shared__ WarpStage s_stage[8];
    if (threadIdx.x < 16) s_lut[threadIdx.x] = sc.sub[threadIdx.x];
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (uint64_t i = blockIdx.x * 8ull + w; i < n; i += (uint64_t)gridDim.x * 8) {
        const uint32_t t = tp[i], q = qp[i];
        if ((uint64_t)t + L > T.len || (uint64_t)q + L > Q.len) {
            if (lane == 0) ok[i] = 0;
            continue;
        }
        const LaneExt r = extend_warp(T, Q, t, q, L, sc.xdrop, s_lut, sc.ambig, &s_stage[w]);
        if (lane == 0) {
            ok[i] = r.score >= sc.hspthresh ? 1 : 0;
            Hsp o;
            o.t_start = t - r.lext; o.q_start = q - r.lext; o.length = L + r.lext + r.rext; o.score = r.score;
            out[i] = o;
        }
    }
}

void launch_extend_hits(SeqView T, SeqView Q, Score sc, const uint32_t* tpos, const uint32_t* qpos, uint64_t n,
                        uint32_t seed_len, uint32_t mode, Hsp* out, uint8_t* ok, cudaStream_t st) {
    if (!n) return;
    if (mode == 1) {
        const int blocks = (int)umin64((n + 7) / 8, 148 * 8);
        count_launch();
        k_extend_warp<<<blocks, 256, 0, st>>>(T, Q, sc, tpos, qpos, n, seed_len, out, ok);
    } else {
        const int blocks = (int)umin64((n + 255) / 256, 148 * 8);
        count_launch();
        k_extend_lane<<<blocks, 256, 0, st>>>(T, Q, sc, tpos, qpos, n, seed_len, out, ok);
    }
}

}  // namespace gxy
