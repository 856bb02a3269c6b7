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
__device__ __forceinline__ uint64_t spread_bits_to_pairs(uint32_t x) {
    uint64_t v = x;
    v = (v | (v << 16)) & 0x0000FFFF0000FFFFull;
    v = (v | (v << 8)) & 0x00FF00FF00FF00FFull;
    v = (v | (v << 4)) & 0x0F0F0F0F0F0F0F0Full;
    v = (v | (v << 2)) & 0x3333333333333333ull;
    v = (v | (v << 1)) & 0x5555555555555555ull;
    return v * 3;   // each set bit -> a set 2-bit pair
}

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

// SeedExtractor::word_at (src/seeds.rs:208-222) at view-local position p
// (the caller guarantees p + L <= len): seedable iff every care position is
// valid and unmasked; the leftmost care position lands in the top bits.
__device__ __forceinline__ bool word_at(const SeqView& S, const Pattern& pat, uint32_t p, uint32_t& word) {
    const uint64_t gp = S.base + p;
    const uint32_t ok = load_bits32(S.valid, gp) & ~load_bits32(S.mask, gp);
    if ((ok & pat.care_mask) != pat.care_mask) return false;
    const uint64_t c = load_codes32(S.codes, gp);
    uint32_t w = 0;
#pragma unroll
    for (int i = 0; i < kMaxWeight; i++) {
        if ((uint32_t)i >= pat.weight) break;
        w = (w << 2) | ((uint32_t)(c >> (2 * pat.care[i])) & 3u);
    }
    word = w;
    return true;
}

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
// Screen: fused hit enumeration + capped lane-per-hit x-drop.
//
// Each warp runs a producer and 32 consumers over a shared-memory queue of
// hits (t, q, unit).
//  - Producer (warp-cooperative): takes tiles of 32 consecutive query windows
//    of one unit from a global work counter, forms each window's seed word
//    and its transition variants (src/seed_search.rs:303-316), and pushes the
//    hits of each variant's bucket (src/pos_table.rs:102-108) into the queue.
//  - Consumers (one lane per hit): every iteration an idle lane takes the
//    next queued hit, and every busy lane advances its own hit by one chunk of
//    up to 32 columns -- the seed footprint, then the right side, then the
//    left side of extend_hit (src/hsp.rs:98-195).  All phases run the same
//    chunk code, so lanes in different phases do not diverge.
// A hit is extended up to `cap` columns per side:
//  - ended below hspthresh: dropped.  Such a hit can never change the output:
//    search() only records diagonal cover for a hit whose HSP passes
//    (src/seed_search.rs:321-340), so whether it was admitted is irrelevant.
//  - ended at or above hspthresh, or still running at the cap: kept as a
//    candidate for the walk, which applies the diagonal rule in order.
// ---------------------------------------------------------------------------
constexpr int kRefillBelow = 96;  // the producer runs while fewer hits are queued

enum : uint32_t { kIdle = 0, kSeed = 1, kRight = 2, kLeft = 3 };

__device__ __forceinline__ uint64_t rev_pairs64(uint64_t c) {
    c = __brevll(c);
    return ((c >> 1) & 0x5555555555555555ull) | ((c & 0x5555555555555555ull) << 1);
}

template <int WARPS, int MINB>
__global__ __launch_bounds__(WARPS * 32, MINB) void k_screen(const __grid_constant__ ScreenArgs a) {
    constexpr int kQCap = WARPS >= 16 ? 128 : 256;   // queued hits per warp
    __shared__ int32_t s_lut[16];
    __shared__ uint32_t s_qt[WARPS][kQCap];
    __shared__ uint32_t s_qq[WARPS][kQCap];
    __shared__ uint32_t s_qu[WARPS][kQCap];
    __shared__ uint32_t s_ex[WARPS][32];
    __shared__ uint32_t s_b[WARPS][32];
    __shared__ uint32_t s_qw[WARPS][32];
    if (threadIdx.x < 16) s_lut[threadIdx.x] = a.sc.sub[threadIdx.x];
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t lt = lanemask_lt();
    const uint32_t L = a.pat.len;
    const int32_t ambig = a.sc.ambig, xdrop = a.sc.xdrop, thresh = a.sc.hspthresh;
    unsigned long long n_windows = 0, n_raw = 0, n_cols = 0;

    // ---- producer state (warp-uniform, except the per-lane window data) ----
    uint32_t head = 0, tail = 0;
    bool exhausted = false, have_tile = false;
    uint32_t pu = 0, v = 0, done_v = 0, total_v = 0, maxc = 0;
    const uint32_t* p_starts = nullptr;
    const uint32_t* p_pos = nullptr;
    uint32_t word = 0, qwin = 0, my_b = 0, my_cnt = 0, my_ex = 0;
    bool wv = false;

    // ---- consumer state (per lane) ----
    uint32_t phase = kIdle, ht = 0, hq = 0, hu = 0xffffffffu;
    uint32_t pos_t = 0, pos_q = 0, rem = 0, ext = 0, bext = 0, rext = 0;
    int32_t run = 0, best = 0, seed = 0, rbest = 0;
    SeqView T{}, Q{};
    uint32_t cur_unit = 0xffffffffu;

    auto load_variant = [&]() {
        my_b = 0;
        my_cnt = 0;
        if (wv) {
            const uint32_t vw = word ^ a.var_xor[v];
            my_b = __ldg(p_starts + vw);
            my_cnt = __ldg(p_starts + vw + 1) - my_b;
        }
        uint32_t incl = my_cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(kFull, incl, o);
            if (lane >= o) incl += y;
        }
        total_v = __shfl_sync(kFull, incl, 31);
        my_ex = incl - my_cnt;
        maxc = my_cnt;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) maxc = max(maxc, __shfl_xor_sync(kFull, maxc, o));
        done_v = 0;
        n_raw += lane == 0 ? total_v : 0;
    };

    for (;;) {
        // ---------------- produce ----------------
        while (!exhausted && tail - head < (uint32_t)kRefillBelow) {
            if (!have_tile) {
                uint32_t tile = 0;
                if (lane == 0) tile = atomicAdd(a.tile_counter, 1u);
                tile = __shfl_sync(kFull, tile, 0);
                if (tile >= a.n_tiles) {
                    exhausted = true;
                    break;
                }
                uint32_t lo = 0, hi = a.n_units;
                while (hi - lo > 1) {
                    const uint32_t mid = (lo + hi) >> 1;
                    if (a.units[mid].tile_base <= tile) lo = mid;
                    else hi = mid;
                }
                pu = lo;
                const UnitDev U = a.units[pu];
                p_starts = U.starts;
                p_pos = U.positions;
                const uint32_t k = (tile - U.tile_base) * 32 + lane;
                qwin = k * a.step;
                wv = false;
                if (k < U.nwin) wv = word_at(a.qsegs[U.qseg], a.pat, qwin, word);
                n_windows += wv ? 1 : 0;
                s_qw[w][lane] = qwin;
                v = 0;
                load_variant();
                have_tile = true;
            }
            while (done_v == total_v) {
                if (++v == a.n_var) {
                    have_tile = false;
                    break;
                }
                load_variant();
            }
            if (!have_tile) continue;
            const uint32_t room = (uint32_t)kQCap - (tail - head);
            const uint32_t np = min(room, total_v - done_v);
            if (done_v == 0 && np == total_v && maxc <= 8) {
                // Typical case: each lane copies its own short bucket.
                for (uint32_t j = 0; j < my_cnt; j++) {
                    const uint32_t slot = (tail + my_ex + j) % kQCap;
                    s_qt[w][slot] = __ldg(p_pos + my_b + j);
                    s_qq[w][slot] = qwin;
                    s_qu[w][slot] = pu;
                }
            } else {
                // Hot buckets: all lanes copy; owner = last lane with ex <= idx.
                s_ex[w][lane] = my_ex;
                s_b[w][lane] = my_b;
                __syncwarp();
                for (uint32_t j = lane; j < np; j += 32) {
                    const uint32_t idx = done_v + j;
                    uint32_t lo2 = 0, hi2 = 32;
                    while (hi2 - lo2 > 1) {
                        const uint32_t mid = (lo2 + hi2) >> 1;
                        if (s_ex[w][mid] <= idx) lo2 = mid;
                        else hi2 = mid;
                    }
                    const uint32_t slot = (tail + j) % kQCap;
                    s_qt[w][slot] = __ldg(p_pos + s_b[w][lo2] + (idx - s_ex[w][lo2]));
                    s_qq[w][slot] = s_qw[w][lo2];
                    s_qu[w][slot] = pu;
                }
            }
            __syncwarp();
            tail += np;
            done_v += np;
        }

        // ---------------- assign ----------------
        const bool idle = phase == kIdle;
        const uint32_t im = __ballot_sync(kFull, idle);
        const uint32_t avail = tail - head;
        const uint32_t take = min((uint32_t)__popc(im), avail);
        if (idle) {
            const uint32_t rk = __popc(im & lt);
            if (rk < take) {
                const uint32_t slot = (head + rk) % kQCap;
                ht = s_qt[w][slot];
                hq = s_qq[w][slot];
                hu = s_qu[w][slot];
                if (hu != cur_unit) {
                    cur_unit = hu;
                    const UnitDev U = a.units[hu];
                    T = a.tsegs[U.tseg];
                    Q = a.qsegs[U.qseg];
                }
                phase = kSeed;
            }
        }
        head += take;
        const bool busy = phase != kIdle;
        if (!__any_sync(kFull, busy)) {
            if (exhausted && tail == head) break;
            continue;
        }

        // ---------------- one chunk ----------------
        uint64_t tg = 0, qg = 0;
        uint32_t n = 0;
        int32_t xd = INT32_MAX;
        const bool fwd = phase != kLeft;
        if (phase == kSeed) {
            tg = T.base + ht;
            qg = Q.base + hq;
            n = L;
        } else if (phase == kRight) {
            tg = T.base + pos_t;
            qg = Q.base + pos_q;
            n = min(32u, rem);
            xd = xdrop;
        } else if (phase == kLeft) {
            tg = T.base + pos_t - 31;
            qg = Q.base + pos_q - 31;
            n = min(32u, rem);
            xd = xdrop;
        }
        uint64_t tc = 0, qc = 0;
        uint32_t vv = 0;
        if (busy) {
            tc = load_codes32(T.codes, tg);
            qc = load_codes32(Q.codes, qg);
            vv = load_bits32(T.valid, tg) & load_bits32(Q.valid, qg);
            if (!fwd) {
                tc = rev_pairs64(tc);
                qc = rev_pairs64(qc);
                vv = __brev(vv);
            }
        }
        int32_t r = phase == kSeed ? 0 : run;
        int32_t b = best;
        uint32_t be = bext;
        bool alive = busy;
        bool ended = false;
#pragma unroll
        for (int g = 0; g < 4; g++) {
            if (!__any_sync(kFull, alive && (uint32_t)(g * 8) < n)) break;
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const int k = g * 8 + i;
                if (alive && (uint32_t)k < n) {
                    r += col_score(tc, qc, vv, k, s_lut, ambig);
                    if (r > b) {
                        b = r;
                        be = ext + k + 1;
                    } else if (b - r > xd) {
                        alive = false;
                        ended = true;
                        n_cols += (unsigned long long)(k + 1);
                    }
                }
            }
        }

        // Columns examined this chunk (the break column included), for the
        // algorithmic byte count.
        if (busy) n_cols += phase == kSeed ? n : (ended ? 0 : n);
        // ---------------- bookkeeping ----------------
        bool finish = false, cand = false, is_long = false;
        int32_t score = 0;
        uint32_t lext_out = 0;
        if (busy) {
            if (phase == kSeed) {
                seed = r;
                phase = kRight;
                pos_t = ht + L;
                pos_q = hq + L;
                rem = min(T.len - ht - L, Q.len - hq - L);
                run = 0; best = 0; bext = 0; ext = 0;
            } else {
                run = r; best = b; bext = be;
                ext += n;
                rem -= n;
                const bool side_done = ended || rem == 0;
                if (!side_done && ext >= a.cap) {
                    finish = true;      // still extending at the cap: defer to the walk
                    cand = true;
                    is_long = true;
                } else if (!side_done) {
                    if (phase == kRight) { pos_t += n; pos_q += n; }
                    else { pos_t -= n; pos_q -= n; }
                } else if (phase == kRight) {
                    rbest = best;
                    rext = bext;
                    phase = kLeft;
                    pos_t = ht - 1;
                    pos_q = hq - 1;
                    rem = min(ht, hq);
                    run = 0; best = 0; bext = 0; ext = 0;
                } else {
                    finish = true;
                    score = seed + best + rbest;
                    lext_out = bext;
                    cand = score >= thresh;
                }
            }
            // An empty right side goes straight to the left; an empty left side finishes.
            if (!finish && phase == kRight && rem == 0) {
                rbest = 0; rext = 0;
                phase = kLeft;
                pos_t = ht - 1;
                pos_q = hq - 1;
                rem = min(ht, hq);
                run = 0; best = 0; bext = 0; ext = 0;
            }
            if (!finish && phase == kLeft && rem == 0) {
                finish = true;
                score = seed + rbest;
                lext_out = 0;
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
                    const uint32_t tk = T.key_base + ht, qk = Q.key_base + hq;
                    a.cand_keys[slot] = ((uint64_t)(tk - qk + a.qkey_total) << 32) | tk;
                    a.cand_vals[slot] = slot;
                    Cand c;
                    c.unit = hu; c.t = ht; c.q = hq;
                    c.flags = is_long ? kCandLong : 0u;
                    c.lext = lext_out; c.rext = rext; c.score = score; c.pad_ = 0;
                    a.cands[slot] = c;
                }
            }
        }
        if (finish) phase = kIdle;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        n_windows += __shfl_xor_sync(kFull, n_windows, o);
        n_cols += __shfl_xor_sync(kFull, n_cols, o);
    }
    if (lane == 0) {
        atomicAdd(&a.stats[0], n_windows);
        atomicAdd(&a.stats[1], n_raw);
        atomicAdd(&a.stats[2], n_cols);
    }
}

void launch_screen(const ScreenArgs& a, int warps, int blocks, cudaStream_t st) {
    switch (warps) {
        case 4: count_launch(); k_screen<4, 4><<<blocks, 128, 0, st>>>(a); break;
        case 16: count_launch(); k_screen<16, 1><<<blocks, 512, 0, st>>>(a); break;
        default: count_launch(); k_screen<8, 2><<<blocks, 256, 0, st>>>(a); break;
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
    const uint32_t gw = blockIdx.x * WARPS + w, nwarps = gridDim.x * WARPS;
    const uint32_t L = a.seed_len;
    for (uint32_t r = gw; (uint64_t)r * 32 < n; r += nwarps) {
        const uint32_t i = r * 32 + lane;
        bool head = false;
        if (i < n) head = (i == 0) || ((a.keys[i] >> 32) != (a.keys[i - 1] >> 32));
        uint32_t hb = __ballot_sync(kFull, head);
        while (hb) {
            const uint32_t h = r * 32 + (uint32_t)(__ffs(hb) - 1);
            hb &= hb - 1;
            const uint32_t segkey = (uint32_t)(a.keys[h] >> 32);
            uint32_t j = h;
            uint32_t cover = 0, cur_unit = 0xffffffffu;
            for (;;) {
                const uint32_t jj = j + lane;
                const bool inseg = jj < n && (uint32_t)(a.keys[jj] >> 32) == segkey;
                Cand c;
                c.unit = 0xffffffffu; c.t = 0;
                if (inseg) c = a.cands[a.idx[jj]];
                const bool elig = inseg && (c.unit != cur_unit || c.t >= cover);
                const uint32_t be = __ballot_sync(kFull, !inseg);
                const uint32_t bc = __ballot_sync(kFull, elig);
                const uint32_t stop = be ? (uint32_t)(__ffs(be) - 1) : 32u;
                const uint32_t first = bc ? (uint32_t)(__ffs(bc) - 1) : 32u;
                if (first < stop) {
                    const uint32_t unit = __shfl_sync(kFull, c.unit, first);
                    const uint32_t t = __shfl_sync(kFull, c.t, first);
                    const uint32_t q = __shfl_sync(kFull, c.q, first);
                    const uint32_t flags = __shfl_sync(kFull, c.flags, first);
                    int32_t score = __shfl_sync(kFull, c.score, first);
                    uint32_t lext = __shfl_sync(kFull, c.lext, first);
                    uint32_t rext = __shfl_sync(kFull, c.rext, first);
                    if (unit != cur_unit) {
                        cur_unit = unit;
                        cover = 0;
                    }
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
