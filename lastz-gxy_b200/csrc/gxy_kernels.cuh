// gxy_kernels.cuh -- launch interfaces of the seed->HSP kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "gxy_device.cuh"

namespace gxy {

// Seed pattern as the kernels read it (src/seeds.rs:20-100).
struct Pattern {
    uint32_t len;         // L <= 32
    uint32_t weight;      // care positions, <= kMaxWeight
    uint32_t care_mask;   // bit i set when offset i is a care position
    uint8_t care[16];     // care offsets, leftmost first
};

// SeedExtractor::word_at (src/seeds.rs:133-147) at view-local position p
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

// --- packing -----------------------------------------------------------------
// PackedSeq::from_ascii (src/sequences.rs:89-131): n ASCII bytes -> a device
// sequence laid out as gxy_device.cuh describes.
void launch_pack_ascii(const uint8_t* ascii, uint64_t n, uint64_t* codes, uint32_t* valid, uint32_t* mask,
                       cudaStream_t st);
// PackedSeq::reverse_complement (src/sequences.rs:303-318).
void launch_reverse_complement(const uint64_t* icodes, const uint32_t* ivalid, const uint32_t* imask,
                               uint64_t n, uint64_t* ocodes, uint32_t* ovalid, uint32_t* omask,
                               cudaStream_t st);

// --- table build (src/pos_table.rs:35-136) -----------------------------------
// Seed words of the windows k*step of a view; key = word, or num_words for a
// window that is not seedable; val = view-local position.  counts[word]++.
void launch_seed_words(SeqView view, Pattern pat, uint32_t step, uint32_t nwin, uint32_t num_words_sentinel,
                       uint32_t* keys, uint32_t* vals, uint32_t* counts, cudaStream_t st);
// prune_hot_words: counts2[w] = bucket size when <= limit, else 0.
void launch_prune_counts(const uint32_t* starts, uint64_t num_words, uint32_t limit, uint32_t* counts2,
                         cudaStream_t st);
// Moves the kept buckets into the compacted table (one thread per bucket;
// kept buckets hold at most `limit` positions).
void launch_prune_copy(const uint32_t* positions, const uint32_t* starts, uint64_t num_words,
                       const uint32_t* new_starts, uint32_t limit, uint32_t* new_positions, cudaStream_t st);

// --- search ------------------------------------------------------------------
// A raw seed hit: target position t, query window q, unit.  unit kNoUnit
// marks a slot of a hit-buffer reservation that failed (skipped by readers).
struct Hit {
    uint32_t t;
    uint32_t q;
    uint32_t unit;
};
constexpr uint32_t kNoUnit = 0xffffffffu;

// Layout of a worker's device counters (u32 indices).  The ones every warp
// hits with atomics sit 1-4 KB apart so that they fall in different L2
// slices.
//  - per launch: [kCTile] tile cursor, [kCPass] passes run, [kCCand]
//    candidates, [kCHsps] HSPs, [kCRecs] records, u64 [kCStats] statistics,
//    [kCRedoN + 0/1] redo-list lengths, u64 [kCMaxFail] largest tile that
//    did not fit the hit buffer, flags [kCSurvOver] and [kCRedoOver],
//    [kCWorkPasses] passes that found raw hits, [kCWalk] walk cursor;
//  - per pass (reset by k_pass_reset): u64 [kCHits] raw hits, u64 [kCSurv]
//    survivors, [kCHitNext] screen cursor, [kCFiltNext] filter cursor,
//    [kCRedoTake] redo-list cursor, [kCStop] the hit buffer is full.
constexpr uint32_t kCTile = 0, kCHsps = 2, kCRecs = 4, kCStats = 8, kCPass = 128, kCStop = 160, kCRedoN = 192,
                   kCMaxFail = 224, kCSurvOver = 256, kCRedoOver = 288, kCWorkPasses = 320, kCCand = 1024,
                   kCHitNext = 2048, kCRedoTake = 2560, kCHits = 3072, kCSurv = 3328, kCWalk = 3584,
                   kCFiltNext = 3840;
constexpr uint32_t kCounterWords = 4096;
// Tiles a pass can hand to the next one (two lists of this many).
constexpr uint32_t kRedoCap = 1u << 16;

struct ScreenArgs {
    const UnitDev* units;
    const SeqView* tsegs;
    const SeqView* qsegs;
    uint32_t n_units;
    uint32_t tile_lo;      // this pass enumerates tiles [tile_lo, tile_hi)
    uint32_t tile_hi;
    uint32_t* tile_counter;
    Pattern pat;
    uint32_t step;
    uint32_t n_var;
    uint32_t var_xor[kMaxVariants];
    Score sc;
    uint32_t cap;          // columns per side before a hit is deferred
    uint32_t qkey_total;   // size of the query key axis
    Hit* hits;             // raw hits of this pass
    uint64_t hit_cap;
    unsigned long long* hit_count;   // hits enumerated (may exceed hit_cap: then the pass is redone smaller)
    uint32_t* hit_next;    // x-drop work counter
    uint64_t* cand_keys;
    uint32_t* cand_vals;
    Cand* cands;
    uint32_t cand_cap;
    uint32_t* cand_count;
    unsigned long long* stats;   // [0] windows, [1] raw hits, [2] columns examined, [3] filter columns
    // The upper-bound filter (gxy_filter.cu, filter_bounds).
    int32_t fub[4];        // per class x = t_code ^ q_code: the largest score of that class
    uint64_t f_inv;        // class word given to the columns where either base is invalid
    uint64_t f_end;        // class word given to the columns past a side's end
    int32_t f_seed_max;    // seed length x the largest class bound
    uint32_t f_cap;        // columns per side after which a hit survives unexamined
    uint32_t f_claim;      // raw hits a filter warp claims at a time (0: sized from the hit count)
    // Passes that resume on the device: the worker's counters (layout
    // above) and the two redo lists of tiles that did not fit the hit buffer.
    uint32_t* ctl;
    uint32_t* redo;
};
// Seed-hit enumeration: one warp per tile of 32 query windows; writes the
// hits of every (window, variant) bucket to a.hits.  A pass takes the tiles
// the previous pass could not fit first, then fresh tiles from a.tile_counter
// until the hit buffer is full; a tile that does not fit goes to the next
// pass's list.
void launch_enumerate(const ScreenArgs& a, int sm_count, cudaStream_t st);
// Starts a pass: flags survivor overflow of the previous pass (its count above
// surv_cap), advances the pass counter and resets the per-pass counters.
void launch_pass_reset(uint32_t* ctl, uint64_t surv_cap, cudaStream_t st);
// Capped lane-per-hit x-drop over a.hits; keeps the candidates.  grid = persistent.
void launch_screen(const ScreenArgs& a, int warps_per_block, int blocks, cudaStream_t st);
// The upper-bound x-drop filter between enumeration and the exact screen
// (gxy_filter.cu).  filter_bounds fills a's fub/f_inv/f_end/f_seed_max from
// a.sc and a.pat and returns false when the scoring admits no such bound
// (then the exact screen takes every raw hit).
bool filter_bounds(ScreenArgs& a);
// The bounded x-drop over a raw-hit array: reads
// io.raw[0, *io.raw_count) (nothing when that count exceeds io.raw_cap) and
// writes the survivors to a.hits / a.hit_count / a.hit_cap.
struct FilterIO {
    const Hit* raw;
    const unsigned long long* raw_count;
    uint64_t raw_cap;
    uint32_t* cursor;      // zeroed by the caller
};
void launch_filter_hits(const ScreenArgs& a, const FilterIO& io, int sm_count, cudaStream_t st);
// Per-device kernel attributes of the filter (its shared-memory table); call
// once with the device current, before any stream capture.
void filter_init();
// Bucket occupancy bitmap of a table: bit (w & 31) of occ[w >> 5] is set iff
// bucket w holds a position.
void launch_occupancy(const uint32_t* starts, uint64_t num_words, uint32_t* occ, cudaStream_t st);

struct WalkArgs {
    const uint64_t* keys;      // candidate keys in sorted order
    const uint32_t* idx;       // candidate index per sorted position
    const Cand* cands;
    const uint32_t* n_dev;     // candidate count (clamped to n_cap)
    uint32_t n_cap;
    const UnitDev* units;
    const SeqView* tsegs;
    const SeqView* qsegs;
    uint32_t seed_len;
    Score sc;
    uint32_t has_entropy;
    int32_t entropy_thr;
    uint8_t* out_flag;         // per sorted position: 1 = emitted and kept
    Hsp* out_hsp;              // per sorted position
    uint32_t* chunk_next;      // work counter: chunks of 32 sorted positions (zeroed by the caller)
    uint32_t n_units;          // units of the launch (one unit: every segment is walked in one pass)
};
// Diagonal suppression (src/diag_hash.rs:34-53 as used at
// src/seed_search.rs:92-116) over the candidates sorted by (diagonal, t),
// one warp per diagonal segment.
void launch_walk(const WalkArgs& a, int warps_per_block, int blocks, cudaStream_t st);

// Gathers the kept HSPs: out[offsets[i]] = hsp[i], out_unit likewise.
void launch_compact(const uint8_t* flag, const uint32_t* offsets, const Hsp* hsp, const uint32_t* idx,
                    const Cand* cands, const uint32_t* n_dev, uint32_t n_cap, Hsp* out, uint32_t* out_unit,
                    int blocks, cudaStream_t st);
// Orders each (unit, diagonal) run by (t_start, length, score).
void launch_fixup(Hsp* hsp, const uint32_t* unit, const uint32_t* n_dev, uint32_t n_cap, uint8_t* head_scratch,
                  int blocks, cudaStream_t st);
// Gathers records by a permutation.
void launch_gather_hsp(const Hsp* in, const uint32_t* in_unit, const uint32_t* perm, const uint32_t* n_dev,
                       uint32_t n_cap, Hsp* out, uint32_t* out_unit, int blocks, cudaStream_t st);
void launch_iota(uint32_t* v, const uint32_t* n_dev, uint32_t n_cap, int blocks, cudaStream_t st);

// --- driver records (src/driver.rs:371-391, :437-468) --------------------------
// Where a unit's HSPs go: the output group (the driver's (target, query,
// strand) rank) and the chunk's global start added to t_start.
struct Place {
    uint32_t group;
    uint32_t t_offset;
};
// One ungapped record: t_span = q_span = span.  unit = the unit it came from.
struct Record {
    uint32_t group;
    uint32_t t_start;
    uint32_t q_start;
    uint32_t span;
    int32_t score;
    uint32_t unit;
};
// Sort keys of the records.  mode 0: (group, t, q, span) packed into one u64
// with the given shifts (span at bit 0); mode 1: (q << 32) | span; mode 2:
// (group << 32) | t.  t = t_start + the unit's t_offset.  HSP i is
// hsp[perm[i]] (perm may be null: the identity); val[i] = that index.
void launch_record_keys(const Hsp* hsp, const uint32_t* unit, const Place* place, const uint32_t* perm,
                        const uint32_t* n_dev, uint32_t n_cap, int mode, int sh_g, int sh_t, int sh_q, uint64_t* key,
                        uint32_t* val, int blocks, cudaStream_t st);
// flag[i] = 1 when record perm[i] differs from record perm[i-1] in (group,
// t, q, span) (dedup_by, src/driver.rs:381-387, keeps the first).
void launch_record_heads(const Hsp* hsp, const uint32_t* unit, const Place* place, const uint32_t* perm,
                         const uint32_t* n_dev, uint32_t n_cap, uint8_t* flag, int blocks, cudaStream_t st);
// out[offsets[i]] = the record of perm[i] for every flagged i.
void launch_record_emit(const Hsp* hsp, const uint32_t* unit, const Place* place, const uint32_t* perm,
                        const uint8_t* flag, const uint32_t* offsets, const uint32_t* n_dev, uint32_t n_cap,
                        Record* out, int blocks, cudaStream_t st);

// --- x-drop of given hits (test entry) ---------------------------------------
void launch_extend_hits(SeqView T, SeqView Q, Score sc, const uint32_t* tpos, const uint32_t* qpos, uint64_t n,
                        uint32_t seed_len, uint32_t mode, Hsp* out, uint8_t* ok, cudaStream_t st);

}  // namespace gxy
