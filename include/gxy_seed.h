/*
 * gxy_seed.h -- C ABI of the B200 seed->HSP stage for lastz-gxy.
 *
 * The stage replaces, bit for bit, what the reference computes in
 *   PosTable::build            src/pos_table.rs:35-83
 *   PosTable::prune_hot_words  src/pos_table.rs:113-136
 *   seed_search::search        src/seed_search.rs:45-125
 *     (DiagHash src/diag_hash.rs:34-53, extend_hit src/hsp.rs:66-211,
 *      extend_hit_avx2 src/hsp_simd.rs:27-243, entropy gate src/entropy.rs:27-67)
 * and is called where the reference's driver calls them (src/driver.rs:212-240,
 * src/tweener.rs:111-126).  Paths are relative to the nekrut/lastz-gxy root.
 *
 * Conventions: every entry point returns a gxy_status; on failure
 * gxy_last_error() returns a message for the calling thread.  No torch or CUDA
 * types appear in the signatures.  Sequences cross the boundary in the
 * reference's PackedSeq layout (src/sequences.rs:53-66):
 *   codes: 2-bit A=0 C=1 G=2 T=3, 4 per byte, position i at bits 2*(i&3) of byte i>>2
 *   valid: bit i&7 of byte i>>3 set when position i is unambiguous ACGT
 *   mask : bit i&7 of byte i>>3 set when position i was soft-masked (lowercase)
 * Coordinates in returned HSPs are those of the sequences passed in (chunk-local
 * target, strand-local query), exactly like the reference's Vec<Hsp>.
 */
#ifndef GXY_SEED_H
#define GXY_SEED_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

typedef enum {
    GXY_OK = 0,
    GXY_EINVAL = 1,         /* bad argument (reference: a panic or a parse error) */
    GXY_ENOMEM = 2,         /* device or host allocation failed */
    GXY_EUNSUPPORTED = 3,   /* outside the exact envelope (seed weight > 15, i32 overflow risk) */
    GXY_ETIMEDOUT = 4,      /* a bounded device or host wait ran out */
    GXY_ECUDA = 5,          /* CUDA runtime error */
    GXY_ENOTREADY = 6,      /* serving: request not finished yet */
    GXY_EOVERFLOW = 7,      /* a caller-provided buffer is too small; *needed is set */
    GXY_ECANCELED = 8       /* serving: the request was cancelled before its results were kept */
} gxy_status;

typedef struct gxy_ctx gxy_ctx;       /* one device, its streams and memory pool */
typedef struct gxy_table gxy_table;   /* device-resident PosTable */
typedef struct gxy_dseq gxy_dseq;     /* device-resident PackedSeq */
typedef struct gxy_server gxy_server; /* serving loop */

/* Host view of a PackedSeq (src/sequences.rs:61-66). */
typedef struct {
    const uint8_t* codes;
    const uint8_t* valid;
    const uint8_t* mask;
    uint64_t len;
} gxy_packed_seq;

/* SearchParams{step, hsp: HspParams{x_drop, hsp_threshold}, transitions,
 * entropy_threshold} (src/seed_search.rs:19-30, src/hsp.rs:46-49) plus the
 * ScoringMatrix fields the path reads (src/scoring.rs:32-40):
 * sub[r*4+q] = score of target code r against query code q; ambig = score of
 * a column where either base is not ACGT. */
typedef struct {
    int32_t sub[16];
    int32_t ambig;
    int32_t xdrop;
    int32_t hspthresh;
    uint32_t step;
    uint8_t transitions;   /* 0, 1, >=2 (treated as 2), src/seed_search.rs:69-90 */
    uint8_t has_entropy;   /* entropy_threshold.is_some() */
    uint8_t pad_[2];
    int32_t entropy_thr;
} gxy_search_params;

/* Hsp (src/hsp.rs:19-24), #[repr(C)]-compatible, 16 bytes. */
typedef struct {
    uint32_t t_start;
    uint32_t q_start;
    uint32_t length;
    int32_t score;
} gxy_hsp;

/* Output of a search.  If hsps == NULL on entry the library allocates it
 * (free with gxy_hsp_buf_free).  Otherwise it is a caller buffer of cap
 * entries; when too small the call returns GXY_EOVERFLOW and len holds the
 * number needed.  HSPs come back in canonical order: by diagonal
 * (t_start - q_start), then t_start, length, score -- the reference sorts by
 * (diagonal, t_start) and dedups (src/seed_search.rs:122-123). */
typedef struct {
    gxy_hsp* hsps;
    uint64_t len;
    uint64_t cap;
} gxy_hsp_buf;

/* Counters of one search or batch. */
typedef struct {
    uint64_t windows;      /* seedable query windows */
    uint64_t raw_hits;     /* table entries visited over all variants */
    uint64_t candidates;   /* hits that pass or run past the screen's column cap */
    uint64_t hsps;         /* HSPs returned */
    double device_ms;      /* CUDA-event time of the call's device work */
    double screen_ms;      /* CUDA-event time of the exact x-drop screen kernel (with enumeration and
                              the filter when passes > 1) */
    uint64_t columns;      /* alignment columns the screen scanned on the two sides */
    double enum_ms;        /* CUDA-event time of the hit enumeration kernel (single pass) */
    uint32_t passes;       /* window-range passes the raw hits needed */
    uint32_t reruns;       /* pipeline runs repeated after a buffer had to grow */
    uint64_t survivors;    /* raw hits the upper-bound filter passed on to the exact screen
                              (equal to raw_hits when the filter does not apply) */
    uint64_t filter_columns; /* alignment columns the upper-bound filter scanned on the two sides */
    double filter_ms;      /* CUDA-event time of the upper-bound filter kernel (single pass) */
    uint32_t rounds;       /* host rounds of passes (each ends with the epilogue and one counter copy) */
    uint32_t graph_updates; /* rounds launched by updating the worker's kept CUDA graph in place */
} gxy_stats;

const char* gxy_status_string(gxy_status s);
const char* gxy_last_error(void);
uint32_t gxy_abi_version(void);
/* Number of CUDA kernels this library has launched in this process. */
uint64_t gxy_kernel_launches(void);

/* ---- context ------------------------------------------------------------ */
gxy_status gxy_ctx_create(int device, gxy_ctx** out);
gxy_status gxy_ctx_destroy(gxy_ctx* ctx);
/* Tunables (screen kernel warps per block, column cap per side, screen blocks
 * per SM, walk warps per block, raw hits per pass, the upper-bound filter's
 * column cap and round size).  Zero leaves a field unchanged. */
typedef struct {
    uint32_t screen_warps;
    uint32_t screen_cap;
    uint32_t screen_blocks_per_sm;
    uint32_t walk_warps;
    uint32_t max_hits_per_pass;   /* raw-hit buffer bound; larger searches run in window passes */
    uint32_t initial_candidates;  /* candidate capacity every search starts from (grown on demand);
                                     0 in the context = keep what each stream's buffers grew to */
    uint32_t filter_cap;          /* upper-bound filter: columns per side after which a hit is
                                     passed on unexamined (a multiple of 32, 32..256) */
    uint32_t filter_claim;        /* upper-bound filter: raw hits a warp claims at a time (32..4096;
                                     1 = sized from each launch's hit count, the default) */
    uint32_t gapped_pool_blocks;  /* gapped extension: traceback blocks the first pass may use at most
                                     (0 = no limit: sized by the library); sides that do not fit run
                                     again in an exactly sized second pass */
    uint32_t gapped_cells;        /* gapped extension: cells of a DP row per thread, 4 (the default) or 8 */
} gxy_tuning;
gxy_status gxy_ctx_set_tuning(gxy_ctx* ctx, const gxy_tuning* t);
gxy_status gxy_ctx_get_tuning(gxy_ctx* ctx, gxy_tuning* t);
/* Device timing on the context's primary stream -- the stream every call
 * made from one host thread at a time runs on.  gxy_ctx_mark records CUDA
 * event `slot` (0..15) there; gxy_ctx_elapsed_ms waits for event b and
 * returns the milliseconds between events a and b. */
gxy_status gxy_ctx_mark(gxy_ctx* ctx, uint32_t slot);
gxy_status gxy_ctx_elapsed_ms(gxy_ctx* ctx, uint32_t a, uint32_t b, double* ms);

/* ---- device-resident sequences ------------------------------------------- */
/* Copies a host PackedSeq to the device. */
gxy_status gxy_dseq_upload(gxy_ctx* ctx, const gxy_packed_seq* host, gxy_dseq** out);
/* Packs ASCII bases on the device: PackedSeq::from_ascii / push_ascii with
 * encode_base (src/sequences.rs:89-131, src/dna.rs:12-20). */
gxy_status gxy_dseq_from_ascii(gxy_ctx* ctx, const uint8_t* ascii, uint64_t n, gxy_dseq** out);
/* PackedSeq::reverse_complement on the device (src/sequences.rs:303-318). */
gxy_status gxy_dseq_reverse_complement(gxy_ctx* ctx, const gxy_dseq* in, gxy_dseq** out);
/* Copies a device sequence back into host buffers of ceil(len/4), ceil(len/8),
 * ceil(len/8) bytes; any pointer may be NULL. */
gxy_status gxy_dseq_download(const gxy_dseq* s, uint8_t* codes, uint8_t* valid, uint8_t* mask);
uint64_t gxy_dseq_len(const gxy_dseq* s);
/* Frees a device sequence; valid before or after its context is destroyed. */
gxy_status gxy_dseq_free(gxy_dseq* s);

/* ---- input formats (src/sequences.rs:338-377, src/bit2.rs:73-163) -------- */
/* Sequences parsed from a file's bytes straight into device sequences. */
typedef struct {
    uint64_t n;          /* sequences */
    gxy_dseq** seqs;     /* device sequences; a caller that keeps one sets its slot to NULL */
    char** names;        /* NUL-terminated names */
} gxy_seq_set;
/* parse_fasta (src/sequences.rs:338-377): records start at lines whose first
 * byte is '>' (name = first whitespace-delimited token; an empty one is
 * GXY_EINVAL), ASCII whitespace is skipped, bases before the first header
 * join the first record, and each record is packed like
 * PackedSeq::from_ascii.  Input below 4 GiB. */
gxy_status gxy_parse_fasta(gxy_ctx* ctx, const uint8_t* bytes, uint64_t n, gxy_seq_set* out);
/* parse_2bit (src/bit2.rs:73-163): UCSC 2bit, either byte order; N blocks
 * become invalid bases (code 0), mask blocks soft-mask the valid ones.  Bad
 * magic, version or a truncated file are GXY_EINVAL with the reason in
 * gxy_last_error. */
gxy_status gxy_parse_2bit(gxy_ctx* ctx, const uint8_t* bytes, uint64_t n, gxy_seq_set* out);
/* Frees the names and every non-NULL device sequence of the set. */
void gxy_seq_set_free(gxy_seq_set* set);

/* ---- position table (src/pos_table.rs) --------------------------------- */
/* PosTable::build(seq, pattern, step) followed, when max_word_count > 0, by
 * prune_hot_words(max_word_count) as the driver does (src/driver.rs:212-215).
 * pattern01 is the 0/1 seed pattern (src/seeds.rs:38-51), at most 32
 * positions; weight <= 15 (2^30 buckets) is supported. */
gxy_status gxy_table_build(gxy_ctx* ctx, const gxy_packed_seq* target, const char* pattern01,
                           uint32_t step, uint32_t max_word_count, gxy_table** out);
/* Same over a device sequence, restricted to the view [lo, hi) -- the
 * driver's per-chunk table over chunk.seq (src/driver.rs:178, :212); the
 * table's positions are view-local like the reference's chunk copy. */
gxy_status gxy_table_build_view(gxy_ctx* ctx, const gxy_dseq* target, uint64_t lo, uint64_t hi,
                                const char* pattern01, uint32_t step, uint32_t max_word_count,
                                gxy_table** out);
/* gxy_table_build_view for n views [lo[i], hi[i]) of one device sequence at
 * once -- every chunk table of the driver (src/driver.rs:156-215) -- by one
 * sort over all the views' windows.  out[i] (n entries) receives view i's
 * table, equal to gxy_table_build_view of that view.  The tables share their
 * device arrays, which go when the last of them is freed; each is freed with
 * gxy_table_free as usual. */
gxy_status gxy_table_build_views(gxy_ctx* ctx, const gxy_dseq* target, uint32_t n, const uint64_t* lo,
                                 const uint64_t* hi, const char* pattern01, uint32_t step,
                                 uint32_t max_word_count, gxy_table** out);
/* PosTable::prune_hot_words(limit) (src/pos_table.rs:113-136) on a built
 * table: drops every bucket with more than limit positions. */
gxy_status gxy_table_prune_hot_words(gxy_table* t, uint32_t limit);
/* PosTable::build(seq, pattern, step) for callers that cannot allocate
 * device memory -- their memory belongs to another allocator (a framework's
 * caching allocator or a fixed serving arena) or they cannot afford the
 * device synchronisation an allocation implies.  This entry point has no
 * counterpart in the reference; it exists only for those callers.
 * It allocates nothing: the caller passes device buffers starts_out
 * (starts_cap >= 4^weight + 1 entries) and positions_out (positions_cap >=
 * the target's window count), and the staged target and every intermediate
 * live in one fixed device array of about 17 MiB inside this library, held
 * by each GPU that loads it until the process exits.  Limits: target length
 * at most 1,048,576 bp (longer targets are rejected with GXY_EINVAL); no hot
 * word pruning.  Runs on the calling thread's current device and the legacy
 * default stream and returns when the table is complete; *n_positions
 * receives starts[num_words].  The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress); make that first call before
 * any stream capture.  All calls share the array: builds from one process
 * are serialised per device, and calls from elsewhere that overlap on the
 * GPU would race on it. */
gxy_status gxy_table_build_static(const gxy_packed_seq* target, const char* pattern01, uint32_t step,
                                  uint32_t* starts_out, uint64_t starts_cap, uint32_t* positions_out,
                                  uint64_t positions_cap, uint64_t* n_positions);
gxy_status gxy_table_info(const gxy_table* t, uint64_t* num_words, uint64_t* n_positions,
                          uint32_t* pattern_len, uint32_t* weight);
/* Copies starts (num_words + 1 entries) and positions to host buffers; either
 * may be NULL. */
gxy_status gxy_table_download(const gxy_table* t, uint32_t* starts, uint32_t* positions);
/* Frees a table; valid before or after its context is destroyed, and for
 * the tables of one gxy_table_build_views call in any order. */
gxy_status gxy_table_free(gxy_table* t);

/* ---- the drop-in search (src/seed_search.rs:45-125) --------------------- */
/* seed_search::search(&table, &target, &query, &matrix, &params).  The
 * target must be the sequence the table was built from (the reference's
 * driver and tweener always pass the same one); it is re-read from host only
 * when its pointers or length differ from the build's.  Thread-safe: calls
 * from several host threads on one table run on separate streams. */
gxy_status gxy_search(gxy_ctx* ctx, const gxy_table* table, const gxy_packed_seq* target,
                      const gxy_packed_seq* query, const gxy_search_params* params,
                      gxy_hsp_buf* out, gxy_stats* stats);
/* Same with device-resident sequences (the table's own target is used). */
gxy_status gxy_search_dseq(gxy_ctx* ctx, const gxy_table* table, const gxy_dseq* query,
                           const gxy_search_params* params, gxy_hsp_buf* out, gxy_stats* stats);
void gxy_hsp_buf_free(gxy_hsp_buf* buf);

/* ---- batched: many (table, query, strand) units in one launch ------------ */
/* One unit is one reference search() call: the driver's
 * (chunk, query, strand) triple (src/driver.rs:210-240).  strand 1 searches
 * the reverse complement of the query, computed once per query on the device
 * (the reference recomputes it per chunk, src/driver.rs:221).  When
 * primary_hi > primary_lo the unit keeps only HSPs whose t_start lies in
 * [primary_lo, primary_hi), the driver's chunk filter (src/driver.rs:250-256). */
typedef struct {
    uint32_t table;
    uint32_t query;
    uint32_t strand;
    uint32_t primary_lo;
    uint32_t primary_hi;
} gxy_unit;

typedef struct {
    gxy_hsp* hsps;          /* all units' HSPs, unit-major, canonical within a unit */
    uint64_t* unit_offsets; /* n_units + 1 */
    uint64_t n_hsps;
    uint32_t n_units;
} gxy_batch_result;

typedef struct {
    uint32_t use_graph;     /* capture the batch's device work in a CUDA graph */
    uint32_t reserved_[7];
} gxy_batch_opts;

gxy_status gxy_batch_search(gxy_ctx* ctx, uint32_t n_tables, const gxy_table* const* tables,
                            uint32_t n_queries, const gxy_dseq* const* queries,
                            uint32_t n_units, const gxy_unit* units,
                            const gxy_search_params* params, const gxy_batch_opts* opts,
                            gxy_batch_result* out, gxy_stats* stats);
void gxy_batch_result_free(gxy_batch_result* r);

/* ---- driver records: the batch's HSPs as the driver's ungapped records ---- */
/* gxy_batch_search plus the driver's post-processing on the device
 * (build_ungapped_record src/driver.rs:437-468; grouping, sort and dedup
 * :370-391): every HSP of unit i becomes a record of group places[i].group
 * with t_start + places[i].t_offset (the chunk's global start); records are
 * ordered by (group, t_start, q_start, span) and repeats of those four fields
 * are dropped, keeping the first (lowest unit).  Groups stand for the
 * driver's (target, query, strand) triples in its output order; one group
 * may collect the units of every chunk of its target (their primary regions
 * are disjoint, so the order across chunks is the reference's chunk order).
 * Records carry coordinates, span and score; names, lengths and the ASCII
 * bases are the caller's, by group and coordinates. */
typedef struct {
    uint32_t group;      /* < 2^32 - 1 */
    uint32_t t_offset;   /* added to t_start; t_offset + target length <= 2^32 */
} gxy_unit_place;

typedef struct {
    uint32_t group;
    uint32_t t_start;    /* global target coordinate */
    uint32_t q_start;
    uint32_t span;       /* t_span = q_span = the HSP length */
    int32_t score;
    uint32_t unit;       /* the unit that produced it */
} gxy_record;

typedef struct {
    gxy_record* records;       /* group-major, each group by (t_start, q_start, span) */
    uint64_t* group_offsets;   /* n_groups + 1 (n_groups = 1 + the largest group named) */
    uint64_t n_records;
    uint32_t n_groups;
} gxy_record_result;

gxy_status gxy_batch_records(gxy_ctx* ctx, uint32_t n_tables, const gxy_table* const* tables,
                             uint32_t n_queries, const gxy_dseq* const* queries,
                             uint32_t n_units, const gxy_unit* units, const gxy_unit_place* places,
                             const gxy_search_params* params, const gxy_batch_opts* opts,
                             gxy_record_result* out, gxy_stats* stats);
void gxy_record_result_free(gxy_record_result* r);

/* chunk_target (src/driver.rs:156-194): writes up to cap chunks as
 * (chunk_lo, chunk_hi, primary_lo_local, primary_hi_local) quadruples and
 * returns the count in *n (always set, even when cap is too small). */
gxy_status gxy_chunk_plan(uint64_t target_len, uint32_t primary_bp, uint32_t halo_bp,
                          uint64_t* quads, uint64_t cap, uint64_t* n);

/* ---- x-drop extension of given hits (src/hsp.rs:66-148) ------------------ */
/* Extends n seed hits (t_pos[i], q_pos[i]) of seed_len columns exactly like
 * extend_hit: ok[i] = 1 and out[i] set when the HSP reaches hspthresh.
 * mode 0 = one lane per hit, mode 1 = one warp per hit (shuffle prefix-max). */
gxy_status gxy_extend_hits(gxy_ctx* ctx, const gxy_dseq* target, const gxy_dseq* query,
                           const gxy_search_params* params, uint64_t n, const uint32_t* t_pos,
                           const uint32_t* q_pos, uint32_t seed_len, uint32_t mode,
                           gxy_hsp* out, uint8_t* ok);

/* ---- consumers of the HSP list (src/anchor.rs, src/chain.rs) ------------- */
/* choose_anchor (src/anchor.rs:25-69) for n HSPs of (target, query) on the
 * device: t_pos[i], q_pos[i] = the midpoint of the highest-scoring window of
 * min(max(window, 1), length) columns along HSP i (first window on ties).
 * Scores from params->sub / ambig.  Empty or out-of-range HSPs: GXY_EINVAL. */
gxy_status gxy_choose_anchors(gxy_ctx* ctx, const gxy_dseq* target, const gxy_dseq* query,
                              const gxy_search_params* params, const gxy_hsp* hsps, uint64_t n, uint32_t window,
                              uint32_t* t_pos, uint32_t* q_pos);
/* best_chain (src/chain.rs:19-69): the highest-scoring chain of HSPs that is
 * strictly increasing on both axes, in t_start order, with the reference's
 * tie rules; out holds up to n HSPs, *out_n receives the chain length.  Host
 * code, O(n log n) (the reference scans O(n^2)); empty HSPs: GXY_EINVAL. */
gxy_status gxy_best_chain(const gxy_hsp* hsps, uint64_t n, gxy_hsp* out, uint64_t* out_n);
/* best_chain (src/chain.rs:19-69) for n_groups groups at once on the device
 * (the driver's --chain applies it per (target, query, strand) group,
 * src/driver.rs).  Group g is hsps[group_offsets[g] .. group_offsets[g+1]);
 * group_offsets has n_groups + 1 entries, starts at 0 and does not decrease.
 * Group g's chain goes to out[group_offsets[g] ..] in t_start order (the rest
 * of its range is zeroed) and its length to chain_len[g].  The reference's
 * O(n^2) scan, one block per group, with its tie rules; any HSP length is
 * accepted.  Host buffers; fewer than 2^31 HSPs in all. */
gxy_status gxy_best_chain_groups(gxy_ctx* ctx, const gxy_hsp* hsps, const uint64_t* group_offsets,
                                 uint32_t n_groups, gxy_hsp* out, uint64_t* chain_len);

/* ---- gapped extension (src/gapped_extend.rs:78-460) ---------------------- */
/* GappedParams (src/gapped_extend.rs:27-31) plus the ScoringMatrix's affine
 * gap costs (src/scoring.rs:35-36): a gap of k columns costs
 * gap_open + k * gap_extend. */
typedef struct {
    int32_t gap_open;
    int32_t gap_extend;
    int32_t y_drop;
    int32_t gapped_threshold;
} gxy_gapped_params;

/* GappedAlignment (src/gapped_extend.rs:54-63) of one anchor.  passed = 1 when
 * extend() returns Some (total >= gapped_threshold); then the coordinates are
 * set (t_start in the target view's coordinates) and the edit script is
 * runs[script_off .. script_off + script_len) of the result.  passed = 0 is
 * None: score holds the total, everything else is 0. */
typedef struct {
    uint32_t t_start;
    uint32_t q_start;
    uint32_t t_len;
    uint32_t q_len;
    int32_t score;
    uint32_t passed;
    uint64_t script_off;
    uint32_t script_len;
    uint32_t pad_;
} gxy_gapped_aln;

/* One call's alignments (one per anchor, in anchor order) and their edit
 * scripts (EditScript, src/edit_script.rs:47-74): a run is count << 2 | op,
 * op 0 = Match, 1 = InsertQuery (gap in the target), 2 = DeleteQuery (gap in
 * the query); adjacent runs never share an op.  Free with
 * gxy_gapped_result_free. */
typedef struct {
    gxy_gapped_aln* alns;
    uint32_t* runs;
    uint64_t n_alns;
    uint64_t n_runs;
} gxy_gapped_result;

typedef struct {
    uint64_t rows;                 /* DP rows of all sides (each side's DP once) */
    uint64_t cells;                /* DP cells of all sides (the band's width summed over the rows) */
    double device_ms;              /* CUDA-event time of the DP kernel (last run) */
    uint32_t reruns;               /* first passes repeated after the run buffer had to grow */
    uint32_t warps_per_side;       /* warps of the block that runs one side (8 cells of a row a thread) */
    uint64_t max_side_rows;        /* rows of the longest side (sides run in parallel; rows are sequential) */
    uint64_t second_pass_sides;    /* sides run again with exactly sized traceback storage */
    uint32_t cells_per_thread;     /* cells of a DP row one thread holds (4 or 8) */
    uint32_t pad_;
    uint64_t second_pass_cells;    /* DP cells computed again by the second pass (not in cells) */
} gxy_gapped_stats;

/* extend (src/gapped_extend.rs:78-132) for n anchors (t_pos[i], q_pos[i]) on
 * the device, all against target[t_lo, t_hi) (the driver's chunk,
 * src/driver.rs:395-414; t_lo = t_hi = 0: the whole target) and the whole
 * query.  Scores: params->sub / ambig.  Every anchor is extended on its own,
 * as one extend() call; results are bit-exact to the reference's, script
 * included.  Anchors outside a sequence: GXY_EINVAL.  Outside the exact
 * envelope (|scores| > 2^16, gap_open > 2^20, gap_extend > 2^16,
 * y_drop > 2^27, a band wider than 2048 cells, or the largest positive
 * score x the shorter sequence >= 2^31 - 2^20): GXY_EUNSUPPORTED.  stats may
 * be NULL. */
gxy_status gxy_gapped_extend(gxy_ctx* ctx, const gxy_dseq* target, uint64_t t_lo, uint64_t t_hi,
                             const gxy_dseq* query, const gxy_search_params* params, const gxy_gapped_params* gp,
                             const uint32_t* t_pos, const uint32_t* q_pos, uint64_t n, gxy_gapped_result* out,
                             gxy_gapped_stats* stats);
void gxy_gapped_result_free(gxy_gapped_result* r);

/* ---- serving loop ---------------------------------------------------------- */
/* Keeps the given tables resident, admits submitted queries while device
 * memory is below max_device_bytes and in-flight units below max_units, and
 * runs them in overlapping batches on max_streams streams. */
typedef struct {
    uint64_t max_device_bytes;
    uint32_t max_units;
    uint32_t max_streams;
    uint32_t max_batch_units;
    uint32_t both_strands;
    /* Query bases (counted once per strand) one batch takes at most, so that
     * a batch stays short and requests behind it wait less; 0 = 16 Mbp. */
    uint64_t max_batch_bases;
    /* Requests with at least big_bases query bases are "big": each runs in a
     * batch of its own, at most max_big_inflight of them at a time, and
     * while that many run, the smaller requests queued behind them are
     * admitted ahead of them.  big_bases 0 = 1 Mbp; max_big_inflight 0 = 1. */
    uint64_t big_bases;
    uint32_t max_big_inflight;
    uint32_t reserved_;
    /* When > 0, each dispatcher sizes every buffer a batch uses at start for
     * a query of this many bases against the largest resident table, and a
     * batch then takes at most this many query bases (per strand) besides its
     * first request: no request that size or smaller waits for a device
     * allocation (growing a buffer by gigabytes took up to 0.7 s on a B200). */
    uint64_t warm_bases;
} gxy_server_opts;

gxy_status gxy_server_create(gxy_ctx* ctx, uint32_t n_tables, const gxy_table* const* tables,
                             const gxy_search_params* params, const gxy_server_opts* opts,
                             gxy_server** out);
/* Copies the query and queues it against table; returns its id. */
gxy_status gxy_server_submit(gxy_server* s, uint32_t table, const gxy_packed_seq* query,
                             uint64_t* request_id);
/* Waits up to timeout_ms for request_id.  On completion fills plus/minus
 * (library-allocated) and the request's submit->done latency. */
gxy_status gxy_server_wait(gxy_server* s, uint64_t request_id, uint32_t timeout_ms,
                           gxy_hsp_buf* plus, gxy_hsp_buf* minus, double* latency_ms);
typedef struct {
    uint64_t submitted;
    uint64_t completed;
    uint64_t batches;
    uint64_t max_inflight_units;
    uint64_t bytes_in_use;
    uint64_t reruns;        /* batches' pipeline runs repeated after a buffer had to grow */
    double busy_ms;         /* summed device time of the batches */
    uint64_t failed;        /* requests that completed with an error status */
    uint64_t canceled;      /* requests cancelled before their results were kept */
    uint64_t isolated;      /* failed batches whose requests were rerun one by one */
    uint64_t mem_refreshes; /* free-device-memory queries since creation */
} gxy_server_stats;
gxy_status gxy_server_get_stats(gxy_server* s, gxy_server_stats* st);
/* Cancels a request.  A queued request leaves the queue at once; one already
 * in a running batch finishes on the device but its results are dropped.
 * Either way gxy_server_wait then returns GXY_ECANCELED for it.  A request
 * that has already completed keeps its results (the call still returns
 * GXY_OK); an unknown id (never submitted, or already waited for) is
 * GXY_EINVAL. */
gxy_status gxy_server_cancel(gxy_server* s, uint64_t request_id);
/* Test hook (fault injection on the host): every batch that holds
 * request_id fails with `status` before any device work, as a failed device
 * allocation would.  A failed batch of several requests is rerun one request
 * at a time, so only the faulty request completes with that status.
 * status GXY_OK clears the fault.  Ids are handed out in submission order
 * starting at 1, so a fault can be set for an id not yet submitted (it then
 * holds from the moment that request is queued). */
gxy_status gxy_server_inject_fault(gxy_server* s, uint64_t request_id, gxy_status status);
gxy_status gxy_server_destroy(gxy_server* s);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif
#endif
