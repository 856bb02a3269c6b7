/*
 * oracle.h -- CPU restatement of the lastz-gxy seed->HSP path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA path is
 * compared against (tests/, __graft_entry__.smoke()) and the CPU baseline that
 * bench.py times (its cpu_baseline leg and its --impl reference arm).  Nothing
 * in the product path links or calls it.
 *
 * Every function names the reference file:line it restates (paths relative to
 * the nekrut/lastz-gxy project root).  The reference is Rust; it cannot be
 * compiled in this image (no cargo/rustc), so this C restatement is the oracle.
 * It is pinned by the reference's own known-answer tests (ported in
 * tests/test_oracle_kats.py) and by the reference's differential property test
 * shape (scalar == AVX2, src/hsp.rs:283-314).
 */
#ifndef GXY_ORACLE_H
#define GXY_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* PackedSeq (src/sequences.rs:61-66): 2-bit codes, 4 per byte, position i at
 * bits 2*(i&3) of byte i>>2; valid and mask bitsets, bit i&7 of byte i>>3. */
typedef struct {
    const uint8_t* codes;
    const uint8_t* valid;
    const uint8_t* mask;
    uint64_t len;
} orc_seq;

/* Hsp (src/hsp.rs:19-24). */
typedef struct {
    uint32_t t_start;
    uint32_t q_start;
    uint32_t length;
    int32_t score;
} orc_hsp;

/* SearchParams + HspParams + ScoringMatrix (src/seed_search.rs:19-30,
 * src/hsp.rs:46-49, src/scoring.rs:32-40).  sub[r*4+q] is the score of target
 * (reference) code r against query code q. */
typedef struct {
    int32_t sub[16];
    int32_t ambig;
    int32_t xdrop;
    int32_t hspthresh;
    uint32_t step;
    uint8_t transitions;
    uint8_t has_entropy;
    uint8_t pad_[2];
    int32_t entropy_thr;
} orc_params;

/* Position table (src/pos_table.rs:24-28). */
typedef struct {
    uint32_t* starts;     /* num_words + 1 */
    uint32_t* positions;  /* starts[num_words] */
    uint64_t num_words;
    uint32_t pattern_len;
    uint32_t weight;
    uint8_t care[32];     /* care offsets, leftmost first */
} orc_table;

typedef struct {
    uint64_t windows;     /* valid query windows */
    uint64_t raw_hits;    /* bucket entries visited (all variants) */
    uint64_t extended;    /* hits admitted by the diagonal filter */
    uint64_t hsps;        /* HSPs emitted (before sort/dedup) */
} orc_stats;

/* ---- packing (src/dna.rs:12-20, src/sequences.rs:89-131, :277-318) ---- */
void orc_pack_ascii(const uint8_t* ascii, uint64_t n, uint8_t* codes, uint8_t* valid,
                    uint8_t* mask);
void orc_reverse_complement(const orc_seq* in, uint8_t* codes, uint8_t* valid, uint8_t* mask);
void orc_slice(const orc_seq* in, uint64_t start, uint64_t end, uint8_t* codes, uint8_t* valid,
               uint8_t* mask);

/* ---- seeds (src/seeds.rs:38-51, :208-236) ---- */
/* Parses a 0/1 pattern; returns the pattern length, or -1 on a bad char, empty
 * or longer than 32 positions. */
int orc_pattern_parse(const char* pattern01, uint8_t* care, uint32_t* weight);
/* Returns 1 and stores the word when the window at pos is seedable, else 0. */
int orc_word_at(const orc_seq* s, const char* pattern01, uint64_t pos, uint64_t* word);

/* ---- position table (src/pos_table.rs:35-83, :113-136) ---- */
/* Returns 0 on success, -1 bad pattern / weight > 15, -2 step 0, -3 > 4 G
 * positions, -4 out of memory. */
int orc_table_build(const orc_seq* s, const char* pattern01, uint32_t step, orc_table* out);
void orc_table_prune(orc_table* t, uint32_t limit);
void orc_table_free(orc_table* t);

/* ---- x-drop extension (src/hsp.rs:98-211; src/hsp_simd.rs:27-243) ---- */
/* Returns 1 and fills *out when the HSP reaches hspthresh, else 0. */
int orc_extend_hit_scalar(const orc_seq* t, const orc_seq* q, const orc_params* p,
                          uint32_t t_pos, uint32_t q_pos, uint32_t seed_len, orc_hsp* out);
int orc_extend_hit_avx2(const orc_seq* t, const orc_seq* q, const orc_params* p,
                        uint32_t t_pos, uint32_t q_pos, uint32_t seed_len, orc_hsp* out);
/* 1 when this build and CPU can run the AVX2 restatement. */
int orc_has_avx2(void);

/* ---- entropy gate (src/entropy.rs:27-67) ---- */
double orc_shannon_entropy(const orc_seq* s, uint64_t start, uint64_t end);
int orc_passes_entropy_gate(const orc_seq* s, uint32_t t_start, uint32_t t_end, int32_t score,
                            int32_t threshold);

/* ---- search (src/seed_search.rs:45-125 with src/diag_hash.rs:34-53) ---- */
/* use_avx2 selects extend_hit_avx2 (the reference's dispatch on x86 with an
 * i8-safe matrix, src/hsp.rs:66-87) instead of extend_hit_scalar.  Output is
 * malloc'd, sorted canonically by (diagonal, t_start, length, score) and
 * deduplicated; free with orc_free.  Returns 0, or -1 on out of memory. */
int orc_search(const orc_table* table, const orc_seq* target, const orc_seq* query,
               const orc_params* p, int use_avx2, orc_hsp** out, uint64_t* n_out,
               orc_stats* stats);

/* Runs orc_search over n_units independent (table, target, query) units with
 * up to n_threads POSIX threads (the reference fans out over chunks with
 * rayon, src/driver.rs:210).  out[i]/n_out[i] receive unit i's HSPs. */
int orc_search_units(int n_units, const orc_table* const* tables, const orc_seq* targets,
                     const orc_seq* queries, const orc_params* p, int use_avx2, int n_threads,
                     orc_hsp** out, uint64_t* n_out, orc_stats* stats);

/* DiagHash (src/diag_hash.rs:19-53) on its own, for the reference's KATs. */
void* orc_diag_new(void);
int orc_diag_admit(void* h, uint32_t t_pos, uint32_t q_pos);
void orc_diag_mark_covered(void* h, uint32_t t_end, uint32_t q_end);
void orc_diag_free(void* h);

/* best_chain (src/chain.rs:19-69) in the reference's O(n^2) form: the chain
 * into out (up to n HSPs) in t_start order; returns its length. */
uint64_t orc_best_chain(const orc_hsp* hsps, uint64_t n, orc_hsp* out);

/* ---- gapped extension (src/gapped_extend.rs:78-460) ---- */
/* GappedParams (src/gapped_extend.rs:27-31) plus the ScoringMatrix gap
 * fields (src/scoring.rs:35-36). */
typedef struct {
    int32_t gap_open;
    int32_t gap_extend;
    int32_t y_drop;
    int32_t gapped_threshold;
} orc_gapped_params;

/* GappedAlignment (src/gapped_extend.rs:54-63); runs = the EditScript,
 * count << 2 | op with op 0 = Match, 1 = InsertQuery, 2 = DeleteQuery
 * (src/edit_script.rs:17-22).  left/right_score: the two sides' DP bests,
 * set whether or not the total passes. */
typedef struct {
    uint32_t t_start, q_start, t_len, q_len;
    int32_t score;
    uint32_t n_runs;
    uint32_t* runs;   /* malloc'd; free with orc_free */
    int32_t left_score, right_score;
    uint64_t cells;   /* DP cells of both sides (the bands' widths summed over the rows) */
} orc_gapped_aln;

/* extend(): 1 = Some (out filled), 0 = None (total below gapped_threshold),
 * -1 = out of memory, -2 = anchor outside a sequence. */
int orc_gapped_extend(const orc_seq* t, const orc_seq* q, const orc_params* p, const orc_gapped_params* gp,
                      uint32_t t_pos, uint32_t q_pos, orc_gapped_aln* out);
/* n anchors over n_threads POSIX threads; rc[i] = orc_gapped_extend's return. */
int orc_gapped_extend_many(const orc_seq* t, const orc_seq* q, const orc_params* p, const orc_gapped_params* gp,
                           const uint32_t* t_pos, const uint32_t* q_pos, uint64_t n, int n_threads,
                           orc_gapped_aln* out, int* rc);

void orc_free(void* p);

#ifdef __cplusplus
}
#endif
#endif
