/*
 * oracle.c -- CPU restatement of the lastz-gxy seed->HSP path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path and the timed CPU
 * baseline.  Each function cites the reference file:line it restates.  The
 * arithmetic is kept in the reference's order and widths: i32 saturating adds
 * for scores, u32 positions, i64 diagonals.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <pthread.h>

#if defined(__x86_64__)
#include <immintrin.h>
#endif

/* ------------------------------------------------------------------------ */
/* PackedSeq accessors (src/sequences.rs:136-150).                          */
/* ------------------------------------------------------------------------ */
static inline uint32_t s_code(const orc_seq* s, uint64_t i) {
    return (s->codes[i >> 2] >> ((i & 3) * 2)) & 3u;
}
static inline int s_valid(const orc_seq* s, uint64_t i) { return (s->valid[i >> 3] >> (i & 7)) & 1; }
static inline int s_masked(const orc_seq* s, uint64_t i) { return (s->mask[i >> 3] >> (i & 7)) & 1; }

static inline int32_t sat_add(int32_t a, int32_t b) {
    int64_t r = (int64_t)a + (int64_t)b;
    if (r > INT32_MAX) return INT32_MAX;
    if (r < INT32_MIN) return INT32_MIN;
    return (int32_t)r;
}
static inline int32_t sat_sub(int32_t a, int32_t b) {
    int64_t r = (int64_t)a - (int64_t)b;
    if (r > INT32_MAX) return INT32_MAX;
    if (r < INT32_MIN) return INT32_MIN;
    return (int32_t)r;
}

/* encode_base, src/dna.rs:12-20. */
static inline void encode_base(uint8_t b, uint32_t* code, int* valid) {
    switch (b) {
        case 'A': case 'a': *code = 0; *valid = 1; return;
        case 'C': case 'c': *code = 1; *valid = 1; return;
        case 'G': case 'g': *code = 2; *valid = 1; return;
        case 'T': case 't': case 'U': case 'u': *code = 3; *valid = 1; return;
        default: *code = 0; *valid = 0; return;
    }
}

/* PackedSeq::push_ascii, src/sequences.rs:107-131, applied over a buffer
 * (from_ascii, :89-95).  Output buffers must be zeroed by the caller's size:
 * codes ceil(n/4), valid and mask ceil(n/8) bytes. */
void orc_pack_ascii(const uint8_t* ascii, uint64_t n, uint8_t* codes, uint8_t* valid,
                    uint8_t* mask) {
    memset(codes, 0, (n + 3) / 4);
    memset(valid, 0, (n + 7) / 8);
    memset(mask, 0, (n + 7) / 8);
    for (uint64_t i = 0; i < n; i++) {
        uint32_t c; int v;
        uint8_t b = ascii[i];
        encode_base(b, &c, &v);
        codes[i >> 2] |= (uint8_t)((c & 3u) << ((i & 3) * 2));
        if (v) valid[i >> 3] |= (uint8_t)(1u << (i & 7));
        if (v && b >= 'a' && b <= 'z') mask[i >> 3] |= (uint8_t)(1u << (i & 7));
    }
}

/* PackedSeq::reverse_complement, src/sequences.rs:303-318: position len-1-i of
 * the output is the complement (!c & 3) of input position i; an invalid input
 * position is pushed as 'N' (code 0, not valid, not masked); the mask bit
 * moves with its base. */
void orc_reverse_complement(const orc_seq* in, uint8_t* codes, uint8_t* valid, uint8_t* mask) {
    uint64_t n = in->len;
    memset(codes, 0, (n + 3) / 4);
    memset(valid, 0, (n + 7) / 8);
    memset(mask, 0, (n + 7) / 8);
    for (uint64_t o = 0; o < n; o++) {
        uint64_t i = n - 1 - o;
        if (!s_valid(in, i)) continue;
        uint32_t c = (~s_code(in, i)) & 3u;
        codes[o >> 2] |= (uint8_t)(c << ((o & 3) * 2));
        valid[o >> 3] |= (uint8_t)(1u << (o & 7));
        if (s_masked(in, i)) mask[o >> 3] |= (uint8_t)(1u << (o & 7));
    }
}

/* PackedSeq::slice_to_new, src/sequences.rs:277-298: invalid positions become
 * 'N' (code 0, mask 0); valid positions keep their code and mask bit. */
void orc_slice(const orc_seq* in, uint64_t start, uint64_t end, uint8_t* codes, uint8_t* valid,
               uint8_t* mask) {
    uint64_t n = end - start;
    memset(codes, 0, (n + 3) / 4);
    memset(valid, 0, (n + 7) / 8);
    memset(mask, 0, (n + 7) / 8);
    for (uint64_t o = 0; o < n; o++) {
        uint64_t i = start + o;
        if (!s_valid(in, i)) continue;
        codes[o >> 2] |= (uint8_t)(s_code(in, i) << ((o & 3) * 2));
        valid[o >> 3] |= (uint8_t)(1u << (o & 7));
        if (s_masked(in, i)) mask[o >> 3] |= (uint8_t)(1u << (o & 7));
    }
}

/* ------------------------------------------------------------------------ */
/* Seeds (src/seeds.rs).                                                    */
/* ------------------------------------------------------------------------ */

/* SeedPattern::parse + SeedPattern::new (src/seeds.rs:26-51), and
 * SeedExtractor::new's care-offset list (:187-195). */
int orc_pattern_parse(const char* pattern01, uint8_t* care, uint32_t* weight) {
    int len = 0;
    uint32_t w = 0;
    for (const char* c = pattern01; *c; c++) {
        if (*c != '0' && *c != '1') return -1;
        if (len >= 32) return -1;
        if (*c == '1') care[w++] = (uint8_t)len;
        len++;
    }
    if (len == 0) return -1;
    *weight = w;
    return len;
}

/* SeedExtractor::word_at, src/seeds.rs:133-147: None when the window runs past
 * the end or any care position is invalid or soft-masked; the leftmost care
 * position lands in the most significant bits. */
static inline int word_at(const orc_seq* s, const uint8_t* care, uint32_t weight, uint32_t plen,
                          uint64_t pos, uint64_t* word) {
    uint64_t end = pos + plen;
    if (end > s->len) return 0;
    uint64_t w = 0;
    for (uint32_t i = 0; i < weight; i++) {
        uint64_t p = pos + care[i];
        if (!s_valid(s, p) || s_masked(s, p)) return 0;
        w = (w << 2) | s_code(s, p);
    }
    *word = w;
    return 1;
}

int orc_word_at(const orc_seq* s, const char* pattern01, uint64_t pos, uint64_t* word) {
    uint8_t care[32]; uint32_t weight;
    int plen = orc_pattern_parse(pattern01, care, &weight);
    if (plen < 0) return 0;
    return word_at(s, care, weight, (uint32_t)plen, pos, word);
}

/* ------------------------------------------------------------------------ */
/* PosTable (src/pos_table.rs).                                             */
/* ------------------------------------------------------------------------ */

/* PosTable::build, src/pos_table.rs:35-83.  Windows come from
 * iter_with_stride (src/seeds.rs:151-161): pos = 0, step, ... <= len-L (with
 * len-L saturating at 0).  Count per word, exclusive prefix into starts,
 * then scatter in ascending position order. */
int orc_table_build(const orc_seq* s, const char* pattern01, uint32_t step, orc_table* out) {
    memset(out, 0, sizeof(*out));
    int plen = orc_pattern_parse(pattern01, out->care, &out->weight);
    if (plen < 0 || out->weight > 15) return -1;
    if (step < 1) return -2;
    out->pattern_len = (uint32_t)plen;
    uint64_t nw = 1ull << (2 * out->weight);
    out->num_words = nw;
    uint32_t* counts = (uint32_t*)calloc(nw, sizeof(uint32_t));
    out->starts = (uint32_t*)malloc((nw + 1) * sizeof(uint32_t));
    if (!counts || !out->starts) { free(counts); free(out->starts); return -4; }
    uint64_t max_start = s->len > (uint64_t)plen ? s->len - (uint64_t)plen : 0;
    uint64_t nwin = 0;
    for (uint64_t pos = 0; pos <= max_start; pos += step) {
        uint64_t w;
        if (word_at(s, out->care, out->weight, (uint32_t)plen, pos, &w)) { counts[w]++; nwin++; }
    }
    if (nwin > 0xFFFFFFFFull) { free(counts); free(out->starts); return -3; }
    uint32_t acc = 0;
    for (uint64_t i = 0; i < nw; i++) { out->starts[i] = acc; acc += counts[i]; }
    out->starts[nw] = acc;
    out->positions = (uint32_t*)malloc((acc ? acc : 1) * sizeof(uint32_t));
    if (!out->positions) { free(counts); free(out->starts); return -4; }
    for (uint64_t i = 0; i < nw; i++) counts[i] = out->starts[i];
    for (uint64_t pos = 0; pos <= max_start; pos += step) {
        uint64_t w;
        if (word_at(s, out->care, out->weight, (uint32_t)plen, pos, &w))
            out->positions[counts[w]++] = (uint32_t)pos;
    }
    free(counts);
    return 0;
}

/* PosTable::prune_hot_words, src/pos_table.rs:113-136: drop every bucket
 * whose multiplicity exceeds limit and rebuild starts/positions compactly. */
void orc_table_prune(orc_table* t, uint32_t limit) {
    uint64_t nw = t->num_words;
    uint32_t acc = 0;
    uint32_t prev_start = t->starts[0];
    for (uint64_t w = 0; w < nw; w++) {
        uint32_t s = prev_start, e = t->starts[w + 1];
        prev_start = e;
        t->starts[w] = acc;
        if (e - s <= limit) {
            memmove(t->positions + acc, t->positions + s, (size_t)(e - s) * sizeof(uint32_t));
            acc += e - s;
        }
    }
    t->starts[nw] = acc;
}

void orc_table_free(orc_table* t) {
    free(t->starts);
    free(t->positions);
    t->starts = NULL;
    t->positions = NULL;
}

/* ------------------------------------------------------------------------ */
/* Scalar x-drop extension (src/hsp.rs).                                    */
/* ------------------------------------------------------------------------ */

/* column_score, src/hsp.rs:198-211. */
static inline int32_t column_score(const orc_seq* t, const orc_seq* q, const orc_params* p,
                                   int64_t ti, int64_t qi) {
    if (!s_valid(t, (uint64_t)ti) || !s_valid(q, (uint64_t)qi)) return p->ambig;
    return p->sub[s_code(t, (uint64_t)ti) * 4 + s_code(q, (uint64_t)qi)];
}

/* extend_one_side, src/hsp.rs:160-195. */
static void extend_one_side(const orc_seq* t, const orc_seq* q, const orc_params* p, int64_t st,
                            int64_t sq, int64_t dir, int32_t* best_out, uint32_t* ext_out) {
    int64_t tl = (int64_t)t->len, ql = (int64_t)q->len;
    int32_t running = 0, best = 0;
    uint32_t best_ext = 0, ext = 0;
    int64_t ti = st, qi = sq;
    for (;;) {
        if (ti < 0 || qi < 0 || ti >= tl || qi >= ql) break;
        ext++;
        running = sat_add(running, column_score(t, q, p, ti, qi));
        if (running > best) {
            best = running;
            best_ext = ext;
        } else if ((int64_t)best - (int64_t)running > (int64_t)p->xdrop) {
            break;
        }
        ti += dir;
        qi += dir;
    }
    *best_out = best;
    *ext_out = best_ext;
}

/* extend_hit_scalar, src/hsp.rs:98-148. */
int orc_extend_hit_scalar(const orc_seq* t, const orc_seq* q, const orc_params* p,
                          uint32_t t_pos, uint32_t q_pos, uint32_t seed_len, orc_hsp* out) {
    int64_t tp = t_pos, qp = q_pos, L = seed_len;
    if (tp + L > (int64_t)t->len || qp + L > (int64_t)q->len) return 0;
    int32_t seed = 0;
    for (int64_t k = 0; k < L; k++) seed = sat_add(seed, column_score(t, q, p, tp + k, qp + k));
    int32_t rb, lb;
    uint32_t re, le;
    extend_one_side(t, q, p, tp + L, qp + L, 1, &rb, &re);
    extend_one_side(t, q, p, tp - 1, qp - 1, -1, &lb, &le);
    int32_t score = sat_add(sat_add(seed, lb), rb);
    if (score < p->hspthresh) return 0;
    out->t_start = (uint32_t)(tp - le);
    out->q_start = (uint32_t)(qp - le);
    out->length = (uint32_t)(L + le + re);
    out->score = score;
    return 1;
}

/* ------------------------------------------------------------------------ */
/* AVX2 x-drop extension (src/hsp_simd.rs) -- the CPU baseline's extender.  */
/* ------------------------------------------------------------------------ */

#if defined(__x86_64__)
/* UNPACK_LUT, src/sequences.rs:24-35: byte -> its four 2-bit codes. */
static uint8_t g_unpack_lut[256][4];
static int g_unpack_ready = 0;
static void unpack_lut_init(void) {
    if (g_unpack_ready) return;
    for (int i = 0; i < 256; i++)
        for (int k = 0; k < 4; k++) g_unpack_lut[i][k] = (uint8_t)((i >> (2 * k)) & 3);
    g_unpack_ready = 1;
}

/* PackedSeq::codes_batch, src/sequences.rs:174-212: up to 16 codes from
 * start -- the head of an unaligned first byte, then 4 codes per LUT load,
 * then a per-position tail. */
static inline uint32_t codes_batch(const orc_seq* s, uint64_t start, uint8_t out[16]) {
    uint64_t n = s->len > start ? s->len - start : 0;
    if (n > 16) n = 16;
    if (n == 0) return 0;
    uint64_t off = start & 3, base = start >> 2, filled = 0;
    if (off != 0) {
        uint8_t byte = s->codes[base];
        for (uint64_t k = off; k < 4 && k < off + n; k++) out[filled++] = (byte >> (k * 2)) & 3;
        base++;
    }
    while (filled + 4 <= n) {
        memcpy(out + filled, g_unpack_lut[s->codes[base]], 4);
        base++;
        filled += 4;
    }
    while (filled < n) {
        uint64_t pos = start + filled;
        out[filled++] = (s->codes[pos >> 2] >> ((pos & 3) * 2)) & 3;
    }
    return (uint32_t)n;
}
/* PackedSeq::valid_mask_batch, src/sequences.rs:220-240. */
static inline uint32_t valid_mask_batch(const orc_seq* s, uint64_t start) {
    uint64_t n = s->len > start ? s->len - start : 0;
    if (n > 16) n = 16;
    uint32_t m = 0;
    uint64_t i = 0;
    while (i < n) {
        uint64_t pos = start + i;
        uint32_t byte = s->valid[pos >> 3];
        uint32_t off = pos & 7;
        uint64_t take = n - i < 8 - off ? n - i : 8 - off;
        uint32_t chunk = (byte >> off) & ((1u << take) - 1u);
        m |= chunk << i;
        i += take;
    }
    return m;
}

/* extend_side, src/hsp_simd.rs:113-243: PSHUFB lookup of 16 columns against
 * the i8 LUT (src/scoring.rs:102-112), blend invalid columns to the i8 ambig
 * score, then the scalar prefix/x-drop scan. */
__attribute__((target("avx2,sse4.1,ssse3")))
static void extend_side_avx2(const orc_seq* t, const orc_seq* q, __m128i lut, int8_t ambig_i8,
                             int32_t xdrop, int64_t st, int64_t sq, int64_t dir,
                             int32_t* best_out, uint32_t* ext_out) {
    int64_t tl = (int64_t)t->len, ql = (int64_t)q->len;
    uint64_t max_ext;
    if (dir > 0) {
        if (st >= tl || sq >= ql) max_ext = 0;
        else max_ext = (uint64_t)((tl - st) < (ql - sq) ? (tl - st) : (ql - sq));
    } else {
        if (st < 0 || sq < 0) max_ext = 0;
        else max_ext = (uint64_t)((st + 1) < (sq + 1) ? (st + 1) : (sq + 1));
    }
    *best_out = 0;
    *ext_out = 0;
    if (max_ext == 0) return;
    const __m128i ambig_v = _mm_set1_epi8(ambig_i8);
    const __m128i low4 = _mm_set1_epi8(0x0F);
    int32_t running = 0, best = 0;
    uint32_t best_ext = 0, ext = 0;
    uint64_t off = 0;
    while (off < max_ext) {
        uint64_t chunk = max_ext - off < 16 ? max_ext - off : 16;
        uint8_t tc[16] = {0}, qc[16] = {0}, inv[16] = {0};
        if (dir > 0) {
            uint64_t ts = (uint64_t)(st + (int64_t)off), qs = (uint64_t)(sq + (int64_t)off);
            codes_batch(t, ts, tc);
            codes_batch(q, qs, qc);
            uint32_t both = valid_mask_batch(t, ts) & valid_mask_batch(q, qs);
            for (uint64_t i = 0; i < chunk; i++)
                if (((both >> i) & 1u) == 0) inv[i] = 0xFF;
        } else {
            for (uint64_t i = 0; i < chunk; i++) {
                int64_t ti = st - (int64_t)(off + i), qi = sq - (int64_t)(off + i);
                tc[i] = (uint8_t)s_code(t, (uint64_t)ti);
                qc[i] = (uint8_t)s_code(q, (uint64_t)qi);
                if (!s_valid(t, (uint64_t)ti) || !s_valid(q, (uint64_t)qi)) inv[i] = 0xFF;
            }
        }
        for (uint64_t i = chunk; i < 16; i++) inv[i] = 0xFF;
        __m128i tv = _mm_loadu_si128((const __m128i*)tc);
        __m128i qv = _mm_loadu_si128((const __m128i*)qc);
        __m128i idx = _mm_and_si128(_mm_or_si128(_mm_slli_epi16(tv, 2), qv), low4);
        __m128i sc = _mm_shuffle_epi8(lut, idx);
        __m128i blended = _mm_blendv_epi8(sc, ambig_v, _mm_loadu_si128((const __m128i*)inv));
        int8_t d[16];
        _mm_storeu_si128((__m128i*)d, blended);
        for (uint64_t i = 0; i < chunk; i++) {
            ext++;
            running = sat_add(running, (int32_t)d[i]);
            if (running > best) {
                best = running;
                best_ext = ext;
            } else if (sat_sub(best, running) > xdrop) {
                *best_out = best;
                *ext_out = best_ext;
                return;
            }
        }
        off += chunk;
    }
    *best_out = best;
    *ext_out = best_ext;
}

static int i8_safe(const orc_params* p) {
    for (int i = 0; i < 16; i++)
        if (p->sub[i] < -128 || p->sub[i] > 127) return 0;
    return p->ambig >= -128 && p->ambig <= 127;
}

/* extend_hit_avx2, src/hsp_simd.rs:27-95. */
__attribute__((target("avx2,sse4.1,ssse3")))
int orc_extend_hit_avx2(const orc_seq* t, const orc_seq* q, const orc_params* p,
                        uint32_t t_pos, uint32_t q_pos, uint32_t seed_len, orc_hsp* out) {
    int64_t tp = t_pos, qp = q_pos, L = seed_len;
    if (tp + L > (int64_t)t->len || qp + L > (int64_t)q->len) return 0;
    unpack_lut_init();
    int8_t lutb[16];
    for (int r = 0; r < 4; r++)
        for (int c = 0; c < 4; c++) lutb[(r << 2) | c] = (int8_t)p->sub[r * 4 + c];
    __m128i lut = _mm_loadu_si128((const __m128i*)lutb);
    int32_t seed = 0;
    for (int64_t k = 0; k < L; k++) seed = sat_add(seed, column_score(t, q, p, tp + k, qp + k));
    int32_t rb, lb;
    uint32_t re, le;
    extend_side_avx2(t, q, lut, (int8_t)p->ambig, p->xdrop, tp + L, qp + L, 1, &rb, &re);
    extend_side_avx2(t, q, lut, (int8_t)p->ambig, p->xdrop, tp - 1, qp - 1, -1, &lb, &le);
    int32_t score = sat_add(sat_add(seed, lb), rb);
    if (score < p->hspthresh) return 0;
    out->t_start = (uint32_t)(tp - le);
    out->q_start = (uint32_t)(qp - le);
    out->length = (uint32_t)(L + le + re);
    out->score = score;
    return 1;
}

int orc_has_avx2(void) { return __builtin_cpu_supports("avx2") ? 1 : 0; }
#else
int orc_extend_hit_avx2(const orc_seq* t, const orc_seq* q, const orc_params* p,
                        uint32_t t_pos, uint32_t q_pos, uint32_t seed_len, orc_hsp* out) {
    return orc_extend_hit_scalar(t, q, p, t_pos, q_pos, seed_len, out);
}
int orc_has_avx2(void) { return 0; }
static int i8_safe(const orc_params* p) { (void)p; return 0; }
#endif

/* ------------------------------------------------------------------------ */
/* Entropy gate (src/entropy.rs:27-67).                                     */
/* ------------------------------------------------------------------------ */
double orc_shannon_entropy(const orc_seq* s, uint64_t start, uint64_t end) {
    uint32_t counts[4] = {0, 0, 0, 0};
    uint32_t total = 0;
    uint64_t e = end < s->len ? end : s->len;
    for (uint64_t i = start; i < e; i++)
        if (s_valid(s, i)) { counts[s_code(s, i)]++; total++; }
    if (total == 0) return 0.0;
    double tt = (double)total, h = 0.0;
    for (int k = 0; k < 4; k++) {
        if (counts[k] == 0) continue;
        double pk = (double)counts[k] / tt;
        h -= pk * log2(pk);
    }
    return h;
}

int orc_passes_entropy_gate(const orc_seq* s, uint32_t t_start, uint32_t t_end, int32_t score,
                            int32_t threshold) {
    double h = orc_shannon_entropy(s, t_start, t_end);
    double scaled = (double)score * (h / 2.0);
    return scaled >= (double)threshold;
}

/* ------------------------------------------------------------------------ */
/* DiagHash (src/diag_hash.rs:19-53): map diagonal -> next admissible t.     */
/* Open addressing over i64 keys; only get/insert are used, as in the       */
/* reference, so the container's iteration order never matters.            */
/* ------------------------------------------------------------------------ */
typedef struct {
    int64_t* keys;
    uint32_t* vals;
    uint8_t* used;
    uint64_t cap, n;
} diag_hash;

static inline uint64_t mix64(uint64_t x) {
    x ^= x >> 30; x *= 0xbf58476d1ce4e5b9ull;
    x ^= x >> 27; x *= 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}
static int dh_init(diag_hash* h, uint64_t cap) {
    h->cap = cap; h->n = 0;
    h->keys = (int64_t*)malloc(cap * sizeof(int64_t));
    h->vals = (uint32_t*)malloc(cap * sizeof(uint32_t));
    h->used = (uint8_t*)calloc(cap, 1);
    return h->keys && h->vals && h->used ? 0 : -1;
}
static void dh_free(diag_hash* h) { free(h->keys); free(h->vals); free(h->used); }
static inline uint64_t dh_find(const diag_hash* h, int64_t k) {
    uint64_t i = mix64((uint64_t)k) & (h->cap - 1);
    while (h->used[i] && h->keys[i] != k) i = (i + 1) & (h->cap - 1);
    return i;
}
/* admit, src/diag_hash.rs:34-37. */
static inline int dh_admit(const diag_hash* h, uint32_t t, uint32_t q) {
    int64_t d = (int64_t)t - (int64_t)q;
    uint64_t i = dh_find(h, d);
    return !h->used[i] || t >= h->vals[i];
}
static int dh_grow(diag_hash* h) {
    diag_hash g;
    if (dh_init(&g, h->cap * 2)) return -1;
    for (uint64_t i = 0; i < h->cap; i++)
        if (h->used[i]) {
            uint64_t j = dh_find(&g, h->keys[i]);
            g.used[j] = 1; g.keys[j] = h->keys[i]; g.vals[j] = h->vals[i]; g.n++;
        }
    dh_free(h);
    *h = g;
    return 0;
}
/* mark_covered, src/diag_hash.rs:43-53. */
static inline int dh_mark_covered(diag_hash* h, uint32_t t_end, uint32_t q_end) {
    if ((h->n + 1) * 2 > h->cap && dh_grow(h)) return -1;
    int64_t d = (int64_t)t_end - (int64_t)q_end;
    uint64_t i = dh_find(h, d);
    if (h->used[i]) {
        if (t_end > h->vals[i]) h->vals[i] = t_end;
    } else {
        h->used[i] = 1; h->keys[i] = d; h->vals[i] = t_end; h->n++;
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* search (src/seed_search.rs:45-125).                                     */
/* ------------------------------------------------------------------------ */
static int hsp_cmp(const void* a, const void* b) {
    const orc_hsp* x = (const orc_hsp*)a;
    const orc_hsp* y = (const orc_hsp*)b;
    int64_t dx = (int64_t)x->t_start - (int64_t)x->q_start;
    int64_t dy = (int64_t)y->t_start - (int64_t)y->q_start;
    if (dx != dy) return dx < dy ? -1 : 1;
    if (x->t_start != y->t_start) return x->t_start < y->t_start ? -1 : 1;
    if (x->length != y->length) return x->length < y->length ? -1 : 1;
    if (x->score != y->score) return x->score < y->score ? -1 : 1;
    return 0;
}

int orc_search(const orc_table* table, const orc_seq* target, const orc_seq* query,
               const orc_params* p, int use_avx2, orc_hsp** out, uint64_t* n_out,
               orc_stats* stats) {
    const uint32_t L = table->pattern_len, w = table->weight;
    orc_stats st = {0, 0, 0, 0};
    *out = NULL;
    *n_out = 0;
    /* shifts, src/seed_search.rs:63. */
    uint32_t shifts[32];
    for (uint32_t i = 0; i < w; i++) shifts[i] = 2 * (w - 1 - i);
    /* variants capacity, src/seed_search.rs:69-73. */
    uint32_t vcap = p->transitions == 0 ? 1 : (p->transitions == 1 ? 1 + w : 1 + w + w * (w ? w - 1 : 0) / 2);
    uint64_t* variants = (uint64_t*)malloc(vcap * sizeof(uint64_t));
    uint32_t bounds[2 * (1 + 15 + 105)];
    uint64_t cap = 1024, n = 0;
    orc_hsp* res = (orc_hsp*)malloc(cap * sizeof(orc_hsp));
    diag_hash dh;
    if (!variants || !res || dh_init(&dh, 1024)) { free(variants); free(res); return -1; }
    if (use_avx2 && !(orc_has_avx2() && i8_safe(p))) use_avx2 = 0;
    uint32_t step = p->step ? p->step : 1;
    uint64_t max_start = query->len > L ? query->len - L : 0;
    for (uint64_t qpos = 0; qpos <= max_start; qpos += step) {
        uint64_t word;
        if (!word_at(query, table->care, w, L, qpos, &word)) continue;
        st.windows++;
        /* variant order, src/seed_search.rs:76-90. */
        uint32_t nv = 0;
        variants[nv++] = word;
        if (p->transitions >= 1)
            for (uint32_t i = 0; i < w; i++) variants[nv++] = word ^ (2ull << shifts[i]);
        if (p->transitions >= 2)
            for (uint32_t i = 0; i < w; i++)
                for (uint32_t j = i + 1; j < w; j++)
                    variants[nv++] = word ^ (2ull << shifts[i]) ^ (2ull << shifts[j]);
        /* src/seed_search.rs:92-116.  The bucket bounds of all variants are
         * read first (independent loads the CPU can overlap); the hits are
         * then visited in the reference's order. */
        for (uint32_t v = 0; v < nv; v++) {
            uint64_t vw = variants[v];
            bounds[2 * v] = table->starts[vw];
            bounds[2 * v + 1] = table->starts[vw + 1];
        }
        for (uint32_t v = 0; v < nv; v++) {
            uint32_t b = bounds[2 * v], e = bounds[2 * v + 1];
            st.raw_hits += e - b;
            for (uint32_t j = b; j < e; j++) {
                uint32_t tpos = table->positions[j];
                if (!dh_admit(&dh, tpos, (uint32_t)qpos)) continue;
                st.extended++;
                orc_hsp h;
                int ok = use_avx2 ? orc_extend_hit_avx2(target, query, p, tpos, (uint32_t)qpos, L, &h)
                                  : orc_extend_hit_scalar(target, query, p, tpos, (uint32_t)qpos, L, &h);
                if (!ok) continue;
                if (p->has_entropy &&
                    !orc_passes_entropy_gate(target, h.t_start, h.t_start + h.length, h.score,
                                             p->entropy_thr))
                    continue;
                if (dh_mark_covered(&dh, h.t_start + h.length, h.q_start + h.length)) goto oom;
                if (n == cap) {
                    cap *= 2;
                    orc_hsp* r2 = (orc_hsp*)realloc(res, cap * sizeof(orc_hsp));
                    if (!r2) goto oom;
                    res = r2;
                }
                res[n++] = h;
                st.hsps++;
            }
        }
    }
    /* sort by (diagonal, t_start) + dedup, src/seed_search.rs:122-123; the
     * oracle breaks key ties by (length, score) so its order is canonical. */
    qsort(res, n, sizeof(orc_hsp), hsp_cmp);
    {
        uint64_t m = 0;
        for (uint64_t i = 0; i < n; i++)
            if (m == 0 || hsp_cmp(&res[m - 1], &res[i]) != 0) res[m++] = res[i];
        n = m;
    }
    dh_free(&dh);
    free(variants);
    *out = res;
    *n_out = n;
    if (stats) *stats = st;
    return 0;
oom:
    dh_free(&dh);
    free(variants);
    free(res);
    return -1;
}

typedef struct {
    int n_units;
    const orc_table* const* tables;
    const orc_seq* targets;
    const orc_seq* queries;
    const orc_params* p;
    int use_avx2;
    orc_hsp** out;
    uint64_t* n_out;
    orc_stats* stats;
    int next;       /* next unit to run; taken under the lock */
    int err;
    pthread_mutex_t mu;
} units_job;

static void* units_worker(void* arg) {
    units_job* j = (units_job*)arg;
    for (;;) {
        pthread_mutex_lock(&j->mu);
        int u = j->next++;
        pthread_mutex_unlock(&j->mu);
        if (u >= j->n_units) break;
        orc_stats s;
        int r = orc_search(j->tables[u], &j->targets[u], &j->queries[u], j->p, j->use_avx2, &j->out[u],
                           &j->n_out[u], &s);
        if (j->stats) j->stats[u] = s;
        if (r) {
            pthread_mutex_lock(&j->mu);
            j->err = 1;
            pthread_mutex_unlock(&j->mu);
        }
    }
    return NULL;
}

int orc_search_units(int n_units, const orc_table* const* tables, const orc_seq* targets,
                     const orc_seq* queries, const orc_params* p, int use_avx2, int n_threads,
                     orc_hsp** out, uint64_t* n_out, orc_stats* stats) {
    units_job j;
    j.n_units = n_units; j.tables = tables; j.targets = targets; j.queries = queries; j.p = p;
    j.use_avx2 = use_avx2; j.out = out; j.n_out = n_out; j.stats = stats; j.next = 0; j.err = 0;
    pthread_mutex_init(&j.mu, NULL);
    if (n_threads < 1) n_threads = 1;
    if (n_threads > n_units) n_threads = n_units > 0 ? n_units : 1;
    pthread_t th[256];
    if (n_threads > 256) n_threads = 256;
    int started = 0;
    for (int i = 1; i < n_threads; i++)
        if (pthread_create(&th[started], NULL, units_worker, &j) == 0) started++;
    units_worker(&j);
    for (int i = 0; i < started; i++) pthread_join(th[i], NULL);
    pthread_mutex_destroy(&j.mu);
    return j.err ? -1 : 0;
}

void* orc_diag_new(void) {
    diag_hash* h = (diag_hash*)malloc(sizeof(diag_hash));
    if (!h) return NULL;
    if (dh_init(h, 64)) { free(h); return NULL; }
    return h;
}
int orc_diag_admit(void* h, uint32_t t_pos, uint32_t q_pos) { return dh_admit((diag_hash*)h, t_pos, q_pos); }
void orc_diag_mark_covered(void* h, uint32_t t_end, uint32_t q_end) { dh_mark_covered((diag_hash*)h, t_end, q_end); }
void orc_diag_free(void* h) {
    if (!h) return;
    dh_free((diag_hash*)h);
    free(h);
}

void orc_free(void* ptr) { free(ptr); }

/* ------------------------------------------------------------------------ */
/* best_chain (src/chain.rs:19-69): stable sort by (t_start, q_start)       */
/* (:28-29), weighted longest-increasing-chain DP with the first            */
/* predecessor of the largest best (strict >, :37-46), the first terminal   */
/* of the largest best (:49-56), traceback (:58-66).                        */
/* ------------------------------------------------------------------------ */
static int chain_cmp(const void* a, const void* b) {
    const orc_hsp* x = *(const orc_hsp* const*)a;
    const orc_hsp* y = *(const orc_hsp* const*)b;
    if (x->t_start != y->t_start) return x->t_start < y->t_start ? -1 : 1;
    if (x->q_start != y->q_start) return x->q_start < y->q_start ? -1 : 1;
    return x < y ? -1 : (x > y);   /* input order: a stable sort */
}

uint64_t orc_best_chain(const orc_hsp* hsps, uint64_t n, orc_hsp* out) {
    if (n == 0) return 0;
    const orc_hsp** srt = (const orc_hsp**)malloc(n * sizeof(*srt));
    int64_t* best = (int64_t*)malloc(n * sizeof(int64_t));
    int64_t* parent = (int64_t*)malloc(n * sizeof(int64_t));
    for (uint64_t i = 0; i < n; i++) srt[i] = &hsps[i];
    qsort(srt, n, sizeof(*srt), chain_cmp);
    for (uint64_t i = 0; i < n; i++) {
        best[i] = srt[i]->score;
        parent[i] = -1;
    }
    for (uint64_t i = 1; i < n; i++) {
        int64_t bp = 0, bi = -1;
        const uint32_t ti = srt[i]->t_start, qi = srt[i]->q_start;
        for (uint64_t j = 0; j < i; j++) {
            const orc_hsp* h = srt[j];
            if (h->t_start + h->length <= ti && h->q_start + h->length <= qi && best[j] > bp) {
                bp = best[j];
                bi = (int64_t)j;
            }
        }
        best[i] = bp + srt[i]->score;
        parent[i] = bi;
    }
    uint64_t end = 0;
    for (uint64_t i = 1; i < n; i++)
        if (best[i] > best[end]) end = i;
    uint64_t len = 0;
    for (int64_t c = (int64_t)end; c >= 0; c = parent[c]) len++;
    uint64_t k = len;
    for (int64_t c = (int64_t)end; c >= 0; c = parent[c]) out[--k] = *srt[c];
    free(srt);
    free(best);
    free(parent);
    return len;
}

/* ------------------------------------------------------------------------ */
/* Gapped extension (src/gapped_extend.rs:78-460): the banded 3-state       */
/* affine x-drop DP of extend_one_side (:178-412) run to the right of the   */
/* anchor and, on reversed inputs, to its left; the traceback's edit script */
/* (src/edit_script.rs:47-104: run-length runs, push merges equal ops).     */
/* Rows are allocated as the DP reaches them instead of (n+1) rows up front */
/* (:236-243), and the scores of only the previous and the current row are */
/* kept (the recurrences and the prune read no others); every row starts as */
/* NEG_INF / State::M like the reference's preallocated storage, so the    */
/* values read are the same.  The back-pointers are kept for every row.    */
/* ------------------------------------------------------------------------ */
#define G_NEG_INF (INT32_MIN / 4)   /* src/gapped_extend.rs:44 */
enum { G_M = 0, G_X = 1, G_Y = 2 };  /* State (:46-51) */

typedef struct {
    uint32_t* runs;   /* count << 2 | op */
    uint32_t n, cap;
} g_script;

/* EditScript::push (src/edit_script.rs:63-74). */
static int g_push(g_script* s, uint32_t op, uint32_t cnt) {
    if (cnt == 0) return 0;
    if (s->n && (s->runs[s->n - 1] & 3u) == op) {
        s->runs[s->n - 1] += cnt << 2;
        return 0;
    }
    if (s->n == s->cap) {
        uint32_t nc = s->cap ? s->cap * 2 : 16;
        uint32_t* r = (uint32_t*)realloc(s->runs, (size_t)nc * 4);
        if (!r) return -1;
        s->runs = r;
        s->cap = nc;
    }
    s->runs[s->n++] = (cnt << 2) | op;
    return 0;
}

/* pair_score (:160-166) on (code, valid) of the sliced inputs. */
static inline int32_t g_pair(const orc_seq* t, int64_t ti, const orc_seq* q, int64_t qi, const orc_params* p) {
    if (s_valid(t, (uint64_t)ti) && s_valid(q, (uint64_t)qi))
        return p->sub[s_code(t, (uint64_t)ti) * 4 + s_code(q, (uint64_t)qi)];
    return p->ambig;
}

typedef struct {
    int32_t score;
    uint32_t t_span, q_span;
    g_script script;   /* root-to-tip, as OneSide.script */
    uint64_t cells;    /* DP cells computed: the band's width summed over the rows */
} g_side;

/* extend_one_side (:178-412).  The sliced input of the reference is target
 * element i-1 = T[t0 + dir*i] and query element j-1 = Q[q0 + dir*j]
 * (dir +1: the right slice from anchor+1; dir -1: the reversed left slice). */
static int g_one_side(const orc_seq* T, int64_t t0, int64_t n, const orc_seq* Q, int64_t q0, int64_t m, int dir,
                      const orc_params* p, const orc_gapped_params* gp, g_side* out) {
    memset(out, 0, sizeof(*out));
    if (n == 0 || m == 0) return 0;
    const int32_t goe = gp->gap_open + gp->gap_extend, ge = gp->gap_extend, ydrop = gp->y_drop;
    int64_t radius;
    if (ge > 0) {
        int32_t r = sat_sub(ydrop, goe) / ge;
        radius = (r > 0 ? r : 0) + 2;
    } else {
        radius = m + 1;
    }
    int64_t bw = 4 * radius + 4;
    if (bw > m + 1) bw = m + 1;
    /* Back-pointer rows grow on demand; scores: rows i & 1 (two rows). */
    int64_t rows_cap = 0;
    int64_t* row_lo = NULL;
    int32_t* mm = (int32_t*)malloc((size_t)(2 * bw) * 4);
    int32_t* xx = (int32_t*)malloc((size_t)(2 * bw) * 4);
    int32_t* yy = (int32_t*)malloc((size_t)(2 * bw) * 4);
    uint8_t *mf = NULL, *xf = NULL, *yf = NULL;
    int rc = 0;
    if (!mm || !xx || !yy) {
        rc = -1;
        goto done;
    }
#define G_GROW(i)                                                                                      \
    if ((i) >= rows_cap) {                                                                             \
        int64_t nc = rows_cap ? rows_cap * 2 : 64;                                                     \
        if (nc > n + 1) nc = n + 1;                                                                    \
        int64_t* a = (int64_t*)realloc(row_lo, (size_t)nc * 8);                                        \
        if (a) row_lo = a;                                                                             \
        uint8_t* c1 = (uint8_t*)realloc(mf, (size_t)(nc * bw));                                        \
        if (c1) mf = c1;                                                                               \
        uint8_t* c2 = (uint8_t*)realloc(xf, (size_t)(nc * bw));                                        \
        if (c2) xf = c2;                                                                               \
        uint8_t* c3 = (uint8_t*)realloc(yf, (size_t)(nc * bw));                                        \
        if (c3) yf = c3;                                                                               \
        if (!a || !c1 || !c2 || !c3) {                                                                 \
            rc = -1;                                                                                   \
            goto done;                                                                                 \
        }                                                                                              \
        for (int64_t k = rows_cap * bw; k < nc * bw; k++) mf[k] = xf[k] = yf[k] = G_M;                 \
        rows_cap = nc;                                                                                 \
    }
    for (int64_t k = 0; k < 2 * bw; k++) mm[k] = xx[k] = yy[k] = G_NEG_INF;
    G_GROW(0);
    mm[0] = 0;
    int32_t best_score = 0;
    int64_t bi = 0, bj = 0;
    int best_state = G_M;
    int64_t lo = 0, hi = 0;
    row_lo[0] = 0;
    for (int64_t i = 0; i <= n; i++) {
        G_GROW(i);
        if (i >= 2)   /* row i's score storage was row i-2's: back to NEG_INF, as a fresh row */
            for (int64_t k = (i & 1) * bw; k < (i & 1) * bw + bw; k++) mm[k] = xx[k] = yy[k] = G_NEG_INF;
        const int64_t j_lo = lo > radius ? lo - radius : 0;
        int64_t j_hi = hi + radius;
        if (j_hi > m) j_hi = m;
        if (j_hi > j_lo + bw - 1) j_hi = j_lo + bw - 1;
        row_lo[i] = j_lo;
        out->cells += (uint64_t)(j_hi - j_lo + 1);
        const int64_t lo_this = j_lo;
        const int64_t lo_prev = i >= 1 ? row_lo[i - 1] : 0;
        const int64_t hi_prev_excl = lo_prev + bw;
        const int64_t base_this = (i & 1) * bw, base_prev = i >= 1 ? ((i - 1) & 1) * bw : 0;
        const int64_t tb_this = i * bw;   /* back-pointers of row i */
        for (int64_t j = j_lo; j <= j_hi; j++) {
            if (i == 0 && j == 0) continue;
            int32_t best = G_NEG_INF;
            const int64_t here = base_this + (j - lo_this);
            if (i >= 1) {   /* X: gap in query (:282-302) */
                int32_t pm = G_NEG_INF, px = G_NEG_INF;
                if (j >= lo_prev && j < hi_prev_excl) {
                    const int64_t off = base_prev + (j - lo_prev);
                    pm = mm[off];
                    px = xx[off];
                }
                const int32_t fm = pm - goe, fx = px - ge;
                const int32_t v = fm >= fx ? fm : fx;
                xx[here] = v;
                xf[tb_this + (j - lo_this)] = fm >= fx ? G_M : G_X;
                if (v > best) best = v;
            }
            if (j >= 1) {   /* Y: gap in target (:305-327) */
                int32_t pm = G_NEG_INF, py = G_NEG_INF;
                if (j - 1 >= lo_this) {
                    const int64_t off = base_this + (j - 1 - lo_this);
                    pm = mm[off];
                    py = yy[off];
                }
                const int32_t fm = pm - goe, fy = py - ge;
                const int32_t v = fm >= fy ? fm : fy;
                yy[here] = v;
                yf[tb_this + (j - lo_this)] = fm >= fy ? G_M : G_Y;
                if (v > best) best = v;
            }
            if (i >= 1 && j >= 1) {   /* M (:330-350) */
                const int32_t s = g_pair(T, t0 + dir * i, Q, q0 + dir * j, p);
                int32_t fm = G_NEG_INF, fx = G_NEG_INF, fy = G_NEG_INF;
                if (j - 1 >= lo_prev && j - 1 < hi_prev_excl) {
                    const int64_t off = base_prev + (j - 1 - lo_prev);
                    fm = mm[off];
                    fx = xx[off];
                    fy = yy[off];
                }
                int32_t prev;
                uint8_t from;
                if (fm >= fx && fm >= fy) {
                    prev = fm;
                    from = G_M;
                } else if (fx >= fy) {
                    prev = fx;
                    from = G_X;
                } else {
                    prev = fy;
                    from = G_Y;
                }
                const int32_t v = prev + s;
                mm[here] = v;
                mf[tb_this + (j - lo_this)] = from;
                if (v > best) best = v;
            }
            if (best > best_score) {   /* :353-363 */
                best_score = best;
                best_state = mm[here] == best ? G_M : (xx[here] == best ? G_X : G_Y);
                bi = i;
                bj = j;
            }
        }
        /* x-drop prune of the touched cells (:366-398). */
        const int32_t threshold = sat_sub(best_score, ydrop);
        int64_t new_lo = -1, new_hi = 0;
        for (int64_t j = j_lo; j <= j_hi; j++) {
            const int64_t here = base_this + (j - row_lo[i]);
            int32_t alive = mm[here] > xx[here] ? mm[here] : xx[here];
            if (yy[here] > alive) alive = yy[here];
            if (alive >= threshold) {
                if (new_lo < 0) new_lo = j;
                new_hi = j;
            } else {
                mm[here] = xx[here] = yy[here] = G_NEG_INF;
            }
        }
        if (new_lo < 0) break;
        lo = new_lo;
        hi = new_hi;
    }
    /* Traceback from the best cell (:404-437), emitted tip to root, then
     * reversed (:439). */
    {
        int64_t i = bi, j = bj;
        int st = best_state;
        g_script tip = {0};
        while (i > 0 || j > 0) {
            const int64_t h = i * bw + (j - row_lo[i]);
            if (st == G_M) {
                if (g_push(&tip, 0, 1)) { rc = -1; break; }
                st = mf[h];
                i--;
                j--;
            } else if (st == G_X) {
                if (g_push(&tip, 2, 1)) { rc = -1; break; }
                st = xf[h];
                i--;
            } else {
                if (g_push(&tip, 1, 1)) { rc = -1; break; }
                st = yf[h];
                j--;
            }
        }
        if (rc == 0) {
            for (uint32_t k = tip.n; k-- > 0;) {
                if (g_push(&out->script, tip.runs[k] & 3u, tip.runs[k] >> 2)) { rc = -1; break; }
            }
        }
        free(tip.runs);
    }
    out->score = best_score;
    out->t_span = (uint32_t)bi;
    out->q_span = (uint32_t)bj;
done:
#undef G_GROW
    free(row_lo);
    free(mm);
    free(xx);
    free(yy);
    free(mf);
    free(xf);
    free(yf);
    return rc;
}

/* extend (src/gapped_extend.rs:78-132). */
int orc_gapped_extend(const orc_seq* t, const orc_seq* q, const orc_params* p, const orc_gapped_params* gp,
                      uint32_t t_pos, uint32_t q_pos, orc_gapped_aln* out) {
    memset(out, 0, sizeof(*out));
    if ((uint64_t)t_pos >= t->len || (uint64_t)q_pos >= q->len) return -2;
    const int32_t col = g_pair(t, t_pos, q, q_pos, p);
    g_side right, left;
    if (g_one_side(t, t_pos, (int64_t)t->len - t_pos - 1, q, q_pos, (int64_t)q->len - q_pos - 1, 1, p, gp, &right))
        return -1;
    if (g_one_side(t, t_pos, t_pos, q, q_pos, q_pos, -1, p, gp, &left)) {
        free(right.script.runs);
        return -1;
    }
    const int32_t total = sat_add(sat_add(col, left.score), right.score);
    int rc = 0;
    if (total >= gp->gapped_threshold) {
        g_script s = {0};
        int bad = 0;
        for (uint32_t k = left.script.n; k-- > 0 && !bad;)   /* left_raw.script.reversed() */
            bad = g_push(&s, left.script.runs[k] & 3u, left.script.runs[k] >> 2);
        if (!bad) bad = g_push(&s, 0, 1);   /* the anchor column */
        for (uint32_t k = 0; k < right.script.n && !bad; k++)
            bad = g_push(&s, right.script.runs[k] & 3u, right.script.runs[k] >> 2);
        if (bad) {
            free(s.runs);
            rc = -1;
        } else {
            out->t_start = t_pos - left.t_span;
            out->q_start = q_pos - left.q_span;
            out->t_len = left.t_span + 1 + right.t_span;
            out->q_len = left.q_span + 1 + right.q_span;
            out->score = total;
            out->n_runs = s.n;
            out->runs = s.runs;
            rc = 1;
        }
    }
    out->left_score = left.score;
    out->cells = left.cells + right.cells;
    out->right_score = right.score;
    free(right.script.runs);
    free(left.script.runs);
    return rc;
}

typedef struct {
    const orc_seq *t, *q;
    const orc_params* p;
    const orc_gapped_params* gp;
    const uint32_t *tp, *qp;
    orc_gapped_aln* out;
    int* rc;
    uint64_t n;
    int nth, me;
} g_job;

static void* g_worker(void* arg) {
    g_job* J = (g_job*)arg;
    for (uint64_t i = (uint64_t)J->me; i < J->n; i += (uint64_t)J->nth)
        J->rc[i] = orc_gapped_extend(J->t, J->q, J->p, J->gp, J->tp[i], J->qp[i], &J->out[i]);
    return NULL;
}

int orc_gapped_extend_many(const orc_seq* t, const orc_seq* q, const orc_params* p, const orc_gapped_params* gp,
                           const uint32_t* t_pos, const uint32_t* q_pos, uint64_t n, int n_threads,
                           orc_gapped_aln* out, int* rc) {
    if (n_threads < 1) n_threads = 1;
    pthread_t th[256];
    g_job jobs[256];
    if (n_threads > 256) n_threads = 256;
    for (int k = 0; k < n_threads; k++) {
        jobs[k] = (g_job){t, q, p, gp, t_pos, q_pos, out, rc, n, n_threads, k};
        if (pthread_create(&th[k], NULL, g_worker, &jobs[k])) return -1;
    }
    for (int k = 0; k < n_threads; k++) pthread_join(th[k], NULL);
    return 0;
}
