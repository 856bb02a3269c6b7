"""The oracle against the reference's own known-answer tests (CPU only).

Each test names the reference test it ports (file:line).  These pin the C
restatement in oracle/oracle.c; the GPU tests then compare the CUDA path with
the oracle."""
import numpy as np
import pytest

import oracle as O
from helpers import rand_ascii

HOX = O.params


# ---- src/dna.rs:43-74 via packing -------------------------------------------------
def test_encode_and_case():
    s = O.pack_ascii(b"ACGTacgtUuN")
    codes = [(int(s.codes[i >> 2]) >> ((i & 3) * 2)) & 3 for i in range(11)]
    valid = [(int(s.valid[i >> 3]) >> (i & 7)) & 1 for i in range(11)]
    mask = [(int(s.mask[i >> 3]) >> (i & 7)) & 1 for i in range(11)]
    assert codes[:10] == [0, 1, 2, 3, 0, 1, 2, 3, 3, 3]
    assert valid == [1] * 10 + [0]
    assert mask == [0, 0, 0, 0, 1, 1, 1, 1, 0, 1, 0]


def test_ambiguous_bases_are_invalid():
    s = O.pack_ascii(b"NnRrYyMmKkSsWwBbDdHhVv?-")
    assert not any((int(s.valid[i >> 3]) >> (i & 7)) & 1 for i in range(24))


# ---- src/sequences.rs:396-577 -------------------------------------------------------
def to_ascii(s):
    out = []
    for i in range(s.len):
        if (int(s.valid[i >> 3]) >> (i & 7)) & 1:
            out.append(b"ACGT"[(int(s.codes[i >> 2]) >> ((i & 3) * 2)) & 3])
        else:
            out.append(ord("N"))
    return bytes(out)


def masked(s, i):
    return bool((int(s.mask[i >> 3]) >> (i & 7)) & 1)


def test_packed_roundtrip_and_rc():
    assert to_ascii(O.pack_ascii(b"ACGTACGTNACG")) == b"ACGTACGTNACG"          # :396-402
    rc = O.reverse_complement(O.pack_ascii(b"ACGTACGT"))
    assert to_ascii(rc) == b"ACGTACGT"                                            # :413-419
    assert to_ascii(O.reverse_complement(rc)) == b"ACGTACGT"
    assert to_ascii(O.reverse_complement(O.pack_ascii(b"ACCGTTNAG"))) == b"CTNAACGGT"  # :422-426


def test_soft_mask_and_slice():
    p = O.pack_ascii(b"ACgtAC")                                                   # :457-465
    assert [masked(p, i) for i in range(6)] == [False, False, True, True, False, False]
    s = O.slice_to_new(O.pack_ascii(b"ACgtNACGT"), 2, 7)                          # :478-488
    assert s.len == 5 and to_ascii(s) == b"GTNAC"
    assert masked(s, 0) and masked(s, 1) and not masked(s, 3) and not masked(s, 4)
    rc = O.reverse_complement(O.pack_ascii(b"ACgtAC"))                            # :567-577
    assert masked(rc, 2) and masked(rc, 3) and not any(masked(rc, i) for i in (0, 1, 4, 5))


# ---- src/seeds.rs:185-281 -----------------------------------------------------------
def test_seed_words():
    assert O.word_at(O.pack_ascii(b"ACGT"), "1111", 0) == 0x1B                  # :291-299
    assert O.word_at(O.pack_ascii(b"ACGT"), "1001", 0) == 0b0011                # :301-309
    assert O.word_at(O.pack_ascii(b"AcG"), "111", 0) is None                    # :311-318
    assert O.word_at(O.pack_ascii(b"AcG"), "101", 0) is not None                # :320-328
    assert O.word_at(O.pack_ascii(b"ACG"), "1111", 0) is None                   # :330-336


def test_iter_with_stride():
    s = O.pack_ascii(b"ACGNNACGT")                                              # :338-347
    assert [p for p in range(7) if O.word_at(s, "111", p) is not None] == [0, 5, 6]
    t = O.Table(O.pack_ascii(b"ACGTACGT"), "11", 3)                             # :349-356
    pos = sorted(t.positions().tolist())
    assert pos == [0, 3, 6]


# ---- src/pos_table.rs:143-225 -------------------------------------------------------
def test_pos_table_known_buckets():
    s = O.pack_ascii(b"ACGTACGT")
    t = O.Table(s, "111", 1)
    w = {k: O.word_at(s, "111", p) for k, p in (("acg", 0), ("cgt", 1), ("gta", 2), ("tac", 3))}
    assert t.lookup(w["acg"]) == [0, 4] and t.lookup(w["cgt"]) == [1, 5]          # :144-161
    assert t.lookup(w["gta"]) == [2] and t.lookup(w["tac"]) == [3]
    a = O.Table(O.pack_ascii(b"ACGACGACGACG"), "111", 1)                          # :164-175
    st, pos = a.starts(), a.positions()
    for i in range(a.num_words):
        b = pos[st[i]:st[i + 1]]
        assert all(b[k] < b[k + 1] for k in range(len(b) - 1))
    s16 = O.pack_ascii(b"ACGTACGTACGTACGT")                                       # :177-187
    assert len(O.Table(s16, "111", 3).positions()) < len(O.Table(s16, "111", 1).positions())
    assert O.Table(s16, "111", 3).lookup(w["acg"]) == [0, 12]
    assert O.Table(O.pack_ascii(b"ACGNACG"), "111", 1).lookup(w["acg"]) == [0, 4]  # :190-197
    hot = O.pack_ascii(b"AAAAAAAAAAACG")                                          # :200-211
    assert len(O.Table(hot, "111", 1).lookup(0)) >= 9
    pr = O.Table(hot, "111", 1, max_word_count=4)
    assert pr.lookup(0) == [] and pr.lookup(O.word_at(hot, "111", 10)) == [10]
    m = O.Table(O.pack_ascii(b"ACGTACGTACGT"), "1111", 1)                         # :214-225
    st = m.starts()
    assert np.all(np.diff(st.astype(np.int64)) >= 0) and st[-1] == len(m.positions())


# ---- src/diag_hash.rs:73-102 --------------------------------------------------------
def test_diag_hash():
    assert O.DiagHash().admit(10, 5)
    h = O.DiagHash()
    h.mark_covered(100, 50)
    assert not h.admit(80, 30) and h.admit(200, 150)
    assert h.admit(100, 49)
    g = O.DiagHash()
    g.mark_covered(200, 100)
    g.mark_covered(150, 50)
    assert not g.admit(199, 99) and g.admit(200, 100)


# ---- src/hsp.rs:222-324 -------------------------------------------------------------
def test_extend_hit_known_answers():
    s = O.pack_ascii(b"ACGTACGTACGTACGT")
    h = O.extend_hit(s, s, HOX(xdrop=100, hspthresh=100), 2, 2, 4)               # :222-232
    assert h[0] == 0 and h[1] == 0 and h[2] == 16 and h[3] >= 100
    t, q = O.pack_ascii(b"TTTACGTTTT"), O.pack_ascii(b"AAAACGAAAA")              # :234-245
    assert O.extend_hit(t, q, HOX(xdrop=50, hspthresh=50), 3, 3, 3)[:3] == (3, 3, 3)
    assert O.extend_hit(O.pack_ascii(b"ACGT"), O.pack_ascii(b"TTTT"),            # :247-253
                        HOX(xdrop=100, hspthresh=10000), 0, 0, 4) is None
    a = O.pack_ascii(b"ACGT")                                                     # :255-261
    assert O.extend_hit(a, a, HOX(), 2, 2, 10) is None
    hh = O.extend_hit(O.pack_ascii(b"ACGTACGT"), O.pack_ascii(b"ACNTACGT"),      # :263-271
                      HOX(xdrop=500, hspthresh=200), 4, 4, 4)
    assert hh is not None and hh[2] >= 4
    c = O.pack_ascii(b"CCCCCCAAAAAACCCCCC")                                       # :316-324
    h2 = O.extend_hit(c, c, HOX(xdrop=500, hspthresh=100), 8, 8, 2)
    assert 8 - h2[0] == h2[0] + h2[2] - 10


@pytest.mark.parametrize("seed", [0, 1])
def test_avx2_matches_scalar(seed):
    # The shape of the proptest simd_matches_scalar, src/hsp.rs:283-314.
    if not O.lib().orc_has_avx2():
        pytest.skip("no AVX2 on this host")
    rng = np.random.default_rng(seed)
    for _ in range(200):
        tb = rand_ascii(rng, int(rng.integers(32, 200)), b"ACGTN")
        qb = rand_ascii(rng, int(rng.integers(32, 200)), b"ACGTN")
        L = int(rng.integers(4, 12))
        xd = int(rng.integers(50, 2000))
        T, Q = O.pack_ascii(tb), O.pack_ascii(qb)
        p = HOX(xdrop=xd, hspthresh=0)
        tp, qp = (len(tb) - L) // 2, (len(qb) - L) // 2
        assert O.extend_hit(T, Q, p, tp, qp, L) == O.extend_hit(T, Q, p, tp, qp, L, avx2=True)


# ---- src/seed_search.rs:136-280 -----------------------------------------------------
def search(t, q, pattern, xdrop, thresh, transitions):
    T, Q = O.pack_ascii(t), O.pack_ascii(q)
    h, _ = O.search(O.Table(T, pattern, 1), T, Q, HOX(xdrop=xdrop, hspthresh=thresh, transitions=transitions))
    return [tuple(int(x) for x in r) for r in h]


def test_search_known_answers():
    h = search(b"AAAAAGATTACACATGGCATGAAAAA", b"GATTACACATGGCATG", "1" * 8, 500, 1000, 0)   # :362-387
    assert len(h) == 1 and h[0][:3] == (5, 0, 16)
    assert search(b"AAAAACGTAAAAA", b"ACATA", "1" * 5, 500, 50, 0) == []                 # :389-426
    assert search(b"AAAAACGTAAAAA", b"ACATA", "1" * 5, 500, 50, 1) != []
    assert search(b"AAAAAAAAAA", b"CCCCCCCCCC", "1" * 5, 100, 100, 0) == []              # :428-447
    d = search(b"AAAAAGATTACACATGGCATGTCGAAAAAA", b"GATTACACATGGCATGTCGA", "1" * 7, 500, 500, 0)
    assert len(d) == len({x[0] - x[1] for x in d}) and (5, 0, 20) in [x[:3] for x in d]  # :449-479
    two = search(b"AAAAGATTACACATGGAAAAAAAAAAAAGATTACACATGGTTTTT", b"GATTACACATGG", "1" * 8, 500, 500, 0)
    assert len({x[0] - x[1] for x in two}) >= 2                                          # :481-506


def test_fixture_smoke_hsp_level():
    # tests/fixture_smoke.rs:15-51 (t_start 11, q_start 0, span 20) before gapped extension.
    h = search(b"AAAAAAAAAAAGATTACACATGGCATGTCGAATTTTTTTTTTT", b"GATTACACATGGCATGTCGA", "1" * 12,
               910, 500, 1)
    assert (11, 0, 20) in [x[:3] for x in h]


# ---- src/entropy.rs:72-122 ----------------------------------------------------------
def test_entropy():
    assert abs(O.shannon_entropy(O.pack_ascii(b"ACGTACGTACGTACGT"), 0, 16) - 2.0) < 1e-9
    assert O.shannon_entropy(O.pack_ascii(b"AAAAAAAAAA"), 0, 10) == 0.0
    assert abs(O.shannon_entropy(O.pack_ascii(b"ATATATATAT"), 0, 10) - 1.0) < 1e-9
    s = O.pack_ascii(b"NNNNACGTACGT")
    assert abs(O.shannon_entropy(s, 0, 12) - 2.0) < 1e-9
    assert not O.passes_entropy_gate(O.pack_ascii(b"AAAAAAAAAA"), 0, 10, 10_000, 1_000)
    b = O.pack_ascii(b"ACGTACGTACGT")
    assert O.passes_entropy_gate(b, 0, 12, 1_000, 1_000) and not O.passes_entropy_gate(b, 0, 12, 999, 1_000)
    a = O.pack_ascii(b"ATATATATAT")
    assert not O.passes_entropy_gate(a, 0, 10, 1_000, 1_000) and O.passes_entropy_gate(a, 0, 10, 2_000, 1_000)


# ---- input formats: src/sequences.rs:440-454, src/bit2.rs:321-449 -------------------
from helpers import write_2bit  # noqa: E402


def test_parse_fasta_blank_lines_and_case():
    seqs = O.parse_fasta(b">a\n\nacgt\nACGT\n")                                      # sequences.rs:441-454
    assert len(seqs) == 1 and seqs[0][0] == "a"
    s = O.pack_ascii(seqs[0][1])
    assert to_ascii(s) == b"ACGTACGT"
    assert [masked(s, i) for i in range(8)] == [True] * 4 + [False] * 4


def test_2bit_known_answers():
    with pytest.raises(O.InputError):
        O.parse_2bit(bytes(32))                                                        # bit2.rs:321-325
    for be in (False, True):                                                           # :327-354
        p = O.parse_2bit(write_2bit([("chr1", b"ACGTACGT")], big_endian=be))
        assert p == [("chr1", b"ACGTACGT")]
    assert O.parse_2bit(write_2bit([("chr1", b"ACGTACGTACGT")])) == [("chr1", b"ACGTACGTACGT")]   # :356-364
    multi = [("chrA", b"ACGT"), ("chrB", b"TTTT"), ("chrC", b"GATTACACATG")]          # :366-382
    assert O.parse_2bit(write_2bit(multi)) == multi
    n = O.pack_ascii(O.parse_2bit(write_2bit([("chr1", b"ACGTNNNNACGT")]))[0][1])     # :384-393
    assert to_ascii(n) == b"ACGTNNNNACGT"
    assert not any((int(n.valid[i >> 3]) >> (i & 7)) & 1 for i in range(4, 8))
    mk = O.pack_ascii(O.parse_2bit(write_2bit([("chr1", b"ACGTacgtACGT")]))[0][1])    # :395-412
    assert to_ascii(mk) == b"ACGTACGTACGT"
    assert [masked(mk, i) for i in range(12)] == [False] * 4 + [True] * 4 + [False] * 4
    ov = O.pack_ascii(O.parse_2bit(write_2bit([("chr1", b"ACntACGT")]))[0][1])        # :414-424
    assert not (int(ov.valid[0]) >> 2) & 1 and (int(ov.valid[0]) >> 3) & 1 and masked(ov, 3)
    short = [("chr1", b"A"), ("chr2", b"AC"), ("chr3", b"ACG"), ("chr4", b"ACGT"), ("chr5", b"ACGTA")]
    assert O.parse_2bit(write_2bit(short)) == short                                    # :426-439
    with pytest.raises(O.InputError):                                                  # :441-447
        O.parse_2bit(write_2bit([("chr1", b"ACGT")])[:-2])


# ---- HSP consumers: src/chain.rs:78-138, src/anchor.rs:79-126 --------------------------
def test_best_chain_known_answers():
    h = lambda t, q, l, s: (t, q, l, s)  # noqa: E731
    assert O.best_chain([]) == []                                                         # chain.rs:79-82
    assert O.best_chain([h(10, 20, 30, 1000)]) == [h(10, 20, 30, 1000)]                   # :84-88
    a, b, c = h(0, 0, 20, 500), h(40, 40, 20, 500), h(80, 10, 20, 700)                    # :90-105
    assert O.best_chain([a, b, c]) == [a, b]
    a, b, c, d = h(0, 0, 10, 100), h(20, 20, 10, 100), h(40, 40, 10, 100), h(60, 60, 10, 500)
    assert O.best_chain([a, b, c, d]) == [a, b, c, d]                                     # :107-117
    a, b = h(0, 50, 10, 1000), h(20, 0, 10, 800)                                          # :119-128
    assert O.best_chain([a, b]) == [a]
    a, b = h(10, 10, 5, 100), h(0, 0, 5, 100)                                             # :130-137
    assert O.best_chain([a, b]) == [b, a]


def test_choose_anchor_known_answers():
    sub = [row[:] for row in HOXD70_ROWS]
    s = O.pack_ascii(b"ACGTACGTACGTACGT")                                                 # anchor.rs:79-88
    assert O.choose_anchor((0, 0, 16, 0), s, s, sub, -100, 4) == (2, 2)
    t, q = O.pack_ascii(b"AACCCCAA"), O.pack_ascii(b"TTCCCCTT")                           # :90-102
    assert O.choose_anchor((0, 0, 8, 0), t, q, sub, -100, 4) == (4, 4)
    a = O.pack_ascii(b"ACGT")                                                             # :104-110
    assert O.choose_anchor((0, 0, 4, 0), a, a, sub, -100, 1000)[0] == 2


HOXD70_ROWS = [[91, -114, -31, -123], [-114, 100, -125, -31], [-31, -125, 100, -114], [-123, -31, -114, 91]]


def test_driver_records_order_dedup_and_filter():
    """The driver's record post-processing (src/driver.rs:250-256, :370-391,
    :437-468): primary filter, global t, per-unit sort by (t, q, t_span,
    q_span) and keep-first dedup, units in (target, query, strand) order."""
    import oracle as O
    entries = [
        # (ti, qi, strand, chunk_start, plo, phi, hsps (t, q, len, score))
        (0, 0, 1, 0, 0, 100, [(5, 7, 20, 3100)]),
        (0, 0, 0, 100, 10, 60, [(30, 2, 20, 3200), (10, 1, 20, 3000), (9, 0, 20, 9999), (60, 0, 20, 9999),
                                 (10, 1, 20, 3000), (10, 1, 21, 3050)]),
        (0, 0, 0, 0, 0, 50, [(40, 3, 20, 3300)]),
        (1, 0, 0, 0, 0, 100, []),
    ]
    got = O.driver_records(entries)
    assert got == [
        # (0,0,0): the chunk at 100 first (it completed first), then the chunk at 0
        (0, 0, 0, 110, 1, 20, 3000), (0, 0, 0, 110, 1, 21, 3050), (0, 0, 0, 130, 2, 20, 3200),
        (0, 0, 0, 40, 3, 20, 3300),
        (0, 0, 1, 5, 7, 20, 3100),
    ]


def test_driver_records_chunk_order_equals_one_sort_per_group():
    """With chunks completing in target order, the reference's per-unit sort
    and concatenation equals one sort of each (target, query, strand) group:
    primary regions are disjoint and ascending, so no record crosses a chunk
    boundary.  This is the order gxy_batch_records produces."""
    import random
    import oracle as O
    rng = random.Random(5)
    primary, halo, tlen = 1000, 150, 4500
    chunks = []
    ps = 0
    while ps < tlen:
        pe = min(ps + primary, tlen)
        lo, hi = max(ps - halo, 0), min(pe + halo, tlen)
        chunks.append((lo, hi, ps - lo, pe - lo))
        ps = pe
    entries = []
    for lo, hi, plo, phi in chunks:
        for strand in (0, 1):
            # Equal coordinates carry equal scores, as extensions of the same columns do.
            hs = []
            for _ in range(40):
                t, q, ln = rng.randrange(0, hi - lo), rng.randrange(0, 3000), rng.randrange(19, 60)
                hs.append((t, q, ln, 3000 + (t * 7 + q * 3 + ln) % 6000))
            hs += hs[:5]   # repeats
            entries.append((0, 0, strand, lo, plo, phi, hs))
    got = O.driver_records(entries)
    want = []
    for strand in (0, 1):
        recs = set()
        for ti, qi, sd, lo, plo, phi, hs in entries:
            if sd != strand:
                continue
            for t, q, ln, sc in hs:
                if plo <= t < phi:
                    recs.add((t + lo, q, ln, sc))
        want.extend((0, 0, strand, t, q, ln, sc) for t, q, ln, sc in sorted(recs))
    assert got == want


# ---- src/gapped_extend.rs:462-602 (gapped extension) ---------------------------------
def _gx(t: bytes, q: bytes, hsp_t: int, hsp_q: int, offset: int, y_drop: int, thr: int):
    # anchor_from_hsp (:470-476): the anchor sits `offset` columns into the HSP.
    T, Q = O.pack_ascii(t), O.pack_ascii(q)
    return O.gapped_extend(T, Q, HOX(), O.gapped_params(y_drop=y_drop, gapped_threshold=thr),
                           hsp_t + offset, hsp_q + offset)


def _spans(runs):
    tsp = sum(r >> 2 for r in runs if (r & 3) in (0, 2))
    qsp = sum(r >> 2 for r in runs if (r & 3) in (0, 1))
    return tsp, qsp


def test_gapped_perfect_match_stays_ungapped():   # :478-490
    s = b"ACGTACGTACGTACGT"
    a = _gx(s, s, 0, 0, 8, 500, 100)
    assert (a["t_start"], a["q_start"], a["t_len"], a["q_len"]) == (0, 0, 16, 16)
    assert O.cigar(a["runs"]) == "16M"


def test_gapped_single_insertion_is_recovered():   # :492-510
    a = _gx(b"ACGTACGTACGT", b"ACGTACGGTACGT", 0, 0, 3, 1000, 100)
    assert a["t_len"] == 12 and a["q_len"] == 13
    assert "1I" in O.cigar(a["runs"])
    assert _spans(a["runs"]) == (12, 13)


def test_gapped_single_deletion_is_recovered():   # :512-525
    a = _gx(b"ACGTACGGTACGT", b"ACGTACGTACGT", 0, 0, 3, 1000, 100)
    assert a["t_len"] == 13 and a["q_len"] == 12
    assert "1D" in O.cigar(a["runs"])


def test_gapped_below_threshold_returns_none():   # :527-534
    assert _gx(b"ACGT", b"ACGT", 0, 0, 1, 500, 100_000) is None


def test_gapped_extension_stops_at_diverging_tail():   # :536-550
    a = _gx(b"TTTTTTTTACGTACGTACGTACGTACGTACGTTTTTTTTT", b"AAAAAAAAACGTACGTACGTACGTACGTACGTAAAAAAAA",
            8, 8, 12, 300, 500)
    assert 24 <= a["t_len"] <= 32


def test_gapped_banded_dp_accommodates_large_gap():   # :552-585
    core = b"GATTACACATGGCATGTCGAATGCCTAGCATGTCA"
    t = core + core
    q = core + b"AGCTAGCTAGCTAGCTAGCTAGCTAGCTAGCTAGCTAGCTAGCTAGCTAG" + core
    a = _gx(t, q, 0, 0, 5, 9400, 500)
    assert a["t_len"] >= 60 and a["q_len"] >= 110
    assert "I" in O.cigar(a["runs"])


def test_gapped_script_spans_equal_reported_lengths():   # :587-600
    a = _gx(b"AAAGATTACACATGGCATGTCGATTTT", b"GATACACATGGCAGTCGA", 3, 0, 3, 5000, 100)
    assert _spans(a["runs"]) == (a["t_len"], a["q_len"])


def test_gapped_many_threads_equals_one():
    # The threaded batch form is the same function per anchor.
    rng = np.random.default_rng(5)
    t = rand_ascii(rng, 3000, b"ACGT")
    q = bytearray(t)
    for i in rng.choice(len(q), 300, replace=False):
        q[i] = b"ACGT"[rng.integers(4)]
    q = bytes(q[:1500] + q[1510:])
    T, Q = O.pack_ascii(t), O.pack_ascii(q)
    tp = rng.integers(0, 1400, 40)
    qp = tp + rng.integers(-3, 3, 40).clip(0)
    gp = O.gapped_params(gapped_threshold=0)
    many = O.gapped_extend_many(T, Q, HOX(), gp, tp, qp, threads=4)
    one = [O.gapped_extend(T, Q, HOX(), gp, int(a), int(b)) for a, b in zip(tp, qp)]
    assert many == one
    assert any(a is not None for a in many)


def _py_extend(t: bytes, q: bytes, tp: int, qp: int, go: int, ge: int, ydrop: int, thr: int, cells_out=None):
    """A second, direct restatement of extend() (src/gapped_extend.rs:78-132,
    :178-460) with the reference's up-front (n+1) x band_width storage, for
    small cases: checks the C oracle's on-demand rows and run merging."""
    sub = [[91, -114, -31, -123], [-114, 100, -125, -31], [-31, -125, 100, -114], [-123, -31, -114, 91]]
    enc = {ord(c): i for i, c in enumerate("ACGT")}
    enc.update({ord(c): i for i, c in enumerate("acgt")})
    NEG = -(2 ** 31) // 4

    def pair(a, b):
        return sub[enc[a]][enc[b]] if a in enc and b in enc else -100

    ncells = [0]

    def one_side(T, Q):
        n, m = len(T), len(Q)
        if n == 0 or m == 0:
            return 0, 0, 0, []
        goe = go + ge
        radius = (max(int((ydrop - goe) / ge), 0) + 2) if ge > 0 else m + 1
        bw = min(4 * radius + 4, m + 1)
        row_lo = [0] * (n + 1)
        size = (n + 1) * bw
        mm, xx, yy = [NEG] * size, [NEG] * size, [NEG] * size
        mf, xf, yf = [0] * size, [0] * size, [0] * size
        mm[0] = 0
        best_score, best_cell = 0, (0, 0, 0)
        lo = hi = 0
        for i in range(n + 1):
            j_lo = max(lo - radius, 0)
            j_hi = min(hi + radius, m, j_lo + bw - 1)
            row_lo[i] = j_lo
            ncells[0] += j_hi - j_lo + 1
            lo_prev = row_lo[i - 1] if i >= 1 else 0
            for j in range(j_lo, j_hi + 1):
                if i == 0 and j == 0:
                    continue
                best = NEG
                here = i * bw + (j - j_lo)
                inb = lambda jj: lo_prev <= jj < lo_prev + bw
                if i >= 1:
                    pm, px = (mm[(i - 1) * bw + j - lo_prev], xx[(i - 1) * bw + j - lo_prev]) if inb(j) else (NEG, NEG)
                    fm, fx = pm - goe, px - ge
                    xx[here], xf[here] = (fm, 0) if fm >= fx else (fx, 1)
                    best = max(best, xx[here])
                if j >= 1:
                    pm, py = (mm[here - 1], yy[here - 1]) if j - 1 >= j_lo else (NEG, NEG)
                    fm, fy = pm - goe, py - ge
                    yy[here], yf[here] = (fm, 0) if fm >= fy else (fy, 2)
                    best = max(best, yy[here])
                if i >= 1 and j >= 1:
                    s = pair(T[i - 1], Q[j - 1])
                    o = (i - 1) * bw + j - 1 - lo_prev
                    fm, fx, fy = (mm[o], xx[o], yy[o]) if inb(j - 1) else (NEG, NEG, NEG)
                    if fm >= fx and fm >= fy:
                        prev, fr = fm, 0
                    elif fx >= fy:
                        prev, fr = fx, 1
                    else:
                        prev, fr = fy, 2
                    mm[here], mf[here] = prev + s, fr
                    best = max(best, mm[here])
                if best > best_score:
                    best_score = best
                    st = 0 if mm[here] == best else (1 if xx[here] == best else 2)
                    best_cell = (i, j, st)
            thr_ = best_score - ydrop
            new_lo, new_hi = None, 0
            for j in range(j_lo, j_hi + 1):
                h = i * bw + (j - j_lo)
                if max(mm[h], xx[h], yy[h]) >= thr_:
                    new_lo = j if new_lo is None else new_lo
                    new_hi = j
                else:
                    mm[h] = xx[h] = yy[h] = NEG
            if new_lo is None:
                break
            lo, hi = new_lo, new_hi
        i, j, st = best_cell
        ops = []
        while i > 0 or j > 0:
            h = i * bw + (j - row_lo[i])
            if st == 0:
                ops.append(0); st = mf[h]; i -= 1; j -= 1
            elif st == 1:
                ops.append(2); st = xf[h]; i -= 1
            else:
                ops.append(1); st = yf[h]; j -= 1
        return best_score, best_cell[0], best_cell[1], ops[::-1]

    R = one_side(t[tp + 1:], q[qp + 1:])
    L = one_side(t[:tp][::-1], q[:qp][::-1])
    total = pair(t[tp], q[qp]) + L[0] + R[0]
    if cells_out is not None:
        cells_out.append(ncells[0])
    if total < thr:
        return None
    ops = L[3][::-1] + [0] + R[3]
    runs = []
    for op in ops:
        if runs and (runs[-1] & 3) == op:
            runs[-1] += 4
        else:
            runs.append(4 | op)
    return {"t_start": tp - L[1], "q_start": qp - L[2], "t_len": L[1] + 1 + R[1], "q_len": L[2] + 1 + R[2],
            "score": total, "runs": runs}


@pytest.mark.parametrize("go,ge,ydrop", [(400, 30, 9400), (400, 30, 300), (400, 30, 1200), (0, 30, 700), (400, 0, 500),
                                         (50, 5, 2000)])
def test_gapped_c_oracle_equals_direct_restatement(go, ge, ydrop):
    rng = np.random.default_rng(go + ge + ydrop)
    for case in range(12):
        n = int(rng.integers(1, 160))
        t = bytearray(rand_ascii(rng, n, b"ACGTACGTacgtN"))
        q = bytearray(t)
        for _ in range(int(rng.integers(0, 6))):   # indels and substitutions
            k = int(rng.integers(0, len(q)))
            r = rng.integers(3)
            if r == 0:
                q[k:k] = rand_ascii(rng, int(rng.integers(1, 9)), b"ACGT")
            elif r == 1:
                del q[k:k + int(rng.integers(1, 9))]
            else:
                q[k] = b"ACGTN"[rng.integers(5)]
        if not q:
            q = bytearray(b"A")
        t, q = bytes(t), bytes(q)
        tp, qp = int(rng.integers(0, len(t))), int(rng.integers(0, len(q)))
        pc = []
        want = _py_extend(t, q, tp, qp, go, ge, ydrop, -10 ** 6, pc)
        got = O.gapped_extend(O.pack_ascii(t), O.pack_ascii(q), HOX(),
                              O.gapped_params(go, ge, ydrop, -10 ** 6), tp, qp)
        assert got == want, (case, t, q, tp, qp)
        cc = []
        O.gapped_extend_many(O.pack_ascii(t), O.pack_ascii(q), HOX(), O.gapped_params(go, ge, ydrop, -10 ** 6),
                             [tp], [qp], cells=cc)
        assert cc == pc   # the DP cells: the band widths summed over the rows of both sides
