"""GPU parity: the CUDA path against the oracle, bit for bit.

Shapes follow the reference's own tests (src/seed_search.rs:137-280,
src/pos_table.rs:139-225, src/hsp.rs:213-324, tests/fixture_smoke.rs) plus the
seeded synthetic workloads."""
import zlib

import numpy as np
import pytest

import oracle as O
from helpers import as_tuples, homologous_pair, oracle_search, oracle_seq, orc_params, rand_ascii

pytestmark = pytest.mark.gpu

P12 = "1110100110010101111"


def gpu_search(gxy, ctx, target: bytes, query: bytes, pattern, sp, matrix=None, max_word_count=0, stats=None):
    matrix = matrix or gxy.ScoringMatrix.hoxd70()
    T = gxy.PackedSeq.from_ascii(target)
    Q = gxy.PackedSeq.from_ascii(query)
    tab = gxy.PosTable.build(T, pattern, sp.step, ctx=ctx)
    if max_word_count:
        tab.prune_hot_words(max_word_count)
    return gxy.search(tab, T, Q, matrix, sp, stats=stats)


def both(gxy, ctx, target, query, pattern, sp, matrix=None, max_word_count=0):
    matrix = matrix or gxy.ScoringMatrix.hoxd70()
    g = gpu_search(gxy, ctx, target, query, pattern, sp, matrix, max_word_count)
    o, _ = oracle_search(target, query, pattern, matrix, sp, max_word_count)
    return as_tuples(g), as_tuples(o)


# ---- known answers of src/seed_search.rs:137-280 --------------------------------
def test_exact_match_coordinates(gxy, ctx):
    sp = gxy.SearchParams(1, gxy.HspParams(500, 1000), 0)
    g, o = both(gxy, ctx, b"AAAAAGATTACACATGGCATGAAAAA", b"GATTACACATGGCATG", "1" * 8, sp)
    assert g == o
    assert len(g) == 1 and g[0][:3] == (5, 0, 16)


def test_transition_variants(gxy, ctx):
    hp = gxy.HspParams(500, 50)
    g0, o0 = both(gxy, ctx, b"AAAAACGTAAAAA", b"ACATA", "1" * 5, gxy.SearchParams(1, hp, 0))
    g1, o1 = both(gxy, ctx, b"AAAAACGTAAAAA", b"ACATA", "1" * 5, gxy.SearchParams(1, hp, 1))
    assert g0 == o0 == []
    assert g1 == o1 and len(g1) > 0


def test_no_match(gxy, ctx):
    g, o = both(gxy, ctx, b"AAAAAAAAAA", b"CCCCCCCCCC", "1" * 5, gxy.SearchParams(1, gxy.HspParams(100, 100), 0))
    assert g == o == []


def test_diag_collapse(gxy, ctx):
    sp = gxy.SearchParams(1, gxy.HspParams(500, 500), 0)
    g, o = both(gxy, ctx, b"AAAAAGATTACACATGGCATGTCGAAAAAA", b"GATTACACATGGCATGTCGA", "1" * 7, sp)
    assert g == o
    assert (5, 0, 20) in [x[:3] for x in g]
    assert len({x[0] - x[1] for x in g}) == len(g)


def test_two_diagonals(gxy, ctx):
    sp = gxy.SearchParams(1, gxy.HspParams(500, 500), 0)
    g, o = both(gxy, ctx, b"AAAAGATTACACATGGAAAAAAAAAAAAGATTACACATGGTTTTT", b"GATTACACATGG", "1" * 8, sp)
    assert g == o and len({x[0] - x[1] for x in g}) >= 2


def test_fixture_tiny(gxy, ctx):
    # tests/fixture_smoke.rs:15-51 at the HSP level: t_start 11, span 20.
    sp = gxy.SearchParams(1, gxy.HspParams(910, 500), 1)
    g, o = both(gxy, ctx, b"AAAAAAAAAAAGATTACACATGGCATGTCGAATTTTTTTTTTT", b"GATTACACATGGCATGTCGA", "1" * 12, sp)
    assert g == o
    assert (11, 0, 20) in [x[:3] for x in g]


# ---- table build (src/pos_table.rs) -------------------------------------------
@pytest.mark.parametrize("pattern,step,mwc", [("111", 1, 0), ("1111", 1, 0), ("111", 3, 0), ("1101", 2, 0),
                                               (P12, 1, 0), (P12, 3, 0), ("111", 1, 4), (P12, 1, 2),
                                               ("11111111101111111111"[:14], 1, 0)])
def test_table_bit_exact(gxy, ctx, pattern, step, mwc):
    rng = np.random.default_rng(zlib.crc32(f"{pattern}/{step}/{mwc}".encode()))
    s = rand_ascii(rng, 20000, b"ACGTACGTacgtN", None) + b"AAAAAAAAAAAAAAAAAAAAAAAACG"
    T = gxy.PackedSeq.from_ascii(s)
    tab = gxy.PosTable.build(T, pattern, step, ctx=ctx)
    if mwc:
        tab.prune_hot_words(mwc)
    starts, pos = tab.arrays()
    ot = O.Table(O.pack_ascii(s), pattern, step, mwc)
    assert np.array_equal(starts, ot.starts())
    assert np.array_equal(pos, ot.positions())


# The build is a stable radix sort of the windows by word, so every bucket
# holds its positions in ascending order straight from the build -- small
# buckets, buckets of thousands (a poly-A run, a tandem repeat) -- against the
# oracle, after a search on the same table.
@pytest.mark.parametrize("pattern,step", [("111", 1), ("11011", 1), (P12, 1), ("111", 2)])
def test_table_bucket_orders(gxy, ctx, pattern, step):
    rng = np.random.default_rng(7 + step + len(pattern))
    s = (rand_ascii(rng, 30000, b"ACGTacgtN", None) + b"A" * 13000 + b"ACGTT" * 900 +
         rand_ascii(rng, 5000, b"ACGT", None))
    T = gxy.PackedSeq.from_ascii(s)
    tab = gxy.PosTable.build(T, pattern, step, ctx=ctx)
    q = s[2000:12000]   # random part: few raw hits even for the dense patterns
    sp = gxy.SearchParams(step, gxy.HspParams(910, 3000), 1)
    got = gxy.search(tab, T, gxy.PackedSeq.from_ascii(q), gxy.ScoringMatrix.hoxd70(), sp)
    starts, pos = tab.arrays()
    ot = O.Table(O.pack_ascii(s), pattern, step)
    assert np.array_equal(starts, ot.starts())
    assert np.array_equal(pos, ot.positions())
    assert int(np.diff(starts.astype(np.int64)).max()) > 4096
    want, _ = O.search(ot, O.pack_ascii(s), O.pack_ascii(q), orc_params(gxy.ScoringMatrix.hoxd70(), sp))
    assert as_tuples(got) == as_tuples(want) and len(want) > 0
    # A query inside the tandem repeat: its windows hit buckets of hundreds
    # of positions (the warp-cooperative copy in the enumeration).
    q2 = s[43000 + 100:43000 + 400] + s[3000:3300]
    got2 = gxy.search(tab, T, gxy.PackedSeq.from_ascii(q2), gxy.ScoringMatrix.hoxd70(), sp)
    want2, _ = O.search(ot, O.pack_ascii(s), O.pack_ascii(q2), orc_params(gxy.ScoringMatrix.hoxd70(), sp))
    assert as_tuples(got2) == as_tuples(want2) and len(want2) > 0


def test_table_bucket_size_classes(gxy, ctx):
    # Random 40 bp units each repeated k times (k = 2 .. 5000) between random
    # spacers: buckets of every size class the build orders differently
    # (2-3 in place, 4-32 a warp, 33-4096 a block, larger the radix sort),
    # one table and as views, against the oracle.
    rng = np.random.default_rng(12)
    parts = []
    for k in (2, 3, 4, 5, 9, 16, 31, 32, 33, 40, 100, 1000, 4096, 4097, 5000):
        unit = rand_ascii(rng, 40, b"ACGT", None)
        parts.append(rand_ascii(rng, 300, b"ACGT", None) + unit * k)
    s = b"".join(parts)
    T = gxy.PackedSeq.from_ascii(s)
    tab = gxy.PosTable.build(T, P12, 1, ctx=ctx)
    starts, pos = tab.arrays()
    ot = O.Table(O.pack_ascii(s), P12, 1)
    assert np.array_equal(starts, ot.starts()) and np.array_equal(pos, ot.positions())
    assert int(np.diff(starts.astype(np.int64)).max()) > 4096
    tab.free()
    dT = T.to_device(ctx)
    half = len(s) // 2
    views = gxy.PosTable.build_views(dT, [(0, half), (half - 1000, len(s))], P12, 1, ctx=ctx)
    for (lo, hi), t in zip([(0, half), (half - 1000, len(s))], views):
        st2, p2 = t.arrays()
        o2 = O.Table(O.pack_ascii(s[lo:hi]), P12, 1)
        assert np.array_equal(st2, o2.starts()) and np.array_equal(p2, o2.positions()), (lo, hi)
        t.free()
    dT.free()


def test_table_full_size_bit_exact(gxy, ctx):
    # A 10 Mbp chromosome-style target (repeat families, soft-masked runs,
    # N blocks), 12of19 and step 1, and a 2 Mbp target at step 2: starts and
    # positions equal the reference's stable scatter, bucket order included.
    from lastz_gxy_b200 import synth
    for n, step in ((10_000_000, 1), (2_000_000, 2)):
        s = synth.chromosome(np.random.default_rng(n + step), n, families=n // 5000, nblocks=20).tobytes()
        T = gxy.PackedSeq.from_ascii(s)
        tab = gxy.PosTable.build(T, P12, step, ctx=ctx)
        starts, pos = tab.arrays()
        ot = O.Table(O.pack_ascii(s), P12, step)
        assert np.array_equal(starts, ot.starts())
        assert np.array_equal(pos, ot.positions())
        assert int(np.diff(starts.astype(np.int64)).max()) > 5
        tab.free()


@pytest.mark.parametrize("mwc", [0, 3])
def test_table_build_views(gxy, ctx, mwc):
    # Overlapping chunk views of one device sequence (chunk_target's shape,
    # src/driver.rs:156-194), an empty view and one shorter than the pattern,
    # built by one sort: each equals its own build_view and the oracle's
    # table of the sliced chunk; freeing them in any order leaves the rest
    # intact.
    from lastz_gxy_b200 import synth
    s = synth.chromosome(np.random.default_rng(41), 3_000_000, families=600, nblocks=4).tobytes()
    dT = gxy.PackedSeq.from_ascii(s).to_device(ctx)
    ranges = [(lo, hi) for lo, hi, _, _ in gxy.chunk_target(len(s), 400_000, 20_000)]
    ranges += [(1000, 1000), (5000, 5010), (0, len(s))]
    tabs = gxy.PosTable.build_views(dT, ranges, P12, 1, mwc, ctx=ctx)
    assert len(tabs) == len(ranges)
    gone = (3, 0, len(ranges) - 1)
    for i in gone:
        tabs[i].free()
    for i, ((lo, hi), t) in enumerate(zip(ranges, tabs)):
        if i in gone:
            continue
        starts, pos = t.arrays()
        one = gxy.PosTable.build_view(dT, lo, hi, P12, 1, mwc, ctx=ctx)
        s1, p1 = one.arrays()
        one.free()
        assert np.array_equal(starts, s1) and np.array_equal(pos, p1), (lo, hi)
        if i in (1, len(ranges) - 3, len(ranges) - 2):
            ot = O.Table(O.pack_ascii(s[lo:hi]), P12, 1, mwc)
            assert np.array_equal(starts, ot.starts()) and np.array_equal(pos, ot.positions()), (lo, hi)
        t.free()
    dT.free()


def test_tiny_weight_tables(gxy, ctx):
    # Weight 1 and 2 (4 and 16 words): every bucket is large.
    rng = np.random.default_rng(5)
    t, q = homologous_pair(rng, 3000, 0.9)
    for pattern in ("1", "101", "11"):
        sp = gxy.SearchParams(1, gxy.HspParams(910, 300), 0)
        g, o = both(gxy, ctx, t, q, pattern, sp)
        assert g == o, pattern


def test_table_known_buckets(gxy, ctx):
    # src/pos_table.rs:144-161, :177-187, :190-197, :200-211
    T = gxy.PackedSeq.from_ascii(b"ACGTACGT")
    tab = gxy.PosTable.build(T, "111", 1, ctx=ctx)
    acg = O.word_at(O.pack_ascii(b"ACGTACGT"), "111", 0)
    assert list(tab.lookup(acg)) == [0, 4]
    tab3 = gxy.PosTable.build(gxy.PackedSeq.from_ascii(b"ACGTACGTACGTACGT"), "111", 3, ctx=ctx)
    assert list(tab3.lookup(acg)) == [0, 12]
    tabn = gxy.PosTable.build(gxy.PackedSeq.from_ascii(b"ACGNACG"), "111", 1, ctx=ctx)
    assert list(tabn.lookup(acg)) == [0, 4]
    tp = gxy.PosTable.build(gxy.PackedSeq.from_ascii(b"AAAAAAAAAAACG"), "111", 1, ctx=ctx)
    assert len(tp.lookup(0)) >= 9
    tp.prune_hot_words(4)
    assert len(tp.lookup(0)) == 0
    assert list(tp.lookup(acg)) == [10]


# ---- packing ------------------------------------------------------------------
@pytest.mark.parametrize("n", [0, 1, 7, 31, 32, 33, 100, 4096, 100003])
def test_pack_and_revcomp(gxy, ctx, n):
    rng = np.random.default_rng(n)
    s = rand_ascii(rng, n, b"ACGTUacgtuNnRYx-", None)
    d = gxy.DeviceSeq.from_ascii(s, ctx=ctx)
    h = d.to_host()
    o = O.pack_ascii(s)
    nb4, nb8 = (n + 3) // 4, (n + 7) // 8
    assert bytes(h.codes[:nb4]) == bytes(o.codes[:nb4])
    assert bytes(h.valid[:nb8]) == bytes(o.valid[:nb8])
    assert bytes(h.mask[:nb8]) == bytes(o.mask[:nb8])
    r = d.reverse_complement().to_host()
    orr = O.reverse_complement(o)
    assert bytes(r.codes[:nb4]) == bytes(orr.codes[:nb4])
    assert bytes(r.valid[:nb8]) == bytes(orr.valid[:nb8])
    assert bytes(r.mask[:nb8]) == bytes(orr.mask[:nb8])


# ---- x-drop differential, the shape of src/hsp.rs:283-314 ------------------------
@pytest.mark.parametrize("mode", [0, 1])
def test_extend_matches_scalar(gxy, ctx, mode):
    rng = np.random.default_rng(283 + mode)
    m = gxy.ScoringMatrix.hoxd70()
    for case in range(200):
        tb = rand_ascii(rng, int(rng.integers(32, 200)), b"ACGTN")
        qb = rand_ascii(rng, int(rng.integers(32, 200)), b"ACGTN")
        L = int(rng.integers(4, 12))
        xd = int(rng.integers(50, 2000))
        tmax, qmax = len(tb) - L, len(qb) - L
        tp, qp = tmax // 2, qmax // 2
        T = gxy.DeviceSeq.from_ascii(tb, ctx=ctx)
        Q = gxy.DeviceSeq.from_ascii(qb, ctx=ctx)
        h, ok = gxy.extend_hits(T, Q, m, gxy.HspParams(xd, 0), [tp], [qp], L, mode)
        o = O.extend_hit(O.pack_ascii(tb), O.pack_ascii(qb), O.params(xdrop=xd, hspthresh=0), tp, qp, L)
        got = (int(h[0]["t_start"]), int(h[0]["q_start"]), int(h[0]["length"]), int(h[0]["score"])) if ok[0] else None
        assert got == o, (case, tb, qb, L, xd)


def test_extend_long_homology(gxy, ctx):
    # Long extensions cross many 32-column steps and warp stage refills.
    rng = np.random.default_rng(5)
    m = gxy.ScoringMatrix.hoxd70()
    for ident in (1.0, 0.97, 0.9, 0.8):
        t, q = homologous_pair(rng, 6000, ident)
        L = 12
        n = min(len(t), len(q)) - L
        tp = rng.integers(0, n, 64)
        T, Q = gxy.DeviceSeq.from_ascii(t, ctx=ctx), gxy.DeviceSeq.from_ascii(q, ctx=ctx)
        OT, OQ = O.pack_ascii(t), O.pack_ascii(q)
        for mode in (0, 1):
            h, ok = gxy.extend_hits(T, Q, m, gxy.HspParams(910, 0), tp, tp, L, mode)
            for i in range(len(tp)):
                o = O.extend_hit(OT, OQ, O.params(xdrop=910, hspthresh=0), int(tp[i]), int(tp[i]), L)
                got = tuple(int(h[i][k]) for k in ("t_start", "q_start", "length", "score")) if ok[i] else None
                assert got == o


# ---- whole searches -------------------------------------------------------------
@pytest.mark.parametrize("seed,transitions,step,lower,nfrac", [(1, 1, 1, 0.0, 0.0), (2, 0, 1, 0.2, 0.01),
                                                                (3, 2, 1, 0.1, 0.0), (4, 1, 3, 0.0, 0.02),
                                                                (5, 1, 2, 0.3, 0.005)])
def test_random_homology(gxy, ctx, seed, transitions, step, lower, nfrac):
    rng = np.random.default_rng(seed)
    t, q = homologous_pair(rng, 40000, 0.8, lower=lower, nfrac=nfrac)
    sp = gxy.SearchParams(step, gxy.HspParams(910, 3000), transitions)
    g, o = both(gxy, ctx, t, q, P12, sp)
    assert g == o
    assert len(o) > 0


# The screen packs a side's run and extent into one i32 when scores, x-drop
# and the column cap allow it, else it runs the unpacked kernel: both must
# equal the oracle, on both sides of each bound.
@pytest.mark.parametrize("scale,xdrop,thresh,cap", [
    (1, 0, 300, 0),                 # x-drop 0: breaks on the first non-improving column
    (1, 1, 300, 0),
    (1, 910, 3000, 192),            # largest packed cap
    (1, 910, 3000, 224),            # cap above the packed bound
    (131, 910 * 131, 3000 * 131, 0),   # |score| 16375: packed
    (132, 910 * 132, 3000 * 132, 0),   # |score| 16500: unpacked
    (1, 1 << 22, 3000, 0),          # largest packed x-drop
    (1, (1 << 22) + 1, 3000, 0),    # unpacked
    (1, -1, 200, 0),                # negative x-drop: unpacked
])
def test_screen_envelopes(gxy, scale, xdrop, thresh, cap):
    rng = np.random.default_rng(91)
    t, q = homologous_pair(rng, 30000, 0.8, lower=0.05, nfrac=0.003)
    base = gxy.ScoringMatrix.hoxd70()
    m = gxy.ScoringMatrix(sub=[[v * scale for v in row] for row in base.sub], ambig_score=base.ambig_score * scale)
    sp = gxy.SearchParams(1, gxy.HspParams(xdrop, thresh), 1)
    c2 = gxy.Context(0)
    try:
        if cap:
            c2.set_tuning(screen_cap=cap)
        g, o = both(gxy, c2, t, q, P12, sp, matrix=m)
    finally:
        c2.close()
    assert g == o
    assert len(o) > 0


def test_entropy_gate(gxy, ctx):
    rng = np.random.default_rng(11)
    t, q = homologous_pair(rng, 30000, 0.85)
    t = t + b"ATATATATATATATATATATATATATATATATATATATATATATATATATATATAT" * 4
    q = q + b"ATATATATATATATATATATATATATATATATATATATATATATATATATATATAT" * 4
    sp = gxy.SearchParams(1, gxy.HspParams(910, 2000), 1, entropy_threshold=2500)
    g, o = both(gxy, ctx, t, q, P12, sp)
    assert g == o


@pytest.mark.parametrize("thr", [500, 2200, 5000])
def test_entropy_gate_thresholds(gxy, ctx, thr):
    # The gate (src/entropy.rs:27-67, applied at src/seed_search.rs:102-112)
    # decides which passing HSPs set the diagonal's cover, so it changes which
    # later hits are admitted: sequences mixing random stretches with di- and
    # tri-nucleotide repeats and homopolymer runs (entropies from 0 to 2 bits)
    # at a sweep of thresholds, in f64 on both sides.
    rng = np.random.default_rng(40 + thr)
    parts_t, parts_q = [], []
    for k in range(24):
        kind = k % 4
        if kind == 0:
            t, q = homologous_pair(rng, 1500, 0.9)
        else:
            unit = [b"AT", b"CAG", b"A", b"GC"][int(rng.integers(4))] if kind != 3 else b"ACGTTGCA"
            t = (unit * (900 // len(unit) + 1))[:900]
            q = bytearray(t)
            for i in rng.choice(len(q), 30, replace=False):
                q[i] = b"ACGT"[rng.integers(4)]
            q = bytes(q)
        parts_t.append(t)
        parts_q.append(q)
    t, q = b"".join(parts_t), b"".join(parts_q)
    sp = gxy.SearchParams(1, gxy.HspParams(910, 1500), 1, entropy_threshold=thr)
    g, o = both(gxy, ctx, t, q, P12, sp)
    assert g == o
    assert len(o) > 0


def test_max_word_count(gxy, ctx):
    rng = np.random.default_rng(12)
    t, q = homologous_pair(rng, 30000, 0.85)
    sp = gxy.SearchParams(1, gxy.HspParams(910, 3000), 1)
    g, o = both(gxy, ctx, t, q, P12, sp, max_word_count=1)
    assert g == o


def test_edge_cases(gxy, ctx):
    sp = gxy.SearchParams(1, gxy.HspParams(910, 100), 1)
    cases = [(b"ACGT" * 10, b""), (b"ACGT" * 10, b"ACG"), (b"", b"ACGT" * 10), (b"N" * 500, b"N" * 500),
             (b"acgt" * 200, b"ACGT" * 200), (b"ACGTACGTACGTACGTACG", b"ACGTACGTACGTACGTACG")]
    for t, q in cases:
        g, o = both(gxy, ctx, t, q, P12, sp)
        assert g == o, (t[:20], q[:20])


def test_c1_both_strands(gxy, ctx):
    from lastz_gxy_b200 import synth
    pr = synth.c1()
    t, q = pr.target.tobytes(), pr.query.tobytes()
    sp = gxy.SearchParams()
    T = gxy.PackedSeq.from_ascii(t)
    Q = gxy.PackedSeq.from_ascii(q)
    tab = gxy.PosTable.build(T, P12, 1, ctx=ctx)
    Qr = Q.reverse_complement(ctx)
    m = gxy.ScoringMatrix.hoxd70()
    OT, OQ = O.pack_ascii(t), O.pack_ascii(q)
    ot = O.Table(OT, P12, 1)
    for qq, oq in ((Q, OQ), (Qr, O.reverse_complement(OQ))):
        g = as_tuples(gxy.search(tab, T, qq, m, sp))
        o = as_tuples(O.search(ot, OT, oq, orc_params(m, sp))[0])
        assert g == o


def test_window_passes_match_single_pass(gxy):
    # A tiny raw-hit buffer forces the search into many window-range passes,
    # including redone passes; the HSPs must not change.
    rng = np.random.default_rng(21)
    t, q = homologous_pair(rng, 400000, 0.8, lower=0.1)
    sp = gxy.SearchParams()
    c2 = gxy.Context(0)
    try:
        T, Q = gxy.PackedSeq.from_ascii(t), gxy.PackedSeq.from_ascii(q)
        tab = gxy.PosTable.build(T, P12, 1, ctx=c2)
        m = gxy.ScoringMatrix.hoxd70()
        st1 = {}
        ref = gxy.search(tab, T, Q, m, sp, stats=st1)
        assert st1["raw_hits"] > 3 * 4096
        c2.set_tuning(max_hits_per_pass=4096)
        st2 = {}
        got = gxy.search(tab, T, Q, m, sp, stats=st2)
        assert st2["passes"] > 1
        assert got.tobytes() == ref.tobytes()
        assert st1["raw_hits"] == st2["raw_hits"] and st1["windows"] == st2["windows"]
        # A tiny candidate capacity as well: candidates overflow inside a pass,
        # the arrays grow keeping earlier passes' candidates and the pass is redone.
        assert st1["candidates"] > 4 * 1024
        c2.set_tuning(initial_candidates=1024)
        st3 = {}
        got3 = gxy.search(tab, T, Q, m, sp, stats=st3)
        assert st3["passes"] > 1 and got3.tobytes() == ref.tobytes()
        assert st3["candidates"] == st1["candidates"]
        # Single pass with the tiny candidate capacity: grown and rerun whole.
        c2.set_tuning(max_hits_per_pass=1 << 30)
        st4 = {}
        assert gxy.search(tab, T, Q, m, sp, stats=st4).tobytes() == ref.tobytes()
        assert st4["passes"] == 1 and st4["candidates"] == st1["candidates"]
        tab.free()
    finally:
        c2.close()


@pytest.mark.parametrize("case", ["hoxd70", "ambig_high", "no_negative_class", "asymmetric"])
def test_filter_bounds_cases(gxy, ctx, case):
    # The upper-bound filter between enumeration and the exact screen takes
    # each class x = t ^ q at its largest score (at least the ambiguous one);
    # it is off when no class is <= 0 (a bounded side would never break).
    # Whatever the matrix, the output must equal the oracle's: a matrix with
    # the ambiguous score above the transversions (invalid columns in every
    # class), one with no non-positive class (filter off: every raw hit goes
    # to the exact screen), and an asymmetric one (sub[t][q] != sub[q][t]).
    rng = np.random.default_rng(41)
    t, q = homologous_pair(rng, 40000, 0.8, lower=0.05, nfrac=0.01)
    base = gxy.ScoringMatrix.hoxd70()
    sp = gxy.SearchParams(1, gxy.HspParams(910, 3000), 1)
    if case == "hoxd70":
        m = base
    elif case == "ambig_high":
        m = gxy.ScoringMatrix(sub=[row[:] for row in base.sub], ambig_score=-20)
    elif case == "no_negative_class":
        # Transitions score +5: every class has a positive member.
        sub = [row[:] for row in base.sub]
        for a, b in ((0, 2), (2, 0), (1, 3), (3, 1), (0, 1), (1, 0), (2, 3), (3, 2), (0, 3), (3, 0), (1, 2), (2, 1)):
            sub[a][b] = 5 if (a ^ b) == 2 else sub[a][b]
        sub[0][1] = 1   # class 1 gets a positive member
        sub[0][3] = 1   # class 3 too
        m = gxy.ScoringMatrix(sub=sub, ambig_score=-100)
        sp = gxy.SearchParams(1, gxy.HspParams(910, 6000), 1)
    else:
        sub = [row[:] for row in base.sub]
        sub[0][2], sub[2][0] = -20, -60
        sub[1][0], sub[0][1] = -90, -130
        m = gxy.ScoringMatrix(sub=sub, ambig_score=-100)
    g, o = both(gxy, ctx, t, q, P12, sp, matrix=m)
    assert g == o
    assert len(o) > 0
