"""Batched launches: many (table, query, strand) units in one pass through the
pipeline must give each unit exactly the reference search() result.

Shapes: uneven query lengths, both strands, several targets, the driver's
chunk/halo split with its primary-region filter (src/driver.rs:156-256), and
the CUDA-graph capture of the batch."""
import numpy as np
import pytest

import oracle as O
from helpers import homologous_pair, rand_ascii

pytestmark = pytest.mark.gpu
P12 = "1110100110010101111"


def make_queries(rng, target: bytes, n: int, lo=1000, hi=30000):
    from lastz_gxy_b200 import synth
    t = np.frombuffer(target, np.uint8)
    out = []
    for i in range(n):
        L = int(rng.integers(lo, hi))
        s = int(rng.integers(0, len(t) - L))
        ident = float(rng.uniform(0.65, 0.95))
        out.append(synth.evolve(rng, t[s:s + L].copy(), ident, 0.005).tobytes())
    return out


def oracle_units(target: bytes, queries, units, pattern=P12, mwc=0, sp=None):
    T = O.pack_ascii(target)
    tab = O.Table(T, pattern, 1, mwc)
    p = O.params() if sp is None else sp
    res = []
    for (ti, qi, strand) in units:
        Q = O.pack_ascii(queries[qi])
        if strand:
            Q = O.reverse_complement(Q)
        h, _ = O.search(tab, T, Q, p)
        res.append(h)
    return res


@pytest.mark.parametrize("use_graph", [False, True])
def test_batch_matches_per_unit_search(gxy, ctx, use_graph):
    rng = np.random.default_rng(31)
    target = rand_ascii(rng, 200_000, b"ACGTACGTACGTacgtN")
    queries = make_queries(rng, target, 12)
    T = gxy.PackedSeq.from_ascii(target)
    tab = gxy.PosTable.build(T, P12, 1, ctx=ctx)
    dq = [gxy.PackedSeq.from_ascii(q).to_device(ctx) for q in queries]
    units = [(0, qi, s) for qi in range(len(queries)) for s in (0, 1)]
    st = {}
    got = gxy.batch_search([tab], dq, units, gxy.ScoringMatrix.hoxd70(), gxy.SearchParams(),
                           use_graph=use_graph, stats=st)
    want = oracle_units(target, queries, units)
    assert sum(len(w) for w in want) > 0
    for u, (g, w) in enumerate(zip(got, want)):
        assert g.tobytes() == w.tobytes(), u


def test_batch_graph_repeat_is_identical(gxy, ctx):
    rng = np.random.default_rng(32)
    target = rand_ascii(rng, 100_000, b"ACGT")
    queries = make_queries(rng, target, 6, 2000, 20000)
    tab = gxy.PosTable.build(gxy.PackedSeq.from_ascii(target), P12, 1, ctx=ctx)
    dq = [gxy.PackedSeq.from_ascii(q).to_device(ctx) for q in queries]
    units = [(0, qi, s) for qi in range(len(queries)) for s in (0, 1)]
    m, sp = gxy.ScoringMatrix.hoxd70(), gxy.SearchParams()
    a = gxy.batch_search([tab], dq, units, m, sp, use_graph=True)
    b = gxy.batch_search([tab], dq, units, m, sp, use_graph=True)
    c = gxy.batch_search([tab], dq, units, m, sp, use_graph=False)
    for x, y, z in zip(a, b, c):
        assert x.tobytes() == y.tobytes() == z.tobytes()


def test_batch_several_targets(gxy, ctx):
    rng = np.random.default_rng(33)
    targets = [rand_ascii(rng, n, b"ACGTACGTacgt") for n in (60_000, 150_000, 90_000)]
    queries, units = [], []
    for ti, t in enumerate(targets):
        for q in make_queries(rng, t, 3, 1000, 20000):
            units.append((ti, len(queries), 0))
            units.append((ti, len(queries), 1))
            queries.append(q)
    tabs = [gxy.PosTable.build(gxy.PackedSeq.from_ascii(t), P12, 1, ctx=ctx) for t in targets]
    dq = [gxy.PackedSeq.from_ascii(q).to_device(ctx) for q in queries]
    got = gxy.batch_search(tabs, dq, units, gxy.ScoringMatrix.hoxd70(), gxy.SearchParams())
    for u, (ti, qi, s) in enumerate(units):
        want = oracle_units(targets[ti], queries, [(0, qi, s)])[0]
        assert got[u].tobytes() == want.tobytes(), u


@pytest.mark.parametrize("transitions,mwc", [(1, 0), (0, 0), (1, 3)])
def test_chunked_batch_matches_driver_semantics(gxy, ctx, transitions, mwc):
    # driver.rs:156-256: per chunk a table over the chunk copy (extension stops
    # at the chunk edges), per (chunk, query, strand) a search, then the
    # primary-region filter on t_start.
    rng = np.random.default_rng(40 + transitions + mwc)
    target, query = homologous_pair(rng, 130_000, 0.85, lower=0.1, nfrac=0.002)
    primary, halo = 30_000, 5_000
    chunks = gxy.chunk_target(len(target), primary, halo)
    assert len(chunks) > 3
    dT = gxy.PackedSeq.from_ascii(target).to_device(ctx)
    tabs = [gxy.PosTable.build_view(dT, lo, hi, P12, 1, max_word_count=mwc, ctx=ctx) for lo, hi, _, _ in chunks]
    dq = [gxy.PackedSeq.from_ascii(query).to_device(ctx)]
    units = [(ci, 0, s, chunks[ci][2], chunks[ci][3]) for ci in range(len(chunks)) for s in (0, 1)]
    sp = gxy.SearchParams(transitions=transitions)
    got = gxy.batch_search(tabs, dq, units, gxy.ScoringMatrix.hoxd70(), sp)
    OT = O.pack_ascii(target)
    OQ = O.pack_ascii(query)
    total = 0
    for u, (ci, _, s, plo, phi) in enumerate(units):
        lo, hi = chunks[ci][0], chunks[ci][1]
        CS = O.slice_to_new(OT, lo, hi)
        tab = O.Table(CS, P12, 1, mwc)
        h, _ = O.search(tab, CS, O.reverse_complement(OQ) if s else OQ, O.params(transitions=transitions))
        h = h[(h["t_start"] >= plo) & (h["t_start"] < phi)]
        total += len(h)
        assert got[u].tobytes() == h.tobytes(), u
    assert total > 0


def test_concurrent_searches_share_one_table(gxy, ctx):
    # src/driver.rs:210-240 calls search() from rayon threads on one shared
    # table; every concurrent call must give its sequential result.
    import threading
    rng = np.random.default_rng(34)
    target = rand_ascii(rng, 150_000, b"ACGTACGTacgtN")
    queries = make_queries(rng, target, 16, 1000, 20000)
    T = gxy.PackedSeq.from_ascii(target)
    tab = gxy.PosTable.build(T, P12, 1, ctx=ctx)
    m, sp = gxy.ScoringMatrix.hoxd70(), gxy.SearchParams()
    packed = [gxy.PackedSeq.from_ascii(q) for q in queries]
    want = [gxy.search(tab, T, q, m, sp) for q in packed]
    got = [None] * len(packed)
    errors = []

    def worker(k):
        try:
            for i in range(k, len(packed), 4):
                got[i] = gxy.search(tab, T, packed[i], m, sp)
        except Exception as e:   # surfaced below
            errors.append(e)
    threads = [threading.Thread(target=worker, args=(k,)) for k in range(4)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors
    for i, (g, w) in enumerate(zip(got, want)):
        assert g.tobytes() == w.tobytes(), i
    assert sum(len(w) for w in want) > 0


def test_batch_repeated_and_split_units(gxy, ctx):
    """Units that share (table, query, strand) -- the same unit twice, and one
    chunk's primary range split over two units -- share one diagonal key range,
    so their candidates interleave on each diagonal; each unit must still get
    exactly its own search() result (its own diagonal cover)."""
    rng = np.random.default_rng(33)
    target, query = homologous_pair(rng, 120_000, 0.85)
    T = gxy.PackedSeq.from_ascii(target)
    tab = gxy.PosTable.build(T, P12, 1, ctx=ctx)
    dq = [gxy.PackedSeq.from_ascii(query).to_device(ctx)]
    cut = 50_000
    units = [(0, 0, 0), (0, 0, 1), (0, 0, 0), (0, 0, 0, 0, cut), (0, 0, 0, cut, len(target)), (0, 0, 1)]
    got = gxy.batch_search([tab], dq, units, gxy.ScoringMatrix.hoxd70(), gxy.SearchParams())
    want = oracle_units(target, [query], [(0, 0, 0), (0, 0, 1)])
    plus, minus = want
    assert len(plus) > 20
    assert got[0].tobytes() == plus.tobytes()
    assert got[1].tobytes() == minus.tobytes()
    assert got[2].tobytes() == plus.tobytes()
    lo = plus[plus["t_start"] < cut]
    hi = plus[plus["t_start"] >= cut]
    assert len(lo) > 0 and len(hi) > 0
    assert got[3].tobytes() == lo.tobytes()
    assert got[4].tobytes() == hi.tobytes()
    assert got[5].tobytes() == minus.tobytes()


def test_graph_multi_pass_and_kept_graph(gxy):
    # A raw-hit buffer far smaller than the launch's hits: the passes resume
    # on the device (tiles that do not fit go to the next pass) inside one
    # CUDA graph, with further rounds when the graph's passes fall short.
    # The graph stays with the worker across calls: the same shape is
    # updated in place, another shape (more passes, other units) is
    # instantiated anew.  Every result must equal the oracle's.
    rng = np.random.default_rng(33)
    target = rand_ascii(rng, 150_000, b"ACGT" * 12 + b"aN")   # 33k raw hits, 27k in the first 9 units
    queries = make_queries(rng, target, 8, 3000, 30000)
    c2 = gxy.Context(0)
    try:
        tab = gxy.PosTable.build(gxy.PackedSeq.from_ascii(target), P12, 1, ctx=c2)
        dq = [gxy.PackedSeq.from_ascii(q).to_device(c2) for q in queries]
        m, sp = gxy.ScoringMatrix.hoxd70(), gxy.SearchParams()
        units = [(0, qi, s) for qi in range(len(queries)) for s in (0, 1)]
        want = oracle_units(target, queries, units)
        assert sum(len(w) for w in want) > 0
        c2.set_tuning(max_hits_per_pass=4096)
        for k, sub in enumerate((units, units, units[:9], units)):
            st = {}
            got = gxy.batch_search([tab], dq, sub, m, sp, use_graph=True, stats=st, ctx=c2)
            assert st["raw_hits"] > 3 * 4096 and st["passes"] > 1
            if k == 1:
                # the same shape again: the kept graph is updated in place
                assert st["graph_updates"] >= 1, st
            for u, g in zip(sub, got):
                assert g.tobytes() == want[units.index(u)].tobytes(), u
        for d in dq:
            d.free()
        tab.free()
    finally:
        c2.close()


def test_objects_freed_after_their_context(gxy, ctx):
    # Device sequences and tables keep their device ordinal, so freeing them
    # after their context was destroyed touches no freed host memory; the
    # default context keeps working afterwards.
    c2 = gxy.Context(0)
    t = gxy.PackedSeq.from_ascii(b"ACGTTGCAAC" * 3000)
    dq = t.to_device(c2)
    tab = gxy.PosTable.build(t, P12, 1, ctx=c2)
    c2.close()
    dq.free()
    tab.free()
    T = gxy.PackedSeq.from_ascii(b"ACGTACGGTCAGTTACGATC" * 2000)
    tab2 = gxy.PosTable.build(T, P12, 1, ctx=ctx)
    h = gxy.search(tab2, T, T, gxy.ScoringMatrix.hoxd70(), gxy.SearchParams())
    assert len(h) > 0
    tab2.free()
