"""Gapped extension on the device (src/gapped_extend.rs:78-460) against the
oracle: the reference's own cases, random small cases over the band and gap
parameters (N's, anchors at the sequence ends, one-sided extensions), and
every anchor of real searches over planted homologous segments with indels,
in a whole target and in a chunk of it.  Equality is exact: score,
coordinates and every run of the edit script."""
import numpy as np
import pytest

import oracle as O
from helpers import rand_ascii

pytestmark = pytest.mark.gpu
P12 = "1110100110010101111"


def orc_result(a):
    if a is None:
        return None
    return (a["t_start"], a["q_start"], a["t_len"], a["q_len"], a["score"], list(a["runs"]))


def gpu_result(a):
    if a is None:
        return None
    return (a.t_start, a.q_start, a.t_len, a.q_len, a.score, [int(r) for r in a.script])


def both(gxy, ctx, t: bytes, q: bytes, anchors, go=400, ge=30, ydrop=9400, thr=3000, view=None, threads=8):
    m = gxy.ScoringMatrix.hoxd70()
    m.gap_open, m.gap_extend = go, ge
    dT = gxy.PackedSeq.from_ascii(t).to_device(ctx)
    dQ = gxy.PackedSeq.from_ascii(q).to_device(ctx)
    st = {}
    got = gxy.gapped_extend(dT, dQ, anchors, m, gxy.GappedParams(ydrop, thr), t_view=view, ctx=ctx, stats=st)
    tt = t if view is None else t[view[0]:view[1]]
    OT, OQ = O.pack_ascii(tt), O.pack_ascii(q)
    a = np.asarray(anchors, np.int64).reshape(-1, 2)
    cells = []
    want = O.gapped_extend_many(OT, OQ, O.params(), O.gapped_params(go, ge, ydrop, thr), a[:, 0], a[:, 1],
                                threads=threads, cells=cells)
    st["oracle_cells"] = sum(cells)
    return [gpu_result(x) for x in got], [orc_result(x) for x in want], st


def test_gapped_known_answers(gxy, ctx):
    # src/gapped_extend.rs:478-600, anchors = HSP start + offset.
    cases = [
        (b"ACGTACGTACGTACGT", b"ACGTACGTACGTACGT", 8, 8, 500, 100),
        (b"ACGTACGTACGT", b"ACGTACGGTACGT", 3, 3, 1000, 100),
        (b"ACGTACGGTACGT", b"ACGTACGTACGT", 3, 3, 1000, 100),
        (b"ACGT", b"ACGT", 1, 1, 500, 100000),
        (b"TTTTTTTTACGTACGTACGTACGTACGTACGTTTTTTTTT", b"AAAAAAAAACGTACGTACGTACGTACGTACGTAAAAAAAA", 20, 20, 300, 500),
        (b"AAAGATTACACATGGCATGTCGATTTT", b"GATACACATGGCAGTCGA", 6, 3, 5000, 100),
    ]
    core = b"GATTACACATGGCATGTCGAATGCCTAGCATGTCA"
    cases.append((core + core, core + b"AGCTAGCTAGCTAGCTAGCTAGCTAGCTAGCTAGCTAGCTAGCTAGCTAG" + core, 5, 5, 9400, 500))
    for t, q, tp, qp, yd, thr in cases:
        g, w, _ = both(gxy, ctx, t, q, [(tp, qp)], ydrop=yd, thr=thr)
        assert g == w, (t, q)
    g, _, _ = both(gxy, ctx, b"ACGTACGTACGTACGT", b"ACGTACGTACGTACGT", [(8, 8)], ydrop=500, thr=100)
    assert gxy.cigar(g[0][5]) == "16M"
    g, _, _ = both(gxy, ctx, core + core, core + b"AGCTAGCTAGCTAGCTAGCTAGCTAGCTAGCTAGCTAGCTAGCTAGCTAG" + core, [(5, 5)],
                   ydrop=9400, thr=500)
    assert g[0][2] >= 60 and g[0][3] >= 110 and "I" in gxy.cigar(g[0][5])


def _mutate(rng, s: bytes, nedits: int) -> bytes:
    q = bytearray(s)
    for _ in range(nedits):
        if not q:
            break
        k = int(rng.integers(0, len(q)))
        r = rng.integers(3)
        if r == 0:
            q[k:k] = rand_ascii(rng, int(rng.integers(1, 12)), b"ACGT")
        elif r == 1:
            del q[k:k + int(rng.integers(1, 12))]
        else:
            q[k] = b"ACGTN"[rng.integers(5)]
    return bytes(q) or b"A"


@pytest.mark.parametrize("go,ge,ydrop", [(400, 30, 9400), (400, 30, 300), (400, 30, 1500), (0, 30, 700),
                                         (400, 0, 500), (50, 5, 2000), (400, 30, 0)])
def test_gapped_random_small(gxy, ctx, go, ge, ydrop):
    # Short sequences (bands as wide as the query, m + 1 cells), anchors
    # anywhere including both ends, N's and soft-masked bases.
    rng = np.random.default_rng(1000 + go + ge + ydrop)
    for case in range(8):
        n = int(rng.integers(1, 400))
        t = rand_ascii(rng, n, b"ACGTACGTacgtN")
        q = _mutate(rng, t, int(rng.integers(0, 12)))
        anchors = [(int(rng.integers(0, len(t))), int(rng.integers(0, len(q)))) for _ in range(24)]
        anchors += [(0, 0), (len(t) - 1, len(q) - 1), (0, len(q) - 1), (len(t) - 1, 0)]
        g, w, _ = both(gxy, ctx, t, q, anchors, go, ge, ydrop, thr=-10 ** 6)
        assert g == w, case


def planted(rng, n: int, segs: int, seg_len=(300, 3000), identity=(0.78, 0.95)):
    """A random target and query sharing `segs` diverged segments (substitutions
    and indels, half of them reverse-complemented), elsewhere unrelated."""
    from lastz_gxy_b200 import synth
    t = np.frombuffer(rand_ascii(rng, n, b"ACGT"), np.uint8).copy()
    q = np.frombuffer(rand_ascii(rng, n, b"ACGT"), np.uint8).copy()
    for _ in range(segs):
        ln = int(rng.integers(*seg_len))
        a = int(rng.integers(0, n - ln))
        b = int(rng.integers(0, n - ln))
        ev = synth.evolve(rng, t[a:a + ln].copy(), float(rng.uniform(*identity)), 0.01)[:ln]
        if rng.random() < 0.5:   # half of them on the minus strand
            ev = np.frombuffer(ev.tobytes().translate(bytes.maketrans(b"ACGT", b"TGCA"))[::-1], np.uint8)
        q[b:b + len(ev)] = ev
    low = rng.random(n) < 0.05
    t[low] = np.where((t[low] >= 65) & (t[low] <= 90), t[low] + 32, t[low])
    q[rng.random(n) < 0.002] = ord("N")
    return t.tobytes(), q.tobytes()


def search_anchors(gxy, ctx, t: bytes, q: bytes, view=None):
    tt = t if view is None else t[view[0]:view[1]]
    T, Q = gxy.PackedSeq.from_ascii(tt), gxy.PackedSeq.from_ascii(q)
    m = gxy.ScoringMatrix.hoxd70()
    tab = gxy.PosTable.build(T, P12, 1, ctx=ctx)
    hsps = gxy.search(tab, T, Q, m, gxy.SearchParams(1, gxy.HspParams(910, 2000), 1))
    dT, dQ = T.to_device(ctx), Q.to_device(ctx)
    return gxy.choose_anchors(dT, dQ, hsps, m, 31, ctx), hsps


@pytest.mark.parametrize("seed", [1, 2])
def test_gapped_on_search_anchors(gxy, ctx, seed):
    # The driver's step: HSPs -> choose_anchor -> extend, every anchor
    # (src/driver.rs:395-414), both strands of the query.
    rng = np.random.default_rng(70 + seed)
    t, q = planted(rng, 60000, 14)
    rc = q.translate(bytes.maketrans(b"ACGTacgtN", b"TGCAtgcaN"))[::-1]
    for qq in (q, rc):
        anchors, hsps = search_anchors(gxy, ctx, t, qq)
        assert len(anchors) > 10
        g, w, st = both(gxy, ctx, t, qq, anchors)
        assert g == w
        assert sum(x is not None for x in g) > 5
        assert st["rows"] > 0 and st["cells"] >= st["rows"]
        assert st["cells"] == st["oracle_cells"]   # the same bands, row by row


def test_gapped_in_a_chunk_view(gxy, ctx):
    # Extension bounded by a chunk of the target (the driver extends against
    # chunk.seq, src/driver.rs:299-310): anchors in chunk coordinates.
    rng = np.random.default_rng(91)
    t, q = planted(rng, 80000, 16)
    view = (17000, 61000)
    anchors, _ = search_anchors(gxy, ctx, t, q, view)
    assert len(anchors) > 5
    g, w, _ = both(gxy, ctx, t, q, anchors, view=view)
    assert g == w


def test_gapped_long_alignment(gxy, ctx):
    # One 40 kbp homologous stretch: a side of thousands of rows (a deep chain
    # of traceback blocks) and a long edit script.
    from lastz_gxy_b200 import synth
    rng = np.random.default_rng(5)
    t = np.frombuffer(rand_ascii(rng, 40000, b"ACGT"), np.uint8).copy()
    q = synth.evolve(rng, t.copy(), 0.9, 0.005)
    t, q = t.tobytes(), q.tobytes()
    anchors, hsps = search_anchors(gxy, ctx, t, q)
    top = np.argsort(-hsps["score"], kind="stable")[:3]
    g, w, st = both(gxy, ctx, t, q, anchors[top], thr=0)
    assert g == w
    assert max(x[2] for x in g if x) > 20000


@pytest.mark.parametrize("name", ["scaled", "asymmetric"])
def test_gapped_other_matrices(gxy, ctx, name):
    # Substitution scores other than HOXD70 (a uniform match/mismatch matrix
    # and an asymmetric one, each with its own ambiguous score): the column
    # scores enter M through the same per-row lookup as the defaults.
    if name == "scaled":
        sub = [[150 if r == c else -120 for c in range(4)] for r in range(4)]
        ambig = -80
    else:
        sub = [[91, -114, -31, -123], [-100, 100, -125, -31], [-40, -110, 100, -114], [-123, -20, -114, 80]]
        ambig = -150
    rng = np.random.default_rng(7 if name == "scaled" else 8)
    m = gxy.ScoringMatrix.hoxd70()
    m.sub = [row[:] for row in sub]
    m.ambig_score = ambig
    gp = O.gapped_params(400, 30, 3000, -10 ** 6)
    flat = [x for row in sub for x in row]
    for case in range(6):
        t = rand_ascii(rng, int(rng.integers(50, 2000)), b"ACGTACGTacgtN")
        q = _mutate(rng, t, int(rng.integers(0, 20)))
        anchors = [(int(rng.integers(0, len(t))), int(rng.integers(0, len(q)))) for _ in range(12)]
        dT = gxy.PackedSeq.from_ascii(t).to_device(ctx)
        dQ = gxy.PackedSeq.from_ascii(q).to_device(ctx)
        got = gxy.gapped_extend(dT, dQ, anchors, m, gxy.GappedParams(3000, -10 ** 6), ctx=ctx)
        a = np.asarray(anchors, np.int64)
        want = O.gapped_extend_many(O.pack_ascii(t), O.pack_ascii(q), O.params(sub=flat, ambig=ambig), gp,
                                    a[:, 0], a[:, 1], threads=4)
        assert [gpu_result(x) for x in got] == [orc_result(x) for x in want], case


def test_gapped_eight_cells_per_thread(gxy):
    # The layout with 8 cells of a row per thread (half the warps per side of
    # the default 4): the same results as the oracle on search anchors and on
    # short pairs.
    c = gxy.Context(0)
    c.set_tuning(gapped_cells=8)
    rng = np.random.default_rng(23)
    t, q = planted(rng, 60000, 14)
    anchors, _ = search_anchors(gxy, c, t, q)
    g, w, st = both(gxy, c, t, q, anchors)
    assert g == w and st["cells_per_thread"] == 8
    for case in range(6):
        tt = rand_ascii(rng, int(rng.integers(1, 500)), b"ACGTACGTacgtN")
        qq = _mutate(rng, tt, int(rng.integers(0, 12)))
        anchors = [(int(rng.integers(0, len(tt))), int(rng.integers(0, len(qq)))) for _ in range(16)]
        g, w, _ = both(gxy, c, tt, qq, anchors, thr=-10 ** 6)
        assert g == w, case


def test_gapped_second_pass(gxy):
    # A first pass with room for only a few traceback blocks: the sides that
    # ran out are extended again with exactly sized storage, and every result
    # still equals the oracle's.
    c = gxy.Context(0)
    c.set_tuning(gapped_pool_blocks=40)
    rng = np.random.default_rng(17)
    t, q = planted(rng, 60000, 14)
    anchors, _ = search_anchors(gxy, c, t, q)
    g, w, st = both(gxy, c, t, q, anchors)
    assert g == w
    assert st["second_pass_sides"] > 0
    c.set_tuning(gapped_pool_blocks=0xffffffff)
    g2, _, st2 = both(gxy, c, t, q, anchors)
    assert g2 == w and st2["second_pass_sides"] == 0


def test_gapped_rejects(gxy, ctx):
    dT = gxy.PackedSeq.from_ascii(b"ACGTACGTAC").to_device(ctx)
    m = gxy.ScoringMatrix.hoxd70()
    with pytest.raises(gxy.GxyError):   # anchor outside the target
        gxy.gapped_extend(dT, dT, [(10, 0)], m, gxy.GappedParams(), ctx=ctx)
    big = gxy.PackedSeq.from_ascii(b"ACGT" * 2000).to_device(ctx)
    m2 = gxy.ScoringMatrix.hoxd70()
    m2.gap_extend = 1   # band of 4 * 9000 cells: wider than the device DP holds
    with pytest.raises(gxy.GxyError) as e:
        gxy.gapped_extend(big, big, [(10, 10)], m2, gxy.GappedParams(), ctx=ctx)
    assert e.value.status == 3
    assert gxy.gapped_extend(dT, dT, np.zeros((0, 2), np.uint32), m, gxy.GappedParams(), ctx=ctx) == []


def test_gapped_plain_workload_full_size(gxy, ctx):
    # The 10 Mbp plain workload, plus strand: the 24 highest-scoring anchors
    # (sides of up to ~280 k rows, long chains of pool blocks) and 24 more
    # spread over the ranked list, extended in one call and compared with the
    # oracle run on the host threads.
    import os
    from lastz_gxy_b200 import synth
    pr = synth.c2()
    t, q = pr.target.tobytes(), pr.query.tobytes()
    m = gxy.ScoringMatrix.hoxd70()
    T, Q = gxy.PackedSeq.from_ascii(t), gxy.PackedSeq.from_ascii(q)
    dT, dQ = T.to_device(ctx), Q.to_device(ctx)
    tab = gxy.PosTable.build(dT, P12, 1, ctx=ctx)
    hsps = gxy.search_device(tab, dQ, m, gxy.SearchParams())
    anchors = gxy.choose_anchors(dT, dQ, hsps, m, 31, ctx)
    order = np.argsort(-hsps["score"], kind="stable")
    pick = np.concatenate([order[:24], order[np.linspace(24, len(order) - 1, 24).astype(int)]])
    A = np.ascontiguousarray(anchors[pick])
    st = {}
    got = gxy.gapped_extend(dT, dQ, A, m, gxy.GappedParams(), ctx=ctx, stats=st)
    OT, OQ = O.pack_ascii(t), O.pack_ascii(q)
    want = O.gapped_extend_many(OT, OQ, O.params(), O.gapped_params(), A[:, 0], A[:, 1],
                                threads=max(1, min(16, os.cpu_count() or 1)))
    assert [gpu_result(x) for x in got] == [orc_result(x) for x in want]
    assert st["max_side_rows"] > 50_000
