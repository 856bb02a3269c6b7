"""choose_anchor on the device (src/anchor.rs:25-69) against the oracle, on
the reference's own cases and on every HSP of real searches (windows from 1
to longer than the HSPs, sequences with N and soft-masked runs)."""
import numpy as np
import pytest

import oracle as O
from helpers import homologous_pair

pytestmark = pytest.mark.gpu
P12 = "1110100110010101111"
HOX = [[91, -114, -31, -123], [-114, 100, -125, -31], [-31, -125, 100, -114], [-123, -31, -114, 91]]


def anchors_both(gxy, ctx, t: bytes, q: bytes, hsps, window):
    dT = gxy.PackedSeq.from_ascii(t).to_device(ctx)
    dQ = gxy.PackedSeq.from_ascii(q).to_device(ctx)
    got = gxy.choose_anchors(dT, dQ, hsps, gxy.ScoringMatrix.hoxd70(), window, ctx)
    OT, OQ = O.pack_ascii(t), O.pack_ascii(q)
    want = [O.choose_anchor(h, OT, OQ, HOX, -100, window) for h in hsps]
    return [tuple(int(x) for x in r) for r in got], want


def test_anchor_known_answers(gxy, ctx):
    mk = lambda rows: np.array(rows, gxy.HSP_DTYPE)  # noqa: E731
    g, w = anchors_both(gxy, ctx, b"ACGTACGTACGTACGT", b"ACGTACGTACGTACGT", mk([(0, 0, 16, 0)]), 4)
    assert g == w == [(2, 2)]
    g, w = anchors_both(gxy, ctx, b"AACCCCAA", b"TTCCCCTT", mk([(0, 0, 8, 0)]), 4)
    assert g == w == [(4, 4)]
    g, w = anchors_both(gxy, ctx, b"ACGT", b"ACGT", mk([(0, 0, 4, 0)]), 1000)
    assert g == w and g[0][0] == 2


@pytest.mark.parametrize("window", [1, 2, 4, 31, 32, 33, 100, 1000])
def test_anchor_on_search_hsps(gxy, ctx, window):
    rng = np.random.default_rng(60 + window)
    t, q = homologous_pair(rng, 60000, 0.8, lower=0.1, nfrac=0.01)
    T, Q = gxy.PackedSeq.from_ascii(t), gxy.PackedSeq.from_ascii(q)
    tab = gxy.PosTable.build(T, P12, 1, ctx=ctx)
    hsps = gxy.search(tab, T, Q, gxy.ScoringMatrix.hoxd70(), gxy.SearchParams(1, gxy.HspParams(910, 1000), 1))
    assert len(hsps) > 20
    g, w = anchors_both(gxy, ctx, t, q, hsps, window)
    assert g == w


def test_anchor_rejects_bad_hsps(gxy, ctx):
    dT = gxy.PackedSeq.from_ascii(b"ACGTACGT").to_device(ctx)
    for bad in ([(0, 0, 0, 5)], [(4, 0, 8, 5)]):
        with pytest.raises(gxy.GxyError):
            gxy.choose_anchors(dT, dT, np.array(bad, gxy.HSP_DTYPE), gxy.ScoringMatrix.hoxd70(), 4, ctx)


# ---------------------------------------------------------------------------
# best_chain (src/chain.rs:19-69) for many groups on the device.
# ---------------------------------------------------------------------------
def _rows(a):
    return [tuple(int(x) for x in r) for r in a]


def test_chain_groups_known_answers(gxy, ctx):
    # The reference's own cases (src/chain.rs:78-138), one group each, in one launch.
    h = lambda t, q, n, s: (t, q, n, s)  # noqa: E731
    cases = [([], []),                                                                     # chain.rs:79-82
             ([h(10, 20, 30, 1000)], [h(10, 20, 30, 1000)])]                               # :84-88
    a, b, c = h(0, 0, 20, 500), h(40, 40, 20, 500), h(80, 10, 20, 700)                    # :90-105
    cases.append(([a, b, c], [a, b]))
    a, b, c, d = h(0, 0, 10, 100), h(20, 20, 10, 100), h(40, 40, 10, 100), h(60, 60, 10, 500)
    cases.append(([a, b, c, d], [a, b, c, d]))                                             # :107-117
    a, b = h(0, 50, 10, 1000), h(20, 0, 10, 800)                                          # :119-128
    cases.append(([a, b], [a]))
    a, b = h(10, 10, 5, 100), h(0, 0, 5, 100)                                             # :130-137
    cases.append(([a, b], [b, a]))
    arrs = [np.array(g, gxy.HSP_DTYPE).reshape(-1) for g, _ in cases]
    got = gxy.best_chain_groups(arrs, ctx)
    for g, (_, want) in zip(got, cases):
        assert _rows(g) == want


def _random_group(rng, gxy, n, span, ties):
    g = np.zeros(n, gxy.HSP_DTYPE)
    g["t_start"] = rng.integers(0, span, n)
    g["q_start"] = rng.integers(0, span, n)
    g["length"] = rng.integers(0, 40, n)
    g["score"] = rng.integers(-20, 400, n)
    if ties and n > 4:
        # duplicate (t_start, q_start) pairs and equal scores: the tie rules
        k = n // 4
        g[:k]["t_start"] = g[k:2 * k]["t_start"]
        g[:k]["q_start"] = g[k:2 * k]["q_start"]
        g["score"][::3] = 100
    return g


def test_chain_groups_random_vs_oracle(gxy, ctx):
    rng = np.random.default_rng(71)
    sizes = [0, 1, 2, 3, 7, 31, 32, 33, 255, 256, 257, 1000, 4095, 4096, 4097, 6000] + \
        [int(x) for x in rng.integers(0, 200, 300)]
    groups = [_random_group(rng, gxy, n, max(64, n * 8), ties=i % 2 == 0) for i, n in enumerate(sizes)]
    got = gxy.best_chain_groups(groups, ctx)
    assert len(got) == len(groups)
    for i, (g, arr) in enumerate(zip(got, groups)):
        want = O.best_chain_c(arr)
        assert g.tobytes() == want.tobytes(), (i, len(arr))


def test_chain_groups_on_search_hsps(gxy, ctx):
    # Chains of the HSPs of real searches: one group per (target, strand),
    # against the oracle's O(n^2) form and the host's O(n log n) form.
    rng = np.random.default_rng(72)
    groups = []
    for k in range(6):
        t, q = homologous_pair(rng, 40000 + 10000 * k, 0.75 + 0.02 * k, lower=0.1, nfrac=0.01)
        T, Q = gxy.PackedSeq.from_ascii(t), gxy.PackedSeq.from_ascii(q)
        tab = gxy.PosTable.build(T, P12, 1, ctx=ctx)
        for QQ in (Q, Q.reverse_complement()):
            groups.append(gxy.search(tab, T, QQ, gxy.ScoringMatrix.hoxd70(),
                                     gxy.SearchParams(1, gxy.HspParams(910, 1000), 1)))
    assert sum(len(g) for g in groups) > 100
    got = gxy.best_chain_groups(groups, ctx)
    for g, arr in zip(got, groups):
        assert g.tobytes() == O.best_chain_c(arr).tobytes()
        assert g.tobytes() == gxy.best_chain(arr).tobytes()


def test_chain_groups_rejects_bad_offsets(gxy, ctx):
    from lastz_gxy_b200._lib import lib
    h = np.zeros(4, gxy.HSP_DTYPE)
    out = np.zeros(4, gxy.HSP_DTYPE)
    ln = np.zeros(2, np.uint64)
    for off in ([0, 3, 2], [1, 2, 4]):
        o = np.array(off, np.uint64)
        assert lib().gxy_best_chain_groups(ctx.h, h.ctypes.data, o.ctypes.data, 2, out.ctypes.data,
                                           ln.ctypes.data) != 0
