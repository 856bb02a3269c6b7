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
