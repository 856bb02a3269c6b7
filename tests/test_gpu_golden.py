"""GPU against the committed golden fixtures, up to the full 10 Mbp size."""
import hashlib
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
P12 = "1110100110010101111"


def run_both_strands(gxy, pr, ctx):
    T = gxy.PackedSeq.from_ascii(pr.target.tobytes())
    dT = T.to_device(ctx)
    dQ = gxy.PackedSeq.from_ascii(pr.query.tobytes()).to_device(ctx)
    tab = gxy.PosTable.build(dT, P12, 1, ctx=ctx)
    m, sp = gxy.ScoringMatrix.hoxd70(), gxy.SearchParams()
    out = []
    for q in (dQ, dQ.reverse_complement()):
        st = {}
        out.append((gxy.search_device(tab, q, m, sp, stats=st), st))
    return out


def test_c1_golden(gxy, ctx):
    from lastz_gxy_b200 import synth
    g = np.load(os.path.join(HERE, "golden", "golden_c1.npz"))
    (plus, _), (minus, _) = run_both_strands(gxy, synth.c1(), ctx)
    assert plus.tobytes() == g["plus"].tobytes() and minus.tobytes() == g["minus"].tobytes()


def test_c2_full_size_golden_hash(gxy, ctx):
    # 10 Mbp x 10 Mbp, both strands: sha256 of the canonical HSP arrays.
    from lastz_gxy_b200 import synth
    g = json.load(open(os.path.join(HERE, "golden", "golden_c2.json")))
    (plus, sp), (minus, sm) = run_both_strands(gxy, synth.c2(), ctx)
    assert len(plus) == g["plus"]["n"] and len(minus) == g["minus"]["n"]
    assert hashlib.sha256(plus.tobytes()).hexdigest() == g["plus"]["sha256"]
    assert hashlib.sha256(minus.tobytes()).hexdigest() == g["minus"]["sha256"]
    assert sp["raw_hits"] == g["plus"]["raw_hits"] and sm["raw_hits"] == g["minus"]["raw_hits"]
    assert sp["windows"] == g["plus"]["windows"]


def test_gapped_golden(gxy, ctx):
    # Every anchor of golden_gapped.npz (the 30 kbp workload's plus-strand
    # HSPs, choose_anchor window 31) extended on the device in one call.
    from lastz_gxy_b200 import synth
    g = np.load(os.path.join(HERE, "golden", "golden_gapped.npz"))
    pr = synth.c1()
    dT = gxy.PackedSeq.from_ascii(pr.target.tobytes()).to_device(ctx)
    dQ = gxy.PackedSeq.from_ascii(pr.query.tobytes()).to_device(ctx)
    got = gxy.gapped_extend(dT, dQ, g["anchors"], gxy.ScoringMatrix.hoxd70(), gxy.GappedParams(), ctx=ctx)
    assert len(got) == len(g["anchors"])
    for k, a in enumerate(got):
        row = g["alns"][k]
        if row[5] == 0:
            assert a is None
            continue
        assert (a.t_start, a.q_start, a.t_len, a.q_len, a.score) == tuple(int(x) for x in row[:5])
        assert [int(x) for x in a.script] == [int(x) for x in g["runs"][g["offsets"][k]:g["offsets"][k + 1]]]
