"""Golden fixtures and generator stability (CPU only)."""
import hashlib
import json
import os

import numpy as np

import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
P12 = "1110100110010101111"


def sha(b):
    return hashlib.sha256(b).hexdigest()


def test_c1_golden_reproduced_by_oracle():
    from lastz_gxy_b200 import synth
    g = np.load(os.path.join(HERE, "golden", "golden_c1.npz"))
    pr = synth.c1()
    assert sha(pr.target.tobytes()) == str(g["target_sha"]) and sha(pr.query.tobytes()) == str(g["query_sha"])
    T, Q = O.pack_ascii(pr.target.tobytes()), O.pack_ascii(pr.query.tobytes())
    tab = O.Table(T, P12, 1)
    plus, _ = O.search(tab, T, Q, O.params())
    minus, _ = O.search(tab, T, O.reverse_complement(Q), O.params())
    assert plus.tobytes() == g["plus"].tobytes() and minus.tobytes() == g["minus"].tobytes()
    assert len(plus) > 0


def test_c2_inputs_stable():
    # The 10 Mbp workload must regenerate byte for byte; the GPU test compares
    # its HSP hashes against golden_c2.json.
    from lastz_gxy_b200 import synth
    g = json.load(open(os.path.join(HERE, "golden", "golden_c2.json")))
    pr = synth.c2()
    assert sha(pr.target.tobytes()) == g["target_sha"] and sha(pr.query.tobytes()) == g["query_sha"]


def _gapped_golden():
    return np.load(os.path.join(HERE, "golden", "golden_gapped.npz"))


def test_gapped_golden_reproduced_by_oracle():
    # golden_gapped.npz: every plus-strand HSP's anchor of the 30 kbp workload
    # and its extend() (src/gapped_extend.rs:78-132); a spread of them redone.
    from lastz_gxy_b200 import synth
    g = _gapped_golden()
    pr = synth.c1()
    assert sha(pr.target.tobytes()) == str(g["target_sha"]) and sha(pr.query.tobytes()) == str(g["query_sha"])
    T, Q = O.pack_ascii(pr.target.tobytes()), O.pack_ascii(pr.query.tobytes())
    hsps, _ = O.search(O.Table(T, P12, 1), T, Q, O.params())
    hox = [O.HOXD70[4 * r:4 * r + 4] for r in range(4)]
    assert len(hsps) == len(g["anchors"]) > 0
    pick = np.linspace(0, len(hsps) - 1, 12).astype(int)
    for k in pick:
        assert tuple(O.choose_anchor(hsps[k], T, Q, hox, -100, 31)) == tuple(int(x) for x in g["anchors"][k])
    got = O.gapped_extend_many(T, Q, O.params(), O.gapped_params(), g["anchors"][pick, 0], g["anchors"][pick, 1],
                               threads=4)
    for k, a in zip(pick, got):
        row = g["alns"][k]
        assert a is not None and row[5] == 1
        assert (a["t_start"], a["q_start"], a["t_len"], a["q_len"], a["score"]) == tuple(int(x) for x in row[:5])
        assert a["runs"] == [int(x) for x in g["runs"][g["offsets"][k]:g["offsets"][k + 1]]]
