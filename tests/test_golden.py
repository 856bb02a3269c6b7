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
