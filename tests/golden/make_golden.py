"""Writes the golden fixtures of tests/golden/ from the oracle.

The reference publishes no HSP goldens for this path (its end-to-end goldens
are upstream-lastz MAF files fetched over the network), so the fixtures are
the oracle's output on the seeded synthetic workloads.  The oracle itself is
pinned by the reference's known-answer tests (tests/test_oracle_kats.py).

    python tests/golden/make_golden.py

golden_c1.npz   the 30 kbp workload: both strands' full HSP sets + input hashes
golden_c2.json  the 10 Mbp workload: per strand, HSP count and sha256 of the
                canonical HSP array (16 bytes per HSP) + input hashes
"""
import hashlib
import importlib.util
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

P12 = "1110100110010101111"


def _synth():
    d = os.path.join(ROOT, "lastz-gxy_b200")
    spec = importlib.util.spec_from_file_location("gxy_synth", os.path.join(d, "synth.py"))
    m = importlib.util.module_from_spec(spec)
    sys.modules["gxy_synth"] = m
    spec.loader.exec_module(m)
    return m


def sha(b: bytes) -> str:
    return hashlib.sha256(b).hexdigest()


def run(pr, threads=2):
    import oracle as O
    t, q = pr.target.tobytes(), pr.query.tobytes()
    T, Q = O.pack_ascii(t), O.pack_ascii(q)
    tab = O.Table(T, P12, 1)
    res, stats = O.search_units([(tab, T, Q), (tab, T, O.reverse_complement(Q))], O.params(), avx2=False,
                                threads=threads)
    return t, q, res, stats


def main():
    import numpy as np
    synth = _synth()
    t0 = time.time()
    t, q, (plus, minus), st = run(synth.c1())
    np.savez_compressed(os.path.join(HERE, "golden_c1.npz"), plus=plus, minus=minus,
                        target_sha=sha(t), query_sha=sha(q))
    print("c1", len(plus), len(minus), round(time.time() - t0, 2), "s")
    t0 = time.time()
    t, q, (plus, minus), st = run(synth.c2())
    out = {"workload": "10 Mbp chromosome target (seed 2) vs ~70% identity query, 12of19, transitions 1, "
                       "HOXD70 910/3000",
           "target_sha": sha(t), "query_sha": sha(q), "target_len": len(t), "query_len": len(q),
           "plus": {"n": int(len(plus)), "sha256": sha(plus.tobytes()), "raw_hits": int(st[0]["raw_hits"]),
                    "windows": int(st[0]["windows"])},
           "minus": {"n": int(len(minus)), "sha256": sha(minus.tobytes()), "raw_hits": int(st[1]["raw_hits"]),
                     "windows": int(st[1]["windows"])}}
    with open(os.path.join(HERE, "golden_c2.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("c2", out["plus"]["n"], out["minus"]["n"], round(time.time() - t0, 2), "s")


if __name__ == "__main__":
    main()
