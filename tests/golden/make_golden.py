"""Writes the golden fixtures of tests/golden/ from the oracle.

The reference publishes no HSP goldens for this path (its end-to-end goldens
are upstream-lastz MAF files fetched over the network), so the fixtures are
the oracle's output on the seeded synthetic workloads.  The oracle itself is
pinned by the reference's known-answer tests (tests/test_oracle_kats.py).

    python tests/golden/make_golden.py

golden_c1.npz   the 30 kbp workload: both strands' full HSP sets + input hashes
golden_c2.json  the 10 Mbp workload: per strand, HSP count and sha256 of the
                canonical HSP array (16 bytes per HSP) + input hashes
golden_gapped.npz  the 30 kbp workload's gapped extension (`python
                tests/golden/make_golden.py gapped`): the anchor of every
                plus-strand HSP (choose_anchor, window 31) and the oracle's
                extend() of each -- coordinates, score and edit-script runs
golden_scale.json  sampled units of the three large workloads at their full
                size (`python tests/golden/make_golden.py scale`, ~15 min on 8
                cores): the uneven batch (the longest contig and 15 more,
                both strands), the chunked chromosome (two whole chunks, both
                strands, transitions 1 and 0, after the primary-region
                filter) and the serving trace (8 requests, both strands); per
                unit the HSP count and sha256, plus input hashes
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


def _hsp_rec(h):
    return {"n": int(len(h)), "sha256": sha(h.tobytes())}


def scale(threads=None):
    """Oracle HSP hashes for sampled units of the full-size uneven-batch,
    chunked and serving workloads (the whole launch runs on the GPU; these
    units are checked against the oracle's search() of the same unit)."""
    import numpy as np
    import oracle as O
    synth = _synth()
    threads = threads or os.cpu_count() or 4
    p1 = O.params()
    out = {"seed": P12, "hoxd70": True, "xdrop": 910, "hspthresh": 3000}

    # Uneven batch: 4,096 log-normal contigs vs one 50 Mbp target.
    t0 = time.time()
    tgt, queries = synth.c3()
    T = O.pack_ascii(tgt.tobytes())
    tab = O.Table(T, P12, 1)
    order = sorted(range(len(queries)), key=lambda i: (len(queries[i]), i))
    pick = sorted(set([order[-1]] + [order[(k * (len(order) - 1)) // 15] for k in range(15)]))
    units, keys = [], []
    for qi in pick:
        Q = O.pack_ascii(queries[qi].tobytes())
        units += [(tab, T, Q), (tab, T, O.reverse_complement(Q))]
        keys.append(qi)
    res, _ = O.search_units(units, p1, avx2=False, threads=threads)
    out["uneven_batch"] = {
        "target_sha": sha(tgt.tobytes()), "n_queries": len(queries),
        "queries_sha": sha(b"".join(hashlib.sha256(q.tobytes()).digest() for q in queries)),
        "units": [{"query": qi, "len": int(len(queries[qi])), "plus": _hsp_rec(res[2 * k]),
                   "minus": _hsp_rec(res[2 * k + 1])} for k, qi in enumerate(keys)]}
    print("uneven batch", len(keys), "contigs", round(time.time() - t0, 1), "s", flush=True)
    del tab, units, res

    # Chunked chromosome: 250 Mbp x 250 Mbp, --chunk-size 10 Mbp --halo 50 kbp.
    t0 = time.time()
    pr = synth.c4()
    T = O.pack_ascii(pr.target.tobytes())
    Q = O.pack_ascii(pr.query.tobytes())
    Qr = O.reverse_complement(Q)
    chunks = O.chunk_target(len(pr.target), 10_000_000, 50_000)
    sel = [0, len(chunks) // 2]
    entries = []
    for tr in (1, 0):
        p = O.params(transitions=tr)
        units, meta = [], []
        for ci in sel:
            lo, hi, plo, phi = chunks[ci]
            S = O.slice_to_new(T, lo, hi)
            ctab = O.Table(S, P12, 1)
            for strand, qq in ((0, Q), (1, Qr)):
                units.append((ctab, S, qq))
                meta.append((ci, strand, plo, phi))
        res, _ = O.search_units(units, p, avx2=False, threads=threads)
        for (ci, strand, plo, phi), h in zip(meta, res):
            h = h[(h["t_start"] >= plo) & (h["t_start"] < phi)]
            entries.append({"transitions": tr, "chunk": ci, "strand": strand, **_hsp_rec(h)})
        print("chunked transitions", tr, round(time.time() - t0, 1), "s", flush=True)
    out["chunked"] = {"target_sha": sha(pr.target.tobytes()), "query_sha": sha(pr.query.tobytes()),
                      "chunks": [list(c) for c in chunks], "units": entries}
    del T, Q, Qr, pr

    # Serving trace: 3 x 100 Mbp targets, 200 requests (Poisson, seed 7).
    t0 = time.time()
    targets = synth.c5_targets()
    reqs = synth.c5_requests(targets, n_requests=200)
    lens = [len(r.query) for r in reqs]
    big = int(np.argmax(lens))
    small = int(np.argmin(lens))
    pick = []
    for i in [big, small, 0, 25, 50, 100, 150, 199]:
        if i not in pick:
            pick.append(i)
    k = 1
    while len(pick) < 8:
        if k not in pick:
            pick.append(k)
        k += 1
    packed = [O.pack_ascii(t.tobytes()) for t in targets]
    tabs = {}
    units = []
    for i in pick:
        r = reqs[i]
        if r.target not in tabs:
            tabs[r.target] = O.Table(packed[r.target], P12, 1)
        Qp = O.pack_ascii(r.query.tobytes())
        units += [(tabs[r.target], packed[r.target], Qp), (tabs[r.target], packed[r.target], O.reverse_complement(Qp))]
    res, _ = O.search_units(units, p1, avx2=False, threads=threads)
    out["serving"] = {
        "targets_sha": [sha(t.tobytes()) for t in targets], "n_requests": len(reqs),
        "requests_sha": sha(b"".join(hashlib.sha256(r.query.tobytes()).digest() for r in reqs)),
        "units": [{"request": i, "target": reqs[i].target, "len": lens[i], "plus": _hsp_rec(res[2 * k]),
                   "minus": _hsp_rec(res[2 * k + 1])} for k, i in enumerate(pick)]}
    print("serving", len(pick), "requests", round(time.time() - t0, 1), "s", flush=True)
    with open(os.path.join(HERE, "golden_scale.json"), "w") as f:
        json.dump(out, f, indent=1)


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


def gapped(threads=None):
    """The 30 kbp workload's gapped extension (src/gapped_extend.rs:78-132):
    every plus-strand HSP's anchor, extended by the oracle with HOXD70's gap
    costs and GappedParams::default()."""
    import numpy as np
    import oracle as O
    synth = _synth()
    threads = threads or os.cpu_count() or 4
    t0 = time.time()
    pr = synth.c1()
    t, q = pr.target.tobytes(), pr.query.tobytes()
    T, Q = O.pack_ascii(t), O.pack_ascii(q)
    hsps, _ = O.search(O.Table(T, P12, 1), T, Q, O.params())
    hox = [O.HOXD70[4 * r:4 * r + 4] for r in range(4)]
    anchors = np.array([O.choose_anchor(h, T, Q, hox, -100, 31) for h in hsps], np.uint32).reshape(-1, 2)
    res = O.gapped_extend_many(T, Q, O.params(), O.gapped_params(), anchors[:, 0], anchors[:, 1], threads=threads)
    alns = np.zeros((len(res), 6), np.int64)   # t_start, q_start, t_len, q_len, score, passed
    runs, offs = [], [0]
    for k, a in enumerate(res):
        if a is not None:
            alns[k] = (a["t_start"], a["q_start"], a["t_len"], a["q_len"], a["score"], 1)
            runs += a["runs"]
        offs.append(len(runs))
    np.savez_compressed(os.path.join(HERE, "golden_gapped.npz"), target_sha=sha(t), query_sha=sha(q),
                        anchors=anchors, alns=alns, runs=np.array(runs, np.uint32), offsets=np.array(offs, np.int64))
    print("gapped", len(res), "anchors", sum(a is not None for a in res), "passed", round(time.time() - t0, 1), "s")


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "scale":
        scale()
    elif len(sys.argv) > 1 and sys.argv[1] == "gapped":
        gapped()
    else:
        main()
