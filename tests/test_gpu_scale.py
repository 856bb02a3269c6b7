"""The three large workloads at their full configured size, checked unit by
unit against the oracle.

Each test runs the whole launch on the GPU -- every unit of the uneven batch
(4,096 contigs x 2 strands against a 50 Mbp target), every (chunk, strand)
unit of the 250 Mbp chunked chromosome for transitions 1 and 0, every request
of the 200-request serving trace -- and compares the sampled units' HSP arrays
with the oracle's sha256 in tests/golden/golden_scale.json (written by
`python tests/golden/make_golden.py scale`).  The sampled units include the
longest contig, whole 10 Mbp chunks and the largest request, i.e. the
multi-pass, candidate-growth and long-diagonal regimes.  The chunked units
are compared after the driver's primary-region filter, the way the
reference's chunked == unchunked test does (tests/fixture_smoke.rs:161-236).
Tolerance: none (bit-identical HSP arrays in canonical order)."""
import hashlib
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
P12 = "1110100110010101111"


def sha(b: bytes) -> str:
    return hashlib.sha256(b).hexdigest()


@pytest.fixture(scope="module")
def golden():
    with open(os.path.join(HERE, "golden", "golden_scale.json")) as f:
        return json.load(f)


def check(h, rec, what):
    assert len(h) == rec["n"], f"{what}: {len(h)} HSPs, oracle {rec['n']}"
    assert sha(h.tobytes()) == rec["sha256"], f"{what}: HSPs differ from the oracle"


def test_uneven_batch_full_size(gxy, ctx, golden):
    from lastz_gxy_b200 import synth
    g = golden["uneven_batch"]
    tgt, queries = synth.c3()
    assert sha(tgt.tobytes()) == g["target_sha"] and len(queries) == g["n_queries"]
    assert sha(b"".join(hashlib.sha256(q.tobytes()).digest() for q in queries)) == g["queries_sha"]
    m, sp = gxy.ScoringMatrix.hoxd70(), gxy.SearchParams()
    dT = gxy.PackedSeq.from_ascii(tgt.tobytes()).to_device(ctx)
    tab = gxy.PosTable.build(dT, P12, 1, ctx=ctx)
    dq = [gxy.PackedSeq.from_ascii(q.tobytes()).to_device(ctx) for q in queries]
    units = [(0, qi, st) for qi in range(len(queries)) for st in (0, 1)]
    st = {}
    out = gxy.batch_search([tab], dq, units, m, sp, use_graph=True, stats=st, ctx=ctx)
    assert len(out) == len(units)
    for u in g["units"]:
        qi = u["query"]
        check(out[2 * qi], u["plus"], f"contig {qi} ({u['len']} bp) plus")
        check(out[2 * qi + 1], u["minus"], f"contig {qi} ({u['len']} bp) minus")
    for q in dq:
        q.free()


def test_chunked_full_size(gxy, ctx, golden):
    from lastz_gxy_b200 import synth
    g = golden["chunked"]
    pr = synth.c4()
    assert sha(pr.target.tobytes()) == g["target_sha"] and sha(pr.query.tobytes()) == g["query_sha"]
    chunks = gxy.chunk_target(len(pr.target), 10_000_000, 50_000)
    assert [list(c) for c in chunks] == g["chunks"]
    m = gxy.ScoringMatrix.hoxd70()
    dT = gxy.PackedSeq.from_ascii(pr.target.tobytes()).to_device(ctx)
    dQ = gxy.PackedSeq.from_ascii(pr.query.tobytes()).to_device(ctx)
    # Every chunk's table from one build over the shared bucket space (the
    # path the chunked bench takes).
    tabs = gxy.PosTable.build_views(dT, [(lo, hi) for lo, hi, _, _ in chunks], P12, 1, ctx=ctx)
    units = [(ci, 0, st, chunks[ci][2], chunks[ci][3]) for ci in range(len(chunks)) for st in (0, 1)]
    for tr in (1, 0):
        st = {}
        out = gxy.batch_search(tabs, [dQ], units, m, gxy.SearchParams(transitions=tr), stats=st, ctx=ctx)
        if tr == 1:
            assert st["passes"] > 1   # the multi-pass regime is exercised
        for u in g["units"]:
            if u["transitions"] != tr:
                continue
            k = 2 * u["chunk"] + u["strand"]
            check(out[k], u, f"chunk {u['chunk']} strand {u['strand']} transitions {tr}")
    for t in tabs:
        t.free()


def test_serving_trace_full_size(gxy, ctx, golden):
    from lastz_gxy_b200 import synth
    g = golden["serving"]
    targets = synth.c5_targets()
    assert [sha(t.tobytes()) for t in targets] == g["targets_sha"]
    reqs = synth.c5_requests(targets, n_requests=g["n_requests"])
    assert sha(b"".join(hashlib.sha256(r.query.tobytes()).digest() for r in reqs)) == g["requests_sha"]
    m, sp = gxy.ScoringMatrix.hoxd70(), gxy.SearchParams()
    tabs = [gxy.PosTable.build(gxy.PackedSeq.from_ascii(t.tobytes()).to_device(ctx), P12, 1, ctx=ctx)
            for t in targets]
    srv = gxy.Server(tabs, m, sp, max_streams=2, max_batch_units=64)
    try:
        # Every request is queued at once: the admission and batching see the
        # whole trace in flight.
        ids = [srv.submit(r.target, gxy.PackedSeq.from_ascii(r.query.tobytes())) for r in reqs]
        res = [srv.wait(i, timeout_ms=600_000) for i in ids]
        stats = srv.stats()
    finally:
        srv.close()
    assert stats["completed"] == len(reqs) and stats["batches"] > 1
    for u in g["units"]:
        i = u["request"]
        plus, minus = res[i][0], res[i][1]
        check(plus, u["plus"], f"request {i} ({u['len']} bp) plus")
        check(minus, u["minus"], f"request {i} ({u['len']} bp) minus")
    for t in tabs:
        t.free()
