"""Serving loop: resident tables, requests admitted by device memory and batched
as they arrive.  Each request's HSPs must be the same whether it ran alone or
in the mix (the tolerance is zero: bit-identical), and equal the reference
search() on both strands."""
import numpy as np
import pytest

import oracle as O
from helpers import rand_ascii

pytestmark = pytest.mark.gpu
P12 = "1110100110010101111"


def requests(rng, targets, n):
    from lastz_gxy_b200 import synth
    out = []
    for i in range(n):
        ti = int(rng.integers(0, len(targets)))
        t = np.frombuffer(targets[ti], np.uint8)
        L = int(rng.integers(500, 40000))
        s = int(rng.integers(0, len(t) - L))
        out.append((ti, synth.evolve(rng, t[s:s + L].copy(), float(rng.uniform(0.6, 0.95)), 0.005).tobytes()))
    return out


@pytest.fixture(scope="module")
def setup(gxy, ctx):
    rng = np.random.default_rng(77)
    targets = [rand_ascii(rng, 200_000, b"ACGTACGTacgtN"), rand_ascii(rng, 120_000, b"ACGTacgt")]
    tables = [gxy.PosTable.build(gxy.PackedSeq.from_ascii(t), P12, 1, ctx=ctx) for t in targets]
    return targets, tables, requests(rng, targets, 24)


def run_server(gxy, tables, reqs, mode, **opts):
    srv = gxy.Server(tables, gxy.ScoringMatrix.hoxd70(), gxy.SearchParams(), **opts)
    try:
        out = {}
        if mode == "alone":
            for i, (ti, q) in enumerate(reqs):
                rid = srv.submit(ti, gxy.PackedSeq.from_ascii(q))
                out[i] = srv.wait(rid)
        else:
            ids = [srv.submit(ti, gxy.PackedSeq.from_ascii(q)) for ti, q in reqs]
            for i, rid in enumerate(ids):
                out[i] = srv.wait(rid)
        return out, srv.stats()
    finally:
        srv.close()


def test_mix_equals_alone_equals_reference(gxy, setup):
    targets, tables, reqs = setup
    alone, _ = run_server(gxy, tables, reqs, "alone")
    mix, st = run_server(gxy, tables, reqs, "mix", max_streams=2, max_batch_units=8)
    assert st["completed"] == len(reqs) and st["batches"] > 1
    total = 0
    for i, (ti, q) in enumerate(reqs):
        T = O.pack_ascii(targets[ti])
        tab = O.Table(T, P12, 1)
        Q = O.pack_ascii(q)
        wp, _ = O.search(tab, T, Q, O.params())
        wm, _ = O.search(tab, T, O.reverse_complement(Q), O.params())
        for got in (alone[i], mix[i]):
            assert got[0].tobytes() == wp.tobytes() and got[1].tobytes() == wm.tobytes(), i
        total += len(wp) + len(wm)
    assert total > 0


def test_admission_by_memory_budget(gxy, setup):
    # A budget below one request's estimate admits one request at a time;
    # results do not change.
    targets, tables, reqs = setup
    few = reqs[:6]
    ref, _ = run_server(gxy, tables, few, "mix")
    tight, st = run_server(gxy, tables, few, "mix", max_device_bytes=1 << 20, max_streams=2)
    assert st["completed"] == len(few) and st["batches"] == len(few)
    for i in range(len(few)):
        assert ref[i][0].tobytes() == tight[i][0].tobytes() and ref[i][1].tobytes() == tight[i][1].tobytes()


def test_big_requests_run_alone_and_small_ones_go_ahead(gxy, setup):
    # With big_bases below most request sizes, the big requests each run in a
    # batch of their own, one at a time; results do not change.
    targets, tables, reqs = setup
    ref, _ = run_server(gxy, tables, reqs, "alone")
    lens = sorted(len(q) for _, q in reqs)
    cut = lens[len(lens) // 3]
    n_big = sum(1 for _, q in reqs if len(q) >= cut)
    mix, st = run_server(gxy, tables, reqs, "mix", max_streams=2, max_batch_units=64, big_bases=cut,
                         max_big_inflight=1)
    assert st["completed"] == len(reqs)
    # Every big request is a batch; the small ones share the others.
    assert st["batches"] >= n_big + 1
    for i in range(len(reqs)):
        assert ref[i][0].tobytes() == mix[i][0].tobytes() and ref[i][1].tobytes() == mix[i][1].tobytes(), i


def test_warm_buffers_and_stats(gxy, setup):
    # warm_bases sizes every dispatcher's buffers at creation; results do not
    # change, and no batch has to rerun after a buffer grew.
    targets, tables, reqs = setup
    ref, _ = run_server(gxy, tables, reqs[:8], "alone")
    warm, st = run_server(gxy, tables, reqs[:8], "mix", max_streams=2, warm_bases=max(len(q) for _, q in reqs))
    assert st["completed"] == 8 and st["reruns"] == 0 and st["busy_ms"] > 0
    for i in range(8):
        assert ref[i][0].tobytes() == warm[i][0].tobytes() and ref[i][1].tobytes() == warm[i][1].tobytes()


def test_wait_timeout_and_unknown_id(gxy, setup):
    _, tables, reqs = setup
    srv = gxy.Server(tables, gxy.ScoringMatrix.hoxd70(), gxy.SearchParams())
    try:
        with pytest.raises(gxy.GxyError):
            srv.wait(987654, timeout_ms=10)
        rid = srv.submit(0, gxy.PackedSeq.from_ascii(reqs[0][1]))
        srv.wait(rid, timeout_ms=120000)
    finally:
        srv.close()
