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


# ---- failure handling: faults are made on the host (a test hook, an input
# outside the exact envelope, a cancel); no GPU fault is involved. ----------

def test_injected_fault_fails_only_its_request(gxy, setup):
    # Request 3 of a batch fails as a device allocation would (GXY_ENOMEM,
    # injected on the host before any device work).  The batch is rerun one
    # request at a time: the others complete with the same HSPs as alone.
    from lastz_gxy_b200 import _lib
    targets, tables, reqs = setup
    few = [r for r in reqs if r[0] == 0][:6]
    ref, _ = run_server(gxy, tables, few, "alone")
    srv = gxy.Server(tables, gxy.ScoringMatrix.hoxd70(), gxy.SearchParams(), max_streams=1, max_batch_units=64)
    try:
        srv.inject_fault(3, _lib.GXY_ENOMEM)          # ids start at 1: the third request
        ids = [srv.submit(ti, gxy.PackedSeq.from_ascii(q)) for ti, q in few]
        assert ids[2] == 3
        out = [srv.wait_status(i) for i in ids]
        st = srv.stats()
    finally:
        srv.close()
    assert out[2][0] == _lib.GXY_ENOMEM
    for i in range(len(few)):
        if i == 2:
            continue
        assert out[i][0] == _lib.GXY_OK
        assert out[i][1].tobytes() == ref[i][0].tobytes() and out[i][2].tobytes() == ref[i][1].tobytes(), i
    assert st["failed"] == 1 and st["completed"] == len(few)


def test_bad_input_mid_stream_fails_alone(gxy, ctx):
    # Scores scaled x100: a 200 kbp query against a 250 kbp target can leave
    # the i32 envelope (GXY_EUNSUPPORTED), 20 kbp queries cannot.  Queued
    # together, the long one fails alone; its batch-mates equal the oracle.
    from lastz_gxy_b200 import _lib
    rng = np.random.default_rng(5)
    target = rand_ascii(rng, 250_000, b"ACGTACGTacgt")
    tab = gxy.PosTable.build(gxy.PackedSeq.from_ascii(target), P12, 1, ctx=ctx)
    m = gxy.ScoringMatrix(sub=[[x * 100 for x in row] for row in gxy.ScoringMatrix.hoxd70().sub], ambig_score=-10000)
    sp = gxy.SearchParams(hsp=gxy.HspParams(x_drop=91000, hsp_threshold=300000))
    t = np.frombuffer(target, np.uint8)
    from lastz_gxy_b200 import synth
    qs = []
    for i, L in enumerate([20_000, 20_000, 20_000, 200_000, 20_000, 20_000]):
        s = int(rng.integers(0, len(t) - L))
        qs.append(synth.evolve(rng, t[s:s + L].copy(), 0.85, 0.005).tobytes())
    srv = gxy.Server([tab], m, sp, max_streams=1, max_batch_units=64)
    try:
        ids = [srv.submit(0, gxy.PackedSeq.from_ascii(q)) for q in qs]
        out = [srv.wait_status(i) for i in ids]
        st = srv.stats()
    finally:
        srv.close()
    assert out[3][0] == _lib.GXY_EUNSUPPORTED
    T = O.pack_ascii(target)
    otab = O.Table(T, P12, 1)
    p = O.params(xdrop=91000, hspthresh=300000, sub=[x * 100 for x in O.HOXD70], ambig=-10000)
    n = 0
    for i, q in enumerate(qs):
        if i == 3:
            continue
        Q = O.pack_ascii(q)
        wp, _ = O.search(otab, T, Q, p)
        wm, _ = O.search(otab, T, O.reverse_complement(Q), p)
        assert out[i][0] == _lib.GXY_OK
        assert out[i][1].tobytes() == wp.tobytes() and out[i][2].tobytes() == wm.tobytes(), i
        n += len(wp) + len(wm)
    assert n > 0 and st["failed"] == 1
    tab.free()


def test_cancel(gxy, setup):
    # One dispatcher busy with a long request; a request queued behind it is
    # cancelled before it reaches the device and waits return GXY_ECANCELED.
    # The others are unaffected; unknown ids are rejected.
    from lastz_gxy_b200 import _lib
    targets, tables, reqs = setup
    big = max(range(len(reqs)), key=lambda i: len(reqs[i][1]))
    order = [big] + [i for i in range(len(reqs)) if i != big][:5]
    ref, _ = run_server(gxy, tables, [reqs[i] for i in order], "alone")
    srv = gxy.Server(tables, gxy.ScoringMatrix.hoxd70(), gxy.SearchParams(), max_streams=1, max_batch_units=2)
    try:
        ids = [srv.submit(reqs[i][0], gxy.PackedSeq.from_ascii(reqs[i][1])) for i in order]
        srv.cancel(ids[-1])
        out = [srv.wait_status(i) for i in ids]
        st = srv.stats()
        with pytest.raises(gxy.GxyError):
            srv.cancel(ids[0])   # already waited for: unknown
    finally:
        srv.close()
    assert out[-1][0] == _lib.GXY_ECANCELED and st["canceled"] == 1
    for k in range(len(order) - 1):
        assert out[k][0] == _lib.GXY_OK
        assert out[k][1].tobytes() == ref[k][0].tobytes() and out[k][2].tobytes() == ref[k][1].tobytes(), k


def test_free_memory_is_refreshed(gxy, setup):
    # The admission estimate is re-based on the device's free memory at a low
    # rate, while the server is idle, by the server's monitor thread.
    import time
    _, tables, _ = setup
    srv = gxy.Server(tables, gxy.ScoringMatrix.hoxd70(), gxy.SearchParams())
    try:
        time.sleep(1.3)
        assert srv.stats()["mem_refreshes"] >= 2
    finally:
        srv.close()
