"""The C ABI driven from C++ the way the reference's driver drives search()
(src/driver.rs:156-256, :362-391): chunk tables built and searched from a
pool of host threads, both strands of a chunk concurrently on its shared
table, then the primary-region filter, global coordinates and the per-group
sort and dedup.  The harness's records must equal the oracle's."""
import os
import subprocess

import numpy as np
import pytest

import oracle as O
from helpers import homologous_pair

pytestmark = pytest.mark.gpu
P12 = "1110100110010101111"
HERE = os.path.dirname(os.path.abspath(__file__))
REC = np.dtype([("query", "<u4"), ("strand", "<u4"), ("t_start", "<u4"), ("q_start", "<u4"),
                ("span", "<u4"), ("score", "<i4")])


@pytest.fixture(scope="module")
def harness(gxy, tmp_path_factory):
    out = str(tmp_path_factory.mktemp("harness") / "driver_harness")
    subprocess.run(["make", "-s", "-C", os.path.join(HERE, "harness"), f"OUT={out}"], check=True)
    return out


def oracle_records(gxy, target: bytes, query: bytes, primary, halo, transitions, mwc):
    OT, OQ = O.pack_ascii(target), O.pack_ascii(query)
    recs = []
    for lo, hi, plo, phi in gxy.chunk_target(len(target), primary, halo):
        CS = O.slice_to_new(OT, lo, hi)
        tab = O.Table(CS, P12, 1, mwc)
        for strand, q in ((0, OQ), (1, O.reverse_complement(OQ))):
            h, _ = O.search(tab, CS, q, O.params(transitions=transitions))
            for r in h:
                if plo <= r["t_start"] < phi:
                    recs.append((0, strand, int(r["t_start"]) + lo, int(r["q_start"]), int(r["length"]),
                                 int(r["score"])))
    recs.sort(key=lambda r: r[:5])
    out = []
    for r in recs:
        if out and out[-1][:5] == r[:5]:
            continue
        out.append(r)
    return out


@pytest.mark.parametrize("transitions,mwc,threads,mode", [(1, 0, 4, 0), (0, 3, 3, 0), (1, 0, 1, 1), (0, 3, 1, 1)])
def test_driver_harness_matches_oracle(gxy, harness, tmp_path, transitions, mwc, threads, mode):
    """mode 0: plain search() calls from a thread pool; mode 1: one
    gxy_batch_records call (filter, global coordinates, order and dedup on
    the device)."""
    rng = np.random.default_rng(90 + transitions)
    target, query = homologous_pair(rng, 140_000, 0.85, lower=0.1, nfrac=0.002)
    tp, qp, op = tmp_path / "t.txt", tmp_path / "q.txt", tmp_path / "out.bin"
    tp.write_bytes(target)
    qp.write_bytes(query)
    primary, halo = 30_000, 5_000
    r = subprocess.run([harness, str(tp), str(qp), str(op), str(primary), str(halo), str(threads),
                        str(transitions), str(mwc), str(mode)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    raw = op.read_bytes()
    n = int(np.frombuffer(raw[:8], np.uint64)[0])
    got = np.frombuffer(raw[8:], REC, count=n)
    want = oracle_records(gxy, target, query, primary, halo, transitions, mwc)
    assert len(want) > 0
    assert [tuple(int(x) for x in g) for g in got] == want


def oracle_group_records(targets, queries, plans, offsets, transitions, mwc):
    """The driver's records over several targets and queries, with the group
    of (target, query, strand) numbered in the driver's output order."""
    OQ = [O.pack_ascii(q) for q in queries]
    OQR = [O.reverse_complement(q) for q in OQ]
    groups = {}
    for ti, target in enumerate(targets):
        OT = O.pack_ascii(target)
        for lo, hi, plo, phi in plans[ti]:
            CS = O.slice_to_new(OT, lo, hi)
            tab = O.Table(CS, P12, 1, mwc)
            for qi in range(len(queries)):
                for strand, q in ((0, OQ[qi]), (1, OQR[qi])):
                    g = (ti * len(queries) + qi) * 2 + strand
                    h, _ = O.search(tab, CS, q, O.params(transitions=transitions))
                    for r in h:
                        if plo <= r["t_start"] < phi:
                            groups.setdefault(g, []).append(
                                (g, (int(r["t_start"]) + lo + offsets[ti]) & 0xFFFFFFFF, int(r["q_start"]),
                                 int(r["length"]), int(r["score"])))
    out = []
    for g in sorted(groups):
        last = None
        for r in sorted(groups[g], key=lambda r: r[:4]):
            if r[:4] != last:
                out.append(r)
            last = r[:4]
    return out


@pytest.mark.parametrize("big_offset", [False, True])
def test_batch_records_groups_match_oracle(gxy, big_offset):
    """Two targets (one chunked), two queries, both strands in one
    batch_records call.  big_offset pushes t past 2^31 so that the record key
    needs more than 64 bits and the two-sort path runs."""
    rng = np.random.default_rng(404)
    t0, q0 = homologous_pair(rng, 90_000, 0.85, lower=0.1, nfrac=0.002)
    t1, q1 = homologous_pair(rng, 50_000, 0.8)
    q0 = q0 + q1[:20_000]
    targets, queries = [t0, t1], [q0, q1]
    plans = [gxy.chunk_target(len(t0), 30_000, 4_000), gxy.chunk_target(len(t1), 0, 0)]
    offsets = [4_000_000_000 if big_offset else 0, 7]
    ctx = gxy.Context.default()
    dT = [gxy.DeviceSeq.from_ascii(t, ctx) for t in targets]
    dQ = [gxy.DeviceSeq.from_ascii(q, ctx) for q in queries]
    tables, units, places = [], [], []
    for ti in range(2):
        for lo, hi, plo, phi in plans[ti]:
            tables.append(gxy.PosTable.build_view(dT[ti], lo, hi, gxy.SeedPattern.twelve_of_nineteen(), 1))
            for qi in range(2):
                for strand in (0, 1):
                    units.append((len(tables) - 1, qi, strand, plo, phi))
                    places.append(((ti * 2 + qi) * 2 + strand, lo + offsets[ti]))
    # Units in an order other than the group order.
    perm = rng.permutation(len(units))
    units = [units[i] for i in perm]
    places = [places[i] for i in perm]
    params = gxy.SearchParams(transitions=1)
    recs, offs = gxy.batch_records(tables, dQ, units, places, gxy.ScoringMatrix.hoxd70(), params)
    want = oracle_group_records(targets, queries, plans, offsets, 1, 0)
    assert len(want) > 100
    got = [(int(r["group"]), int(r["t_start"]), int(r["q_start"]), int(r["span"]), int(r["score"])) for r in recs]
    assert got == want
    assert len(offs) == 9 and int(offs[-1]) == len(recs)
    for g in range(8):
        assert np.all(recs["group"][int(offs[g]):int(offs[g + 1])] == g)
    # Each record's unit names a unit of its group; its t lies in that unit's primary region.
    for r in recs:
        u = units[int(r["unit"])]
        assert places[int(r["unit"])][0] == int(r["group"])
        local = (int(r["t_start"]) - places[int(r["unit"])][1]) & 0xFFFFFFFF
        assert u[3] <= local < u[4]
    # Same records without the graph and with it.
    recs_g, _ = gxy.batch_records(tables, dQ, units, places, gxy.ScoringMatrix.hoxd70(), params, use_graph=True)
    assert np.array_equal(recs_g, recs)
    for t in tables:
        t.free()


def test_batch_records_duplicate_units_dedup(gxy):
    """The same unit twice in one group: every record appears twice before
    the dedup and once after it, attributed to the first unit."""
    rng = np.random.default_rng(405)
    t, q = homologous_pair(rng, 40_000, 0.85)
    ctx = gxy.Context.default()
    dT, dQ = gxy.DeviceSeq.from_ascii(t, ctx), gxy.DeviceSeq.from_ascii(q, ctx)
    tab = gxy.PosTable.build_view(dT, 0, len(t), gxy.SeedPattern.twelve_of_nineteen(), 1)
    m, p = gxy.ScoringMatrix.hoxd70(), gxy.SearchParams(transitions=1)
    one, _ = gxy.batch_records([tab], [dQ], [(0, 0, 0)], [(0, 0)], m, p)
    two, offs = gxy.batch_records([tab], [dQ], [(0, 0, 0), (0, 0, 0), (0, 0, 1)], [(1, 0), (1, 0), (0, 0)], m, p)
    assert len(one) > 10
    g1 = two[int(offs[1]):int(offs[2])]
    assert np.array_equal(g1[["t_start", "q_start", "span", "score"]], one[["t_start", "q_start", "span", "score"]])
    assert np.all(g1["unit"] == 0)
    assert np.all(two[:int(offs[1])]["unit"] == 2)
    # An empty batch and a bad offset.
    e, eo = gxy.batch_records([tab], [dQ], [], [], m, p)
    assert len(e) == 0 and len(eo) == 1
    with pytest.raises(gxy.GxyError):
        gxy.batch_records([tab], [dQ], [(0, 0, 0)], [(0, 2**32 - 100)], m, p)
    tab.free()
