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


@pytest.mark.parametrize("transitions,mwc,threads", [(1, 0, 4), (0, 3, 3)])
def test_driver_harness_matches_oracle(gxy, harness, tmp_path, transitions, mwc, threads):
    rng = np.random.default_rng(90 + transitions)
    target, query = homologous_pair(rng, 140_000, 0.85, lower=0.1, nfrac=0.002)
    tp, qp, op = tmp_path / "t.txt", tmp_path / "q.txt", tmp_path / "out.bin"
    tp.write_bytes(target)
    qp.write_bytes(query)
    primary, halo = 30_000, 5_000
    r = subprocess.run([harness, str(tp), str(qp), str(op), str(primary), str(halo), str(threads),
                        str(transitions), str(mwc)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    raw = op.read_bytes()
    n = int(np.frombuffer(raw[:8], np.uint64)[0])
    got = np.frombuffer(raw[8:], REC, count=n)
    want = oracle_records(gxy, target, query, primary, halo, transitions, mwc)
    assert len(want) > 0
    assert [tuple(int(x) for x in g) for g in got] == want
