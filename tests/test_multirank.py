"""World-size-2 gloo run of the sharded unit path on CPU.

Each rank takes its share of (query x strand) units with shard_units, runs the
reference's search on them (here the oracle stands in for the GPU stage, which
needs a device), and the ranks gather only their results -- the same plumbing
bench.py uses under torchrun with NCCL.  The union must equal the single-rank
result."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "tests"))
    sys.path.insert(0, os.path.join(root, "oracle"))
    import conftest  # noqa: F401  loads the package
    import torch.distributed as dist
    import oracle as O
    from lastz_gxy_b200.shard import shard_units
    from lastz_gxy_b200 import synth
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    rng = np.random.default_rng(5)
    t = synth.iid(rng, 20000, 0.41)
    queries = [synth.evolve(rng, t[i * 3000:i * 3000 + 6000], 0.85, 0.005) for i in range(4)]
    T = O.pack_ascii(t.tobytes())
    tab = O.Table(T, "1110100110010101111", 1)
    units = [(qi, s) for qi in range(len(queries)) for s in (0, 1)]
    mine = shard_units(len(units), rank, world, [len(queries[u[0]]) for u in units])
    res = {}
    for i in mine:
        qi, s = units[i]
        Q = O.pack_ascii(queries[qi].tobytes())
        if s:
            Q = O.reverse_complement(Q)
        h, _ = O.search(tab, T, Q, O.params())
        res[i] = h.tobytes()
    gathered = [None] * world
    dist.all_gather_object(gathered, res)
    dist.destroy_process_group()
    if rank == 0:
        allres = {}
        for g in gathered:
            allres.update(g)
        q.put(allres)


def test_two_rank_gloo_sharding():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=300)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # single-rank reference
    import oracle as O
    from lastz_gxy_b200 import synth
    rng = np.random.default_rng(5)
    t = synth.iid(rng, 20000, 0.41)
    queries = [synth.evolve(rng, t[i * 3000:i * 3000 + 6000], 0.85, 0.005) for i in range(4)]
    T = O.pack_ascii(t.tobytes())
    tab = O.Table(T, "1110100110010101111", 1)
    units = [(qi, s) for qi in range(len(queries)) for s in (0, 1)]
    assert sorted(got) == list(range(len(units)))
    for i, (qi, s) in enumerate(units):
        Q = O.pack_ascii(queries[qi].tobytes())
        if s:
            Q = O.reverse_complement(Q)
        h, _ = O.search(tab, T, Q, O.params())
        assert got[i] == h.tobytes()
    assert any(len(v) for v in got.values())
