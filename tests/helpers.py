"""Helpers shared by the tests: random sequences, oracle <-> package conversions."""
from __future__ import annotations

import numpy as np

import oracle as O


def rand_ascii(rng: np.random.Generator, n: int, alphabet: bytes = b"ACGTacgtN", p=None) -> bytes:
    a = np.frombuffer(alphabet, np.uint8)
    return a[rng.choice(len(a), size=n, p=p)].tobytes()


def homologous_pair(rng: np.random.Generator, n: int, identity: float = 0.85, alphabet=b"ACGT", lower=0.0,
                    nfrac=0.0):
    """A target and a query that share diverged segments, with optional soft-masking and Ns."""
    from lastz_gxy_b200 import synth
    t = np.frombuffer(rand_ascii(rng, n, alphabet), np.uint8).copy()
    q = synth.evolve(rng, t, identity, 0.01)
    for s in (t, q):
        if lower > 0:
            m = rng.random(len(s)) < lower
            up = (s >= ord("A")) & (s <= ord("Z")) & (s != ord("N"))
            s[m & up] += 32
        if nfrac > 0:
            s[rng.random(len(s)) < nfrac] = ord("N")
    return t.tobytes(), q.tobytes()


def oracle_seq(gxy_seq) -> O.Seq:
    """A package PackedSeq as an oracle Seq (same byte layout)."""
    n = len(gxy_seq)
    pad = 8
    return O.Seq(np.concatenate([gxy_seq.codes, np.zeros(pad, np.uint8)]),
                 np.concatenate([gxy_seq.valid, np.zeros(pad, np.uint8)]),
                 np.concatenate([gxy_seq.mask, np.zeros(pad, np.uint8)]), n)


def orc_params(matrix, sp) -> "O.OrcParams":
    sub = [matrix.sub[r][q] for r in range(4) for q in range(4)]
    return O.params(xdrop=sp.hsp.x_drop, hspthresh=sp.hsp.hsp_threshold, step=sp.step, transitions=sp.transitions,
                    entropy=sp.entropy_threshold, sub=sub, ambig=matrix.ambig_score)


def as_tuples(h) -> list:
    return [(int(x["t_start"]), int(x["q_start"]), int(x["length"]), int(x["score"])) for x in h]


def oracle_search(target: bytes, query: bytes, pattern: str, matrix, sp, max_word_count: int = 0):
    T = O.pack_ascii(target)
    Q = O.pack_ascii(query)
    tab = O.Table(T, pattern, sp.step, max_word_count)
    h, st = O.search(tab, T, Q, orc_params(matrix, sp))
    return h, st



def write_2bit(seqs, big_endian: bool = False) -> bytes:
    """A UCSC 2bit file of [(name, ascii)] (lastz_gxy_b200.synth.to_2bit)."""
    from lastz_gxy_b200 import synth
    return synth.to_2bit(seqs, big_endian)
