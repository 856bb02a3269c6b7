"""Seeded synthetic DNA for the seed->HSP workloads.

There is no public dataset for this path, so every workload is generated here
from a documented model with numpy's PCG64 generator:

* iid bases at a given GC fraction (A=T=(1-gc)/2, C=G=gc/2);
* planted repeat families: a consensus of `fam_len` bp copied `copies_lo..hi`
  times, each copy diverged by substitutions at a rate U(div_lo, div_hi), in a
  random orientation, written at a uniform random offset -- later copies
  overwrite earlier ones (the families' total length may exceed the target's);
* soft-masking: alternating unmasked/masked runs, masked runs U(100, 5000) bp,
  unmasked gaps sized so the masked fraction is `mask_frac` (lowercase);
* N-blocks of `nblock_len` bp at uniform random offsets;
* evolution (query from target): substitutions at rate 1 - identity with
  transition:transversion 2:1, indels at `indel_rate` per bp (50/50 insertion
  and deletion, geometric lengths of mean 3), optional replacement of a
  fraction of the length by random segments.  N stays N; a base keeps the
  case of its source position; inserted and replaced bases are uppercase.

The byte sequences are ASCII; PackedSeq.from_ascii packs them.
"""
from __future__ import annotations

import hashlib
from dataclasses import dataclass

import numpy as np

_ACGT = np.frombuffer(b"ACGT", np.uint8)
_acgt = np.frombuffer(b"acgt", np.uint8)
# ASCII -> code for ACGTacgt (others 255)
_CODE = np.full(256, 255, np.uint8)
for _i, _b in enumerate(b"ACGT"):
    _CODE[_b] = _i
    _CODE[_b + 32] = _i


def iid(rng: np.random.Generator, n: int, gc: float) -> np.ndarray:
    at = (1.0 - gc) / 2.0
    cg = gc / 2.0
    codes = rng.choice(4, size=n, p=[at, cg, cg, at]).astype(np.uint8)
    return _ACGT[codes]


def _revcomp_codes(c: np.ndarray) -> np.ndarray:
    return (3 - c)[::-1]


def substitute(rng: np.random.Generator, seq: np.ndarray, rate: float) -> np.ndarray:
    """Substitutions at `rate` per ACGT base, Ts:Tv = 2:1 (A<->G, C<->T are transitions)."""
    out = seq.copy()
    codes = _CODE[out]
    isb = codes != 255
    hit = isb & (rng.random(len(out)) < rate)
    idx = np.nonzero(hit)[0]
    c = codes[idx]
    ts = rng.random(len(idx)) < (2.0 / 3.0)
    tv = np.where(rng.random(len(idx)) < 0.5, 1, 3).astype(np.uint8)
    nc = np.where(ts, c ^ 2, c ^ tv).astype(np.uint8)
    lower = out[idx] >= ord("a")
    out[idx] = np.where(lower, _acgt[nc], _ACGT[nc])
    return out


def plant_repeats(rng: np.random.Generator, seq: np.ndarray, families: int, fam_len: int = 300,
                  copies_lo: int = 5, copies_hi: int = 50, div_lo: float = 0.10, div_hi: float = 0.20,
                  gc: float = 0.41) -> np.ndarray:
    out = seq.copy()
    n = len(out)
    for _ in range(families):
        cons = _CODE[iid(rng, fam_len, gc)]
        k = int(rng.integers(copies_lo, copies_hi + 1))
        for _ in range(k):
            d = rng.uniform(div_lo, div_hi)
            c = cons.copy()
            hit = rng.random(fam_len) < d
            m = int(hit.sum())
            ts = rng.random(m) < (2.0 / 3.0)
            tv = np.where(rng.random(m) < 0.5, 1, 3).astype(np.uint8)
            c[hit] = np.where(ts, c[hit] ^ 2, c[hit] ^ tv)
            if rng.random() < 0.5:
                c = _revcomp_codes(c)
            if n <= fam_len:
                continue
            off = int(rng.integers(0, n - fam_len))
            out[off:off + fam_len] = _ACGT[c]
    return out


def soft_mask(rng: np.random.Generator, seq: np.ndarray, frac: float, run_lo: int = 100,
              run_hi: int = 5000) -> np.ndarray:
    out = seq.copy()
    n = len(out)
    if frac <= 0:
        return out
    mean_run = (run_lo + run_hi) / 2.0
    mean_gap = mean_run * (1.0 - frac) / frac
    pos = int(rng.integers(0, int(mean_gap) + 1))
    lowered = np.zeros(n, bool)
    while pos < n:
        L = int(rng.integers(run_lo, run_hi + 1))
        lowered[pos:pos + L] = True
        pos += L + int(rng.integers(1, int(2 * mean_gap)))
    isu = (out >= ord("A")) & (out <= ord("Z")) & (out != ord("N"))
    out[lowered & isu] += 32
    return out


def n_blocks(rng: np.random.Generator, seq: np.ndarray, count: int, length: int) -> np.ndarray:
    out = seq.copy()
    n = len(out)
    for _ in range(count):
        if n <= length:
            break
        off = int(rng.integers(0, n - length))
        out[off:off + length] = ord("N")
    return out


def evolve(rng: np.random.Generator, seq: np.ndarray, identity: float, indel_rate: float,
           replace_frac: float = 0.0, gc: float = 0.41, indel_mean: float = 3.0) -> np.ndarray:
    """Query = seq evolved to ~identity (see the module docstring)."""
    out = substitute(rng, seq, 1.0 - identity)
    n = len(out)
    if replace_frac > 0 and n > 0:
        covered = 0
        target = int(replace_frac * n)
        while covered < target:
            L = int(rng.integers(500, 5001))
            off = int(rng.integers(0, max(1, n - L)))
            out[off:off + L] = iid(rng, len(out[off:off + L]), gc)
            covered += L
    if indel_rate > 0 and n > 0:
        ev = int(rng.binomial(n, indel_rate))
        pos = np.sort(rng.integers(0, n, size=ev))
        lens = rng.geometric(1.0 / indel_mean, size=ev)
        is_ins = rng.random(ev) < 0.5
        keep = np.ones(n, bool)
        dp, dl = pos[~is_ins], lens[~is_ins]
        if len(dp):
            idx = np.repeat(dp, dl) + (np.arange(dl.sum()) - np.repeat(np.cumsum(dl) - dl, dl))
            keep[idx[idx < n]] = False
        pref = np.concatenate([[0], np.cumsum(keep)])
        kept = out[keep]
        ip, il = pos[is_ins], lens[is_ins]
        ins_at = np.repeat(pref[ip], il)
        ins_bases = iid(rng, int(il.sum()), gc)
        out = np.insert(kept, ins_at, ins_bases)
    return out


def lcg_dna(n: int, seed: int) -> np.ndarray:
    """The reference bench's LCG DNA (benches/hotpath.rs:22-30)."""
    state = seed
    out = np.empty(n, np.uint8)
    a, c, m = 6364136223846793005, 1442695040888963407, (1 << 64) - 1
    acgt = b"ACGT"
    for i in range(n):
        state = (state * a + c) & m
        out[i] = acgt[(state >> 33) & 3]
    return out


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(a.tobytes()).hexdigest()


# ---------------------------------------------------------------------------
# The workloads
# ---------------------------------------------------------------------------
@dataclass
class Pair:
    target: np.ndarray
    query: np.ndarray


def c1(seed: int = 1, length: int = 30_000) -> Pair:
    """30 kbp iid at 38% GC (seed 1), query at ~80% identity, indels 0.5%/bp."""
    rng = np.random.default_rng(seed)
    t = iid(rng, length, 0.38)
    q = evolve(rng, t, 0.80, 0.005, gc=0.38)
    return Pair(t, q)


def chromosome(rng: np.random.Generator, length: int, families: int, nblocks: int, gc: float = 0.41,
               mask_frac: float = 0.45, nblock_len: int = 10_000) -> np.ndarray:
    t = iid(rng, length, gc)
    t = plant_repeats(rng, t, families, gc=gc)
    t = soft_mask(rng, t, mask_frac)
    t = n_blocks(rng, t, nblocks, nblock_len)
    return t


def c2(seed: int = 2, length: int = 10_000_000, families: int = 2000, nblocks: int = 20) -> Pair:
    """10 Mbp chromosome-style target; query at ~70% identity, 1% indels, 5% random segments."""
    rng = np.random.default_rng(seed)
    t = chromosome(rng, length, families, nblocks)
    q = evolve(rng, t, 0.70, 0.01, replace_frac=0.05)
    return Pair(t, q)


def c3(seed: int = 3, target_len: int = 50_000_000, n_queries: int = 4096, total: int = 200_000_000,
       median: int = 20_000, lo: int = 1_000, hi: int = 2_000_000):
    """One chromosome-style target (families scaled by length) and log-normal query contigs,
    each a target slice evolved to U(65%, 95%) identity with 0.5%/bp indels."""
    rng = np.random.default_rng(seed)
    fam = max(1, int(round(2000 * target_len / 10_000_000)))
    nb = max(1, int(round(20 * target_len / 10_000_000)))
    t = chromosome(rng, target_len, fam, nb)
    lens = rng.lognormal(np.log(median), 1.3, size=n_queries)
    lens = np.clip(lens, lo, hi)
    lens = np.clip(lens * (total / lens.sum()), lo, min(hi, target_len))
    lens = lens.astype(np.int64)
    queries = []
    for L in lens:
        s = int(rng.integers(0, max(1, target_len - L)))
        ident = rng.uniform(0.65, 0.95)
        queries.append(evolve(rng, t[s:s + L], ident, 0.005))
    return t, queries


def c4(seed: int = 4, length: int = 250_000_000, families: int = 30_000, nblocks: int = 500) -> Pair:
    """250 Mbp chromosome-style target; query at ~70% identity as in c2."""
    rng = np.random.default_rng(seed)
    t = chromosome(rng, length, families, nblocks)
    q = evolve(rng, t, 0.70, 0.01, replace_frac=0.05)
    return Pair(t, q)


@dataclass
class Request:
    arrival_s: float
    target: int
    query: np.ndarray
    identity: float


def c5_targets(seed: int = 5, n: int = 3, length: int = 100_000_000):
    rng = np.random.default_rng(seed)
    fam = max(1, int(round(2000 * length / 10_000_000)))
    nb = max(1, int(round(20 * length / 10_000_000)))
    return [chromosome(rng, length, fam, nb) for _ in range(n)]


def c5_requests(targets, n_requests: int, seed: int = 7, rate: float = 50.0, lo: int = 10_000,
                hi: int = 5_000_000):
    """Poisson arrivals at `rate`/s; each a target slice of log-uniform length, evolved to U(60%, 95%)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for _ in range(n_requests):
        t += rng.exponential(1.0 / rate)
        ti = int(rng.integers(0, len(targets)))
        L = int(np.exp(rng.uniform(np.log(lo), np.log(hi))))
        L = min(L, len(targets[ti]) - 1)
        s = int(rng.integers(0, max(1, len(targets[ti]) - L)))
        ident = float(rng.uniform(0.60, 0.95))
        out.append(Request(t, ti, evolve(rng, targets[ti][s:s + L], ident, 0.005), ident))
    return out


def to_2bit(seqs, big_endian: bool = False) -> bytes:
    """A UCSC 2bit file of [(name, ascii)] (the format in src/bit2.rs:9-27):
    N/n runs become N blocks, lowercase non-N runs mask blocks, and the packed
    DNA holds T/C/A/G = 0/1/2/3, first base in the high bits (N as T)."""
    import struct
    e = ">" if big_endian else "<"
    lut = np.zeros(256, np.uint8)
    for ch, v in ((b"T", 0), (b"C", 1), (b"A", 2), (b"G", 3)):
        lut[ch[0]] = v
        lut[ch[0] | 0x20] = v

    def runs(flags: np.ndarray):
        f = np.concatenate([[False], flags, [False]]).astype(np.int8)
        d = np.diff(f)
        starts = np.flatnonzero(d == 1)
        ends = np.flatnonzero(d == -1)
        return starts, ends - starts

    def arr(x):
        return np.asarray(x, dtype=e + "u4").tobytes()
    head = struct.pack(e + "IIII", 0x1A412743, 0, len(seqs), 0)
    index_size = sum(1 + len(n) + 4 for n, _ in seqs)
    body, index = [], b""
    off = 16 + index_size
    for name, asc in seqs:
        a_ = np.frombuffer(bytes(asc), np.uint8)
        up = a_ & 0xDF
        is_n = up == ord("N")
        is_low = (a_ >= 97) & (a_ <= 122) & ~is_n
        ns, nz = runs(is_n)
        ms, mz = runs(is_low)
        rec = struct.pack(e + "II", len(a_), len(ns)) + arr(ns) + arr(nz)
        rec += struct.pack(e + "I", len(ms)) + arr(ms) + arr(mz) + struct.pack(e + "I", 0)
        c = lut[a_]
        pad = (-len(c)) % 4
        c = np.concatenate([c, np.zeros(pad, np.uint8)]).reshape(-1, 4)
        pk = (c[:, 0] << 6) | (c[:, 1] << 4) | (c[:, 2] << 2) | c[:, 3]
        rec += pk.astype(np.uint8).tobytes()
        index += bytes([len(name)]) + name.encode() + struct.pack(e + "I", off)
        body.append(rec)
        off += len(rec)
    return head + index + b"".join(body)
