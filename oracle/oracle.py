"""ctypes view of liboracle.so -- the CPU restatement of the reference's seed->HSP path.

TEST INFRASTRUCTURE ONLY.  tests/, __graft_entry__.smoke() and bench.py's CPU
baseline legs load this module as the checker / the timed CPU baseline; the
product path never imports it.  Every wrapped function restates a reference
function, cited in oracle/oracle.c.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")


def build() -> str:
    """Compiles liboracle.so from oracle.c with the Makefile beside it."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


class OrcSeq(C.Structure):
    _fields_ = [("codes", C.c_void_p), ("valid", C.c_void_p), ("mask", C.c_void_p), ("len", C.c_uint64)]


class OrcHsp(C.Structure):
    _fields_ = [("t_start", C.c_uint32), ("q_start", C.c_uint32), ("length", C.c_uint32), ("score", C.c_int32)]


class OrcParams(C.Structure):
    _fields_ = [
        ("sub", C.c_int32 * 16),
        ("ambig", C.c_int32),
        ("xdrop", C.c_int32),
        ("hspthresh", C.c_int32),
        ("step", C.c_uint32),
        ("transitions", C.c_uint8),
        ("has_entropy", C.c_uint8),
        ("pad_", C.c_uint8 * 2),
        ("entropy_thr", C.c_int32),
    ]


class OrcTable(C.Structure):
    _fields_ = [
        ("starts", C.POINTER(C.c_uint32)),
        ("positions", C.POINTER(C.c_uint32)),
        ("num_words", C.c_uint64),
        ("pattern_len", C.c_uint32),
        ("weight", C.c_uint32),
        ("care", C.c_uint8 * 32),
    ]


class OrcStats(C.Structure):
    _fields_ = [("windows", C.c_uint64), ("raw_hits", C.c_uint64), ("extended", C.c_uint64), ("hsps", C.c_uint64)]


class OrcGappedParams(C.Structure):
    _fields_ = [("gap_open", C.c_int32), ("gap_extend", C.c_int32), ("y_drop", C.c_int32),
                ("gapped_threshold", C.c_int32)]


class OrcGappedAln(C.Structure):
    _fields_ = [("t_start", C.c_uint32), ("q_start", C.c_uint32), ("t_len", C.c_uint32), ("q_len", C.c_uint32),
                ("score", C.c_int32), ("n_runs", C.c_uint32), ("runs", C.POINTER(C.c_uint32)),
                ("left_score", C.c_int32), ("right_score", C.c_int32), ("cells", C.c_uint64)]


HSP_DTYPE = np.dtype([("t_start", "<u4"), ("q_start", "<u4"), ("length", "<u4"), ("score", "<i4")])

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        P = C.POINTER
        L.orc_pack_ascii.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_reverse_complement.argtypes = [P(OrcSeq), C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_slice.argtypes = [P(OrcSeq), C.c_uint64, C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_word_at.argtypes = [P(OrcSeq), C.c_char_p, C.c_uint64, P(C.c_uint64)]
        L.orc_word_at.restype = C.c_int
        L.orc_table_build.argtypes = [P(OrcSeq), C.c_char_p, C.c_uint32, P(OrcTable)]
        L.orc_table_build.restype = C.c_int
        L.orc_table_prune.argtypes = [P(OrcTable), C.c_uint32]
        L.orc_table_free.argtypes = [P(OrcTable)]
        for f in (L.orc_extend_hit_scalar, L.orc_extend_hit_avx2):
            f.argtypes = [P(OrcSeq), P(OrcSeq), P(OrcParams), C.c_uint32, C.c_uint32, C.c_uint32, P(OrcHsp)]
            f.restype = C.c_int
        L.orc_has_avx2.restype = C.c_int
        L.orc_shannon_entropy.argtypes = [P(OrcSeq), C.c_uint64, C.c_uint64]
        L.orc_shannon_entropy.restype = C.c_double
        L.orc_passes_entropy_gate.argtypes = [P(OrcSeq), C.c_uint32, C.c_uint32, C.c_int32, C.c_int32]
        L.orc_passes_entropy_gate.restype = C.c_int
        L.orc_search.argtypes = [P(OrcTable), P(OrcSeq), P(OrcSeq), P(OrcParams), C.c_int, P(P(OrcHsp)),
                                 P(C.c_uint64), P(OrcStats)]
        L.orc_search.restype = C.c_int
        L.orc_search_units.argtypes = [C.c_int, P(P(OrcTable)), P(OrcSeq), P(OrcSeq), P(OrcParams), C.c_int,
                                       C.c_int, P(P(OrcHsp)), P(C.c_uint64), P(OrcStats)]
        L.orc_search_units.restype = C.c_int
        L.orc_best_chain.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p]
        L.orc_best_chain.restype = C.c_uint64
        L.orc_free.argtypes = [C.c_void_p]
        L.orc_gapped_extend.argtypes = [P(OrcSeq), P(OrcSeq), P(OrcParams), P(OrcGappedParams), C.c_uint32,
                                        C.c_uint32, P(OrcGappedAln)]
        L.orc_gapped_extend.restype = C.c_int
        L.orc_gapped_extend_many.argtypes = [P(OrcSeq), P(OrcSeq), P(OrcParams), P(OrcGappedParams), C.c_void_p,
                                             C.c_void_p, C.c_uint64, C.c_int, C.c_void_p, C.c_void_p]
        L.orc_gapped_extend_many.restype = C.c_int
        L.orc_diag_new.restype = C.c_void_p
        L.orc_diag_admit.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32]
        L.orc_diag_admit.restype = C.c_int
        L.orc_diag_mark_covered.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32]
        L.orc_diag_free.argtypes = [C.c_void_p]
        _lib = L
    return _lib


# ---------------------------------------------------------------------------
# Sequences: (codes, valid, mask, len) numpy byte arrays in the PackedSeq layout.
# ---------------------------------------------------------------------------
@dataclass
class Seq:
    codes: np.ndarray
    valid: np.ndarray
    mask: np.ndarray
    len: int

    def c(self) -> OrcSeq:
        return OrcSeq(self.codes.ctypes.data, self.valid.ctypes.data, self.mask.ctypes.data, self.len)


def _alloc(n: int):
    return (np.zeros((n + 3) // 4 + 8, np.uint8), np.zeros((n + 7) // 8 + 8, np.uint8),
            np.zeros((n + 7) // 8 + 8, np.uint8))


def pack_ascii(ascii: bytes | str) -> Seq:
    """PackedSeq::from_ascii (src/sequences.rs:89-95)."""
    if isinstance(ascii, str):
        ascii = ascii.encode()
    buf = np.frombuffer(ascii, np.uint8) if len(ascii) else np.zeros(1, np.uint8)
    n = len(ascii)
    c, v, m = _alloc(n)
    lib().orc_pack_ascii(buf.ctypes.data, n, c.ctypes.data, v.ctypes.data, m.ctypes.data)
    return Seq(c, v, m, n)


def reverse_complement(s: Seq) -> Seq:
    c, v, m = _alloc(s.len)
    lib().orc_reverse_complement(C.byref(s.c()), c.ctypes.data, v.ctypes.data, m.ctypes.data)
    return Seq(c, v, m, s.len)


def slice_to_new(s: Seq, start: int, end: int) -> Seq:
    c, v, m = _alloc(end - start)
    lib().orc_slice(C.byref(s.c()), start, end, c.ctypes.data, v.ctypes.data, m.ctypes.data)
    return Seq(c, v, m, end - start)


def word_at(s: Seq, pattern: str, pos: int):
    w = C.c_uint64(0)
    ok = lib().orc_word_at(C.byref(s.c()), pattern.encode(), pos, C.byref(w))
    return int(w.value) if ok else None


HOXD70 = [91, -114, -31, -123, -114, 100, -125, -31, -31, -125, 100, -114, -123, -31, -114, 91]


def params(xdrop=910, hspthresh=3000, step=1, transitions=1, entropy=None, sub=None, ambig=-100) -> OrcParams:
    p = OrcParams()
    for i, x in enumerate(sub if sub is not None else HOXD70):
        p.sub[i] = x
    p.ambig = ambig
    p.xdrop = xdrop
    p.hspthresh = hspthresh
    p.step = step
    p.transitions = transitions
    p.has_entropy = 1 if entropy is not None else 0
    p.entropy_thr = entropy if entropy is not None else 0
    return p


class Table:
    """PosTable::build (+ prune_hot_words), src/pos_table.rs:35-136."""

    def __init__(self, seq: Seq, pattern: str, step: int = 1, max_word_count: int = 0):
        self._t = OrcTable()
        self._seq = seq
        r = lib().orc_table_build(C.byref(seq.c()), pattern.encode(), step, C.byref(self._t))
        if r != 0:
            raise ValueError(f"orc_table_build failed ({r})")
        if max_word_count > 0:
            lib().orc_table_prune(C.byref(self._t), max_word_count)
        self.pattern = pattern
        self.pattern_len = self._t.pattern_len

    @property
    def num_words(self) -> int:
        return int(self._t.num_words)

    def starts(self) -> np.ndarray:
        return np.ctypeslib.as_array(self._t.starts, shape=(self.num_words + 1,)).copy()

    def positions(self) -> np.ndarray:
        n = int(self._t.starts[self.num_words])
        if n == 0:
            return np.zeros(0, np.uint32)
        return np.ctypeslib.as_array(self._t.positions, shape=(n,)).copy()

    def lookup(self, word: int) -> list[int]:
        s = self._t.starts
        return [int(self._t.positions[i]) for i in range(s[word], s[word + 1])]

    def __del__(self):
        try:
            lib().orc_table_free(C.byref(self._t))
        except Exception:
            pass


def extend_hit(t: Seq, q: Seq, p: OrcParams, tpos: int, qpos: int, seed_len: int, avx2: bool = False):
    h = OrcHsp()
    f = lib().orc_extend_hit_avx2 if avx2 else lib().orc_extend_hit_scalar
    ok = f(C.byref(t.c()), C.byref(q.c()), C.byref(p), tpos, qpos, seed_len, C.byref(h))
    return (h.t_start, h.q_start, h.length, h.score) if ok else None


def shannon_entropy(s: Seq, start: int, end: int) -> float:
    return float(lib().orc_shannon_entropy(C.byref(s.c()), start, end))


def passes_entropy_gate(s: Seq, t_start: int, t_end: int, score: int, thr: int) -> bool:
    return bool(lib().orc_passes_entropy_gate(C.byref(s.c()), t_start, t_end, score, thr))


def _to_array(ptr, n: int) -> np.ndarray:
    if n == 0:
        return np.zeros(0, HSP_DTYPE)
    raw = np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_uint8)), shape=(n * 16,))
    return raw.view(HSP_DTYPE).copy()


def search(table: Table, target: Seq, query: Seq, p: OrcParams, avx2: bool = False):
    """seed_search::search (src/seed_search.rs:45-125).  Returns (hsps, stats)."""
    out = C.POINTER(OrcHsp)()
    n = C.c_uint64(0)
    st = OrcStats()
    r = lib().orc_search(C.byref(table._t), C.byref(target.c()), C.byref(query.c()), C.byref(p), 1 if avx2 else 0,
                         C.byref(out), C.byref(n), C.byref(st))
    if r != 0:
        raise MemoryError("orc_search failed")
    arr = _to_array(out, n.value)
    lib().orc_free(out)
    return arr, {"windows": st.windows, "raw_hits": st.raw_hits, "extended": st.extended, "hsps": st.hsps}


def search_units(units, p: OrcParams, avx2: bool = True, threads: int = 1):
    """Runs search over [(table, target, query)] units on `threads` POSIX threads."""
    nu = len(units)
    if nu == 0:
        return [], []
    tabs = (C.POINTER(OrcTable) * nu)(*[C.pointer(u[0]._t) for u in units])
    ts = (OrcSeq * nu)(*[u[1].c() for u in units])
    qs = (OrcSeq * nu)(*[u[2].c() for u in units])
    outs = (C.POINTER(OrcHsp) * nu)()
    ns = (C.c_uint64 * nu)()
    sts = (OrcStats * nu)()
    r = lib().orc_search_units(nu, tabs, ts, qs, C.byref(p), 1 if avx2 else 0, threads, outs, ns, sts)
    if r != 0:
        raise MemoryError("orc_search_units failed")
    res, stats = [], []
    for i in range(nu):
        res.append(_to_array(outs[i], ns[i]))
        lib().orc_free(outs[i])
        stats.append({"windows": sts[i].windows, "raw_hits": sts[i].raw_hits, "extended": sts[i].extended,
                      "hsps": sts[i].hsps})
    return res, stats


class DiagHash:
    """DiagHash (src/diag_hash.rs:19-53)."""

    def __init__(self):
        self.h = lib().orc_diag_new()

    def admit(self, t: int, q: int) -> bool:
        return bool(lib().orc_diag_admit(self.h, t, q))

    def mark_covered(self, t_end: int, q_end: int) -> None:
        lib().orc_diag_mark_covered(self.h, t_end, q_end)

    def __del__(self):
        try:
            lib().orc_diag_free(self.h)
        except Exception:
            pass


# ---- input formats: pure-Python restatements (small inputs only) -------------
class InputError(ValueError):
    """The reference's SeqError::EmptyHeader / Bit2Error variants."""


_WS = b" \t\n\x0c\r"   # u8::is_ascii_whitespace


def parse_fasta(data: bytes) -> list:
    """parse_fasta (src/sequences.rs:338-377): [(name, ascii_bases)].

    Lines split at LF; empty lines skipped; a line starting with '>' starts a
    record named by its first whitespace-delimited token (none: error); every
    other byte except ASCII whitespace is a base.  Bases before the first
    header stay in the buffer and join the first record (:349-356)."""
    seqs = []
    cur_name = None
    cur = bytearray()
    for lineno, line in enumerate(data.split(b"\n")):
        if not line:
            continue
        if line[:1] == b">":
            if cur_name is not None:
                seqs.append((cur_name, bytes(cur)))
                cur = bytearray()
            toks = line[1:].split()
            if not toks:
                raise InputError(f"empty header at line {lineno + 1}")
            cur_name = toks[0].decode()
        else:
            cur.extend(b for b in line if b not in _WS)
    if cur_name is not None:
        seqs.append((cur_name, bytes(cur)))
    return seqs


def parse_2bit(data: bytes) -> list:
    """parse_2bit (src/bit2.rs:73-163): [(name, ascii)] with N blocks as 'N'
    and mask blocks lowercased (N stays N), the ASCII the reference feeds to
    PackedSeq::from_ascii."""
    import struct
    if len(data) < 4:
        raise InputError("truncated")
    m = struct.unpack_from("<I", data, 0)[0]
    if m == 0x1A412743:
        e = "<"
    elif m == 0x4327411A:
        e = ">"
    else:
        raise InputError(f"bad magic 0x{m:08x}")

    def u32(pos):
        if pos + 4 > len(data):
            raise InputError("truncated")
        return struct.unpack_from(e + "I", data, pos)[0]
    if u32(4) != 0:
        raise InputError("bad version")
    count = u32(8)
    pos = 16
    index = []
    for _ in range(count):
        if pos + 1 > len(data):
            raise InputError("truncated")
        ns = data[pos]
        pos += 1
        if pos + ns > len(data):
            raise InputError("truncated")
        name = data[pos:pos + ns].decode()
        pos += ns
        index.append((name, u32(pos)))
        pos += 4
    out = []
    acgt = b"TCAG"
    for name, off in index:
        p = off
        dna = u32(p); p += 4
        blocks = []
        for _ in range(2):
            k = u32(p); p += 4
            st = [u32(p + 4 * j) for j in range(k)]; p += 4 * k
            sz = [u32(p + 4 * j) for j in range(k)]; p += 4 * k
            blocks.append(list(zip(st, sz)))
        p += 4
        nb = (dna + 3) // 4
        if p + nb > len(data):
            raise InputError("truncated")
        packed = data[p:p + nb]
        asc = bytearray(acgt[(packed[i >> 2] >> (6 - (i & 3) * 2)) & 3] for i in range(dna))
        for s, z in blocks[0]:
            for i in range(min(s, dna), min(s + z, dna)):
                asc[i] = ord("N")
        for s, z in blocks[1]:
            for i in range(min(s, dna), min(s + z, dna)):
                if asc[i] != ord("N"):
                    asc[i] = asc[i] | 0x20
        out.append((name, bytes(asc)))
    return out


# ---- gapped extension (src/gapped_extend.rs:78-460) through liboracle -------
OPS = "MID"   # EditOp Match / InsertQuery / DeleteQuery as CIGAR letters (src/edit_script.rs:17-33)


def gapped_params(gap_open=400, gap_extend=30, y_drop=9400, gapped_threshold=3000) -> OrcGappedParams:
    """GappedParams::default() (src/gapped_extend.rs:33-43) with HOXD70's gap
    costs (src/scoring.rs:25-26)."""
    return OrcGappedParams(gap_open, gap_extend, y_drop, gapped_threshold)


def _aln_result(a: OrcGappedAln):
    runs = [int(a.runs[k]) for k in range(a.n_runs)]
    lib().orc_free(C.cast(a.runs, C.c_void_p))
    return {"t_start": a.t_start, "q_start": a.q_start, "t_len": a.t_len, "q_len": a.q_len, "score": a.score,
            "runs": runs}


def gapped_extend(t: Seq, q: Seq, p: OrcParams, gp: OrcGappedParams, t_pos: int, q_pos: int):
    """extend() (src/gapped_extend.rs:78-132): a dict (t_start, q_start,
    t_len, q_len, score, runs) or None when the total is below the gapped
    threshold.  runs: count << 2 | op, op 0 = M, 1 = I, 2 = D."""
    a = OrcGappedAln()
    rc = lib().orc_gapped_extend(C.byref(t.c()), C.byref(q.c()), C.byref(p), C.byref(gp), t_pos, q_pos, C.byref(a))
    if rc < 0:
        raise MemoryError("orc_gapped_extend") if rc == -1 else ValueError("anchor outside a sequence")
    return _aln_result(a) if rc == 1 else None


def gapped_extend_many(t: Seq, q: Seq, p: OrcParams, gp: OrcGappedParams, t_pos, q_pos, threads: int = 1,
                       cells: list | None = None):
    """extend() for many anchors on `threads` host threads: a list of dicts or
    None, as gapped_extend.  `cells`, when given, receives each anchor's DP
    cell count (both sides)."""
    tp = np.ascontiguousarray(t_pos, np.uint32)
    qp = np.ascontiguousarray(q_pos, np.uint32)
    n = len(tp)
    if n == 0:
        return []
    outs = (OrcGappedAln * n)()
    rc = np.zeros(n, np.int32)
    lib().orc_gapped_extend_many(C.byref(t.c()), C.byref(q.c()), C.byref(p), C.byref(gp), tp.ctypes.data,
                                 qp.ctypes.data, n, threads, C.addressof(outs), rc.ctypes.data)
    res = []
    if cells is not None:
        cells.extend(int(outs[k].cells) for k in range(n))
    for k in range(n):
        if rc[k] < 0:
            raise MemoryError("orc_gapped_extend") if rc[k] == -1 else ValueError("anchor outside a sequence")
        res.append(_aln_result(outs[k]) if rc[k] == 1 else None)
    return res


def cigar(runs) -> str:
    """EditScript::to_cigar (src/edit_script.rs:122-129): count + letter per run."""
    return "".join(f"{r >> 2}{OPS[r & 3]}" for r in runs)


# ---- HSP consumers: pure-Python restatements ---------------------------------
def choose_anchor(hsp, t: Seq, q: Seq, sub, ambig: int, window: int):
    """choose_anchor (src/anchor.rs:25-69): (t_pos, q_pos) of the midpoint of
    the first highest-scoring window of clamp(window, 1, length) columns."""
    t0, q0, length = int(hsp[0]), int(hsp[1]), int(hsp[2])
    assert length >= 1
    w = min(max(window, 1), length)

    def col(k):
        ti, qi = t0 + k, q0 + k
        tv = (int(t.valid[ti >> 3]) >> (ti & 7)) & 1
        qv = (int(q.valid[qi >> 3]) >> (qi & 7)) & 1
        if not (tv and qv):
            return ambig
        tc = (int(t.codes[ti >> 2]) >> ((ti & 3) * 2)) & 3
        qc = (int(q.codes[qi >> 2]) >> ((qi & 3) * 2)) & 3
        return sub[tc][qc]
    cols = [col(k) for k in range(length)]
    best_start, best = 0, sum(cols[:w])
    cur = best
    for start in range(1, length - w + 1):
        cur = cur - cols[start - 1] + cols[start + w - 1]
        if cur > best:
            best, best_start = cur, start
    mid = best_start + w // 2
    return t0 + mid, q0 + mid


def best_chain_c(hsps: np.ndarray) -> np.ndarray:
    """best_chain (src/chain.rs:19-69) through liboracle's O(n^2) C form, for
    groups too large for the Python loop below: an HSP record array."""
    h = np.ascontiguousarray(hsps)
    out = np.empty(len(h), h.dtype)
    n = lib().orc_best_chain(h.ctypes.data if len(h) else None, len(h), out.ctypes.data if len(h) else None)
    return out[:n].copy()


def best_chain(hsps) -> list:
    """best_chain (src/chain.rs:19-69), the reference's O(n^2) form: a list of
    (t_start, q_start, length, score) tuples in chain order."""
    hs = [tuple(int(x) for x in h) for h in hsps]
    if not hs:
        return []
    srt = sorted(hs, key=lambda h: (h[0], h[1]))   # stable
    n = len(srt)
    best = [h[3] for h in srt]
    parent = [-1] * n
    for i in range(1, n):
        bp, bi = 0, -1
        ti, qi = srt[i][0], srt[i][1]
        for j in range(i):
            hj = srt[j]
            if hj[0] + hj[2] <= ti and hj[1] + hj[2] <= qi and best[j] > bp:
                bp, bi = best[j], j
        best[i] = bp + srt[i][3]
        parent[i] = bi
    end = 0
    for i in range(n):
        if best[i] > best[end]:
            end = i
    out = []
    c = end
    while c >= 0:
        out.append(srt[c])
        c = parent[c]
    return out[::-1]


def driver_records(entries) -> list:
    """The driver's --nogapped post-processing of search() results.

    entries: (target_index, query_index, strand, chunk_start, primary_lo,
    primary_hi, hsps) per (chunk, query, strand) unit, in the order the units
    completed.  Per unit: keep HSPs whose chunk-local t_start lies in
    [primary_lo, primary_hi) (src/driver.rs:250-256) and build ungapped
    records with t_start + chunk_start and t_span = q_span = length
    (build_ungapped_record, src/driver.rs:437-468).  Units with records are
    then ordered by (target, query, strand), stably (src/driver.rs:370-371),
    and each unit's records are sorted by (t_start, q_start, t_span, q_span)
    and consecutive duplicates of those fields (and the strand) dropped,
    keeping the first (src/driver.rs:373-389), before the units' lists are
    concatenated.  Returns (target, query, strand, t_start, q_start, span,
    score) tuples."""
    grouped = []
    for ti, qi, strand, chunk_start, plo, phi, hsps in entries:
        recs = []
        for h in hsps:
            t, q, length, score = (int(x) for x in h)
            if plo <= t < phi:
                recs.append(((t + chunk_start) & 0xFFFFFFFF, q, length, length, score))
        if recs:
            grouped.append((ti, qi, strand, recs))
    grouped.sort(key=lambda g: (g[0], g[1], g[2]))   # stable, like sort_by_key
    out = []
    for ti, qi, strand, recs in grouped:
        recs.sort(key=lambda r: r[:4])                # stable, like sort_by_key
        kept = []
        for r in recs:
            if kept and kept[-1][:4] == r[:4]:
                continue
            kept.append(r)
        out.extend((ti, qi, strand, r[0], r[1], r[2], r[4]) for r in kept)
    return out


def chunk_target(target_len: int, primary_bp: int, halo_bp: int) -> list:
    """chunk_target (src/driver.rs:156-194): [(chunk_lo, chunk_hi,
    primary_start_local, primary_end_local)].  One chunk covering the whole
    target when chunking is off or the target is at most primary + halo long
    (src/driver.rs:162); otherwise primaries of primary_bp bases, each widened
    by halo_bp on both sides and clamped to the target."""
    if primary_bp == 0 or target_len <= primary_bp + halo_bp:
        return [(0, target_len, 0, target_len)]
    out = []
    ps = 0
    while ps < target_len:
        pe = min(ps + primary_bp, target_len)
        lo = max(ps - halo_bp, 0)
        hi = min(pe + halo_bp, target_len)
        out.append((lo, hi, ps - lo, pe - lo))
        if pe == target_len:
            break
        ps = pe
    return out
