"""B200 seed->HSP stage of lastz-gxy: the reference's PosTable / search API over libgxyseed.so.

The names, argument meanings and error behaviour follow the reference's Rust
API for this path:

    PosTable::build / prune_hot_words   src/pos_table.rs:35-136
    seed_search::search                 src/seed_search.rs:45-125
    SeedPattern                         src/seeds.rs:20-162
    ScoringMatrix::hoxd70               src/scoring.rs:17-58
    HspParams / SearchParams            src/hsp.rs:46-59, src/seed_search.rs:19-41
    PackedSeq                           src/sequences.rs:53-318

All compute runs in the CUDA library; this module only marshals arguments.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._lib import GxyError, check, lib

HSP_DTYPE = np.dtype([("t_start", "<u4"), ("q_start", "<u4"), ("length", "<u4"), ("score", "<i4")])
RECORD_DTYPE = np.dtype([("group", "<u4"), ("t_start", "<u4"), ("q_start", "<u4"), ("span", "<u4"),
                         ("score", "<i4"), ("unit", "<u4")])

__all__ = [
    "GxyError", "HSP_DTYPE", "Context", "parse_fasta", "parse_2bit", "choose_anchors", "best_chain", "best_chain_groups", "PackedSeq", "DeviceSeq", "SeedPattern", "ScoringMatrix", "HspParams",
    "SearchParams", "PosTable", "search", "search_device", "batch_search", "batch_records", "RECORD_DTYPE",
    "chunk_target", "extend_hits", "GappedParams", "GappedAlignment", "gapped_extend", "cigar",
    "Server", "build", "canonical_sort",
]


def build() -> str:
    """Builds libgxyseed.so (sm_100a) in-tree and returns its path."""
    return _lib.build()


# ---------------------------------------------------------------------------
# Context
# ---------------------------------------------------------------------------
class Context:
    """One CUDA device with its streams and workspaces (gxy_ctx)."""

    _default: dict[int, "Context"] = {}

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        check(lib().gxy_ctx_create(device, C.byref(h)))
        self.h = h
        self.device = device

    @classmethod
    def default(cls, device: int = 0) -> "Context":
        if device not in cls._default:
            cls._default[device] = Context(device)
        return cls._default[device]

    def set_tuning(self, screen_warps=0, screen_cap=0, screen_blocks_per_sm=0, walk_warps=0,
                   max_hits_per_pass=0, initial_candidates=0, filter_cap=0, filter_claim=0,
                   gapped_pool_blocks=0, gapped_cells=0) -> None:
        """Zero leaves a field unchanged; gapped_pool_blocks 0xffffffff lifts its limit."""
        t = _lib.TuningC(screen_warps, screen_cap, screen_blocks_per_sm, walk_warps, max_hits_per_pass,
                         initial_candidates, filter_cap, filter_claim, gapped_pool_blocks, gapped_cells)
        check(lib().gxy_ctx_set_tuning(self.h, C.byref(t)))

    def tuning(self) -> dict:
        t = _lib.TuningC()
        check(lib().gxy_ctx_get_tuning(self.h, C.byref(t)))
        return {"screen_warps": t.screen_warps, "screen_cap": t.screen_cap,
                "screen_blocks_per_sm": t.screen_blocks_per_sm, "walk_warps": t.walk_warps,
                "max_hits_per_pass": t.max_hits_per_pass, "initial_candidates": t.initial_candidates,
                "filter_cap": t.filter_cap, "filter_claim": t.filter_claim,
                "gapped_pool_blocks": t.gapped_pool_blocks, "gapped_cells": t.gapped_cells}

    def mark(self, slot: int) -> None:
        """Records CUDA event `slot` on the context's primary stream."""
        check(lib().gxy_ctx_mark(self.h, slot))

    def elapsed_ms(self, a: int, b: int) -> float:
        ms = C.c_double()
        check(lib().gxy_ctx_elapsed_ms(self.h, a, b, C.byref(ms)))
        return ms.value

    def close(self) -> None:
        if self.h:
            lib().gxy_ctx_destroy(self.h)
            self.h = None


# ---------------------------------------------------------------------------
# Sequences
# ---------------------------------------------------------------------------
_CODE = np.zeros(256, np.uint8)
_VALID = np.zeros(256, bool)
for _ch, _c in ((b"A", 0), (b"C", 1), (b"G", 2), (b"T", 3), (b"U", 3)):
    for _b in (_ch[0], _ch.lower()[0]):
        _CODE[_b] = _c
        _VALID[_b] = True
_LOWER = np.zeros(256, bool)
_LOWER[ord("a"):ord("z") + 1] = True


class PackedSeq:
    """Host PackedSeq: 2-bit codes (4/byte, LSB first) + valid + mask bitsets.

    The byte layout is the reference's (src/sequences.rs:53-66), so these
    arrays cross the C boundary unchanged.
    """

    def __init__(self, codes: np.ndarray, valid: np.ndarray, mask: np.ndarray, length: int):
        self.codes = np.ascontiguousarray(codes, np.uint8)
        self.valid = np.ascontiguousarray(valid, np.uint8)
        self.mask = np.ascontiguousarray(mask, np.uint8)
        self.length = int(length)
        if len(self.codes) < (self.length + 3) // 4 or len(self.valid) < (self.length + 7) // 8 \
                or len(self.mask) < (self.length + 7) // 8:
            raise ValueError("PackedSeq buffers shorter than the sequence")

    def __len__(self) -> int:
        return self.length

    @classmethod
    def from_ascii(cls, bases) -> "PackedSeq":
        """PackedSeq::from_ascii (src/sequences.rs:89-131): lowercase ACGT is soft-masked,
        anything but ACGTU (either case) is invalid with code 0."""
        if isinstance(bases, str):
            bases = bases.encode()
        a = np.frombuffer(bytes(bases), np.uint8) if not isinstance(bases, np.ndarray) else bases.astype(np.uint8)
        n = len(a)
        codes = _CODE[a]
        valid = _VALID[a]
        mask = valid & _LOWER[a]
        pad = (-n) % 8
        c = np.concatenate([codes, np.zeros(pad, np.uint8)]).reshape(-1, 4)
        packed = (c[:, 0] | (c[:, 1] << 2) | (c[:, 2] << 4) | (c[:, 3] << 6)).astype(np.uint8)
        return cls(packed[:(n + 3) // 4], np.packbits(valid, bitorder="little")[:(n + 7) // 8],
                   np.packbits(mask, bitorder="little")[:(n + 7) // 8], n)

    def c_struct(self) -> _lib.PackedSeqC:
        return _lib.PackedSeqC(self.codes.ctypes.data, self.valid.ctypes.data, self.mask.ctypes.data, self.length)

    def to_device(self, ctx: Optional[Context] = None) -> "DeviceSeq":
        ctx = ctx or Context.default()
        h = C.c_void_p()
        s = self.c_struct()
        check(lib().gxy_dseq_upload(ctx.h, C.byref(s), C.byref(h)))
        return DeviceSeq(ctx, h, self.length)

    def reverse_complement(self, ctx: Optional[Context] = None) -> "PackedSeq":
        """PackedSeq::reverse_complement (src/sequences.rs:303-318), computed on the device."""
        return self.to_device(ctx).reverse_complement().to_host()

    def code(self, i: int) -> int:
        return int((self.codes[i >> 2] >> ((i & 3) * 2)) & 3)

    def is_valid(self, i: int) -> bool:
        return bool((self.valid[i >> 3] >> (i & 7)) & 1)

    def is_masked(self, i: int) -> bool:
        return bool((self.mask[i >> 3] >> (i & 7)) & 1)

    def clear_masks(self) -> None:
        """--nomasking (src/sequences.rs:154-158, src/main.rs:26-30)."""
        self.mask[:] = 0

    def to_ascii(self) -> bytes:
        n = self.length
        c = np.stack([(self.codes >> s) & 3 for s in (0, 2, 4, 6)], axis=1).reshape(-1)[:n]
        v = np.unpackbits(self.valid, bitorder="little")[:n].astype(bool)
        out = np.frombuffer(b"ACGT", np.uint8)[c]
        out = np.where(v, out, ord("N")).astype(np.uint8)
        return out.tobytes()


class DeviceSeq:
    """A PackedSeq resident in HBM (gxy_dseq)."""

    def __init__(self, ctx: Context, h: C.c_void_p, length: int):
        self.ctx = ctx
        self.h = h
        self.length = length

    def __len__(self) -> int:
        return self.length

    @classmethod
    def from_ascii(cls, bases, ctx: Optional[Context] = None) -> "DeviceSeq":
        """Packs ASCII on the device (encode_base + push_ascii, src/dna.rs:12-20, src/sequences.rs:107-131)."""
        ctx = ctx or Context.default()
        if isinstance(bases, str):
            bases = bases.encode()
        buf = np.frombuffer(bytes(bases), np.uint8) if not isinstance(bases, np.ndarray) else \
            np.ascontiguousarray(bases, np.uint8)
        h = C.c_void_p()
        check(lib().gxy_dseq_from_ascii(ctx.h, buf.ctypes.data if len(buf) else None, len(buf), C.byref(h)))
        return cls(ctx, h, len(buf))

    def reverse_complement(self) -> "DeviceSeq":
        h = C.c_void_p()
        check(lib().gxy_dseq_reverse_complement(self.ctx.h, self.h, C.byref(h)))
        return DeviceSeq(self.ctx, h, self.length)

    def to_host(self) -> PackedSeq:
        n = self.length
        c = np.zeros(max((n + 3) // 4, 1), np.uint8)
        v = np.zeros(max((n + 7) // 8, 1), np.uint8)
        m = np.zeros(max((n + 7) // 8, 1), np.uint8)
        check(lib().gxy_dseq_download(self.h, c.ctypes.data, v.ctypes.data, m.ctypes.data))
        return PackedSeq(c, v, m, n)

    def free(self) -> None:
        if self.h:
            lib().gxy_dseq_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# Seed pattern, scoring, parameters
# ---------------------------------------------------------------------------
class SeedPattern:
    """Spaced seed (src/seeds.rs:20-162): '1' care, '0' don't care, <= 32 positions."""

    def __init__(self, name: str, mask: Sequence[bool]):
        if len(mask) == 0:
            raise ValueError("seed pattern must be non-empty")
        if len(mask) > 32:
            raise ValueError(f"seed pattern length {len(mask)} exceeds 32-position limit")
        self.mask = [bool(x) for x in mask]
        self.name = name

    @classmethod
    def parse(cls, name: str, spec: str) -> "SeedPattern":
        for ch in spec:
            if ch not in "01":
                raise ValueError(f"seed pattern character '{ch}' is not '0' or '1'")
        if not spec:
            raise ValueError("seed pattern is empty")
        return cls(name, [ch == "1" for ch in spec])

    @classmethod
    def twelve_of_nineteen(cls) -> "SeedPattern":
        return cls.parse("12of19", "1110100110010101111")

    @classmethod
    def nineteen_of_twenty(cls) -> "SeedPattern":
        return cls.parse("19of20", "11111111101111111111")

    @classmethod
    def solid(cls, k: int) -> "SeedPattern":
        return cls(f"match{k}", [True] * k)

    def __len__(self) -> int:
        return len(self.mask)

    def weight(self) -> int:
        return sum(self.mask)

    def bit_width(self) -> int:
        return 2 * self.weight()

    def num_words(self) -> int:
        return 1 << self.bit_width()

    def __str__(self) -> str:
        return "".join("1" if c else "0" for c in self.mask)


HOXD70 = [[91, -114, -31, -123], [-114, 100, -125, -31], [-31, -125, 100, -114], [-123, -31, -114, 91]]


@dataclass
class ScoringMatrix:
    """4x4 substitution scores [ref][query] plus the ambiguous-column score (src/scoring.rs:32-40)."""

    sub: list = field(default_factory=lambda: [row[:] for row in HOXD70])
    gap_open: int = 400
    gap_extend: int = 30
    ambig_score: int = -100

    @classmethod
    def hoxd70(cls) -> "ScoringMatrix":
        return cls()

    def score(self, r: int, q: int) -> int:
        return self.sub[r & 3][q & 3]


@dataclass
class HspParams:
    x_drop: int = 910
    hsp_threshold: int = 3000


@dataclass
class SearchParams:
    step: int = 1
    hsp: HspParams = field(default_factory=HspParams)
    transitions: int = 1
    entropy_threshold: Optional[int] = None


def _params_c(matrix: ScoringMatrix, params: SearchParams) -> _lib.SearchParamsC:
    p = _lib.SearchParamsC()
    for r in range(4):
        for q in range(4):
            p.sub[r * 4 + q] = int(matrix.sub[r][q])
    p.ambig = int(matrix.ambig_score)
    p.xdrop = int(params.hsp.x_drop)
    p.hspthresh = int(params.hsp.hsp_threshold)
    p.step = int(params.step)
    p.transitions = min(int(params.transitions), 255)
    p.has_entropy = 0 if params.entropy_threshold is None else 1
    p.entropy_thr = 0 if params.entropy_threshold is None else int(params.entropy_threshold)
    return p


# ---------------------------------------------------------------------------
# Position table
# ---------------------------------------------------------------------------
def _pattern_str(pattern) -> bytes:
    return str(pattern).encode()


class PosTable:
    """Device-resident seed-position index (src/pos_table.rs:24-28)."""

    def __init__(self, ctx: Context, h: C.c_void_p, pattern, target=None):
        self.ctx = ctx
        self.h = h
        self.pattern = pattern
        self._target = target   # keeps host buffers alive for the identity check in search()

    @classmethod
    def build(cls, seq, pattern, step: int, ctx: Optional[Context] = None) -> "PosTable":
        """PosTable::build(seq, pattern, step) (src/pos_table.rs:35-83)."""
        ctx = ctx or Context.default()
        h = C.c_void_p()
        if isinstance(seq, DeviceSeq):
            check(lib().gxy_table_build_view(ctx.h, seq.h, 0, seq.length, _pattern_str(pattern), step, 0,
                                             C.byref(h)))
            return cls(ctx, h, pattern, seq)
        s = seq.c_struct()
        check(lib().gxy_table_build(ctx.h, C.byref(s), _pattern_str(pattern), step, 0, C.byref(h)))
        return cls(ctx, h, pattern, seq)

    @classmethod
    def build_view(cls, dseq: DeviceSeq, lo: int, hi: int, pattern, step: int, max_word_count: int = 0,
                   ctx: Optional[Context] = None) -> "PosTable":
        """Table over dseq[lo:hi] with view-local positions (a driver chunk, src/driver.rs:178, :212)."""
        ctx = ctx or dseq.ctx
        h = C.c_void_p()
        check(lib().gxy_table_build_view(ctx.h, dseq.h, lo, hi, _pattern_str(pattern), step, max_word_count,
                                         C.byref(h)))
        t = cls(ctx, h, pattern, dseq)
        t.view = (lo, hi)
        return t

    @classmethod
    def build_views(cls, dseq: DeviceSeq, ranges, pattern, step: int, max_word_count: int = 0,
                    ctx: Optional[Context] = None) -> list:
        """One table per (lo, hi) view of dseq, built by one sort over all the
        views' windows (the driver's chunk tables, src/driver.rs:156-210);
        each equals build_view of its range."""
        ctx = ctx or dseq.ctx
        n = len(ranges)
        if n == 0:
            return []
        lo = np.array([r[0] for r in ranges], np.uint64)
        hi = np.array([r[1] for r in ranges], np.uint64)
        hs = (C.c_void_p * n)()
        check(lib().gxy_table_build_views(ctx.h, dseq.h, n, lo.ctypes.data, hi.ctypes.data, _pattern_str(pattern),
                                          step, max_word_count, hs))
        out = []
        for i in range(n):
            t = cls(ctx, C.c_void_p(hs[i]), pattern, dseq)
            t.view = (int(lo[i]), int(hi[i]))
            out.append(t)
        return out

    def prune_hot_words(self, limit: int) -> None:
        """PosTable::prune_hot_words(limit) (src/pos_table.rs:113-136)."""
        check(lib().gxy_table_prune_hot_words(self.h, limit))

    def info(self) -> dict:
        nw, npos, L, w = C.c_uint64(), C.c_uint64(), C.c_uint32(), C.c_uint32()
        check(lib().gxy_table_info(self.h, C.byref(nw), C.byref(npos), C.byref(L), C.byref(w)))
        return {"num_words": nw.value, "total_positions": npos.value, "pattern_len": L.value, "weight": w.value}

    def num_words(self) -> int:
        return self.info()["num_words"]

    def total_positions(self) -> int:
        return self.info()["total_positions"]

    def arrays(self):
        """Copies (starts, positions) back to host numpy arrays."""
        inf = self.info()
        starts = np.zeros(inf["num_words"] + 1, np.uint32)
        pos = np.zeros(max(inf["total_positions"], 1), np.uint32)
        check(lib().gxy_table_download(self.h, starts.ctypes.data, pos.ctypes.data))
        return starts, pos[:inf["total_positions"]]

    def lookup(self, word: int) -> np.ndarray:
        """PosTable::lookup (src/pos_table.rs:102-108)."""
        starts, pos = self.arrays()
        return pos[starts[word]:starts[word + 1]]

    def free(self) -> None:
        if self.h:
            lib().gxy_table_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# Search
# ---------------------------------------------------------------------------
def _stats(st: _lib.StatsC) -> dict:
    return {"windows": st.windows, "raw_hits": st.raw_hits, "candidates": st.candidates, "hsps": st.hsps,
            "device_ms": st.device_ms, "screen_ms": st.screen_ms, "columns": st.columns, "enum_ms": st.enum_ms,
            "passes": st.passes, "reruns": st.reruns, "survivors": st.survivors, "filter_columns": st.filter_columns,
            "filter_ms": st.filter_ms, "rounds": st.rounds, "graph_updates": st.graph_updates}


def _take_buf(buf: _lib.HspBufC) -> np.ndarray:
    n = int(buf.len)
    out = np.empty(n, HSP_DTYPE)
    if n:
        C.memmove(out.ctypes.data, buf.hsps, n * HSP_DTYPE.itemsize)
    lib().gxy_hsp_buf_free(C.byref(buf))
    return out


def search(table: PosTable, target: PackedSeq, query: PackedSeq, matrix: ScoringMatrix, params: SearchParams,
           stats: Optional[dict] = None) -> np.ndarray:
    """seed_search::search (src/seed_search.rs:45-125) on the GPU.

    Returns the HSPs as a structured array (t_start, q_start, length, score) in
    canonical (diagonal, t_start, length, score) order."""
    p = _params_c(matrix, params)
    t = target.c_struct()
    q = query.c_struct()
    buf = _lib.HspBufC()
    st = _lib.StatsC()
    check(lib().gxy_search(table.ctx.h, table.h, C.byref(t), C.byref(q), C.byref(p), C.byref(buf), C.byref(st)))
    if stats is not None:
        stats.update(_stats(st))
    return _take_buf(buf)


def search_device(table: PosTable, query: DeviceSeq, matrix: ScoringMatrix, params: SearchParams,
                  stats: Optional[dict] = None) -> np.ndarray:
    """search() with a device-resident query against the table's own target."""
    p = _params_c(matrix, params)
    buf = _lib.HspBufC()
    st = _lib.StatsC()
    check(lib().gxy_search_dseq(table.ctx.h, table.h, query.h, C.byref(p), C.byref(buf), C.byref(st)))
    if stats is not None:
        stats.update(_stats(st))
    return _take_buf(buf)


def batch_search(tables: Sequence[PosTable], queries: Sequence[DeviceSeq], units, matrix: ScoringMatrix,
                 params: SearchParams, use_graph: bool = False, stats: Optional[dict] = None,
                 ctx: Optional[Context] = None) -> list:
    """Runs many reference search() calls in one launch.

    units: iterable of (table_index, query_index, strand[, primary_lo, primary_hi]);
    strand 1 searches the query's reverse complement.  Returns one HSP array per
    unit, each in canonical order."""
    ctx = ctx or tables[0].ctx
    ul = list(units)
    uc = _units_c(ul)
    th = (C.c_void_p * max(len(tables), 1))(*[t.h for t in tables])
    qh = (C.c_void_p * max(len(queries), 1))(*[q.h for q in queries])
    p = _params_c(matrix, params)
    opts = _lib.BatchOptsC()
    opts.use_graph = 1 if use_graph else 0
    res = _lib.BatchResultC()
    st = _lib.StatsC()
    check(lib().gxy_batch_search(ctx.h, len(tables), th, len(queries), qh, len(ul), uc, C.byref(p), C.byref(opts),
                                 C.byref(res), C.byref(st)))
    if stats is not None:
        stats.update(_stats(st))
    n = int(res.n_hsps)
    allh = np.empty(n, HSP_DTYPE)
    if n:
        C.memmove(allh.ctypes.data, res.hsps, n * HSP_DTYPE.itemsize)
    offs = np.zeros(len(ul) + 1, np.uint64)
    if len(ul):
        C.memmove(offs.ctypes.data, res.unit_offsets, (len(ul) + 1) * 8)
    lib().gxy_batch_result_free(C.byref(res))
    return [allh[int(offs[i]):int(offs[i + 1])] for i in range(len(ul))]


def _units_c(ul) -> "C.Array":
    uc = (_lib.UnitC * max(len(ul), 1))()
    for i, u in enumerate(ul):
        uc[i].table, uc[i].query, uc[i].strand = int(u[0]), int(u[1]), int(u[2])
        if len(u) > 3:
            uc[i].primary_lo, uc[i].primary_hi = int(u[3]), int(u[4])
    return uc


def batch_records(tables: Sequence[PosTable], queries: Sequence[DeviceSeq], units, places, matrix: ScoringMatrix,
                  params: SearchParams, use_graph: bool = False, stats: Optional[dict] = None,
                  ctx: Optional[Context] = None):
    """batch_search followed by the driver's record post-processing on the
    device (src/driver.rs:370-391, :437-468).

    units as for batch_search; places: one (group, t_offset) per unit -- the
    output group (the driver's (target, query, strand) rank) and the chunk's
    global start.  Returns (records, group_offsets): a RECORD_DTYPE array in
    (group, t_start, q_start, span) order with repeats of those fields
    dropped, and the n_groups + 1 offsets of each group in it."""
    ctx = ctx or tables[0].ctx
    ul = list(units)
    pl = list(places)
    if len(pl) != len(ul):
        raise ValueError("one place per unit")
    uc = _units_c(ul)
    pc = (_lib.PlaceC * max(len(pl), 1))()
    for i, (g, off) in enumerate(pl):
        pc[i].group, pc[i].t_offset = int(g), int(off)
    th = (C.c_void_p * max(len(tables), 1))(*[t.h for t in tables])
    qh = (C.c_void_p * max(len(queries), 1))(*[q.h for q in queries])
    p = _params_c(matrix, params)
    opts = _lib.BatchOptsC()
    opts.use_graph = 1 if use_graph else 0
    res = _lib.RecordResultC()
    st = _lib.StatsC()
    check(lib().gxy_batch_records(ctx.h, len(tables), th, len(queries), qh, len(ul), uc, pc, C.byref(p),
                                  C.byref(opts), C.byref(res), C.byref(st)))
    if stats is not None:
        stats.update(_stats(st))
    n = int(res.n_records)
    recs = np.empty(n, RECORD_DTYPE)
    if n:
        C.memmove(recs.ctypes.data, res.records, n * RECORD_DTYPE.itemsize)
    offs = np.zeros(int(res.n_groups) + 1, np.uint64)
    C.memmove(offs.ctypes.data, res.group_offsets, (int(res.n_groups) + 1) * 8)
    lib().gxy_record_result_free(C.byref(res))
    return recs, offs


def _take_seq_set(ctx: "Context", st: _lib.SeqSetC) -> list:
    out = []
    try:
        for i in range(int(st.n)):
            h = st.seqs[i]
            name = st.names[i].decode()
            n = int(lib().gxy_dseq_len(h))
            out.append((name, DeviceSeq(ctx, C.c_void_p(h), n)))
            st.seqs[i] = None   # ownership moves to the DeviceSeq
    finally:
        lib().gxy_seq_set_free(C.byref(st))
    return out


def parse_fasta(data: bytes, ctx: Optional[Context] = None) -> list:
    """parse_fasta (src/sequences.rs:338-377) into device sequences: [(name, DeviceSeq)]."""
    ctx = ctx or Context.default()
    st = _lib.SeqSetC()
    data = bytes(data)
    check(lib().gxy_parse_fasta(ctx.h, C.cast(C.c_char_p(data), C.c_void_p), len(data), C.byref(st)))
    return _take_seq_set(ctx, st)


def parse_2bit(data: bytes, ctx: Optional[Context] = None) -> list:
    """parse_2bit (src/bit2.rs:73-163) into device sequences: [(name, DeviceSeq)]."""
    ctx = ctx or Context.default()
    st = _lib.SeqSetC()
    data = bytes(data)
    check(lib().gxy_parse_2bit(ctx.h, C.cast(C.c_char_p(data), C.c_void_p), len(data), C.byref(st)))
    return _take_seq_set(ctx, st)


def choose_anchors(target: DeviceSeq, query: DeviceSeq, hsps: np.ndarray, matrix: ScoringMatrix,
                   window: int, ctx: Optional[Context] = None) -> np.ndarray:
    """choose_anchor (src/anchor.rs:25-69) for every HSP: an (n, 2) array of (t_pos, q_pos)."""
    ctx = ctx or target.ctx
    h = np.ascontiguousarray(np.asarray(hsps, HSP_DTYPE))
    n = len(h)
    t = np.zeros(n, np.uint32)
    q = np.zeros(n, np.uint32)
    p = _params_c(matrix, SearchParams())
    check(lib().gxy_choose_anchors(ctx.h, target.h, query.h, C.byref(p), h.ctypes.data if n else None, n,
                                   int(window), t.ctypes.data if n else None, q.ctypes.data if n else None))
    return np.stack([t, q], axis=1)


def best_chain(hsps: np.ndarray) -> np.ndarray:
    """best_chain (src/chain.rs:19-69): the highest-scoring monotone chain, in t_start order."""
    h = np.ascontiguousarray(np.asarray(hsps, HSP_DTYPE))
    out = np.empty(len(h), HSP_DTYPE)
    n = C.c_uint64()
    check(lib().gxy_best_chain(h.ctypes.data if len(h) else None, len(h),
                               out.ctypes.data if len(h) else None, C.byref(n)))
    return out[:n.value].copy()


def best_chain_groups(groups, ctx: Optional[Context] = None) -> list:
    """best_chain (src/chain.rs:19-69) for every HSP array of `groups` at once
    on the device: one chain (an HSP array in t_start order) per group."""
    ctx = ctx or Context.default()
    arrs = [np.ascontiguousarray(np.asarray(g, HSP_DTYPE)) for g in groups]
    off = np.zeros(len(arrs) + 1, np.uint64)
    if arrs:
        off[1:] = np.cumsum([len(a) for a in arrs])
    h = np.concatenate(arrs) if arrs else np.empty(0, HSP_DTYPE)
    out = np.empty(len(h), HSP_DTYPE)
    ln = np.zeros(max(len(arrs), 1), np.uint64)
    check(lib().gxy_best_chain_groups(ctx.h, h.ctypes.data if len(h) else None, off.ctypes.data, len(arrs),
                                      out.ctypes.data if len(h) else None, ln.ctypes.data))
    return [out[int(off[g]):int(off[g]) + int(ln[g])].copy() for g in range(len(arrs))]


@dataclass
class GappedParams:
    """GappedParams (src/gapped_extend.rs:27-43): upstream lastz's HOXD70 defaults."""
    y_drop: int = 9400
    gapped_threshold: int = 3000


@dataclass
class GappedAlignment:
    """GappedAlignment (src/gapped_extend.rs:54-63); script = EditScript runs
    (count << 2 | op, op 0 = Match, 1 = InsertQuery, 2 = DeleteQuery)."""
    t_start: int
    q_start: int
    t_len: int
    q_len: int
    score: int
    script: np.ndarray

    def t_end(self) -> int:
        return self.t_start + self.t_len

    def q_end(self) -> int:
        return self.q_start + self.q_len


def cigar(script) -> str:
    """EditScript::to_cigar (src/edit_script.rs:122-129)."""
    return "".join(f"{int(r) >> 2}{'MID'[int(r) & 3]}" for r in script)


def gapped_extend(target: DeviceSeq, query: DeviceSeq, anchors, matrix: ScoringMatrix, params: GappedParams,
                  t_view: Optional[tuple] = None, ctx: Optional[Context] = None, stats: Optional[dict] = None) -> list:
    """extend (src/gapped_extend.rs:78-132) for every anchor (t_pos, q_pos) of
    an (n, 2) array, on the device: a list of GappedAlignment, or None where
    the reference returns None.  t_view = (lo, hi) extends within that slice
    of the target (the driver's chunk), anchors in its coordinates."""
    ctx = ctx or target.ctx
    a = np.ascontiguousarray(np.asarray(anchors, np.uint32).reshape(-1, 2))
    tp, qp = np.ascontiguousarray(a[:, 0]), np.ascontiguousarray(a[:, 1])
    n = len(a)
    lo, hi = t_view if t_view is not None else (0, 0)
    sp = _params_c(matrix, SearchParams())
    gp = _lib.GappedParamsC(matrix.gap_open, matrix.gap_extend, params.y_drop, params.gapped_threshold)
    res = _lib.GappedResultC()
    st = _lib.GappedStatsC()
    check(lib().gxy_gapped_extend(ctx.h, target.h, lo, hi, query.h, C.byref(sp), C.byref(gp),
                                  tp.ctypes.data if n else None, qp.ctypes.data if n else None, n, C.byref(res),
                                  C.byref(st)))
    try:
        runs = (np.ctypeslib.as_array(res.runs, (res.n_runs,)).copy() if res.n_runs else np.empty(0, np.uint32))
        out = []
        for k in range(n):
            g = res.alns[k]
            if not g.passed:
                out.append(None)
                continue
            out.append(GappedAlignment(g.t_start, g.q_start, g.t_len, g.q_len, g.score,
                                       runs[g.script_off:g.script_off + g.script_len].copy()))
    finally:
        lib().gxy_gapped_result_free(C.byref(res))
    if stats is not None:
        stats.update(rows=st.rows, cells=st.cells, device_ms=st.device_ms, reruns=st.reruns,
                     warps_per_side=st.warps_per_side, max_side_rows=st.max_side_rows,
                     second_pass_sides=st.second_pass_sides, cells_per_thread=st.cells_per_thread,
                     second_pass_cells=st.second_pass_cells)
    return out


def chunk_target(target_len: int, primary_bp: int, halo_bp: int) -> list:
    """chunk_target (src/driver.rs:156-194): [(chunk_lo, chunk_hi, primary_start_local, primary_end_local)]."""
    n = C.c_uint64()
    lib().gxy_chunk_plan(target_len, primary_bp, halo_bp, None, 0, C.byref(n))
    q = (C.c_uint64 * (4 * max(n.value, 1)))()
    check(lib().gxy_chunk_plan(target_len, primary_bp, halo_bp, q, n.value, C.byref(n)))
    return [tuple(int(q[4 * i + k]) for k in range(4)) for i in range(n.value)]


def extend_hits(target: DeviceSeq, query: DeviceSeq, matrix: ScoringMatrix, hsp: HspParams, t_pos, q_pos,
                seed_len: int, mode: int = 0):
    """extend_hit (src/hsp.rs:66-148) for each (t_pos[i], q_pos[i]); mode 0 lane-per-hit, 1 warp-per-hit.

    Returns (hsps, ok) where ok[i] is False when the reference returns None."""
    t = np.ascontiguousarray(t_pos, np.uint32)
    q = np.ascontiguousarray(q_pos, np.uint32)
    n = len(t)
    out = np.zeros(max(n, 1), HSP_DTYPE)
    ok = np.zeros(max(n, 1), np.uint8)
    p = _params_c(matrix, SearchParams(hsp=hsp))
    check(lib().gxy_extend_hits(target.ctx.h, target.h, query.h, C.byref(p), n, t.ctypes.data, q.ctypes.data,
                                seed_len, mode, out.ctypes.data, ok.ctypes.data))
    return out[:n], ok[:n].astype(bool)


def canonical_sort(h: np.ndarray) -> np.ndarray:
    """Sorts HSPs by (diagonal, t_start, length, score) and drops exact duplicates."""
    if len(h) == 0:
        return h
    d = h["t_start"].astype(np.int64) - h["q_start"].astype(np.int64)
    order = np.lexsort((h["score"], h["length"], h["t_start"], d))
    s = h[order]
    keep = np.ones(len(s), bool)
    keep[1:] = (s[1:] != s[:-1])
    return s[keep]


from .server import Server  # noqa: E402  (needs the names above)
