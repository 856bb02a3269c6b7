"""The allocation-free table build, checked against the regular one.

gxy_table_build_static serves callers that cannot allocate device memory
(their memory belongs to another allocator, or an allocation's device sync is
not acceptable on their path): they pass their own output buffers and the
library works in a fixed static device array.  Here the caller's buffers come
from torch.  Two builds in a row must each equal gxy_table_build's table bit
for bit -- the second also shows that the shared array's leftovers from the
first call do not leak into the next result.  This file is collected last so
that a run stopping at the first failure has already run every other test."""
import ctypes as C

import numpy as np
import pytest

from helpers import rand_ascii

pytestmark = pytest.mark.gpu


def static_build(gxy, seq, pattern: str, step: int):
    import torch
    L, w = len(pattern), pattern.count("1")
    nw = 1 << (2 * w)
    nwin = 0 if len(seq) < L else (len(seq) - L) // step + 1
    starts = torch.full((nw + 1,), 0x7f7f7f7f, dtype=torch.int32, device="cuda:0")
    pos = torch.full((max(nwin, 1),), 0x7f7f7f7f, dtype=torch.int32, device="cuda:0")
    n = C.c_uint64()
    s = seq.c_struct()
    torch.cuda.synchronize()
    gxy.check(gxy.lib().gxy_table_build_static(C.byref(s), pattern.encode(), step, starts.data_ptr(), nw + 1,
                                               pos.data_ptr(), pos.numel(), C.byref(n)))
    st = starts.cpu().numpy().view(np.uint32)
    ps = pos.cpu().numpy().view(np.uint32)[:n.value]
    return st, ps


def check_against_both(gxy, s: bytes, pattern: str, step: int):
    """The static build equals gxy_table_build's table and the oracle's
    PosTable::build (src/pos_table.rs:35-83), bucket order included."""
    import oracle as O
    T = gxy.PackedSeq.from_ascii(s)
    got_starts, got_pos = static_build(gxy, T, pattern, step)
    ref = gxy.PosTable.build(T, pattern, step)
    ref_starts, ref_pos = ref.arrays()
    assert np.array_equal(got_starts, ref_starts)
    assert np.array_equal(got_pos, ref_pos)
    ref.free()
    orc = O.Table(O.pack_ascii(s), pattern, step)
    assert np.array_equal(got_starts, orc.starts())
    assert np.array_equal(got_pos, orc.positions())


@pytest.mark.parametrize("pattern,step", [("1110100110010101111", 1), ("11111111", 2)])
def test_static_build_matches_table_build(gxy, pattern, step):
    import torch
    torch.cuda.init()
    rng = np.random.default_rng(7 + step)
    seqs = [rand_ascii(rng, 300_000, b"ACGTACGTacgtN"), rand_ascii(rng, 170_001, b"ACGTacgN")]
    for s in seqs:   # two calls in a row through the shared static array
        check_against_both(gxy, s, pattern, step)


def test_static_build_edges(gxy):
    # A target shorter than the pattern (no windows: the sort runs on zero
    # keys and every bucket is empty), then one of exactly the size limit
    # (the array's layout at its bound), then a short one again, whose result
    # must not see the large one's leftovers.
    import torch
    torch.cuda.init()
    rng = np.random.default_rng(11)
    check_against_both(gxy, b"ACGTACGTACGTACGTAC", "1110100110010101111", 1)
    check_against_both(gxy, rand_ascii(rng, 1 << 20, b"ACGTACGTacgtN"), "1110100110010101111", 1)
    check_against_both(gxy, rand_ascii(rng, 5_000, b"ACGTacgt"), "1110100110010101111", 1)


def test_static_build_rejects_oversize(gxy):
    # Longer than the fixed array allows: rejected before any device work, so
    # the output pointers are never touched.
    T = gxy.PackedSeq.from_ascii(b"ACGT" * ((1 << 20) // 4 + 1))
    n = C.c_uint64()
    s = T.c_struct()
    st = gxy.lib().gxy_table_build_static(C.byref(s), b"11111111", 1, 16, 1 << 20, 16, 1 << 21, C.byref(n))
    assert st == 1   # GXY_EINVAL
    assert b"too large" in gxy.lib().gxy_last_error()
