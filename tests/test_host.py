"""Host-side logic that needs no GPU: the C ABI's exports, chunk planning, the
Python mirror of the reference types, and unit sharding across ranks."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    txt = open(os.path.join(ROOT, "include", "gxy_seed.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(gxy_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol(gxy):
    lib = gxy.lib()
    names = header_functions()
    assert len(names) >= 30
    for n in names:
        assert hasattr(lib, n), n
    # and the Python binding declares every one of them
    assert set(names) == set(gxy._lib.SIGNATURES)


def chunk_target_ref(t_len, primary, halo):
    # src/driver.rs:156-194 restated for the check.
    if primary == 0 or t_len <= primary + halo:
        return [(0, t_len, 0, t_len)]
    out, ps = [], 0
    while ps < t_len:
        pe = min(ps + primary, t_len)
        lo = max(ps - halo, 0)
        hi = min(pe + halo, t_len)
        out.append((lo, hi, ps - lo, pe - lo))
        if pe == t_len:
            break
        ps = pe
    return out


@pytest.mark.parametrize("t_len,primary,halo", [(2032, 600, 200), (250_000_000, 10_000_000, 50_000),
                                               (100, 0, 50_000), (10_050_000, 10_000_000, 50_000),
                                               (10_050_001, 10_000_000, 50_000), (1, 1, 0)])
def test_chunk_plan(gxy, t_len, primary, halo):
    assert gxy.chunk_target(t_len, primary, halo) == chunk_target_ref(t_len, primary, halo)


def test_chunk_plan_250mbp_has_25_chunks(gxy):
    assert len(gxy.chunk_target(250_000_000, 10_000_000, 50_000)) == 25


def test_reference_types(gxy):
    p = gxy.SeedPattern.twelve_of_nineteen()
    assert len(p) == 19 and p.weight() == 12 and p.bit_width() == 24 and p.num_words() == 1 << 24
    assert gxy.SeedPattern.nineteen_of_twenty().weight() == 19
    assert str(gxy.SeedPattern.parse("custom", "1101")) == "1101"
    with pytest.raises(ValueError):
        gxy.SeedPattern.parse("x", "11X0")
    m = gxy.ScoringMatrix.hoxd70()
    assert m.score(0, 0) == 91 and m.score(1, 1) == 100 and m.ambig_score == -100
    sp = gxy.SearchParams()
    assert (sp.step, sp.hsp.x_drop, sp.hsp.hsp_threshold, sp.transitions) == (1, 910, 3000, 1)
    s = gxy.PackedSeq.from_ascii(b"ACgtNACGT")
    assert s.to_ascii() == b"ACGTNACGT" and s.is_masked(2) and not s.is_valid(4)


def test_packing_matches_oracle(gxy):
    import numpy as np
    import oracle as O
    from helpers import rand_ascii
    rng = np.random.default_rng(3)
    for n in (0, 1, 7, 33, 1000, 4099):
        b = rand_ascii(rng, n, b"ACGTUacgtuNRY-")
        a, o = gxy.PackedSeq.from_ascii(b), O.pack_ascii(b)
        assert bytes(a.codes[:(n + 3) // 4]) == bytes(o.codes[:(n + 3) // 4])
        assert bytes(a.valid[:(n + 7) // 8]) == bytes(o.valid[:(n + 7) // 8])
        assert bytes(a.mask[:(n + 7) // 8]) == bytes(o.mask[:(n + 7) // 8])


def test_no_gpu_fails_loudly(gxy):
    # Without a CUDA device the context cannot be created: no silent CPU path.
    from conftest import has_gpu
    if has_gpu():
        pytest.skip("a GPU is present")
    with pytest.raises(gxy.GxyError):
        gxy.Context(0)


def test_shard_units_partition():
    from lastz_gxy_b200.shard import shard_units
    for world in (1, 2, 3, 8):
        w = [((i * 7919) % 97) + 1 for i in range(50)]
        parts = [shard_units(50, r, world, w) for r in range(world)]
        assert sorted(sum(parts, [])) == list(range(50))
        parts = [shard_units(50, r, world) for r in range(world)]
        assert sorted(sum(parts, [])) == list(range(50))


def test_best_chain_matches_quadratic_reference(gxy):
    # gxy_best_chain (host code, O(n log n)) against the reference's O(n^2)
    # scan restated in the oracle: random HSP sets on a small grid so that
    # equal starts, equal ends, equal scores and equal chain totals are common.
    import oracle as O
    rng = np.random.default_rng(17)
    for trial in range(300):
        n = int(rng.integers(0, 60))
        span = int(rng.integers(5, 200))
        h = np.zeros(n, gxy.HSP_DTYPE)
        h["t_start"] = rng.integers(0, span, n)
        h["q_start"] = rng.integers(0, span, n)
        h["length"] = rng.integers(1, 12, n)
        h["score"] = rng.choice([100, 200, 300, -50, 0], n) if trial % 3 else rng.integers(-100, 1000, n)
        got = [tuple(int(x) for x in r) for r in gxy.best_chain(h)]
        assert got == O.best_chain(h), trial


def test_ctypes_layouts_match_the_header(gxy, tmp_path):
    """Every ctypes mirror of a C ABI struct has the size and field offsets
    that a C compiler gives the struct in include/gxy_seed.h."""
    import ctypes as C
    import subprocess
    from lastz_gxy_b200 import _lib
    pairs = {"gxy_packed_seq": _lib.PackedSeqC, "gxy_search_params": _lib.SearchParamsC, "gxy_hsp": _lib.HspC,
             "gxy_hsp_buf": _lib.HspBufC, "gxy_stats": _lib.StatsC, "gxy_seq_set": _lib.SeqSetC,
             "gxy_tuning": _lib.TuningC, "gxy_unit": _lib.UnitC, "gxy_batch_result": _lib.BatchResultC,
             "gxy_unit_place": _lib.PlaceC, "gxy_record_result": _lib.RecordResultC,
             "gxy_batch_opts": _lib.BatchOptsC, "gxy_server_opts": _lib.ServerOptsC,
             "gxy_server_stats": _lib.ServerStatsC, "gxy_gapped_params": _lib.GappedParamsC,
             "gxy_gapped_aln": _lib.GappedAlnC, "gxy_gapped_result": _lib.GappedResultC,
             "gxy_gapped_stats": _lib.GappedStatsC}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "gxy_seed.h"', 'int main(void) {']
    for cname, py in pairs.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    for cname, dt in (("gxy_hsp", gxy.HSP_DTYPE), ("gxy_record", gxy.RECORD_DTYPE)):
        lines.append(f'printf("{cname} npsize %zu\\n", sizeof({cname}));')
        for fname in dt.names:
            lines.append(f'printf("{cname} np_{fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    inc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")
    subprocess.run(["gcc", "-std=c11", "-I", inc, str(src), "-o", str(exe)], check=True)
    got = {}
    for line in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines():
        a, b, v = line.split()
        got[(a, b)] = int(v)
    for cname, py in pairs.items():
        assert got[(cname, "size")] == C.sizeof(py), cname
        for fname, _ in py._fields_:
            assert got[(cname, fname)] == getattr(py, fname).offset, (cname, fname)
    for cname, dt in (("gxy_hsp", gxy.HSP_DTYPE), ("gxy_record", gxy.RECORD_DTYPE)):
        assert got[(cname, "npsize")] == dt.itemsize, cname
        for fname in dt.names:
            assert got[(cname, "np_" + fname)] == dt.fields[fname][1], (cname, fname)


def test_driver_harness_compiles_against_the_header(gxy, tmp_path):
    """The C++ caller that mirrors the reference's driver builds against
    include/gxy_seed.h and links the library (running it needs a GPU)."""
    import subprocess
    here = os.path.dirname(os.path.abspath(__file__))
    out = str(tmp_path / "driver_harness")
    subprocess.run(["make", "-s", "-C", os.path.join(here, "harness"), f"OUT={out}"], check=True)
    assert os.path.exists(out)
