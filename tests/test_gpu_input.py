"""FASTA and 2bit parsed straight into device sequences must equal the
reference's parse followed by PackedSeq::from_ascii, bit for bit (codes, valid
and mask bytes), names included; malformed inputs fail with GxyError."""
import numpy as np
import pytest

import oracle as O
from helpers import rand_ascii, write_2bit

pytestmark = pytest.mark.gpu


def same(gxy, dev_seqs, want):
    assert [n for n, _ in dev_seqs] == [n for n, _ in want]
    for (name, d), (_, asc) in zip(dev_seqs, want):
        h = d.to_host()
        o = O.pack_ascii(asc)
        assert len(h) == o.len, name
        nb, nv = (o.len + 3) // 4, (o.len + 7) // 8
        assert bytes(h.codes[:nb]) == bytes(np.asarray(o.codes)[:nb]), name
        assert bytes(h.valid[:nv]) == bytes(np.asarray(o.valid)[:nv]), name
        assert bytes(h.mask[:nv]) == bytes(np.asarray(o.mask)[:nv]), name


FASTA_CASES = [
    b">a\n\nacgt\nACGT\n",                                   # src/sequences.rs:441-454
    b">x desc here\nACGTN\nacg\r\n>y\r\nTTTT\n\n>z\n",          # CRLF, description, empty record
    b"ACG\n>first\nTT\n",                                    # bases before the first header join it
    b">a\nAC>GT\n>b\n\tA C\x0cG\n",                          # '>' inside a line is a base; tab/FF/space skipped
    b"no header at all\n",
    b"",
]


@pytest.mark.parametrize("case", range(len(FASTA_CASES)))
def test_fasta_cases(gxy, ctx, case):
    data = FASTA_CASES[case]
    same(gxy, gxy.parse_fasta(data, ctx), O.parse_fasta(data))


def test_fasta_random_records(gxy, ctx):
    rng = np.random.default_rng(3)
    parts = []
    for r in range(40):
        seq = rand_ascii(rng, int(rng.integers(0, 30000)), b"ACGTacgtNnRY")
        width = int(rng.integers(1, 120))
        lines = [seq[i:i + width] for i in range(0, len(seq), width)]
        eol = b"\r\n" if r % 3 == 0 else b"\n"
        parts.append(b">rec%d some text%s" % (r, eol) + eol.join(lines) + eol)
    data = b"".join(parts)
    same(gxy, gxy.parse_fasta(data, ctx), O.parse_fasta(data))


def test_fasta_empty_header_fails(gxy, ctx):
    with pytest.raises(gxy.GxyError):
        gxy.parse_fasta(b">a\nACGT\n>  \nAC\n", ctx)


TWOBIT_CASES = [
    [("chr1", b"ACGTACGTACGT")],
    [("chrA", b"ACGT"), ("chrB", b"TTTT"), ("chrC", b"GATTACACATG")],
    [("chr1", b"ACGTNNNNACGT")],
    [("chr1", b"ACGTacgtACGT")],
    [("chr1", b"ACntACGT")],
    [("chr1", b"A"), ("chr2", b"AC"), ("chr3", b"ACG"), ("chr4", b"ACGT"), ("chr5", b"ACGTA")],
    [("empty", b"")],
]


@pytest.mark.parametrize("case", range(len(TWOBIT_CASES)))
@pytest.mark.parametrize("be", [False, True])
def test_2bit_cases(gxy, ctx, case, be):
    data = write_2bit(TWOBIT_CASES[case], big_endian=be)
    same(gxy, gxy.parse_2bit(data, ctx), O.parse_2bit(data))


def test_2bit_random_blocks(gxy, ctx):
    rng = np.random.default_rng(4)
    seqs = []
    for r in range(6):
        s = bytearray(rand_ascii(rng, int(rng.integers(1, 400000)), b"ACGT"))
        for _ in range(int(rng.integers(0, 60))):       # N runs and soft-masked runs, overlapping
            a = int(rng.integers(0, len(s)))
            b = min(len(s), a + int(rng.integers(1, 5000)))
            if rng.random() < 0.4:
                s[a:b] = b"N" * (b - a)
            else:
                s[a:b] = bytes(s[a:b]).lower()
        seqs.append(("s%d" % r, bytes(s)))
    data = write_2bit(seqs)
    same(gxy, gxy.parse_2bit(data, ctx), O.parse_2bit(data))


@pytest.mark.parametrize("bad", ["magic", "truncated", "version"])
def test_2bit_errors(gxy, ctx, bad):
    data = bytearray(write_2bit([("chr1", b"ACGTACGT")]))
    if bad == "magic":
        data = bytes(32)
    elif bad == "truncated":
        data = bytes(data[:-2])
    else:
        data[4] = 1
        data = bytes(data)
    with pytest.raises(gxy.GxyError):
        gxy.parse_2bit(data, ctx)
