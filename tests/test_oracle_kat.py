"""Known-answer tests of the oracle: canonical form, packing, merged view.

* Canonical form is re-derived here from its definition in the reference
  (src/GetKmer.h:58-82, :181-207): F = the window's bases in reverse read
  order, uncomplemented, left-aligned; C = the complemented bases in read
  order, left-aligned; key = lexicographic min(F, C).  This Python
  restatement is independent of oracle/kmer_oracle.cpp.
* Packing KATs restate tests/test_export_reader.cpp:175-289 of the reference
  (k=33 tail masking, k=64 no tail).
* Merged-histogram KATs restate tests/test_histogram_tool.cpp:211-303.
"""
import numpy as np
import pytest

import oracle

CODE = {"A": 0, "C": 1, "G": 2, "T": 3, "U": 3}


def words_of(bases, nw):
    """MSB-first 2-bit packing, left-aligned in nw 64-bit words."""
    v = 0
    for b in bases:
        v = (v << 2) | b
    v <<= 64 * nw - 2 * len(bases)
    return tuple((v >> (64 * (nw - 1 - i))) & ((1 << 64) - 1) for i in range(nw))


def canonical_py(window, k):
    nw = oracle.words(k)
    codes = [CODE[c.upper()] for c in window]
    F = words_of(list(reversed(codes)), nw)
    C = words_of([3 - c for c in codes], nw)
    return min(F, C)


def naive_keys(seq_lines, k):
    out = []
    valid = set("ACGTUacgtu")
    for s in seq_lines:
        run = 0
        for i, ch in enumerate(s):
            run = run + 1 if ch in valid else 0
            if run >= k:
                out.append(canonical_py(s[i - k + 1:i + 1], k))
    return out


def fq(reads):
    return "".join(f"@r{i}\n{s}\n+\n{'I' * len(s)}\n" for i, s in enumerate(reads)).encode()


@pytest.mark.parametrize("k", [1, 3, 5, 21, 31, 32, 33, 40, 63, 64])
def test_canonical_matches_definition(k):
    rng = np.random.default_rng(k)
    reads = ["".join(rng.choice(list("ACGTNacgtuU"), size=int(rng.integers(0, 140)))) for _ in range(40)]
    reads += ["A" * 80, "T" * 80, "ACGT" * 20, "GATTACA" * 12]
    got = [tuple(int(x) for x in r) for r in oracle.extract(fq(reads), k)]
    assert got == naive_keys(reads, k)


def test_tiny_by_hand():
    # "ACG", k=3: F = pack(G,C,A) = 10 01 00, C = pack(T,G,C) = 11 10 01
    key = oracle.extract(b"@r\nACG\n+\nIII\n", 3)
    assert key.shape == (1, 1)
    assert int(key[0, 0]) == 0b100100 << 58
    # palindromic window ACGT: F = TGCA = 11100100, C = TGCA -> same
    key = oracle.extract(b"@r\nACGT\n+\nIIII\n", 4)
    assert int(key[0, 0]) == 0b11100100 << 56


def test_only_sequence_lines_count():
    # bases in header, plus and quality lines are ignored; CR breaks runs
    data = b"@ACGTACGT\nACGTA\r\n+ACGTACGT\nACGTACGT\n@x\nAC\nGT\n+\nII\n"
    # line 2 of record 2 is "AC"; the next line "GT" is a plus line by count
    keys = oracle.extract(data, 3)
    assert keys.shape[0] == 3  # ACG, CGT, GTA from "ACGTA"; "\r" ends the run


def test_unterminated_last_record():
    assert oracle.extract(b"@r\nACGTACG", 4).shape[0] == 4


def test_pack_k33_tail_masking():
    # tests/test_export_reader.cpp:175-181 inputs; expected = tail word masked to 2 bits
    keys = np.array([[0x0123456789abcdef, 0xc0000000000000ff],
                     [0xfedcba9876543210, 0x8000000000001234],
                     [0x1111222233334444, 0x40000000ffffffff]], dtype=np.uint64)
    raw = oracle.pack(keys, 33)
    assert raw.size == 3 * 9
    assert bytes(raw[:9]) == bytes.fromhex("efcdab8967452301c0")
    back = oracle.unpack(raw, 33)
    exp = keys.copy()
    exp[:, 1] &= np.uint64(0xC000000000000000)
    assert np.array_equal(back, exp)


def test_pack_k64_no_tail():
    keys = np.array([[0x0123456789abcdef, 0xfedcba9876543210],
                     [0xaaaaaaaa55555555, 0x123456789abcdef0]], dtype=np.uint64)
    raw = oracle.pack(keys, 64)
    assert raw.size == 32
    assert np.array_equal(oracle.unpack(raw, 64), keys)


@pytest.mark.parametrize("k,P", [(21, 6), (31, 8), (32, 8), (33, 9), (63, 16), (64, 16), (1, 1), (17, 5)])
def test_packed_sizes(k, P):
    # src/ExportWriter.h:339-342
    assert oracle.packed_bytes(k) == P


def test_histogram_k33_two_phase():
    # tests/test_histogram_tool.cpp:211-235: roots {a:2, c:1, e:4}, low {a,b,c,e}
    a, b, c, e = [(0x0123456789abcdef, 0xc000000000000000), (0x1111111111111111, 0x8000000000000000),
                  (0x2222222222222222, 0x4000000000000000), (0x3333333333333333, 0)]
    low = np.array([a, b, c, e], dtype=np.uint64)
    rk = np.array([a, c, e], dtype=np.uint64)
    rc = np.array([2, 1, 4], dtype=np.uint32)
    _, counts = oracle.merged_counts(oracle.unpack(oracle.pack(low, 33), 33), rk, rc)
    assert list(oracle.histogram(counts, 1, 4)) == [1, 1, 1, 0]


def test_histogram_min_filter():
    # tests/test_histogram_tool.cpp:237-260: roots {g:1, h:2, i:5}, low {g,h,i,j}, range 3..5
    g, h, i, j = [(0x4444444444444444, 0xc000000000000000), (0x5555555555555555, 0x8000000000000000),
                  (0x6666666666666666, 0x4000000000000000), (0x7777777777777777, 0)]
    low = np.array([g, h, i, j], dtype=np.uint64)
    _, counts = oracle.merged_counts(low, np.array([g, h, i], dtype=np.uint64), np.array([1, 2, 5], np.uint32))
    assert list(oracle.histogram(counts, 3, 5)) == [1, 0, 0]


def test_histogram_n1_dispatch():
    # tests/test_histogram_tool.cpp:262-278: k=32, key in root (1) and low -> freq 2
    key = np.array([[0xaaaaaaaa55555555]], dtype=np.uint64)
    _, counts = oracle.merged_counts(oracle.unpack(oracle.pack(key, 32), 32), key, np.array([1], np.uint32))
    assert list(oracle.histogram(counts, 1, 3)) == [0, 1, 0]
