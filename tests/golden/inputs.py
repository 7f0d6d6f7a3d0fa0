"""Deterministic FASTQ inputs for the golden cases.

Each builder returns bytes that depend only on its arguments.  The adversarial
builder exercises every reader/parser rule the reference has
(src/FastqReader.h:140-365, src/FastqParser.h:182-455, src/GetKmer.h:22-82):
lowercase, U/u, N and IUPAC letters, digits and punctuation, CRLF line ends,
reads shorter than k, empty sequence lines, reads longer than the reader's
32 KiB block and 2 MiB file chunk, a record without its final newline, and
padding reads so the file is large enough that the reference's parser
termination race does not drop data (inputs below ~3 MB can lose blocks).
"""
import numpy as np

from kmertreecounter_b200 import synth


def plain_small(seed=1, scale=1.0):
    return synth.fastq(synth.plain_small(seed=seed, scale=scale)).tobytes()


# The benchmark shapes (seeded generator): genome-scale (100 Mbp, 45% GC, 20%
# repeat families, 30x, 3' error ramp, k=31) and large long keys (200 Mbp, 40%
# GC, 30% repeats, 50x, k=63), `scale` shrinking genome and reads together.
# These return numpy arrays (the full genome-scale input is 6.3 GB).
def genome_scale(seed=2, scale=1.0):
    return synth.fastq(synth.genome_scale(seed=seed, scale=scale))


def large_long(seed=5, scale=1.0):
    return synth.fastq(synth.large_long(seed=seed, scale=scale))


def _seq(rng, n, alphabet=b"ACGT"):
    a = np.frombuffer(alphabet, dtype=np.uint8)
    return a[rng.integers(0, a.size, n)].tobytes()


def _record(i, seq, eol=b"\n"):
    qual = bytes([33 + 30]) * len(seq)
    return b"@e" + str(i).encode() + eol + seq + eol + b"+" + eol + qual + eol


def adversarial(seed=11, pad_reads=30000):
    rng = np.random.default_rng(seed)
    genome = _seq(rng, 400_000)
    out = []
    i = 0

    def take(n):
        p = int(rng.integers(0, len(genome) - n))
        return genome[p:p + n]

    kinds = []
    for _ in range(3000):
        kind = int(rng.integers(0, 12))
        L = int(rng.integers(1, 220))
        s = bytearray(take(L))
        if kind == 0:      # lowercase
            s = bytearray(s.lower())
        elif kind == 1:    # mixed case
            for j in range(0, L, 3):
                s[j] = ord(chr(s[j]).lower())
        elif kind == 2:    # U / u for T
            s = bytearray(bytes(s).replace(b"T", b"U"))
            for j in range(0, L, 4):
                if s[j] == ord("U"):
                    s[j] = ord("u")
        elif kind == 3:    # N and IUPAC letters
            for j in rng.integers(0, L, max(1, L // 30)):
                s[int(j)] = b"NRYKMSWBDHVn."[int(rng.integers(0, 13))]
        elif kind == 4:    # digits / punctuation / high bytes
            for j in rng.integers(0, L, max(1, L // 40)):
                s[int(j)] = b"0159-*@+ \t\xc1\xe1\xff"[int(rng.integers(0, 13))]
        elif kind == 5:    # empty sequence line
            s = bytearray()
        kinds.append(kind)
        eol = b"\r\n" if kind == 6 else b"\n"
        out.append(_record(i, bytes(s), eol))
        i += 1
    # reads longer than the reference reader's 32 KiB block and 2 MiB chunk
    for L in (40_000, 70_001, 33_000, 2_500_000):
        s = bytearray(_seq(rng, L))
        s[L // 2] = ord("N")
        out.append(_record(i, bytes(s)))
        i += 1
    for _ in range(pad_reads):
        out.append(_record(i, take(150)))
        i += 1
    # final record without its trailing newline
    last = _record(i, take(120))
    out.append(last[:-1])
    return b"".join(out)
