"""Seeded synthetic workloads (libkc_synth.so, include/kmer_synth.h).

Presets follow the reference benchmark shapes: plain small (5 Mbp i.i.d.
genome, 100k x 150 bp, k=31), genome-scale (100 Mbp, 45% GC, 20% repeat
families, 30x, 3' error ramp, k=31), batched uneven sets, and large long keys
(200 Mbp, 40% GC, 30% repeats, 50x, k=63).  No public dataset exists for the
reference; these generators stand in for one.
"""
import ctypes as C
import math
import os

import numpy as np

from ._native import SYNTH_PATH


class SynthParams(C.Structure):
    _fields_ = [
        ("seed", C.c_uint64), ("genome_len", C.c_uint64), ("gc", C.c_double), ("repeat_frac", C.c_double),
        ("rep_min_len", C.c_uint32), ("rep_max_len", C.c_uint32), ("rep_min_copies", C.c_uint32),
        ("rep_max_copies", C.c_uint32), ("rep_divergence", C.c_double), ("n_reads", C.c_uint64),
        ("read_len_min", C.c_uint32), ("read_len_max", C.c_uint32), ("sub_rate", C.c_double),
        ("sub_profile", C.c_uint32), ("n_rate", C.c_double), ("threads", C.c_uint32),
    ]


def _load():
    if not os.path.exists(SYNTH_PATH):
        raise ImportError(f"{SYNTH_PATH} is missing: run `python -m kmertreecounter_b200.build`")
    lib = C.CDLL(SYNTH_PATH)
    pp = C.POINTER(SynthParams)
    lib.kc_synth_genome.restype = C.c_int
    lib.kc_synth_genome.argtypes = [pp, C.c_void_p]
    lib.kc_synth_fastq_bytes.restype = C.c_uint64
    lib.kc_synth_fastq_bytes.argtypes = [pp]
    lib.kc_synth_fastq.restype = C.c_int64
    lib.kc_synth_fastq.argtypes = [pp, C.c_void_p, C.c_void_p, C.c_uint64]
    return lib


_lib = None


def _synth():
    global _lib
    if _lib is None:
        _lib = _load()
    return _lib


def params(seed=1, genome_len=5_000_000, gc=0.5, repeat_frac=0.0, rep_len=(1000, 10000), rep_copies=(2, 50),
           rep_divergence=0.01, n_reads=100_000, read_len=(150, 150), sub_rate=0.005, sub_profile=0,
           n_rate=0.001, threads=0):
    p = SynthParams()
    p.seed, p.genome_len, p.gc, p.repeat_frac = seed, genome_len, gc, repeat_frac
    p.rep_min_len, p.rep_max_len = rep_len
    p.rep_min_copies, p.rep_max_copies = rep_copies
    p.rep_divergence, p.n_reads = rep_divergence, n_reads
    p.read_len_min, p.read_len_max = read_len
    p.sub_rate, p.sub_profile, p.n_rate, p.threads = sub_rate, sub_profile, n_rate, threads
    return p


# Benchmark shapes.  `scale` shrinks genome and read count together (coverage
# and error structure unchanged) for tests and bounded CPU samples.
def plain_small(seed=1, scale=1.0):
    """5 Mbp i.i.d. genome, 100,000 x 150 bp, 0.5% substitution, 0.1% N; k=31."""
    return params(seed=seed, genome_len=max(1000, int(5_000_000 * scale)), n_reads=max(1, int(100_000 * scale)),
                  sub_rate=0.005, n_rate=0.001)


def genome_scale(seed=2, scale=1.0):
    """100 Mbp, 45% GC, 20% repeat families (1-10 kb x 2-50, 1% diverged),
    30x of 150 bp (20M reads), 1% mean substitution rising toward 3', 0.1% N; k=31."""
    return params(seed=seed, genome_len=max(20_000, int(100_000_000 * scale)), gc=0.45, repeat_frac=0.20,
                  n_reads=max(1, int(20_000_000 * scale)), sub_rate=0.01, sub_profile=1, n_rate=0.001)


def large_long(seed=5, scale=1.0):
    """200 Mbp, 40% GC, 30% repeats, 50x of 150 bp (~67M reads), 1% substitution; k=63."""
    g = max(20_000, int(200_000_000 * scale))
    return params(seed=seed, genome_len=g, gc=0.40, repeat_frac=0.30, n_reads=max(1, int(g * 50 / 150)),
                  sub_rate=0.01, n_rate=0.0)


def batched_sets(n_sets=512, seed=3, scale=1.0):
    """Uneven read sets: genomes 1-20 Mbp, GC 30-70%, reads log-uniform
    10k-2M, length 50-300, substitution 0.5-2%, k 21 or 31 alternating."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_sets):
        g = int(rng.uniform(1e6, 20e6) * scale)
        reads = int(math.exp(rng.uniform(math.log(1e4), math.log(2e6))) * scale)
        lo = int(rng.integers(50, 301))
        p = params(seed=seed * 100003 + i, genome_len=max(1000, g), gc=float(rng.uniform(0.3, 0.7)),
                   n_reads=max(1, reads), read_len=(lo, lo), sub_rate=float(rng.uniform(0.005, 0.02)),
                   n_rate=0.001)
        out.append((p, 21 if i % 2 == 0 else 31))
    return out


def genome(p):
    g = np.empty(p.genome_len, dtype=np.uint8)
    rc = _synth().kc_synth_genome(C.byref(p), g.ctypes.data)
    if rc != 0:
        raise RuntimeError("kc_synth_genome failed")
    return g


def fastq_bytes(p):
    return int(_synth().kc_synth_fastq_bytes(C.byref(p)))


def fastq(p, g=None, out=None):
    """FASTQ bytes of preset p as a uint8 array (or into `out`, a uint8 array
    or an integer host address with enough capacity)."""
    if g is None:
        g = genome(p)
    n = fastq_bytes(p)
    if out is None:
        out = np.empty(n, dtype=np.uint8)
    addr = out if isinstance(out, int) else out.ctypes.data
    w = _synth().kc_synth_fastq(C.byref(p), g.ctypes.data, addr, n)
    if w != n:
        raise RuntimeError(f"kc_synth_fastq wrote {w}, expected {n}")
    return out
