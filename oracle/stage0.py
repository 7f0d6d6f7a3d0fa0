"""CPU restatement of the reference's Stage 0 (test infrastructure only).

The sample (FastqPreReader::pre_read, src/FastqPreReader.h:110-330): at most
256 MiB; a plain file is read in three parts of a third of that, from offset
0, from size/2 - part/2 and from size - part, the last two moved to the first
"\\n@" within 64 KiB (find_next_record_start, :330-346); a read of at least a
part ends its segment, and the read that ends a segment resets the line
state to "header" before it is parsed (so the tail read continues the middle
read's state); reads are max(part, 2 MiB) long.  A gzip file is read as
2 MiB decompressed chunks until the compressed size or 256 MiB is reached
(the read that finds enough is dropped).  Sequence lines (line 1 of 4 from
the last reset) are collected; a reset inside a sequence line lets it run on
into the next collected sequence line.

Counts: canonical k-mers per root prefix (key word 0 >> 56) of the collected
lines (FastqPrefixCounter::count_prefixes), through the oracle's extractor.

Rules (src/main.cpp:38-108, :114-117, :174-186): counts below 1000 become
1000; average = sum // 256; classifier_num from n_thread; per-prefix filter
capacity = max(bit_ceil(int(size/3 * share * 4.81 / 64)), 2^15).  The
longest-processing-time assignment is restated only through its
tie-independent results (the sorted classifier loads).
"""
import gzip
import os

import numpy as np

import oracle

LIMIT = 256 * 1024 * 1024
CHUNK = 2 * 1024 * 1024


def _next_record(data, start):
    window = bytes(data[start:start + 65536])
    if len(window) <= 1:
        return start
    i = window.find(b"\n@")
    return start + i + 1 if i >= 0 else start


def _collect(chunks):
    """Sequence lines of (bytes, reset) chunks, joined by '\\n'."""
    out = bytearray()
    state = 0
    for data, reset in chunks:
        if reset:
            state = 0
        pos = 0
        n = len(data)
        while pos < n:
            nl = data.find(b"\n", pos)
            end = nl if nl >= 0 else n
            if state == 1:
                out += data[pos:end]
            if nl < 0:
                break
            if state == 1:
                out += b"\n"
            state = (state + 1) & 3
            pos = end + 1
    return bytes(out)


def sample_plain(data):
    """(collected sequence lines, sampled bytes) of a plain FASTQ's bytes."""
    data = bytes(data)
    size = len(data)
    need = min(size, LIMIT)
    part = need // 3 or 1
    chunk = max(part, CHUNK)
    offsets = [0, max(size // 2 - part // 2, 0), max(size - part, 0)]
    pos = have = seg_read = seg = 0
    chunks = []
    while True:
        d = data[pos:pos + chunk]
        if not d:
            break
        pos += len(d)
        seg_read += len(d)
        have += len(d)
        reset = False
        if seg_read >= part and seg < 2:
            reset = True
            seg += 1
            seg_read = 0
            pos = _next_record(data, offsets[seg])
        chunks.append((d, reset))
        if have >= need:
            break
    return _collect(chunks), sum(len(d) for d, _ in chunks)


def sample_gzip(raw, compressed_size):
    need = min(compressed_size, LIMIT)
    have = 0
    chunks = []
    while True:
        d = raw[have:have + CHUNK]
        if not d or have >= need:
            break
        chunks.append((d, False))
        have += len(d)
    return _collect(chunks), have


def prefix_counts(lines, k):
    """Canonical k-mers of the collected lines per root prefix."""
    fq = b"".join(b"@\n" + line + b"\n+\n\n" for line in lines.split(b"\n")) if lines else b""
    keys = oracle.extract(np.frombuffer(fq, np.uint8), k)
    if keys.shape[0] == 0:
        return np.zeros(256, np.int64)
    return np.bincount((keys[:, 0] >> np.uint64(56)).astype(np.int64), minlength=256)


def sample_file(path, k):
    with open(path, "rb") as f:
        head = f.read(2)
    size = os.path.getsize(path)
    if head == b"\x1f\x8b":
        with gzip.open(path, "rb") as f:
            raw = f.read()
        lines, sampled = sample_gzip(raw, size)
        est = size * 4
    else:
        with open(path, "rb") as f:
            lines, sampled = sample_plain(f.read())
        est = size
    return prefix_counts(lines, k), est, sampled


def classifiers(n_thread):
    parser = max(n_thread // 8, 1)
    budget = n_thread - 2 - parser
    return max(1, int(budget / 2.0))


def rule(counts, est, n_thread):
    c = np.maximum(np.asarray(counts, np.int64) % (1 << 32), 1000)
    total = int(c.sum())
    caps = []
    for v in c:
        e = int(est // 3 * (int(v) / total) * 4.81 / 64)
        caps.append(max(1 << max(e - 1, 0).bit_length() if e > 1 else 1, 1 << 15))
    # longest processing time: loads as a multiset (independent of ties)
    n = classifiers(n_thread)
    loads = [0] * n
    for v in sorted((int(x) for x in c), reverse=True):
        i = min(range(n), key=lambda j: loads[j])
        loads[i] += v
    return {"average": total // 256, "classifiers": n, "max_capacity": max(caps), "capacity": caps,
            "loads_sorted": sorted(loads)}
