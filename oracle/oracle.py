"""CPU oracle for the exact canonical k-mer counting path.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py as the checker, never by the product.

* extract/count: ctypes calls into oracle/_build/libkmer_oracle.so, a plain
  single-threaded C++ restatement of the reference's reader, parser and
  GetKmer (see oracle/kmer_oracle.cpp for the file:line it follows).
* pack/unpack: the low.bin record layout (src/ExportWriter.h:522-550,
  tool/ExportReader.h:355-391), restated in numpy.
* merged_counts / histogram: the merged view of low.bin + root files that
  tool/histogram_tool.cpp "precise" computes
  (tool/HighFrequencyInsertThreadPool.h:150-177,
  tool/LowFrequencyQueryThreadPool.h:375-432): exact count = root count +
  [key in low.bin].
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libkmer_oracle.so")
REF_TREE = os.path.join(HERE, "_ref", "Tree")
REF_HIST = os.path.join(HERE, "_ref", "histogram_tool")
REF_STAGE0 = os.path.join(HERE, "_ref", "stage0")
REF_POST = os.path.join(HERE, "_ref", "postprocess")
# where build() looks for the reference's sources (absent on machines that
# only carry the prebuilt oracle/_ref binaries)
REF_SRC = os.environ.get("KC_REFERENCE_SRC", "/root/reference")

_lib = None


def build():
    """Compile the restatement (and the reference binaries when its sources
    are present).  Idempotent."""
    src = os.path.join(HERE, "kmer_oracle.cpp")
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", HERE, "oracle"])
    if not all(os.path.exists(p) for p in (REF_TREE, REF_STAGE0, REF_POST)):
        subprocess.call(["make", "-s", "-C", HERE, "ref", f"REF={REF_SRC}"])


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        lib = C.CDLL(LIB)
        u64, u32, vp = C.c_uint64, C.c_uint32, C.c_void_p
        lib.kor_words.restype = u32
        lib.kor_words.argtypes = [u32]
        lib.kor_extract.restype = u64
        lib.kor_extract.argtypes = [vp, u64, u32, vp, u64]
        lib.kor_count.restype = C.c_int64
        lib.kor_count.argtypes = [vp, u64, u32, vp, vp, u64, C.POINTER(u64)]
        lib.kor_packed_bytes.restype = u64
        lib.kor_packed_bytes.argtypes = [u32]
        lib.kor_pack.restype = None
        lib.kor_pack.argtypes = [vp, u64, u32, vp]
        lib.kor_unpack.restype = None
        lib.kor_unpack.argtypes = [vp, u64, u32, vp]
        _lib = lib
    return _lib


def words(k):
    return 1 if k <= 32 else (2 if k <= 64 else 4)


def _as_u8(data):
    if isinstance(data, (bytes, bytearray)):
        return np.frombuffer(data, dtype=np.uint8)
    return np.ascontiguousarray(data, dtype=np.uint8)


def extract(data, k):
    """All canonical keys in emission order, shape (K, N) uint64."""
    lib = _load()
    buf = _as_u8(data)
    K = lib.kor_extract(buf.ctypes.data, buf.size, k, None, 0)
    out = np.empty((K, words(k)), dtype=np.uint64)
    lib.kor_extract(buf.ctypes.data, buf.size, k, out.ctypes.data, K)
    return out


def total_kmers(data, k):
    """K (valid windows) without materialising the keys."""
    lib = _load()
    buf = _as_u8(data)
    return int(lib.kor_extract(buf.ctypes.data, buf.size, k, None, 0))


def count(data, k):
    """Exact counts: (keys (D, N) uint64 sorted lexicographically, counts (D,) uint32, K)."""
    lib = _load()
    buf = _as_u8(data)
    total = C.c_uint64()
    d = lib.kor_count(buf.ctypes.data, buf.size, k, None, None, 0, C.byref(total))
    keys = np.empty((d, words(k)), dtype=np.uint64)
    cnt = np.empty(d, dtype=np.uint32)
    lib.kor_count(buf.ctypes.data, buf.size, k, keys.ctypes.data, cnt.ctypes.data, d, C.byref(total))
    return keys, cnt, int(total.value)


def packed_bytes(k):
    return (k // 32) * 8 + (2 * (k % 32) + 7) // 8


def pack(keys, k):
    """Pack (n, N) uint64 keys into low.bin bytes."""
    lib = _load()
    keys = np.ascontiguousarray(keys, dtype=np.uint64)
    n = keys.shape[0]
    out = np.empty(n * packed_bytes(k), dtype=np.uint8)
    lib.kor_pack(keys.ctypes.data, n, k, out.ctypes.data)
    return out


def unpack(raw, k):
    """low.bin bytes -> (n, N) uint64 keys."""
    lib = _load()
    raw = _as_u8(raw)
    P = packed_bytes(k)
    if raw.size % P:
        raise ValueError(f"Invalid low.bin size: {raw.size} is not divisible by packed k-mer size {P}")
    n = raw.size // P
    out = np.empty((n, words(k)), dtype=np.uint64)
    lib.kor_unpack(raw.ctypes.data, n, k, out.ctypes.data)
    return out


def record_dtype(k):
    return np.dtype([("key", "<u8", (words(k),)), ("count", "<u4"), ("pad", "<u4")])


def read_outputs(out_dir, k):
    """(low keys (L, N), root records structured array with a 'root' column
    implied by file order, per-root counts) from a tmp directory."""
    low = unpack(np.fromfile(os.path.join(out_dir, "low.bin"), dtype=np.uint8), k)
    dt = record_dtype(k)
    parts, counts = [], []
    for r in range(256):
        p = os.path.join(out_dir, f"root_{r}.bin")
        raw = np.fromfile(p, dtype=np.uint8) if os.path.exists(p) else np.empty(0, np.uint8)
        if raw.size % dt.itemsize:
            raise ValueError(f"{p}: size {raw.size} not a multiple of {dt.itemsize}")
        rec = raw.view(dt)
        parts.append(rec)
        counts.append(rec.size)
    return low, (np.concatenate(parts) if parts else np.empty(0, dt)), counts


def _sort_unique(keys, counts):
    """Sort (n, N) keys lexicographically and sum counts of equal keys."""
    if keys.shape[0] == 0:
        return keys.reshape(0, keys.shape[1] if keys.ndim == 2 else 1), counts.astype(np.uint64)
    if keys.shape[1] == 1:
        order = np.argsort(keys[:, 0], kind="stable")
    else:
        order = np.lexsort(tuple(keys[:, i] for i in range(keys.shape[1] - 1, -1, -1)))
    ks, cs = keys[order], counts[order].astype(np.uint64)
    new = np.ones(ks.shape[0], dtype=bool)
    new[1:] = np.any(ks[1:] != ks[:-1], axis=1)
    idx = np.flatnonzero(new)
    return ks[idx], np.add.reduceat(cs, idx)


def merged_counts(low_keys, root_keys, root_counts, nw=None):
    """Exact (key, count) multiset from the two outputs: root count + [in low]."""
    if nw is None:
        nw = low_keys.shape[1] if low_keys.ndim == 2 else (root_keys.shape[1] if root_keys.ndim == 2 else 1)
    lk = low_keys.reshape(-1, nw)
    rk = root_keys.reshape(-1, nw)
    keys = np.concatenate([lk, rk])
    cnt = np.concatenate([np.ones(lk.shape[0], np.uint64), root_counts.astype(np.uint64)])
    return _sort_unique(keys, cnt)


def histogram(counts, min_freq=1, max_freq=10000):
    """freq -> number of keys, for freq in [min_freq, max_freq]
    (tool/histogram_tool.cpp:425-442 writes these as `freq\\tcount` lines)."""
    c = np.asarray(counts, dtype=np.uint64)
    c = c[(c >= min_freq) & (c <= max_freq)]
    h = np.bincount((c - min_freq).astype(np.int64), minlength=max_freq - min_freq + 1)
    return h[: max_freq - min_freq + 1]


def digest(keys, counts):
    """sha256 over the sorted (key words..., count) table: a size-independent
    fingerprint of the exact multiset."""
    import hashlib
    keys = np.ascontiguousarray(keys, dtype=np.uint64)
    h = hashlib.sha256()
    h.update(keys.tobytes())
    h.update(np.ascontiguousarray(counts, dtype=np.uint64).tobytes())
    return h.hexdigest()


def run_reference(fastq_path, k, workdir, threads=8, mem_gb=4, extra=()):
    """Run the reference `Tree` (built from its sources into oracle/_ref) in
    workdir; returns (stdout, returncode).  Outputs land in workdir/tmp/."""
    os.makedirs(os.path.join(workdir, "tmp"), exist_ok=True)
    p = subprocess.run([REF_TREE, str(fastq_path), str(k), str(threads), str(mem_gb), *map(str, extra)],
                       cwd=workdir, capture_output=True, text=True)
    return p.stdout, p.returncode


def reference_total(stdout):
    for line in stdout.splitlines():
        if line.startswith("Total read k-mer count:"):
            return int(line.split(":")[1])
    return None
