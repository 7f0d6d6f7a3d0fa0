"""GPU path (through the C ABI) against the oracle and the reference.

Bit-exact: the merged (canonical k-mer, count) multiset of low.bin + root
files must equal the oracle's, and, for the golden inputs, the digest the
reference's own output produced.  The first-occurrence filter may move a key
between low.bin and its root file only as the reference design allows (a
false positive puts its whole count in the root record)."""
import hashlib
import os
import subprocess

import numpy as np
import pytest

import inputs
import oracle
import parity
from conftest import ROOT

pytestmark = pytest.mark.gpu

kc = pytest.importorskip("kmertreecounter_b200")
from kmertreecounter_b200 import synth  # noqa: E402

_data = {}


def golden_input(golden, name):
    if name not in _data:
        e = golden[name]
        d = getattr(inputs, e["builder"])(**e["kwargs"])
        assert hashlib.sha256(d).hexdigest() == e["fastq_sha256"]
        _data[name] = np.frombuffer(d, np.uint8)
    return _data[name]


GOLDEN = [(n, k) for n, ks in [("plain_small", [31]), ("plain_small_s7", [21, 32, 33, 63, 65, 101, 127, 128]),
                               ("adversarial", [17, 31, 32, 33, 64, 65, 100, 128])] for k in ks]


@pytest.mark.parametrize("name,k", GOLDEN)
def test_golden_digest(golden, name, k):
    g = golden[name]["k"][str(k)]
    data = golden_input(golden, name)
    with kc.Counter(k=k) as c:
        st = c.count_host(data)
        assert st.total_kmers == g["K"]
        low, roots, per_root = parity.gpu_outputs(c, k)
        parity.check_layout(low, roots, per_root, k)
        mk, mc = parity.merged(low, roots, k)
        assert mk.shape[0] == g["D"]
        assert oracle.digest(mk, mc) == g["digest"]
        assert [int(x) for x in oracle.histogram(mc, 1, 64)] == g["hist_1_64"]


@pytest.mark.parametrize("k", [1, 5, 12, 21, 31, 32, 33, 47, 63, 64, 65, 80, 97, 111, 127, 128])
@pytest.mark.parametrize("buckets", [256, 4096])
def test_small_vs_oracle(k, buckets):
    p = synth.plain_small(seed=100 + k, scale=0.05)
    p.sub_rate = 0.02
    data = synth.fastq(p)
    with kc.Counter(k=k, n_buckets=buckets) as c:
        c.count_host(data)
        parity.check_exact(c, data, k)


def test_multi_batch_matches(golden):
    data = golden_input(golden, "adversarial")
    want = oracle.count(data, 31)
    with kc.Counter(k=31, batch_bytes=1 << 20, chunk_bytes=1 << 20) as c:
        st = c.count_host(data)
        assert st.batches == (data.size + (1 << 20) - 1) // (1 << 20)
        parity.check_exact(c, data, 31, want)


def test_forced_rehash_stays_exact():
    p = synth.plain_small(seed=9, scale=0.2)
    data = synth.fastq(p)
    with kc.Counter(k=31, repeat_ratio=1e-7) as c:
        st = c.count_host(data)
        assert st.rehashes > 0
        parity.check_exact(c, data, 31)


def test_device_input_matches_host():
    torch = pytest.importorskip("torch")
    p = synth.plain_small(seed=4, scale=0.1)
    data = synth.fastq(p)
    d = torch.from_numpy(data).cuda()
    want = oracle.count(data, 25)
    with kc.Counter(k=25, batch_bytes=1 << 20) as c:
        c.count_device(d.data_ptr(), d.numel())
        torch.cuda.synchronize()
        parity.check_exact(c, data, 25, want)


@pytest.mark.parametrize("lo,hi", [(2, 2**32 - 1), (1, 3), (3, 10)])
def test_min_max_filter(lo, hi):
    p = synth.plain_small(seed=21, scale=0.1)
    data = synth.fastq(p)
    with kc.Counter(k=21, min_count=lo, max_count=hi) as c:
        c.count_host(data)
        parity.check_filtered(c, data, 21, lo, hi)


@pytest.mark.parametrize("data", [b"", b"@r\n", b"@r\nACG\n+\nIII\n", b"@r\n" + b"N" * 100 + b"\n+\n",
                                  b"@r\nACGTACGTAC", b"\n\n\n\n\n\n\n\n", b"@a\nACGTTGCA\r\n+\r\nIIIIIIII\r\n"])
@pytest.mark.parametrize("k", [4, 31, 40])
def test_edge_inputs(data, k):
    arr = np.frombuffer(data, np.uint8)
    with kc.Counter(k=k) as c:
        c.count_host(arr)
        parity.check_exact(c, arr, k)
        lb, nr, per = c.sizes()
        assert sum(per) == nr


def test_cli_output_read_by_reference_tool(golden, tmp_path):
    """bin/Tree writes ./tmp/low.bin and root_0..255.bin that the reference's
    own histogram_tool reads unchanged and turns into the same histogram."""
    data = golden_input(golden, "adversarial")
    fq = tmp_path / "in.fastq"
    fq.write_bytes(data.tobytes())
    tree = os.path.join(ROOT, "kmertreecounter_b200", "bin", "Tree")
    p = subprocess.run([tree, str(fq), "33", "8", "4"], cwd=tmp_path, capture_output=True, text=True)
    assert p.returncode == 0, p.stderr
    g = golden["adversarial"]["k"]["33"]
    assert f"Total read k-mer count: {g['K']}" in p.stdout
    files = sorted(os.listdir(tmp_path / "tmp"))
    assert "low.bin" in files and all(f"root_{r}.bin" in files for r in range(256))
    low, roots, _ = oracle.read_outputs(str(tmp_path / "tmp"), 33)
    mk, mc = oracle.merged_counts(low, roots["key"], roots["count"])
    assert oracle.digest(mk, mc) == g["digest"]
    if os.path.exists(oracle.REF_HIST):
        h = tmp_path / "hist.tsv"
        subprocess.run([oracle.REF_HIST, "precise", str(tmp_path / "tmp"), "33", "4", "4", str(h), "1", "64"],
                       check=True, capture_output=True)
        assert [int(line.split("\t")[1]) for line in h.read_text().splitlines()] == g["histogram_tool_precise_1_64"]


@pytest.mark.parametrize("k", [21, 31, 32, 45, 63, 64])
def test_sorted_roots(k):
    """sort_output=1: every root file ordered by key (radix sort replacing
    sort/ExportRecordRadixSort.h), same records as unsorted."""
    p = synth.plain_small(seed=60 + k, scale=0.08)
    data = synth.fastq(p)
    with kc.Counter(k=k, sort_output=1) as c:
        c.count_host(data)
        low, roots = parity.check_exact(c, data, k)
        _, _, per_root = c.sizes()
    nw = oracle.words(k)
    rk = roots["key"].reshape(-1, nw)
    off = 0
    for n in per_root:
        seg = rk[off:off + n]
        if n > 1:
            order = np.lexsort(tuple(seg[:, i] for i in range(nw - 1, -1, -1)))
            assert np.array_equal(order, np.arange(n)), "root file not sorted by key"
        off += n


@pytest.mark.parametrize("batch", [1 << 20, 4 << 20, 1 << 30])
def test_stream_sink_matches(golden, batch):
    """kc_count_host_stream: low.bin bytes and root files delivered through
    the sink (copies overlapped with counting) give the exact multiset."""
    import ctypes
    data = golden_input(golden, "adversarial")
    k = 31
    low_parts, roots = [], {}

    def sink(kind, root, addr, nbytes):
        buf = ctypes.string_at(addr, nbytes) if nbytes else b""
        if kind == kc.KC_SINK_LOW:
            low_parts.append(buf)
        else:
            roots.setdefault(root, []).append(buf)
        return 0

    with kc.Counter(k=k, batch_bytes=batch, chunk_bytes=1 << 20) as c:
        st = c.count_host_stream(data.ctypes.data, data.size, sink)
    assert sorted(roots) == list(range(256)), "every root delivered, in order"
    low = oracle.unpack(np.frombuffer(b"".join(low_parts), np.uint8), k)
    dt = kc.record_dtype(k)
    per_root = [sum(len(b) for b in roots[r]) // dt.itemsize for r in range(256)]
    rec = np.frombuffer(b"".join(b"".join(roots[r]) for r in range(256)), dtype=dt)
    parity.check_layout(low, rec, per_root, k)
    mk, mc = parity.merged(low, rec, k)
    g = golden["adversarial"]["k"][str(k)]
    assert st.total_kmers == g["K"] and oracle.digest(mk, mc) == g["digest"]


def test_gzip_input_cli(golden, tmp_path):
    """gzip input is detected by its magic bytes (src/FastqReader.h:93-104)."""
    import gzip
    data = golden_input(golden, "plain_small_s7")
    fq = tmp_path / "in.fastq.gz"
    with gzip.open(fq, "wb", compresslevel=1) as f:
        f.write(data.tobytes())
    tree = os.path.join(ROOT, "kmertreecounter_b200", "bin", "Tree")
    p = subprocess.run([tree, str(fq), "21", "8", "4"], cwd=tmp_path, capture_output=True, text=True)
    assert p.returncode == 0, p.stderr
    low, roots, _ = oracle.read_outputs(str(tmp_path / "tmp"), 21)
    mk, mc = oracle.merged_counts(low, roots["key"], roots["count"])
    assert oracle.digest(mk, mc) == golden["plain_small_s7"]["k"]["21"]["digest"]


def test_cli_missing_input_is_io_error(tmp_path):
    tree = os.path.join(ROOT, "kmertreecounter_b200", "bin", "Tree")
    p = subprocess.run([tree, str(tmp_path / "nope.fastq"), "31", "8", "4"], cwd=tmp_path, capture_output=True,
                       text=True)
    assert p.returncode == 255 and "Failed to open" in p.stderr


@pytest.mark.parametrize("name,k", [("plain_small", 31), ("adversarial", 33), ("plain_small_s7", 63)])
def test_device_histogram(golden, name, k):
    """kc_histogram (device form of histogram_tool precise) reproduces the
    reference's histogram and the distinct count."""
    g = golden[name]["k"][str(k)]
    data = golden_input(golden, name)
    with kc.Counter(k=k, repeat_ratio=0.01) as c:  # small tables: exercises rehash + stale regions
        c.count_host(data)
        h, distinct = c.histogram(1, 64)
        assert [int(x) for x in h] == g["histogram_tool_precise_1_64"]
        assert distinct == g["D"]
        h2, _ = c.histogram(3, 5)  # a second call reuses cleared marks
        assert [int(x) for x in h2] == g["histogram_tool_precise_1_64"][2:5]


def test_k96_keys_are_canonical():
    """k = 96 (256-bit keys, k a multiple of 32 below 128): the reference's
    forward register is masked only in the word that holds the last base
    (src/GetKmer.h, get_next_one and batch_insert: data[kmer_last_index] &=
    back_mask), so bases older than the window drift into key word 3 of its
    F-oriented keys and the same k-mer gets several keys (its low.bin, which
    packs 3 words, drops them again).  This build emits the canonical k-mer
    (word 3 = 0): parity is the oracle's restatement with word 3 cleared and
    equal keys merged."""
    p = synth.plain_small(seed=96, scale=0.05)
    data = synth.fastq(p)
    keys, counts, K = oracle.count(data, 96)
    assert np.count_nonzero(keys[:, 3]) > 0  # the reference behaviour the oracle restates
    keys = keys.copy()
    keys[:, 3] = 0
    keys, counts = oracle._sort_unique(keys, counts.astype(np.uint64))
    with kc.Counter(k=96) as c:
        c.count_host(data)
        parity.check_exact(c, data, 96, (keys, counts, K))


@pytest.mark.parametrize("k", [100, 128])
def test_shared_prefix_keys(k):
    """256-bit slots are claimed by a state word and published after the key
    is written; keys that agree in their first 128 bits meet in the same
    probe sequence and must wait for each other's publication.  Reads here
    share a 200-base stem and end in random 40-base tails, so the windows
    that reach into a tail share their oldest bases (the C orientation's
    leading bits) with every other read's."""
    rng = np.random.default_rng(k)
    acgt = np.frombuffer(b"ACGT", np.uint8)
    stem = acgt[rng.integers(0, 4, 200)]
    recs = []
    for i in range(3000):
        seq = np.concatenate([stem, acgt[rng.integers(0, 4, 40)]]).tobytes()
        recs.append(b"@s%d\n%s\n+\n%s\n" % (i, seq, b"I" * len(seq)))
    data = np.frombuffer(b"".join(recs), np.uint8)
    with kc.Counter(k=k) as c:
        c.count_host(data)
        parity.check_exact(c, data, k)


@pytest.mark.parametrize("buckets", [256, 4096])
@pytest.mark.parametrize("small_tables", [False, True])
def test_windowed_count_matches_global_count(monkeypatch, buckets, small_tables):
    """64-bit keys count in shared-memory table windows (kc_window.cuh) unless
    KC_WINDOW_COUNT=0 selects the global-memory count kernel: both give the
    oracle's exact counts, over several device passes, with buckets of one
    and of many windows, and with tables small enough to overflow (the
    windowed pass leaves overflowed keys to the global retry after growth)."""
    p = synth.genome_scale(seed=12, scale=0.01)
    data = synth.fastq(p)
    want = oracle.count(data, 31)
    for env in ("1", "0"):
        monkeypatch.setenv("KC_WINDOW_COUNT", env)
        # small tables: 1 filter bit and 0.002 repeat keys per k-mer against
        # ~0.04 distinct repeated keys per k-mer at 30x
        knobs = dict(bloom_bits=1.0, repeat_ratio=0.002) if small_tables else {}
        with kc.Counter(k=31, n_buckets=buckets, batch_bytes=16 << 20, **knobs) as c:
            st = c.count_host(data)
            assert st.batches > 1
            if small_tables:
                assert st.rehashes > 0
            parity.check_exact(c, data, 31, want)
