"""Bit-exact parity at the benchmark shapes, through the C ABI.

The reference's own `Tree` (compiled from its sources) counted these inputs
and tests/golden/golden.json holds the sha256 of its merged exact (key,
count) table, its K and distinct count, and its `histogram_tool precise`
output (tests/golden/make_golden.py):

* genome-scale at 5% (100 Mbp x 0.05 genome with 45% GC and 20% repeat
  families, 30x of 150 bp with the 3' error ramp: 1M reads, 313 MB), k=31,
  counted from device memory in one pass and from host memory in 64 MiB
  batches (the ramped batch plan of long host inputs: B/8, B/4, B/2 at both
  ends), and from device memory in 64 MiB passes;
* large long keys at 2% (4 Mbp genome, 40% GC, 30% repeats, 50x: 1.3M reads,
  418 MB), k=63 with 128-bit keys and 4096 buckets, from device memory and
  from host memory in 64 MiB batches;
* genome-scale in full (the benchmark input: 20M reads, 3 Gbases, 6.3 GB),
  k=31, from device memory as the benchmark counts it and through the
  streaming host call the end-to-end benchmark times.

The CPU suite checks the oracle against the same fixtures for the two scaled
inputs (tests/test_oracle_golden.py).
"""
import ctypes
import hashlib

import numpy as np
import pytest

import inputs
import oracle
import parity

pytestmark = pytest.mark.gpu

kc = pytest.importorskip("kmertreecounter_b200")
torch = pytest.importorskip("torch")
from kmertreecounter_b200 import synth  # noqa: E402

MiB = 1 << 20


def plan_batches(n, B, tile=8192):
    """The host path's batch plan (kc_engine.cu plan_batches): B each, except
    that inputs of at least 4 B (B >= 64 MiB) ramp B/8, B/4, B/2 at both ends."""
    al = lambda x: max(tile, x & ~(tile - 1))  # noqa: E731
    if n < 4 * B or B < 64 * MiB:
        return [min(B, n - o) for o in range(0, n, B)]
    ramp = [al(B // 8), al(B // 4), al(B // 2)]
    mid = n - 2 * sum(ramp)
    k = -(-mid // B)
    each = al(mid // k)
    return ramp + [each] * (k - 1) + [mid - (k - 1) * each] + ramp[::-1]


def load(golden, name):
    e = golden[name]
    data = getattr(inputs, e["builder"])(**e["kwargs"])
    assert data.size == e["fastq_bytes"]
    assert hashlib.sha256(data).hexdigest() == e["fastq_sha256"], "input generator drifted"
    return data


def check_against_reference(counter, k, g):
    """The counter's last result (device resident) against the reference's
    fixture: merged digest, K, distinct keys, and the device histogram
    against the reference's histogram_tool precise output."""
    assert counter.stats.total_kmers == g["K"]
    low, roots, per_root = parity.device_outputs(counter, k)
    assert sum(per_root) * (8 * oracle.words(k) + 8) == roots.numel()
    h, distinct = counter.histogram(1, 64)
    assert distinct == g["D"]
    assert [int(x) for x in h] == g["histogram_tool_precise_1_64"]
    keys, counts = parity.merged_on_device(low, roots, k)
    del low, roots
    assert keys.shape[0] == g["D"]
    assert oracle.digest(keys, counts) == g["digest"]


def stream_and_check(counter, host, n, k, g):
    """kc_count_host_stream: collect the sink's pieces, then the merged
    digest of what reached host memory."""
    low_parts, root_parts, order = [], {}, []

    def sink(kind, root, addr, nbytes):
        buf = np.frombuffer(ctypes.string_at(addr, nbytes), np.uint8) if nbytes else np.empty(0, np.uint8)
        if kind == kc.KC_SINK_LOW:
            low_parts.append(buf)
        else:
            if root not in root_parts:
                order.append(root)
            root_parts.setdefault(root, []).append(buf)
        return 0

    st = counter.count_host_stream(host, n, sink)
    assert order == list(range(256)), "every root delivered once, in order"
    assert st.total_kmers == g["K"]
    low = torch.from_numpy(np.concatenate(low_parts)).cuda() if low_parts else torch.empty(0, dtype=torch.uint8,
                                                                                            device="cuda")
    roots = torch.from_numpy(np.concatenate([b for r in range(256) for b in root_parts[r]])).cuda()
    assert low.numel() == st.low_records * kc.packed_bytes(k)
    assert roots.numel() == st.root_records * kc.record_bytes(k)
    keys, counts = parity.merged_on_device(low, roots, k)
    assert keys.shape[0] == g["D"] and oracle.digest(keys, counts) == g["digest"]
    return st


@pytest.fixture(scope="module")
def gs05(golden):
    return load(golden, "genome_scale_s05"), golden["genome_scale_s05"]["k"]["31"]


def test_genome_scale_5pct_device(gs05):
    data, g = gs05
    d = torch.from_numpy(data).cuda()
    with kc.Counter(k=31) as c:
        st = c.count_device(d.data_ptr(), d.numel())
        assert st.batches == 1
        check_against_reference(c, 31, g)


def test_genome_scale_5pct_device_passes(gs05):
    data, g = gs05
    d = torch.from_numpy(data).cuda()
    with kc.Counter(k=31, device_batch_bytes=64 * MiB) as c:
        st = c.count_device(d.data_ptr(), d.numel())
        assert st.batches == -(-data.size // (64 * MiB))
        check_against_reference(c, 31, g)


def test_genome_scale_5pct_host_ramped_batches(gs05):
    data, g = gs05
    plan = plan_batches(data.size, 64 * MiB)
    assert len(plan) > -(-data.size // (64 * MiB)), "the input must engage the ramped plan"
    with kc.Counter(k=31, batch_bytes=64 * MiB, chunk_bytes=16 * MiB) as c:
        st = stream_and_check(c, data.ctypes.data, data.size, 31, g)
        assert st.batches == len(plan)
        # the non-streaming host call on the same plan keeps the result on the device
        st = c.count_host(data)
        assert st.batches == len(plan)
        check_against_reference(c, 31, g)


def test_large_long_2pct_k63_4096_buckets(golden):
    data = load(golden, "large_long_s02")
    g = golden["large_long_s02"]["k"]["63"]
    d = torch.from_numpy(data).cuda()
    with kc.Counter(k=63, n_buckets=4096) as c:
        c.count_device(d.data_ptr(), d.numel())
        check_against_reference(c, 63, g)
    del d
    with kc.Counter(k=63, n_buckets=4096, batch_bytes=64 * MiB, chunk_bytes=16 * MiB) as c:
        st = stream_and_check(c, data.ctypes.data, data.size, 63, g)
        assert st.batches == len(plan_batches(data.size, 64 * MiB))


def test_genome_scale_full_size(golden):
    """The benchmark input itself (6.3 GB, 2.33 G k-mers) against the
    reference's own run on it: device resident in one pass, as the benchmark's
    `value` counts it, and through the streaming host call with the default
    1 GiB ramped batches, as its `e2e` counts it."""
    e = golden["genome_scale_full"]
    g = e["k"]["31"]
    p = synth.genome_scale(**e["kwargs"])
    n = synth.fastq_bytes(p)
    assert n == e["fastq_bytes"]
    host_ptr = kc.host_alloc(n)
    try:
        synth.fastq(p, out=host_ptr)
        host = np.ctypeslib.as_array((ctypes.c_uint8 * n).from_address(host_ptr))
        assert hashlib.sha256(host).hexdigest() == e["fastq_sha256"], "input generator drifted"
        d = torch.empty(n, dtype=torch.uint8, device="cuda")
        d.copy_(torch.from_numpy(host))
        with kc.Counter(k=31) as c:
            st = c.count_device(d.data_ptr(), n)
            assert st.batches == 1 and st.rehashes == 0
            del d
            check_against_reference(c, 31, g)
        torch.cuda.empty_cache()
        with kc.Counter(k=31) as c:
            stream_and_check(c, host_ptr, n, 31, g)
    finally:
        kc.host_free(host_ptr)
