"""The allocation-free entry point kc_count_device_noalloc, through the C ABI.

Some callers cannot allocate device memory on this path (an allocator that
owns the device budget, or a thread that must not stall on cudaMalloc /
cudaFree).  This entry point takes its scratch from a static device array, so
the test checks that (a) its output equals the allocating entry point's
(kc_count_device) on the same input -- the exact merged (k-mer, count)
multiset, the bar every parity test here uses -- on two calls in a row, (b)
free device memory does not change across a call, and (c) oversized input is
rejected with a clear error.  Kept in its own file, collected last.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
import parity

pytestmark = pytest.mark.gpu

kc = pytest.importorskip("kmertreecounter_b200")
torch = pytest.importorskip("torch")
from kmertreecounter_b200 import _native, synth  # noqa: E402


def noalloc(cfg, d_in, n, low_cap, roots_cap):
    d_low = torch.empty(max(low_cap, 1), dtype=torch.uint8, device="cuda")
    d_roots = torch.empty(max(roots_cap, 1), dtype=torch.uint8, device="cuda")
    st = _native.KcStats()
    stream = torch.cuda.current_stream().cuda_stream
    rc = _native.lib.kc_count_device_noalloc(C.byref(cfg), C.c_void_p(d_in.data_ptr()), n,
                                             C.c_void_p(d_low.data_ptr()), low_cap,
                                             C.c_void_p(d_roots.data_ptr()), roots_cap, C.c_void_p(stream),
                                             C.byref(st))
    return rc, st, d_low, d_roots


def merged_from(low_raw, roots_raw, k, n_roots):
    low = oracle.unpack(low_raw, k)
    roots = roots_raw.view(kc.record_dtype(k))[:n_roots]
    nw = oracle.words(k)
    return oracle.merged_counts(low, roots["key"].reshape(-1, nw), roots["count"], nw=nw), low, roots


CASES = [(31, synth.plain_small(seed=41, scale=0.004)), (63, synth.plain_small(seed=42, scale=0.003))]


def test_noalloc_matches_allocating_entry_point():
    for k, p in CASES:  # two calls in a row, different k
        data = synth.fastq(p)
        assert data.size <= _native.NOALLOC_MAX_FASTQ_BYTES
        d_in = torch.from_numpy(data).cuda()
        with kc.Counter(k=k) as c:
            c.count_device(d_in.data_ptr(), d_in.numel())
            want_low, want_roots, _ = parity.gpu_outputs(c, k)
            K = c.stats.total_kmers
        want = parity.merged(want_low, want_roots, k)
        cfg = kc.default_config(k=k)
        P, R = kc.packed_bytes(k), kc.record_bytes(k)
        rc, st, d_low, d_roots = noalloc(cfg, d_in, data.size, data.size * P, data.size * R)
        assert rc == 0, _native.last_error()
        torch.cuda.synchronize()
        assert st.total_kmers == K
        low_raw = d_low.cpu().numpy()[: st.low_records * P]
        roots_raw = d_roots.cpu().numpy()[: st.root_records * R]
        (mk, mc), low, roots = merged_from(low_raw, roots_raw, k, st.root_records)
        parity.check_layout(low, roots, list(st.root_counts), k)
        assert np.array_equal(mk, want[0]) and np.array_equal(mc, want[1])
        keys, counts, K2 = oracle.count(data, k)
        assert K2 == K and np.array_equal(mk, keys)


def test_noalloc_allocates_nothing_and_rejects_oversize():
    k, p = CASES[0]
    data = synth.fastq(p)
    d_in = torch.from_numpy(data).cuda()
    cfg = kc.default_config(k=k)
    P, R = kc.packed_bytes(k), kc.record_bytes(k)
    d_low = torch.empty(data.size * P, dtype=torch.uint8, device="cuda")
    d_roots = torch.empty(data.size * R, dtype=torch.uint8, device="cuda")
    st = _native.KcStats()
    stream = torch.cuda.current_stream().cuda_stream

    def call(n):
        return _native.lib.kc_count_device_noalloc(C.byref(cfg), C.c_void_p(d_in.data_ptr()), n,
                                                   C.c_void_p(d_low.data_ptr()), d_low.numel(),
                                                   C.c_void_p(d_roots.data_ptr()), d_roots.numel(),
                                                   C.c_void_p(stream), C.byref(st))

    assert call(data.size) == 0, _native.last_error()  # set-up call
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    assert call(data.size) == 0, _native.last_error()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free0 == free1
    rc = call(_native.NOALLOC_MAX_FASTQ_BYTES + 1)
    assert rc == kc.KC_ERR_INVALID and "KC_NOALLOC_MAX_FASTQ_BYTES" in _native.last_error()
