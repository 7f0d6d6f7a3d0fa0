"""The allocation-free entry point kc_count_device_noalloc, through the C ABI.

Some callers cannot allocate device memory on this path (an allocator that
owns the device budget, or a thread that must not stall on cudaMalloc /
cudaFree).  This entry point takes its scratch from a static device array, so
the tests check that
  (a) the first call on the device reserves at most that array (it is set up
      lazily, on the first call, under CUDA's default lazy module loading);
  (b) its output equals the allocating entry point's (kc_count_device) on the
      same input -- the exact merged (k-mer, count) multiset, the bar every
      parity test here uses -- and the oracle's, on two calls in a row;
  (c) tables too small for the input grow inside the array (rehashes > 0)
      with the same exact counts;
  (d) free device memory does not change across a call;
  (e) every documented rejection returns KC_ERR_INVALID with its message, and
      a call right after a rejected one is still exact.
Kept in its own file, collected last.
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


def call(cfg, d_in, n, d_low, low_cap, d_roots, roots_cap, st=None, in_ptr=None):
    st = st if st is not None else _native.KcStats()
    stream = torch.cuda.current_stream().cuda_stream
    ptr = in_ptr if in_ptr is not None else d_in.data_ptr()
    return _native.lib.kc_count_device_noalloc(C.byref(cfg), C.c_void_p(ptr), n, C.c_void_p(d_low.data_ptr()),
                                               low_cap, C.c_void_p(d_roots.data_ptr()), roots_cap,
                                               C.c_void_p(stream), C.byref(st))


def noalloc(cfg, d_in, n, low_cap, roots_cap):
    d_low = torch.empty(max(low_cap, 1), dtype=torch.uint8, device="cuda")
    d_roots = torch.empty(max(roots_cap, 1), dtype=torch.uint8, device="cuda")
    st = _native.KcStats()
    rc = call(cfg, d_in, n, d_low, low_cap, d_roots, roots_cap, st)
    return rc, st, d_low, d_roots


def merged_from(low_raw, roots_raw, k, n_roots):
    low = oracle.unpack(low_raw, k)
    roots = roots_raw.view(kc.record_dtype(k))[:n_roots]
    nw = oracle.words(k)
    return oracle.merged_counts(low, roots["key"].reshape(-1, nw), roots["count"], nw=nw), low, roots


CASES = [(31, synth.plain_small(seed=41, scale=0.004)), (63, synth.plain_small(seed=42, scale=0.003))]


def allocating(data, d_in, k):
    """Merged counts and K from the allocating entry point on the same input."""
    with kc.Counter(k=k) as c:
        c.count_device(d_in.data_ptr(), d_in.numel())
        want_low, want_roots, _ = parity.gpu_outputs(c, k)
        return parity.merged(want_low, want_roots, k), c.stats.total_kmers


def check_noalloc(cfg, data, d_in, want, K):
    k = cfg.k
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
    assert K2 == K and np.array_equal(mk, keys) and np.array_equal(mc, counts.astype(mc.dtype))
    return st


def test_first_call_reserves_at_most_the_scratch():
    # the first no-alloc call in this process: under lazy module loading it is
    # the one that reserves the static array (eager loading did it earlier)
    k, p = CASES[0]
    data = synth.fastq(p)
    d_in = torch.from_numpy(data).cuda()
    P, R = kc.packed_bytes(k), kc.record_bytes(k)
    d_low = torch.empty(data.size * P, dtype=torch.uint8, device="cuda")
    d_roots = torch.empty(data.size * R, dtype=torch.uint8, device="cuda")
    cfg = kc.default_config(k=k)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    assert call(cfg, d_in, data.size, d_low, d_low.numel(), d_roots, d_roots.numel()) == 0, _native.last_error()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    # the array plus the module's code and constants (a few MiB)
    assert free0 - free1 <= _native.NOALLOC_SCRATCH_BYTES + (16 << 20), (free0 - free1)


def test_noalloc_matches_allocating_entry_point():
    for k, p in CASES:  # two calls in a row, different k
        data = synth.fastq(p)
        assert data.size <= _native.NOALLOC_MAX_FASTQ_BYTES
        d_in = torch.from_numpy(data).cuda()
        want, K = allocating(data, d_in, k)
        check_noalloc(kc.default_config(k=k), data, d_in, want, K)


def test_noalloc_tables_grow_inside_the_array():
    # tables sized for almost no repeated keys (the 64-slot minimum per bucket)
    # on an input with ~100k repeated keys: buckets overflow and are grown
    # (x4, again if needed) inside the static array
    for k, seed in ((31, 43), (63, 44)):
        p = synth.plain_small(seed=seed, scale=0.02)
        data = synth.fastq(p)
        assert data.size <= _native.NOALLOC_MAX_FASTQ_BYTES
        d_in = torch.from_numpy(data).cuda()
        want, K = allocating(data, d_in, k)
        st = check_noalloc(kc.default_config(k=k, repeat_ratio=0.001), data, d_in, want, K)
        assert st.rehashes > 0


def test_noalloc_allocates_nothing_and_rejects_bad_requests():
    k, p = CASES[0]
    data = synth.fastq(p)
    d_in = torch.from_numpy(data).cuda()
    cfg = kc.default_config(k=k)
    P, R = kc.packed_bytes(k), kc.record_bytes(k)
    d_low = torch.empty(data.size * P, dtype=torch.uint8, device="cuda")
    d_roots = torch.empty(data.size * R, dtype=torch.uint8, device="cuda")

    def run(n=data.size, low_cap=None, roots_cap=None, c=cfg, in_ptr=None):
        return call(c, d_in, n, d_low, d_low.numel() if low_cap is None else low_cap, d_roots,
                    d_roots.numel() if roots_cap is None else roots_cap, in_ptr=in_ptr)

    assert run() == 0, _native.last_error()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    assert run() == 0, _native.last_error()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free0 == free1

    def rejected(rc, text):
        assert rc == kc.KC_ERR_INVALID, (rc, _native.last_error())
        assert text in _native.last_error(), _native.last_error()

    rejected(run(n=_native.NOALLOC_MAX_FASTQ_BYTES + 1), "KC_NOALLOC_MAX_FASTQ_BYTES")
    rejected(run(low_cap=8), "low output buffer too small")
    rejected(run(roots_cap=16), "root output buffer too small")
    rejected(run(c=kc.default_config(k=65)), "k out of range: 1..64")
    rejected(run(c=kc.default_config(k=k, n_buckets=4096)), "256 buckets only")
    rejected(run(n=data.size - 16, in_ptr=d_in.data_ptr() + 8), "16-byte aligned")
    off = _native.lib.kc_count_device_noalloc(C.byref(cfg), C.c_void_p(d_in.data_ptr()), data.size,
                                              C.c_void_p(d_low.data_ptr() + 4), d_low.numel() - 4,
                                              C.c_void_p(d_roots.data_ptr()), d_roots.numel(), None,
                                              C.byref(_native.KcStats()))
    rejected(off, "output buffers must be 16-byte aligned")
    # a call right after the rejections is still exact
    want, K = allocating(data, d_in, k)
    check_noalloc(cfg, data, d_in, want, K)
