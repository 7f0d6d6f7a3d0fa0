"""Parity checks shared by the GPU tests: the GPU path's low.bin + root
records against the oracle, with the invariants the reference's design
guarantees (tool/histogram_tool.cpp precise merge semantics)."""
import numpy as np

import oracle


def unique_rows(a):
    if a.shape[0] < 2:
        return True
    s = a[np.lexsort(tuple(a[:, i] for i in range(a.shape[1] - 1, -1, -1)))]
    return not np.any(np.all(s[1:] == s[:-1], axis=1))


def gpu_outputs(counter, k):
    low = oracle.unpack(counter.low_bytes(), k)
    roots, per_root = counter.root_records()
    return low, roots, per_root


def check_layout(low, roots, per_root, k, min_count=1, max_count=0xFFFFFFFF):
    nw = oracle.words(k)
    assert low.shape[1] == nw
    assert unique_rows(low), "a key was written to low.bin twice"
    rk = roots["key"].reshape(-1, nw)
    assert unique_rows(rk), "a key has two root records"
    assert np.all(roots["pad"] == 0), "ExportRecord padding must be zero"
    assert np.all(roots["count"] >= max(1, min_count)) and np.all(roots["count"] <= max_count)
    # grouping: root file r holds exactly the keys with word0 >> 56 == r
    assert sum(per_root) == roots.shape[0]
    off = 0
    for r, n in enumerate(per_root):
        if n:
            assert np.all((rk[off:off + n, 0] >> np.uint64(56)) == r)
        off += n
    # tail bits below 2k are zero in every key (left-aligned layout, src/kmer.h:15)
    if k % 32:
        lastw = (k - 1) // 32
        mask = np.uint64((1 << (64 - 2 * (k % 32))) - 1)
        assert not np.any(low[:, lastw] & mask) and not np.any(rk[:, lastw] & mask)
    for w in range((k - 1) // 32 + 1, nw):
        assert not np.any(low[:, w]) and not np.any(rk[:, w])


def merged(low, roots, k):
    nw = oracle.words(k)
    return oracle.merged_counts(low, roots["key"].reshape(-1, nw), roots["count"], nw=nw)


def check_exact(counter, data, k, want=None):
    """Full parity with the oracle: same exact (key, count) multiset."""
    low, roots, per_root = gpu_outputs(counter, k)
    check_layout(low, roots, per_root, k)
    mk, mc = merged(low, roots, k)
    if want is None:
        want = oracle.count(data, k)
    keys, counts, K = want
    assert counter.stats.total_kmers == K
    assert mk.shape == keys.shape and np.array_equal(mk, keys)
    assert np.array_equal(mc, counts.astype(np.uint64))
    return low, roots


def check_filtered(counter, data, k, min_count, max_count):
    """min/max apply to the table count (root count), as
    src/NewKmerTree.h:1159-1168: a root record (key, c) exists iff
    c = true_count - [key in low] lies in [min, max]."""
    low, roots, per_root = gpu_outputs(counter, k)
    check_layout(low, roots, per_root, k, min_count, max_count)
    keys, counts, K = oracle.count(data, k)
    nw = oracle.words(k)
    rk = roots["key"].reshape(-1, nw)
    allk = np.concatenate([keys, low, rk])
    _, inv = np.unique(allk, axis=0, return_inverse=True)
    inv = inv.reshape(-1)
    nid = inv.max() + 1 if inv.size else 0
    true = np.zeros(nid, np.int64)
    true[inv[:keys.shape[0]]] = counts
    in_low = np.zeros(nid, bool)
    in_low[inv[keys.shape[0]:keys.shape[0] + low.shape[0]]] = True
    assert np.all(true[inv[keys.shape[0]:keys.shape[0] + low.shape[0]]] >= 1), "low.bin key not in input"
    table = true - in_low.astype(np.int64)
    expect = (table >= min_count) & (table <= max_count) & (table >= 1)
    got = np.zeros(nid, bool)
    rid = inv[keys.shape[0] + low.shape[0]:]
    got[rid] = True
    assert np.array_equal(got, expect)
    assert np.array_equal(roots["count"].astype(np.int64), table[rid])


def merged_on_device(low_raw, roots_raw, k):
    """Merged exact (key, count) table of low.bin bytes and root records held
    in CUDA uint8 tensors, computed on the GPU with torch (for outputs of
    hundreds of millions of keys, where numpy sorting takes minutes): returns
    (keys (D, N) uint64, counts (D,) uint64) as numpy arrays in the oracle's
    lexicographic order, ready for oracle.digest.  Needs packed low.bin
    records of whole words (packed bytes == 8N: k = 31, 32, 63, 64)."""
    import torch
    nw = oracle.words(k)
    if oracle.packed_bytes(k) != 8 * nw:
        raise ValueError("merged_on_device needs whole-word low.bin records")
    rec_words = nw + 1
    lk = low_raw.view(torch.int64).view(-1, nw)
    rr = roots_raw.view(torch.int64).view(-1, rec_words)
    keys = torch.cat([lk, rr[:, :nw]])
    cnt = torch.cat([torch.ones(lk.shape[0], dtype=torch.int64, device=lk.device), rr[:, nw] & 0xFFFFFFFF])
    del lk, rr
    # unsigned lexicographic order: flip the sign bit, stable sorts from the
    # last word to the first
    order = None
    for w in range(nw - 1, -1, -1):
        col = keys[:, w] if order is None else keys[order, w]
        _, idx = torch.sort(col ^ (-(2 ** 63)), stable=True)
        order = idx if order is None else order[idx]
        del col, idx
    keys, cnt = keys[order], cnt[order]
    del order
    new = torch.ones(keys.shape[0], dtype=torch.bool, device=keys.device)
    if keys.shape[0] > 1:
        new[1:] = (keys[1:] != keys[:-1]).any(dim=1)
    seg = torch.cumsum(new.to(torch.int64), 0) - 1
    D = int(seg[-1].item()) + 1 if seg.numel() else 0
    out_c = torch.zeros(D, dtype=torch.int64, device=keys.device).index_add_(0, seg, cnt)
    out_k = keys[new]
    return (out_k.cpu().numpy().view(np.uint64).reshape(-1, nw), out_c.cpu().numpy().view(np.uint64))


def device_outputs(counter, k):
    """The counter's last result copied into CUDA uint8 tensors (low bytes,
    root record bytes) and the per-root record counts."""
    import torch
    lb, nr, per_root = counter.sizes()
    rec = 8 * oracle.words(k) + 8
    low = torch.empty(max(lb, 8), dtype=torch.uint8, device="cuda")[:lb]
    roots = torch.empty(max(nr * rec, 8), dtype=torch.uint8, device="cuda")[:nr * rec]
    if lb:
        counter.copy_low_into(low.data_ptr(), lb)
    if nr:
        counter.copy_roots_into(roots.data_ptr(), nr * rec)
    return low, roots, per_root
