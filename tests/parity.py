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
