"""CPU restatement of the reference's post-processing (test infrastructure
only): PostProcess<N>::merge_all, tool/PostProcess.h:63-139.

  final_root.bin  the root files' records, files 0..255 in order (merge_buckets)
  final_low.bin   low.bin keys that are no root file's key, sorted
                  lexicographically over the key words and unique, each as N
                  raw 64-bit words (process_low_bin, merge_sorted_chunks)
  freq_hist.txt   "count\\tnum_kmers" then "c\\tn" in ascending c: each root
                  record at (count + 1) mod 2^32, each final_low key at 1
                  (load_root_files, write_hist); absent when both are empty
"""
import numpy as np

import oracle


def post_process(low_keys, root_records, k):
    """(final_root bytes, final_low bytes, freq_hist text or None) from
    low.bin keys ((L, N) uint64, any order, repeats allowed) and the root
    records (ExportRecord<N> structured array, files 0..255 in order)."""
    nw = oracle.words(k)
    rk = root_records["key"].reshape(-1, nw)
    final_root = root_records.tobytes()
    lk = np.ascontiguousarray(low_keys, np.uint64).reshape(-1, nw)
    if lk.shape[0]:
        uk, _ = oracle._sort_unique(lk, np.zeros(lk.shape[0], np.uint64))
        if rk.shape[0]:
            allk = np.concatenate([rk, uk])
            _, inv = np.unique(allk, axis=0, return_inverse=True)
            inv = inv.reshape(-1)
            in_root = np.zeros(inv.max() + 1, bool)
            in_root[inv[:rk.shape[0]]] = True
            uk = uk[~in_root[inv[rk.shape[0]:]]]
    else:
        uk = lk
    final_low = np.ascontiguousarray(uk, np.uint64).tobytes()
    hist = {}
    for c in ((root_records["count"].astype(np.uint64) + 1) % (1 << 32)).tolist():
        hist[c] = hist.get(c, 0) + 1
    if uk.shape[0]:
        hist[1] = hist.get(1, 0) + uk.shape[0]
    text = None
    if hist:
        text = "count\tnum_kmers\n" + "".join(f"{c}\t{n}\n" for c, n in sorted(hist.items()))
    return final_root, final_low, text
