"""Post-processing (tool/PostProcess.h merge_all), CPU side: the oracle's
restatement against the REFERENCE's own PostProcess<N> code (header-only,
driven by oracle/postprocess_ref.cpp, built by oracle/Makefile) on output
directories built from the oracle's exact counts, with keys that a filter
false positive put in a root file only and with repeated low.bin keys.  The
device version is compared with both in test_gpu_postprocess.py."""
import os
import subprocess

import numpy as np
import pytest

import oracle
import postprocess
from kmertreecounter_b200 import synth


def build_dir(d, k, seed, fp_every=37, dup_every=0):
    """low.bin + root_{0..255}.bin for the exact counts of a seeded input:
    every key in low.bin except every fp_every-th repeated key (a false
    positive: its whole count in its root record), repeated keys with
    count - 1 in their root file, records shuffled inside each file; with
    dup_every, every dup_every-th low key written twice."""
    data = synth.fastq(synth.plain_small(seed=seed, scale=0.05))
    keys, counts, _ = oracle.count(data, k)
    nw = oracle.words(k)
    rng = np.random.default_rng(seed)
    rep = np.flatnonzero(counts >= 2)
    fp = rep[::fp_every]
    in_low = np.ones(keys.shape[0], bool)
    in_low[fp] = False
    low = keys[in_low]
    if dup_every:
        low = np.concatenate([low, low[::dup_every]])
    low = low[rng.permutation(low.shape[0])]
    os.makedirs(d, exist_ok=True)
    oracle.pack(low, k).tofile(os.path.join(d, "low.bin"))
    root_count = counts.astype(np.int64) - in_low
    sel = np.flatnonzero(root_count >= 1)
    rec = np.zeros(sel.size, oracle.record_dtype(k))
    rec["key"] = keys[sel].reshape(-1, nw)
    rec["count"] = root_count[sel]
    roots = (keys[sel, 0] >> np.uint64(56)).astype(np.int64)
    for r in range(256):
        part = rec[roots == r]
        part = part[rng.permutation(part.size)]
        part.tofile(os.path.join(d, f"root_{r}.bin"))
    return low, rec


def read_root_files(d, k):
    dt = oracle.record_dtype(k)
    return np.concatenate([np.fromfile(os.path.join(d, f"root_{r}.bin"), dt) for r in range(256)])


def reference(d, out, k):
    os.makedirs(out, exist_ok=True)
    subprocess.run([oracle.REF_POST, d + "/", out + "/", str(oracle.words(k))], check=True, capture_output=True)
    files = {}
    for f in ("final_root.bin", "final_low.bin", "freq_hist.txt"):
        p = os.path.join(out, f)
        files[f] = open(p, "rb").read() if os.path.exists(p) else None
    return files


# the reference reads low.bin as raw kmer<N>: only k whose packed size is 8N
@pytest.mark.skipif(not os.path.exists(oracle.REF_POST), reason="reference PostProcess harness not built")
@pytest.mark.parametrize("k,dup", [(31, 0), (32, 5), (63, 0), (64, 7)])
def test_restatement_matches_reference_postprocess(tmp_path, k, dup):
    d = str(tmp_path / "tmp")
    low, _ = build_dir(d, k, seed=70 + k, dup_every=dup)
    ref = reference(d, str(tmp_path / "out"), k)
    root, flow, text = postprocess.post_process(low, read_root_files(d, k), k)
    assert ref["final_root.bin"] == root
    assert ref["final_low.bin"] == flow
    assert ref["freq_hist.txt"].decode() == text


@pytest.mark.skipif(not os.path.exists(oracle.REF_POST), reason="reference PostProcess harness not built")
def test_restatement_matches_reference_on_empty_inputs(tmp_path):
    d = tmp_path / "tmp"
    d.mkdir()
    (d / "low.bin").write_bytes(b"")
    ref = reference(str(d), str(tmp_path / "out"), 31)
    assert ref["final_root.bin"] == b"" and ref["final_low.bin"] == b"" and ref["freq_hist.txt"] is None
    root, flow, text = postprocess.post_process(np.empty((0, 1), np.uint64), np.empty(0, oracle.record_dtype(31)), 31)
    assert (root, flow, text) == (b"", b"", None)
