"""Post-processing on the device (kc_post_process, kc_post_process_dir and
bin/PostProcess) against the REFERENCE's own PostProcess<N>::merge_all
(tool/PostProcess.h:63-139, built by oracle/Makefile) run on the same
low.bin and root files, byte for byte: final_root.bin, final_low.bin and
freq_hist.txt; and against the oracle's restatement for k whose low.bin the
reference cannot read raw (packed size other than 8N)."""
import os
import subprocess

import numpy as np
import pytest

import oracle
import postprocess
from conftest import ROOT
from test_postprocess import build_dir, read_root_files, reference

pytestmark = pytest.mark.gpu

kc = pytest.importorskip("kmertreecounter_b200")
from kmertreecounter_b200 import synth  # noqa: E402

FILES = ("final_root.bin", "final_low.bin", "freq_hist.txt")


def read_out(d):
    return {f: (open(os.path.join(d, f), "rb").read() if os.path.exists(os.path.join(d, f)) else None) for f in FILES}


@pytest.mark.parametrize("k", [21, 31, 32, 45, 63, 64, 100])
def test_device_postprocess_of_a_count(tmp_path, k):
    data = synth.fastq(synth.plain_small(seed=80 + k, scale=0.1))
    with kc.Counter(k=k, bloom_bits=2.0) as c:  # a small filter: some false positives (root-only keys)
        c.count_host(data)
        st = c.post_process(str(tmp_path / "dev"))
        low = oracle.unpack(c.low_bytes(), k)
        roots, _ = c.root_records()
        c.write_outputs(str(tmp_path / "tmp"))
    got = read_out(str(tmp_path / "dev"))
    want_root, want_low, want_hist = postprocess.post_process(low, roots, k)
    assert got["final_root.bin"] == want_root
    assert got["final_low.bin"] == want_low
    assert got["freq_hist.txt"].decode() == want_hist
    assert st.final_low * 8 * oracle.words(k) == len(want_low) and st.root_records == roots.size
    assert st.low_in_roots > 0  # the filter's false positives were exercised
    # the command line on the files the count wrote
    post = os.path.join(ROOT, "kmertreecounter_b200", "bin", "PostProcess")
    p = subprocess.run([post, str(tmp_path / "tmp"), str(tmp_path / "cli"), str(k)], capture_output=True, text=True)
    assert p.returncode == 0, p.stderr
    assert read_out(str(tmp_path / "cli")) == got
    # the reference's own PostProcess on the same files, where it reads low.bin correctly
    if os.path.exists(oracle.REF_POST) and oracle.packed_bytes(k) == 8 * oracle.words(k):
        assert reference(str(tmp_path / "tmp"), str(tmp_path / "ref"), k) == got


@pytest.mark.parametrize("k,dup", [(31, 3), (63, 0)])
def test_device_postprocess_dir_matches_reference(tmp_path, k, dup):
    d = str(tmp_path / "tmp")
    low, _ = build_dir(d, k, seed=90 + k, dup_every=dup)
    kc.post_process_dir(d, str(tmp_path / "dev"), k)
    got = read_out(str(tmp_path / "dev"))
    root, flow, text = postprocess.post_process(low, read_root_files(d, k), k)
    assert got == {"final_root.bin": root, "final_low.bin": flow, "freq_hist.txt": text.encode()}
    if os.path.exists(oracle.REF_POST):
        assert reference(d, str(tmp_path / "ref"), k) == got


def test_device_postprocess_empty(tmp_path):
    with kc.Counter(k=31) as c:
        c.count_host(np.frombuffer(b"@r\nACG\n+\nIII\n", np.uint8))
        st = c.post_process(str(tmp_path / "dev"))
    got = read_out(str(tmp_path / "dev"))
    assert got == {"final_root.bin": b"", "final_low.bin": b"", "freq_hist.txt": None} and st.hist_lines == 0
