"""kc_stage0_file and the command line's Stage-0 lines against the report the
reference printed for the same files (tests/golden/golden.json "stage0"),
and the sample's per-prefix counts against the oracle's restatement of the
reference's sampler (src/FastqPreReader.h:110-330; the sample is counted on
the device by the extraction kernel)."""
import hashlib
import os
import subprocess

import numpy as np
import pytest

import inputs
import stage0 as s0
from conftest import ROOT

pytestmark = pytest.mark.gpu

kc = pytest.importorskip("kmertreecounter_b200")

CASES = [("plain_small", 31), ("plain_small_s7", 21), ("plain_small_s7", 63), ("adversarial", 17),
         ("adversarial", 33), ("genome_scale_s05", 31), ("large_long_s02", 63), ("genome_scale_full", 31)]


def write_input(golden, name, path):
    e = golden[name]
    data = getattr(inputs, e["builder"])(**e["kwargs"])
    assert hashlib.sha256(data).hexdigest() == e["fastq_sha256"]
    path.write_bytes(bytes(data)) if len(data) < (1 << 30) else data.tofile(str(path))


@pytest.mark.parametrize("name,k", CASES)
def test_stage0_file_matches_reference_report(golden, tmp_path, name, k):
    g = golden[name]["k"][str(k)].get("stage0")
    if g is None:
        pytest.skip("no Stage-0 report recorded for this case")
    path = tmp_path / "in.fastq"
    write_input(golden, name, path)
    got = kc.stage0_file(str(path), k=k, n_thread=g["n_thread"])
    assert got.average_prefix_count == g["average"]
    assert got.max_bloom_filter_capacity == g["max_capacity"]
    assert [list(x) for x in got.loads_in_print_order()] == g["loads"]
    if os.path.getsize(path) < (1 << 30):  # the oracle's sampler on the same file (CPU)
        counts, est, sampled = s0.sample_file(str(path), k)
        assert got.estimated_file_size == est and got.sample_bytes == sampled
        assert np.array_equal(np.maximum(counts, 1000), np.array(got.prefix_count, np.int64))
    if name == "plain_small":  # the command line prints the reference's lines
        tree = os.path.join(ROOT, "kmertreecounter_b200", "bin", "Tree")
        p = subprocess.run([tree, str(path), str(k), str(g["n_thread"]), "4"], cwd=tmp_path, capture_output=True,
                           text=True)
        assert p.returncode == 0, p.stderr
        assert f"Average prefix count: {g['average']}" in p.stdout
        for i, load in g["loads"]:
            assert f"Classifier {i} total prefix count: {load}" in p.stdout
        assert f"Max Bloom Filter capacity: {g['max_capacity']}" in p.stdout


def test_stage0_gzip_head(tmp_path):
    """gzip input: the reference samples the first 256 MB-or-file-size of
    decompressed bytes and assumes the raw file is 4x the compressed one."""
    import gzip
    data = inputs.plain_small(seed=3, scale=0.2)
    path = tmp_path / "in.fastq.gz"
    with gzip.open(path, "wb", compresslevel=1) as f:
        f.write(bytes(data))
    got = kc.stage0_file(str(path), k=31, n_thread=8)
    counts, est, sampled = s0.sample_file(str(path), 31)
    assert got.estimated_file_size == est == 4 * os.path.getsize(path)
    assert got.sample_bytes == sampled
    assert np.array_equal(np.maximum(counts, 1000), np.array(got.prefix_count, np.int64))


def test_stage0_side_by_side_report(golden, tmp_path):
    """sizing.stage0_report: the reference's per-prefix filter capacities
    beside this build's sampled and learned rules, on the same file."""
    from kmertreecounter_b200 import sizing
    path = tmp_path / "in.fastq"
    write_input(golden, "plain_small", path)
    model = sizing.MLP.load() if os.path.exists(sizing.MODEL_PATH) else None
    r = sizing.stage0_report(str(path), 31, 8, model)
    g = golden["plain_small"]["k"]["31"]
    assert int(r["reference"].max()) == g["stage0"]["max_capacity"]
    assert int(r["kmers"].sum()) == g["K"] and int(r["distinct"].sum()) == g["D"]
    assert np.all(r["sampled"] >= 256) and np.all((r["sampled"] & (r["sampled"] - 1)) == 0)
    if model is not None:
        assert np.all(r["learned"] >= 256)
