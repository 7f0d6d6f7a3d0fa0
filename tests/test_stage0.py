"""Stage-0 figures of the reference (src/main.cpp:38-108, :114-117, :174-186;
src/FastqPreReader.h:110-330).

CPU tests:
  * the library's rules (kc_stage0_rule) against the reference's OWN rule
    code (lpt and calculate_bloom_filter_capacity from its main.cpp, driven
    by oracle/stage0_ref.cpp and built by oracle/Makefile) on count vectors
    with ties, small counts and skew: owners, capacities, average and the
    classifier loads in print order, exactly;
  * the oracle's restatement of the reference's sampler + the library's rules
    against the report the reference printed for the golden inputs
    (tests/golden/golden.json "stage0", recorded by make_golden.py).
GPU tests (kc_stage0_file, the sample counted by the extraction kernel, and
the command line's printed lines) are in test_gpu_stage0.py.
"""
import hashlib
import os
import subprocess

import numpy as np
import pytest

import inputs
import oracle
import stage0 as s0
import kmertreecounter_b200 as kc


def reference_rule(counts, est, n_thread):
    inp = f"{est} {n_thread} " + " ".join(str(int(c)) for c in counts)
    out = subprocess.run([oracle.REF_STAGE0], input=inp, capture_output=True, text=True, check=True).stdout
    r = {"loads": [], "owner": [0] * 256, "capacity": [0] * 256}
    for line in out.splitlines():
        if line.startswith("Average prefix count:"):
            r["average"] = int(line.split(":")[1])
        elif line.startswith("classifiers "):
            r["classifiers"] = int(line.split()[1])
        elif line.startswith("Classifier "):
            head, val = line.split(":")
            r["loads"].append((int(head.split()[1]), int(val)))
        elif line.startswith("Max Bloom Filter capacity:"):
            r["max_capacity"] = int(line.split(":")[1])
        elif line.startswith("owner "):
            _, p, o = line.split()
            r["owner"][int(p)] = int(o)
        elif line.startswith("capacity "):
            _, p, c = line.split()
            r["capacity"][int(p)] = int(c)
    return r


def vectors():
    rng = np.random.default_rng(7)
    yield np.full(256, 500)                                   # all raised to 1000: every prefix ties
    yield rng.integers(0, 3000, 256)                          # many below 1000
    yield rng.integers(10_000, 10_100, 256)                   # dense ties
    yield (rng.pareto(1.5, 256) * 50_000).astype(np.int64)   # skewed
    v = rng.integers(1_000_000, 2_000_000, 256)
    v[::7] = v[3]                                            # repeated values
    yield v


@pytest.mark.skipif(not os.path.exists(oracle.REF_STAGE0), reason="reference Stage-0 harness not built")
@pytest.mark.parametrize("n_thread", [6, 8, 16, 32, 64])
@pytest.mark.parametrize("est", [1_000, 31_188_890, 6_288_888_890, 21_000_000_000])
def test_rule_matches_reference_code(n_thread, est):
    for counts in vectors():
        ref = reference_rule(counts, est, n_thread)
        got = kc.stage0_rule(counts, est, n_thread)
        assert got.classifier_num == ref["classifiers"]
        assert got.average_prefix_count == ref["average"]
        assert got.max_bloom_filter_capacity == ref["max_capacity"]
        assert list(got.bloom_filter_capacity) == ref["capacity"]
        assert list(got.prefix_owner) == ref["owner"]
        assert got.loads_in_print_order() == ref["loads"]


def test_rule_rejects_too_few_threads():
    with pytest.raises(kc.KcError) as e:
        kc.stage0_rule(np.zeros(256), 1000, 5)
    assert e.value.code == kc.KC_ERR_INVALID


def test_oracle_restatement_against_python_rule():
    # the tie-independent parts of the rule, restated in Python, agree with
    # the library on every vector
    for counts in vectors():
        got = kc.stage0_rule(counts, 6_288_888_890, 16)
        ref = s0.rule(counts, 6_288_888_890, 16)
        assert got.average_prefix_count == ref["average"] and got.max_bloom_filter_capacity == ref["max_capacity"]
        assert list(got.bloom_filter_capacity) == ref["capacity"]
        assert sorted(l for _, l in got.loads_in_print_order()) == ref["loads_sorted"]


STAGE0 = [("plain_small", 31), ("plain_small_s7", 21), ("plain_small_s7", 63), ("adversarial", 17),
          ("adversarial", 33), ("genome_scale_s05", 31), ("large_long_s02", 63)]


@pytest.mark.parametrize("name,k", STAGE0)
def test_sampler_restatement_reproduces_reference_report(golden, tmp_path, name, k):
    g = golden[name]["k"][str(k)].get("stage0")
    if g is None:
        pytest.skip("no Stage-0 report recorded for this case")
    e = golden[name]
    data = getattr(inputs, e["builder"])(**e["kwargs"])
    assert hashlib.sha256(data).hexdigest() == e["fastq_sha256"]
    path = tmp_path / "in.fastq"
    path.write_bytes(bytes(data))
    del data
    counts, est, _ = s0.sample_file(str(path), k)
    got = kc.stage0_rule(counts, est, g["n_thread"])
    assert got.average_prefix_count == g["average"]
    assert got.max_bloom_filter_capacity == g["max_capacity"]
    assert [list(x) for x in got.loads_in_print_order()] == g["loads"]
