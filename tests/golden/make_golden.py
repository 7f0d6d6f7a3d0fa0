"""Generate tests/golden/golden.json from the REFERENCE implementation.

Run in a checkout where the reference sources exist and `make -C oracle ref REF=<reference tree>`
has built oracle/_ref/Tree (the reference's own main.cpp compiled from its
source files).  For every case this script:
  1. builds the FASTQ bytes (tests/golden/inputs.py, deterministic),
  2. runs the reference `Tree <fastq> <k> 8 4` in a scratch directory,
  3. rejects runs whose "Total read k-mer count" differs from the oracle's K
     (the reference's parser can drop blocks on small inputs), retrying,
  4. reads tmp/low.bin + tmp/root_*.bin and records the merged exact
     multiset as (K, D, sha256 digest, count histogram head), plus the
     reference's histogram_tool "precise" output for the same directory.
The oracle itself is NOT used to produce the recorded values; the tests
compare the oracle (CPU) and the GPU path against them.

    python tests/golden/make_golden.py [--only name,name,...] [--stage0-only]

With --only, the named cases are (re)generated and merged into the existing
golden.json; the others are kept as they are.  --stage0-only adds the
reference's Stage-0 report (average prefix count, classifier loads, largest
Bloom filter; src/main.cpp:38-108, :174-186) to the cases of STAGE0_CASES.  The full genome-scale case
needs ~40 GB of host memory and ~20 GB of disk for the reference's outputs.
"""
import hashlib
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

import oracle  # noqa: E402
import inputs  # noqa: E402

CASES = [
    # name, builder, kwargs, k values
    ("plain_small", "plain_small", {"seed": 1}, [31]),
    ("plain_small_s7", "plain_small", {"seed": 7, "scale": 0.3}, [21, 32, 33, 63, 65, 101, 127, 128]),
    ("adversarial", "adversarial", {"seed": 11}, [17, 31, 32, 33, 64, 65, 100, 128]),
    # the benchmark shapes: genome-scale at 5% (1M reads, 313 MB) and in full
    # (20M reads, 3 Gbases, 6.3 GB), large long keys at 2% (1.3M reads, 418 MB)
    ("genome_scale_s05", "genome_scale", {"seed": 2, "scale": 0.05}, [31]),
    ("large_long_s02", "large_long", {"seed": 5, "scale": 0.02}, [63]),
    ("genome_scale_full", "genome_scale", {"seed": 2, "scale": 1.0}, [31]),
]
# host resources for the reference runs of each case (threads, memory_limit_gb)
RESOURCES = {"genome_scale_full": (8, 40)}


def stage0_lines(stdout, threads):
    """The reference's Stage-0 report (src/main.cpp:174-186, :38-108): the
    average prefix count, each classifier's load in print order and the
    largest Bloom filter capacity."""
    out = {"n_thread": threads, "loads": []}
    for line in stdout.splitlines():
        if line.startswith("Average prefix count:"):
            out["average"] = int(line.split(":")[1])
        elif line.startswith("Classifier ") and "total prefix count:" in line:
            head, val = line.split(":")
            out["loads"].append([int(head.split()[1]), int(val)])
        elif line.startswith("Max Bloom Filter capacity:"):
            out["max_capacity"] = int(line.split(":")[1])
    return out


def reference_case(fq, K_oracle, k, workdir, tries=4, threads=8, mem_gb=4):
    for attempt in range(tries):
        tmp = os.path.join(workdir, "tmp")
        if os.path.isdir(tmp):
            for f in os.listdir(tmp):
                os.remove(os.path.join(tmp, f))
        t0 = time.time()
        out, rc = oracle.run_reference(fq, k, workdir, threads=threads, mem_gb=mem_gb)
        wall = time.time() - t0
        K_ref = oracle.reference_total(out)
        total = None
        if rc == 0 and K_ref == K_oracle:
            # the merged counts must account for every k-mer exactly once: a
            # run that lost records in its output files reports the full K on
            # stdout yet sums short (seen with 256-bit keys)
            low, roots, _ = oracle.read_outputs(tmp, k)
            keys, counts = oracle.merged_counts(low, roots["key"], roots["count"], nw=oracle.words(k))
            total = int(counts.sum())
            if total == K_oracle:
                break
        print(f"  reference run rejected (rc={rc}, K={K_ref}, merged total={total}, expected {K_oracle}); retry",
              flush=True)
    else:
        raise RuntimeError("reference never produced a complete run")
    hist_file = os.path.join(workdir, "hist.tsv")
    subprocess.run([oracle.REF_HIST, "precise", tmp, str(k), str(threads), str(mem_gb), hist_file, "1", "64"],
                   check=True, capture_output=True)
    with open(hist_file) as f:
        tool_hist = [int(line.split("\t")[1]) for line in f if line.strip()]
    return {
        "stage0": stage0_lines(out, threads),
        "k": k,
        "K": K_ref,
        "D": int(keys.shape[0]),
        "L_reference": int(low.shape[0]),
        "R_reference": int(roots.shape[0]),
        "digest": oracle.digest(keys, counts),
        "hist_1_64": [int(x) for x in oracle.histogram(counts, 1, 64)],
        "histogram_tool_precise_1_64": tool_hist,
        "reference_wall_s": round(wall, 2),
        "reference_threads": threads,
    }


# (case, k) pairs whose Stage-0 report is recorded by --stage0-only
STAGE0_CASES = [("plain_small", 31), ("plain_small_s7", 21), ("plain_small_s7", 63), ("adversarial", 17),
                ("adversarial", 33), ("genome_scale_s05", 31), ("large_long_s02", 63), ("genome_scale_full", 31)]


def stage0_only(golden, wd):
    """Add the reference's Stage-0 report to existing entries: two reference
    runs must print the same report (its sampling threads could in principle
    drop a block, as its counting threads do on small inputs)."""
    for name, k in STAGE0_CASES:
        if name not in golden or str(k) not in golden[name]["k"]:
            continue
        e = golden[name]
        builder = next(b for n, b, kw, ks in CASES if n == name)
        data = getattr(inputs, builder)(**e["kwargs"])
        assert hashlib.sha256(data).hexdigest() == e["fastq_sha256"], "input generator drifted"
        fq = os.path.join(wd, "in.fastq")
        with open(fq, "wb") as f:
            f.write(data)
        del data
        threads, mem_gb = RESOURCES.get(name, (8, 4))
        reports = []
        for _ in range(4):
            out, rc = oracle.run_reference(fq, k, wd, threads=threads, mem_gb=mem_gb)
            if rc == 0:
                reports.append(stage0_lines(out, threads))
            if len(reports) >= 2 and reports[-1] == reports[-2]:
                break
        else:
            raise RuntimeError(f"{name} k={k}: no two matching Stage-0 reports")
        print(f"{name} k={k}: {reports[-1]['average']} {reports[-1]['loads']} {reports[-1]['max_capacity']}", flush=True)
        e["k"][str(k)]["stage0"] = reports[-1]
        tmp = os.path.join(wd, "tmp")
        for f in os.listdir(tmp):
            os.remove(os.path.join(tmp, f))


def main():
    oracle.build()
    only = None
    if "--only" in sys.argv:
        only = set(sys.argv[sys.argv.index("--only") + 1].split(","))
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.json")
    golden = {}
    if only and os.path.exists(path):
        with open(path) as f:
            golden = json.load(f)
    if "--stage0-only" in sys.argv:
        with open(path) as f:
            golden = json.load(f)
        with tempfile.TemporaryDirectory(dir=os.environ.get("KC_GOLDEN_TMP")) as wd:
            stage0_only(golden, wd)
        with open(path, "w") as f:
            json.dump(golden, f, indent=1, sort_keys=True)
        print("wrote", path)
        return
    with tempfile.TemporaryDirectory(dir=os.environ.get("KC_GOLDEN_TMP")) as wd:
        for name, builder, kw, ks in CASES:
            if only and name not in only:
                continue
            data = getattr(inputs, builder)(**kw)
            entry = {"builder": builder, "kwargs": kw, "fastq_bytes": len(data),
                     "fastq_sha256": hashlib.sha256(data).hexdigest(), "k": {}}
            threads, mem_gb = RESOURCES.get(name, (8, 4))
            fq = os.path.join(wd, "in.fastq")
            with open(fq, "wb") as f:
                f.write(data)
            K_oracle = {k: oracle.total_kmers(np.frombuffer(data, np.uint8), k) for k in ks}
            del data  # the full genome-scale input is 6.3 GB; the reference needs the memory
            for k in ks:
                print(f"{name} k={k}", flush=True)
                entry["k"][str(k)] = reference_case(fq, K_oracle[k], k, wd, threads=threads, mem_gb=mem_gb)
            golden[name] = entry
    with open(path, "w") as f:
        json.dump(golden, f, indent=1, sort_keys=True)
    print("wrote", path)


if __name__ == "__main__":
    main()
