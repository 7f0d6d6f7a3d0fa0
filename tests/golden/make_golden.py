"""Generate tests/golden/golden.json from the REFERENCE implementation.

Run in a checkout where the reference sources exist and `make -C oracle ref`
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

    python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import subprocess
import sys
import tempfile

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
]


def reference_case(data, k, workdir, tries=4):
    fq = os.path.join(workdir, "in.fastq")
    with open(fq, "wb") as f:
        f.write(data)
    K_oracle = int(oracle.extract(np.frombuffer(data, np.uint8), k).shape[0])
    for attempt in range(tries):
        tmp = os.path.join(workdir, "tmp")
        if os.path.isdir(tmp):
            for f in os.listdir(tmp):
                os.remove(os.path.join(tmp, f))
        out, rc = oracle.run_reference(fq, k, workdir, threads=8, mem_gb=4)
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
    subprocess.run([oracle.REF_HIST, "precise", tmp, str(k), "4", "4", hist_file, "1", "64"], check=True,
                   capture_output=True)
    with open(hist_file) as f:
        tool_hist = [int(line.split("\t")[1]) for line in f if line.strip()]
    return {
        "k": k,
        "K": K_ref,
        "D": int(keys.shape[0]),
        "L_reference": int(low.shape[0]),
        "R_reference": int(roots.shape[0]),
        "digest": oracle.digest(keys, counts),
        "hist_1_64": [int(x) for x in oracle.histogram(counts, 1, 64)],
        "histogram_tool_precise_1_64": tool_hist,
    }


def main():
    oracle.build()
    golden = {}
    with tempfile.TemporaryDirectory() as wd:
        for name, builder, kw, ks in CASES:
            data = getattr(inputs, builder)(**kw)
            entry = {"builder": builder, "kwargs": kw, "fastq_bytes": len(data),
                     "fastq_sha256": hashlib.sha256(data).hexdigest(), "k": {}}
            for k in ks:
                print(f"{name} k={k}", flush=True)
                entry["k"][str(k)] = reference_case(data, k, wd)
            golden[name] = entry
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.json")
    with open(path, "w") as f:
        json.dump(golden, f, indent=1, sort_keys=True)
    print("wrote", path)


if __name__ == "__main__":
    main()
