"""The several-GPU driver (kmertreecounter_b200.replicas) in one process on
one GPU: each file counted by kc_count_fastq into its own directory, output
files equal to the oracle's merged counts."""
import numpy as np
import pytest

import oracle
import parity

pytestmark = pytest.mark.gpu

from kmertreecounter_b200 import replicas, synth  # noqa: E402


def test_count_files_matches_oracle(tmp_path):
    files, outs = [], []
    for i, scale in enumerate([0.01, 0.003]):
        path = tmp_path / ("r%d.fastq" % i)
        synth.fastq(synth.plain_small(seed=70 + i, scale=scale)).tofile(path)
        files.append(str(path))
        outs.append(str(tmp_path / ("o%d" % i)))
    res = replicas.count_files(files, outs, k=25)
    for f, o, r in zip(files, outs, res):
        keys, counts, K = oracle.count(np.fromfile(f, np.uint8), 25)
        assert r["total_kmers"] == K and r["rank"] == 0
        low, roots, per_root = oracle.read_outputs(o, 25)
        parity.check_layout(low, roots, per_root, 25)
        mk, mc = parity.merged(low, roots, 25)
        assert np.array_equal(mk, keys) and np.array_equal(mc, counts.astype(np.uint64))
