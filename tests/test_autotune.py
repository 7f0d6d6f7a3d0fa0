"""autotune.passes: the grouping of read sets into kc_count_sets passes
(at most `per_pass` sets and, but for a single set, `max_bytes` FASTQ bytes;
consecutive, covering every set once)."""
import numpy as np

from kmertreecounter_b200 import autotune


def test_passes_cover_every_set_once_within_limits():
    rng = np.random.default_rng(7)
    for _ in range(200):
        n = int(rng.integers(0, 40))
        sets = [(0, int(rng.integers(1, 1000)), 31) for _ in range(n)]
        per = int(rng.integers(1, 12))
        cap = None if rng.random() < 0.3 else int(rng.integers(1, 4000))
        groups = autotune.passes(sets, per, cap)
        assert [i for a, b in groups for i in range(a, b)] == list(range(n))
        for a, b in groups:
            assert 1 <= b - a <= per
            if cap is not None and b - a > 1:
                assert sum(s[1] for s in sets[a:b]) <= cap


def test_passes_keep_an_oversized_set_alone():
    sets = [(0, 10, 21), (0, 5000, 21), (0, 10, 31)]
    assert autotune.passes(sets, 512, 100) == [(0, 1), (1, 2), (2, 3)]
    assert autotune.passes(sets, 2, None) == [(0, 2), (2, 3)]
