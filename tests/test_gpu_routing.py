"""Estimated bucket regions against the oracle.

A batch of at least 4096 extraction tiles (32 MiB) sizes its bucket regions
from a routing histogram of every 32nd 8 KiB tile.  Keys past a region go to
an overflow area after the regions, and a batch whose overflow area fills is
routed again from an exact histogram.  The inputs below use 8 KiB FASTQ
records (one read per extraction tile), so the reads in exactly the sampled
tiles can be made unrepresentative on purpose."""
import numpy as np
import pytest

import oracle
import parity

pytestmark = pytest.mark.gpu

kc = pytest.importorskip("kmertreecounter_b200")
from kmertreecounter_b200 import synth  # noqa: E402

TILE = 8192
READ_LEN = (TILE - 8) // 2  # "@rr\n" + read + "\n+\n" + quality + "\n" = 8192 bytes
STRIDE = 32                 # sampled tiles: 0, 32, 64, ...


def tiled_fastq(kinds, seed):
    """One 8 KiB FASTQ record per kind: 'R' random bases, 'A' poly-A, 'C' poly-C."""
    rng = np.random.default_rng(seed)
    bases = np.frombuffer(b"ACGT", np.uint8)
    out = np.empty(len(kinds) * TILE, np.uint8)
    head = np.frombuffer(b"@rr\n", np.uint8)
    mid = np.frombuffer(b"\n+\n", np.uint8)
    qual = np.full(READ_LEN, ord("I"), np.uint8)
    for i, kind in enumerate(kinds):
        if kind == "R":
            seq = bases[rng.integers(0, 4, READ_LEN)]
        else:
            seq = np.full(READ_LEN, ord(kind), np.uint8)
        rec = np.concatenate([head, seq, mid, qual, np.frombuffer(b"\n", np.uint8)])
        assert rec.size == TILE
        out[i * TILE:(i + 1) * TILE] = rec
    return out


N_TILES = 4160


@pytest.mark.parametrize("k", [31, 63])
def test_overflow_area_absorbs_underestimated_bucket(k):
    # every 64th tile (never a sampled one) is poly-A: bucket 0 holds ~4x its
    # estimate, the excess fits the overflow area
    kinds = ["A" if i % 64 == 5 else "R" for i in range(N_TILES)]
    data = tiled_fastq(kinds, seed=k)
    want = oracle.count(data, k)
    with kc.Counter(k=k) as c:
        st = c.count_host(data)
        assert st.overflow_keys > 0 and st.reroutes == 0
        parity.check_exact(c, data, k, want)


def test_full_overflow_area_reroutes_exactly():
    # the sampled tiles are poly-A, every other tile poly-C: the poly-C bucket
    # is estimated empty and its keys do not fit the overflow area
    kinds = ["A" if i % STRIDE == 0 else "C" for i in range(N_TILES)]
    data = tiled_fastq(kinds, seed=1)
    want = oracle.count(data, 31)
    with kc.Counter(k=31) as c:
        st = c.count_host(data)
        assert st.reroutes == 1
        parity.check_exact(c, data, 31, want)


def test_device_input_above_sampling_threshold():
    torch = pytest.importorskip("torch")
    p = synth.plain_small(seed=31, scale=1.2)
    data = synth.fastq(p)
    assert data.size >= 4096 * TILE
    want = oracle.count(data, 31)
    d = torch.from_numpy(data).cuda()
    with kc.Counter(k=31) as c:
        st = c.count_device(d.data_ptr(), d.numel())
        torch.cuda.synchronize()
        assert st.batches == 1 and st.reroutes == 0
        parity.check_exact(c, data, 31, want)
