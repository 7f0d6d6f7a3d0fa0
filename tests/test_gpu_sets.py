"""Many read sets counted in one pass (kc_count_sets) against the oracle and
against counting each set on its own."""
import numpy as np
import pytest

import oracle
import parity

pytestmark = pytest.mark.gpu

kc = pytest.importorskip("kmertreecounter_b200")
torch = pytest.importorskip("torch")
from kmertreecounter_b200 import synth  # noqa: E402


def make_sets(ks, seed=0):
    rng = np.random.default_rng(seed)
    datas = []
    for i, k in enumerate(ks):
        L = int(rng.integers(50, 301))
        p = synth.params(seed=1000 + seed * 97 + i, genome_len=int(rng.integers(20_000, 300_000)),
                         gc=float(rng.uniform(0.3, 0.7)), n_reads=int(rng.integers(0, 4000)) if i % 5 else 0,
                         read_len=(L, L), sub_rate=float(rng.uniform(0.005, 0.02)))
        datas.append(synth.fastq(p) if p.n_reads else np.zeros(0, np.uint8))
    offs, pos = [], 0
    for d in datas:
        offs.append(pos)
        pos += (d.size + 15) // 16 * 16
    buf = np.full(max(pos, 16), ord("\n"), np.uint8)
    for o, d in zip(offs, datas):
        buf[o:o + d.size] = d
    return buf, [(o, d.size, k) for o, d, k in zip(offs, datas, ks)], datas


def check_sets(c, res, sets, datas):
    low_all = c.low_bytes()
    roots_all, _ = c.root_records()
    for (o, n, k), r, d in zip(sets, res, datas):
        low = oracle.unpack(low_all[r.low_offset:r.low_offset + r.low_bytes], k)
        rec = roots_all[r.root_offset:r.root_offset + r.root_records]
        parity.check_layout(low, rec, list(r.root_counts), k)
        mk, mc = parity.merged(low, rec, k)
        keys, counts, K = oracle.count(d, k)
        assert r.total_kmers == K
        assert np.array_equal(mk, keys) and np.array_equal(mc, counts.astype(np.uint64))


@pytest.mark.parametrize("ks,cfg", [([21, 31] * 12, {}), ([31, 21, 25] * 5, {"repeat_ratio": 1e-6}),
                                    ([33, 63, 47, 64] * 4, {"k": 63}), ([65, 100, 127, 128] * 3, {"k": 101}),
                                    ([70, 99] * 3, {"k": 101, "repeat_ratio": 1e-6})])
def test_sets_match_oracle(ks, cfg):
    buf, sets, datas = make_sets(ks, seed=len(ks))
    d = torch.from_numpy(buf).cuda()
    with kc.Counter(k=cfg.get("k", 31), **{k: v for k, v in cfg.items() if k != "k"}) as c:
        res = c.count_sets(d.data_ptr(), sets)
        if "repeat_ratio" in cfg:
            assert c.stats.rehashes > 0
        check_sets(c, res, sets, datas)


def test_sets_equal_single_counts():
    buf, sets, datas = make_sets([31] * 6, seed=9)
    d = torch.from_numpy(buf).cuda()
    with kc.Counter(k=31) as c:
        res = c.count_sets(d.data_ptr(), sets)
        lows = c.low_bytes()
        roots_all, _ = c.root_records()
    for (o, n, k), r, data in zip(sets, res, datas):
        with kc.Counter(k=k) as single:
            single.count_host(data)
            low1, roots1, _ = parity.gpu_outputs(single, k)
        a = parity.merged(oracle.unpack(lows[r.low_offset:r.low_offset + r.low_bytes], k),
                          roots_all[r.root_offset:r.root_offset + r.root_records], k)
        b = parity.merged(low1, roots1, k)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_sets_graph_is_replayed():
    """The scatter/gap/count graph of kc_count_sets is instantiated once and
    updated for later calls with other sets (same kernels)."""
    buf, sets, datas = make_sets([21, 31] * 4, seed=3)
    d = torch.from_numpy(buf).cuda()
    with kc.Counter(k=31) as c:
        for part in (sets, sets[:5], sets[2:]):
            res = c.count_sets(d.data_ptr(), part)
            check_sets(c, res, part, [datas[sets.index(x)] for x in part])
        assert c.sets_graph_instantiations() == 1


@pytest.mark.parametrize("min_prefix", [0, 1 << 40])
def test_sets_learned_sizing_is_exact(min_prefix):
    """Batched learned sizing (sizing.predict_sets: a batched count of every
    set's first 1%, one network pass, per-set per-bucket rates) sizes the
    tables of kc_count_sets -- every set (min_prefix 0) or none (all keep the
    sampled rule); the counts stay the oracle's."""
    import os
    from kmertreecounter_b200 import sizing
    if not os.path.exists(sizing.MODEL_PATH):
        pytest.skip("no trained sizing model")
    buf, sets, datas = make_sets([21, 31] * 8, seed=5)
    d = torch.from_numpy(buf).cuda()
    model = sizing.MLP.load(max_batch=64)
    with kc.Counter(k=31, sizing=kc.KC_SIZING_LEARNED) as c:
        dist, tab = sizing.predict_sets(c, model, d.data_ptr(), sets, [150] * len(sets), min_prefix_bytes=min_prefix)
        assert dist.shape == (len(sets), 256)
        if min_prefix == 0:
            assert np.all((tab >= 0) & (tab <= model.margin)) and np.all((dist >= 0) & (dist <= 1))
        else:
            assert np.all(tab == -1) and np.all(dist == -1)
        res = c.count_sets(d.data_ptr(), sets)
        check_sets(c, res, sets, datas)


def _tiled_sets(specs, seed):
    """Sets of 8 KiB FASTQ records (one read per extraction tile, so that the
    routing histogram's sampled tiles can be made unrepresentative): specs
    is a list of (kinds or None for a small synthetic set, k)."""
    import test_gpu_routing as tr
    datas = []
    for i, (kinds, k) in enumerate(specs):
        if kinds is None:
            p = synth.params(seed=seed * 31 + i, genome_len=50_000, n_reads=2000, read_len=(150, 150))
            datas.append(synth.fastq(p))
        else:
            datas.append(tr.tiled_fastq(kinds, seed=seed + i))
    offs, pos = [], 0
    for d in datas:
        offs.append(pos)
        pos += (d.size + 15) // 16 * 16
    buf = np.full(pos, ord("\n"), np.uint8)
    for o, d in zip(offs, datas):
        buf[o:o + d.size] = d
    return buf, [(o, d.size, k) for o, d, (_, k) in zip(offs, datas, specs)], datas


def test_sets_estimated_regions_overflow_into_the_set_area():
    """Sets of at least 4096 tiles are routed from a histogram of every 32nd
    tile: a bucket underestimated by the sample (poly-A reads in unsampled
    tiles) spills into that set's own overflow area, a set of random reads is
    estimated well, small sets beside them keep exact regions, and every
    set's counts are the oracle's."""
    n = 4160
    specs = [(["A" if i % 64 == 5 else "R" for i in range(n)], 31), (None, 21), (["R"] * n, 31), (None, 31)]
    buf, sets, datas = _tiled_sets(specs, seed=4)
    d = torch.from_numpy(buf).cuda()
    with kc.Counter(k=31) as c:
        res = c.count_sets(d.data_ptr(), sets)
        assert c.stats.reroutes == 0
        check_sets(c, res, sets, datas)


def test_sets_full_overflow_area_reroutes_exactly():
    """A set whose sampled tiles are all poly-A and the rest poly-C: the
    poly-C bucket is estimated empty and overflows the set's overflow area;
    the pass is routed again with exact regions and stays exact."""
    n = 4160
    specs = [(None, 31), (["A" if i % 32 == 0 else "C" for i in range(n)], 31), (None, 21)]
    buf, sets, datas = _tiled_sets(specs, seed=6)
    d = torch.from_numpy(buf).cuda()
    with kc.Counter(k=31) as c:
        res = c.count_sets(d.data_ptr(), sets)
        assert c.stats.reroutes == 1
        check_sets(c, res, sets, datas)
        res = c.count_sets(d.data_ptr(), sets)  # the next call routes from the sample again
        check_sets(c, res, sets, datas)
