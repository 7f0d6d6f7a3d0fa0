"""One input over several GPUs (kmertreecounter_b200.shard) on the CPU.

Record-boundary slicing, contiguous balanced prefix ranges, and the exchange
run as two gloo ranks: every rank routes its slice, the keys cross in one
all_to_all_single, every rank receives exactly the keys of its prefixes, and
the owners' counts together are the whole input's exact counts.  The oracle's
extraction and counting stand in for the GPU stages (kc_route_device,
kc_count_keys_device) that the product path runs; a failure in one rank's
routing is raised on both ranks before any exchange."""
import datetime
import os
import socket

import numpy as np
import pytest

import oracle
from kmertreecounter_b200 import shard, synth


@pytest.fixture(scope="module")
def reads():
    return synth.fastq(synth.plain_small(seed=77, scale=0.01))


@pytest.mark.parametrize("parts", [1, 2, 3, 7])
def test_record_starts_cut_at_record_boundaries(reads, parts):
    cuts = shard.record_starts(reads, parts, chunk=4096)
    assert cuts[0] == 0 and cuts[-1] == reads.size and cuts == sorted(cuts) and len(cuts) == parts + 1
    for c in cuts[1:-1]:
        assert reads[c - 1] == 10  # a line start
        assert int(np.count_nonzero(reads[:c] == 10)) % 4 == 0  # of a record
    # the slices' k-mers are the input's k-mers (none spans a cut)
    whole = oracle.extract(reads, 25)
    parts_k = [oracle.extract(reads[a:b], 25) for a, b in zip(cuts, cuts[1:])]
    assert sum(p.shape[0] for p in parts_k) == whole.shape[0]


def test_record_starts_tiny_and_ragged():
    d = np.frombuffer(b"@r\nACGT\n+\nIIII\n@s\nAC", np.uint8)
    cuts = shard.record_starts(d, 4)
    assert cuts[0] == 0 and cuts[-1] == d.size
    assert all(c in (0, 15, d.size) for c in cuts)  # 15 = start of the second record


def test_owner_ranges_are_contiguous_and_balanced():
    rng = np.random.default_rng(5)
    for world in (1, 2, 3, 8, 256):
        counts = rng.integers(0, 1000, 256)
        r = shard.owner_ranges(counts, world)
        assert len(r) == world and r[0][0] == 0 and r[-1][1] == 256
        assert all(a[1] == b[0] for a, b in zip(r, r[1:])) and all(lo < hi for lo, hi in r)
        if world <= 8:
            loads = [counts[lo:hi].sum() for lo, hi in r]
            assert max(loads) <= counts.sum() / world + counts.max()
    skew = np.r_[np.zeros(200), np.ones(56)]
    assert shard.owner_ranges(skew, 4) == [(0, 214), (214, 228), (228, 242), (242, 256)]


def _oracle_stages(slice_bytes, k, fail):
    """route/count stand-ins: the oracle's emission-order keys, routed by
    prefix (stable), and np.unique over the owned keys."""
    import torch
    nw = oracle.words(k)

    def route():
        if fail:
            raise OSError("simulated device failure")
        keys = oracle.extract(slice_bytes, k)
        order = np.argsort(keys[:, 0] >> np.uint64(56), kind="stable")
        keys = keys[order]
        counts = np.bincount((keys[:, 0] >> np.uint64(56)).astype(np.int64), minlength=256).astype(np.uint64)
        return torch.from_numpy(keys.reshape(-1).view(np.int64).copy()), counts

    def count(owned, own_counts):
        keys = owned.numpy().view(np.uint64).reshape(-1, nw)
        assert keys.shape[0] == int(own_counts.sum())
        pre = keys[:, 0] >> np.uint64(56)
        got = np.bincount(pre.astype(np.int64), minlength=256).astype(np.uint64)
        assert np.array_equal(got, own_counts)  # exactly the keys of this rank's prefixes
        uk, uc = np.unique(keys, axis=0, return_counts=True)
        return uk, uc.astype(np.uint64), int(keys.shape[0])

    return route, count, nw


def _worker(rank, world, port, data, k, fail_rank, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        cuts = shard.record_starts(data, world)
        route, count, nw = _oracle_stages(data[cuts[rank]:cuts[rank + 1]], k, rank == fail_rank)
        res, ranges, glob = shard.exchange_and_count(route, count, nw, "cpu", dist)
        q.put((rank, "ok", (res, ranges, glob)))
    except RuntimeError as e:
        q.put((rank, "err", str(e)))
    finally:
        dist.destroy_process_group()


def _run(data, k, world=2, fail_rank=-1):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    procs = [ctx.Process(target=_worker, args=(r, world, port, data, k, fail_rank, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=180) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
            pytest.fail("a rank did not exit")
    return sorted(got, key=lambda g: g[0])


@pytest.mark.parametrize("k", [31, 45])
def test_two_ranks_exchange_and_count_exactly(reads, k):
    got = _run(reads, k)
    assert [g[1] for g in got] == ["ok", "ok"]
    (_, _, (r0, ranges, glob)), (_, _, (r1, ranges1, _)) = got
    assert ranges == ranges1 and ranges[0][0] == 0 and ranges[1][1] == 256
    keys = np.concatenate([r0[0], r1[0]])
    counts = np.concatenate([r0[1], r1[1]])
    wk, wc, K = oracle.count(reads, k)
    mk, mc = oracle.merged_counts(keys[:0], keys, counts, nw=oracle.words(k))
    assert r0[2] + r1[2] == K == int(glob.sum())
    assert np.array_equal(mk, wk) and np.array_equal(mc, wc.astype(np.uint64))


def test_routing_failure_on_one_rank_is_raised_on_both(reads):
    got = _run(reads, 31, fail_rank=1)
    assert [g[1] for g in got] == ["err", "err"]
    assert all("rank 1: routing" in g[2] and "simulated device failure" in g[2] for g in got)


def test_merge_outputs(tmp_path):
    dirs = []
    for r in range(2):
        d = tmp_path / f"r{r}"
        d.mkdir()
        (d / "low.bin").write_bytes(bytes([r]) * (3 + r))
        for p in range(256):
            (d / f"root_{p}.bin").write_bytes(bytes([r, p % 256]) if (p < 100) == (r == 0) else b"")
        dirs.append(str(d))
    out = tmp_path / "out"
    shard.merge_outputs(dirs, [(0, 100), (100, 256)], str(out))
    assert (out / "low.bin").read_bytes() == b"\x00" * 3 + b"\x01" * 4
    for p in range(256):
        assert (out / f"root_{p}.bin").read_bytes() == bytes([0 if p < 100 else 1, p])
