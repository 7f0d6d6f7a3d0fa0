"""One input over several GPUs, its device stages on one GPU against the oracle.

kc_route_device leaves exactly the input's canonical k-mers, grouped by root
prefix with the reported per-prefix totals; kc_count_keys_device counts
routed keys exactly; and two slices routed on two contexts, exchanged by
owner range (device copies standing in for the all-to-all) and counted by
two owner contexts, give the whole input's exact counts once the outputs are
merged (low.bin concatenated, root files by owner).  The contexts run one
after another: no kernel waits for another."""
import numpy as np
import pytest

import oracle
import parity

pytestmark = pytest.mark.gpu

kc = pytest.importorskip("kmertreecounter_b200")
from kmertreecounter_b200 import shard, synth  # noqa: E402


def _routed(counter, data, k):
    torch = pytest.importorskip("torch")
    d = torch.from_numpy(data).cuda()
    counts = counter.route_device(d.data_ptr(), d.numel())
    nw = oracle.words(k)
    n = int(counts.sum())
    keys = torch.empty(max(n * nw, 1), dtype=torch.int64, device="cuda")
    counter.copy_routed(keys.data_ptr(), keys.numel() * 8)
    torch.cuda.synchronize()
    return keys[:n * nw], counts


@pytest.mark.parametrize("k", [31, 63])
def test_route_device_emits_every_kmer_by_prefix(k):
    data = synth.fastq(synth.plain_small(seed=41, scale=0.05))
    with kc.Counter(k=k) as c:
        keys, counts = _routed(c, data, k)
    nw = oracle.words(k)
    got = keys.cpu().numpy().view(np.uint64).reshape(-1, nw)
    want = oracle.extract(data, k)
    assert got.shape == want.shape
    pre = got[:, 0] >> np.uint64(56)
    assert np.all(pre[1:] >= pre[:-1])  # prefix order
    assert np.array_equal(np.bincount(pre.astype(np.int64), minlength=256).astype(np.uint64), counts)
    order = lambda a: a[np.lexsort(tuple(a[:, i] for i in range(nw - 1, -1, -1)))]  # noqa: E731
    assert np.array_equal(order(got), order(want))


@pytest.mark.parametrize("k", [21, 31, 63])
def test_count_keys_device_is_exact(k):
    data = synth.fastq(synth.plain_small(seed=42, scale=0.05))
    with kc.Counter(k=k) as c:
        keys, counts = _routed(c, data, k)
        n = int(counts.sum())
        c.count_keys_device(keys.data_ptr(), n, counts)
        parity.check_exact(c, data, k)


def test_count_keys_rejects_bad_totals():
    with kc.Counter(k=31) as c:
        with pytest.raises(kc.KcError) as e:
            c.count_keys_device(0, 5, np.zeros(256, np.uint64))
        assert e.value.code == kc.KC_ERR_INVALID
        with pytest.raises(kc.KcError) as e:
            c.copy_routed(0, 0)
        assert e.value.code == kc.KC_ERR_STATE


@pytest.mark.parametrize("k", [31, 45])
def test_two_owners_on_one_gpu_match_the_oracle(k, tmp_path):
    torch = pytest.importorskip("torch")
    data = synth.fastq(synth.plain_small(seed=43, scale=0.1))
    nw = oracle.words(k)
    cuts = shard.record_starts(data, 2)
    routed = []
    for r in range(2):
        with kc.Counter(k=k) as c:
            routed.append(_routed(c, data[cuts[r]:cuts[r + 1]], k))
    glob = routed[0][1] + routed[1][1]
    ranges = shard.owner_ranges(glob, 2)
    dirs = []
    for d, (lo, hi) in enumerate(ranges):
        parts = []
        for keys, counts in routed:  # what rank r sends to owner d
            a = int(counts[:lo].sum()) * nw
            b = int(counts[:hi].sum()) * nw
            parts.append(keys[a:b])
        owned = torch.cat(parts).contiguous()
        own = np.zeros(256, np.uint64)
        own[lo:hi] = glob[lo:hi]
        with kc.Counter(k=k) as c:
            n = owned.numel() // nw
            st = c.count_keys_device(owned.data_ptr() if n else 0, n, own)
            assert st.total_kmers == int(glob[lo:hi].sum())
            _, per_root = c.root_records()
            assert all(per_root[p] == 0 for p in range(256) if not lo <= p < hi)
            out = tmp_path / f"owner{d}"
            c.write_outputs(str(out))
            dirs.append(str(out))
    merged_dir = tmp_path / "merged"
    shard.merge_outputs(dirs, ranges, str(merged_dir))
    low, roots, _ = oracle.read_outputs(str(merged_dir), k)
    mk, mc = oracle.merged_counts(low, roots["key"].reshape(-1, nw), roots["count"], nw=nw)
    wk, wc, K = oracle.count(data, k)
    assert int(glob.sum()) == K
    assert np.array_equal(mk, wk) and np.array_equal(mc, wc.astype(np.uint64))


def test_shard_command_line_one_rank(tmp_path):
    """The command line end to end under torch.distributed.run with one rank
    (NCCL collectives over one GPU, no peer): merged output == oracle."""
    import os
    import socket
    import subprocess
    import sys
    data = synth.fastq(synth.plain_small(seed=44, scale=0.05))
    path = tmp_path / "reads.fq"
    data.tofile(path)
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = tmp_path / "out"
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "1", "--master-addr",
           "127.0.0.1", "--master-port", str(port), "-m", "kmertreecounter_b200.shard", "--k", "31", "--out", str(out),
           str(path)]
    p = subprocess.run(cmd, cwd=root, capture_output=True, text=True, timeout=300,
                       env=dict(os.environ, PYTHONPATH=root + os.pathsep + os.environ.get("PYTHONPATH", "")))
    assert p.returncode == 0, p.stderr[-2000:]
    low, roots, _ = oracle.read_outputs(str(out), 31)
    mk, mc = oracle.merged_counts(low, roots["key"].reshape(-1, 1), roots["count"], nw=1)
    wk, wc, K = oracle.count(data, 31)
    assert np.array_equal(mk, wk) and np.array_equal(mc, wc.astype(np.uint64))
    assert '"total_kmers": %d' % K in p.stdout


def test_sharded_bench_one_rank():
    """bench.py's several-GPU form (route the slice, one NCCL all-to-all of
    keys sent from the context's own buffer, count the owned prefixes) under
    torch.distributed.run with one rank: its line reports the input's exact
    k-mer total and strong scaling."""
    import json
    import os
    import subprocess
    import sys
    from conftest import ROOT
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "1", "--master-addr",
           "127.0.0.1", "--master-port", "29533", os.path.join(ROOT, "bench.py"), "--gpus", "1", "--shard",
           "--scale", "0.01", "--steps", "2", "--warmup", "1", "--e2e-steps", "1"]
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert p.returncode == 0, p.stderr[-2000:]
    line = json.loads(p.stdout.strip().splitlines()[-1])
    assert line["scaling"] == "strong" and line["config"]["parallelism"].startswith("sharded x1")
    data = synth.fastq(synth.genome_scale(scale=0.01))
    assert line["stats"]["total_kmers"] == oracle.total_kmers(data, 31)
    assert line["gpu_launches"] > 0 and line["e2e"]["h2d_bytes_per_step"] == data.size
