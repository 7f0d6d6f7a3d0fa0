"""Several-GPU host logic (kmertreecounter_b200.replicas) on the CPU.

Two gloo ranks share FASTQ files by the largest-first plan, every file is
counted exactly once, every rank receives every file's result, and a failure
on one rank is raised on both (no rank is left waiting).  The per-file count
here is the CPU oracle, standing in for the GPU count that the product path
runs (kc_count_fastq on the rank's device)."""
import datetime
import functools
import os
import socket

import numpy as np
import pytest

import oracle
from kmertreecounter_b200 import replicas, synth


def test_plan_is_largest_first_to_least_loaded():
    sizes = [5, 9, 1, 7, 3, 3]
    p = replicas.plan(sizes, 2)
    assert sorted(i for r in p for i in r) == list(range(len(sizes)))
    assert p == [[1, 4, 5], [3, 0, 2]]  # 9 | 7, 5 -> 12 | 3 -> 12 | tie, 3 -> 15 | 1 -> 13
    assert replicas.plan(sizes, 1) == [[1, 3, 0, 4, 5, 2]]
    assert replicas.plan([], 3) == [[], [], []]
    assert replicas.plan([4], 3) == [[0], [], []]


def _oracle_count(path, out_dir, k, fail_on=None):
    if fail_on and os.path.basename(path) == fail_on:
        raise OSError("simulated read failure")
    keys, counts, K = oracle.count(np.fromfile(path, np.uint8), k)
    with open(os.path.join(out_dir, "counted"), "a") as f:  # one line per count of this file
        f.write("x\n")
    return {"total_kmers": int(K), "distinct": int(keys.shape[0])}


def _worker(rank, world, port, files, outs, k, fail_on, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        res = replicas.count_files(files, outs, count=functools.partial(_oracle_count, fail_on=fail_on), k=k)
        q.put((rank, "ok", res))
    except RuntimeError as e:
        q.put((rank, "err", str(e)))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _run(files, outs, k, fail_on=None, world=2):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, files, outs, k, fail_on, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=180) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
            pytest.fail("a rank did not exit")
    return sorted(got)


@pytest.fixture(scope="module")
def fastq_files(tmp_path_factory):
    d = tmp_path_factory.mktemp("reads")
    files = []
    for i, scale in enumerate([0.004, 0.02, 0.008, 0.012, 0.002]):
        p = synth.plain_small(seed=40 + i, scale=scale)
        path = d / ("set%d.fastq" % i)
        synth.fastq(p).tofile(path)
        files.append(str(path))
    return files


def test_two_ranks_count_every_file_once(fastq_files, tmp_path):
    outs = [str(tmp_path / ("out%d" % i)) for i in range(len(fastq_files))]
    got = _run(fastq_files, outs, 21)
    assert [g[1] for g in got] == ["ok", "ok"]
    assert got[0][2] == got[1][2]  # every rank holds every file's result
    res = got[0][2]
    sizes = [os.path.getsize(f) for f in fastq_files]
    plan = replicas.plan(sizes, 2)
    for i, f in enumerate(fastq_files):
        keys, counts, K = oracle.count(np.fromfile(f, np.uint8), 21)
        assert res[i]["total_kmers"] == K and res[i]["distinct"] == keys.shape[0]
        assert res[i]["rank"] == (0 if i in plan[0] else 1)
        assert open(os.path.join(outs[i], "counted")).read() == "x\n"
    assert {r["rank"] for r in res} == {0, 1}


def test_failure_on_one_rank_is_raised_on_both(fastq_files, tmp_path):
    outs = [str(tmp_path / ("out%d" % i)) for i in range(len(fastq_files))]
    got = _run(fastq_files, outs, 21, fail_on=os.path.basename(fastq_files[1]))
    assert [g[1] for g in got] == ["err", "err"]
    assert all("set1.fastq" in g[2] and "simulated read failure" in g[2] for g in got)
