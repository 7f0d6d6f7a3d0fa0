"""Several GPUs: one process per GPU, each counting whole inputs of its own.

The counting path has no exchange step between GPUs when the unit of work is
an input file: every file is counted exactly, on one GPU, into its own output
directory (tmp/low.bin + tmp/root_{0..255}.bin), as the reference counts one
file per process.  Files go to ranks largest first, each to the rank with the
least assigned bytes -- the longest-processing-time rule the reference uses to
balance prefix counts over its classifier threads (src/main.cpp:38-86).

Run under torch.distributed (NCCL on GPUs; the tests use gloo on the CPU):

    python -m torch.distributed.run --nproc-per-node 8 --master-addr 127.0.0.1 \\
        -m kmertreecounter_b200.replicas --k 31 --out-root out/ a.fq b.fq ...

Every rank takes the same collective steps in the same order: one
all_gather_object of (per-file stats, error) after its files are done, so a
failure on any rank is raised on every rank instead of leaving the others
waiting.
"""
import argparse
import json
import os
import time


def env():
    """(rank, world size, local rank) from the launcher's environment."""
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def plan(sizes, world):
    """File indices per rank: largest file first to the least-loaded rank
    (ties to the lowest rank).  Deterministic, so every rank computes the same
    plan without communicating."""
    load = [0] * world
    out = [[] for _ in range(world)]
    for i in sorted(range(len(sizes)), key=lambda i: (-sizes[i], i)):
        r = min(range(world), key=lambda r: (load[r], r))
        out[r].append(i)
        load[r] += sizes[i]
    return out


def _dist():
    import torch.distributed as dist
    return dist if dist.is_available() and dist.is_initialized() else None


def max_over_ranks(value, device=None):
    """Largest `value` over all ranks (the timing rule for a multi-GPU step)."""
    dist = _dist()
    if dist is None:
        return value
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _count_on_gpu(path, out_dir, **cfg):
    from ._native import count_fastq
    st = count_fastq(path, out_dir, **cfg)
    return {"total_kmers": int(st.total_kmers), "low_records": int(st.low_records),
            "root_records": int(st.root_records), "device_ms": float(st.device_ms), "wall_ms": float(st.wall_ms)}


def count_files(files, out_dirs, count=None, **cfg):
    """Count every file into its output directory, the files shared over the
    ranks by `plan`.  `count(path, out_dir, **cfg)` returns a JSON-able dict
    (default: the library's kc_count_fastq on this rank's GPU).  Returns the
    per-file results in file order on every rank; raises RuntimeError on every
    rank if any rank failed."""
    if len(files) != len(out_dirs):
        raise ValueError("one output directory per file")
    dist = _dist()
    rank, world = (dist.get_rank(), dist.get_world_size()) if dist else (0, 1)
    if count is None:
        cfg.setdefault("device", env()[2])
        count = _count_on_gpu
    mine = plan([os.path.getsize(f) for f in files], world)[rank]
    results, error = {}, None
    for i in mine:
        try:
            os.makedirs(out_dirs[i], exist_ok=True)
            results[i] = dict(count(files[i], out_dirs[i], **cfg), rank=rank)
        except Exception as e:  # reported to every rank below
            error = f"rank {rank}: {files[i]}: {e}"
            break
    if dist:
        gathered = [None] * world
        dist.all_gather_object(gathered, (results, error))
    else:
        gathered = [(results, error)]
    errors = [e for _, e in gathered if e]
    if errors:
        raise RuntimeError("; ".join(errors))
    merged = {}
    for res, _ in gathered:
        merged.update(res)
    return [merged[i] for i in range(len(files))]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--k", type=int, required=True)
    ap.add_argument("--out-root", required=True, help="one subdirectory per input file")
    ap.add_argument("--min-count", type=int, default=1)
    ap.add_argument("--max-count", type=int, default=0xFFFFFFFF)
    ap.add_argument("files", nargs="+")
    a = ap.parse_args()
    rank, world, local = env()
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    outs = [os.path.join(a.out_root, "%04d_%s" % (i, os.path.basename(f))) for i, f in enumerate(a.files)]
    t0 = time.perf_counter()
    res = count_files(a.files, outs, k=a.k, min_count=a.min_count, max_count=a.max_count)
    wall = max_over_ranks(time.perf_counter() - t0, device="cuda" if world > 1 else None)
    if rank == 0:
        print(json.dumps({"files": len(a.files), "ranks": world, "wall_s": wall, "results": res}))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
