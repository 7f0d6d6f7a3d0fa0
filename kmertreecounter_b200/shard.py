"""One input over several GPUs: root-prefix owners.

Every rank extracts and routes its slice of whole FASTQ records
(kc_route_device), the routed keys are exchanged in one all-to-all so that
rank d receives the keys of the root prefixes [lo_d, hi_d) (key word 0 >> 56),
and each rank counts what it received (kc_count_keys_device).  A rank's root
files are the root files of its prefixes; the low.bin bytes of all ranks,
concatenated in rank order, are the input's low.bin.  The reference
partitions its filters and trees by root prefix the same way
(src/FastqClassifier.h:211-240) and balances prefixes over its classifier
threads by load (src/main.cpp:38-86); here the ranges are contiguous and
balanced by key counts, so that every rank's send buffer is its routed keys
cut at range boundaries.

Slices start at 4-line record boundaries counted from the start of the file
(the reference's reader keeps the line index mod 4, src/FastqReader.h:293-308),
so no k-mer spans two slices and every rank reads its slice as a file of its
own.

Collectives, in this order on every rank (also when a rank failed, so that no
rank waits for good): broadcast_object_list (the slice cuts, found by rank
0), all_gather_object (routing errors), all_reduce (prefix counts),
all_to_all_single (split sizes), all_to_all_single (keys), all_gather_object
(counting errors), barrier (before the merge).

    python -m torch.distributed.run --nproc-per-node 8 --master-addr 127.0.0.1 \\
        -m kmertreecounter_b200.shard --k 31 --out out/ reads.fq
"""
import argparse
import json
import os
import shutil
import time

import numpy as np

N_PREFIX = 256


def record_starts(data, parts, chunk=64 << 20):
    """Byte offsets [0, s_1, .., s_{parts-1}, len(data)] that split `data`
    (FASTQ bytes, any array-like of uint8) into `parts` slices of about equal
    size, each starting at a line whose index from the start of the file is a
    multiple of 4.  Slices may be empty (tiny inputs)."""
    n = len(data)
    out = [0]
    lines = 0  # newlines before `pos`
    pos = 0
    for i in range(1, parts):
        target = max(out[-1], i * n // parts)
        while pos < target:  # count newlines up to the target, in chunks
            end = min(target, pos + chunk)
            lines += int(np.count_nonzero(np.asarray(data[pos:end]) == 10))
            pos = end
        # move to the start of the next line whose index is a multiple of 4:
        # past the next newline while mid-line or on a line of another index
        while pos < n and ((pos > 0 and data[pos - 1] != 10) or lines % 4 != 0):
            step = np.asarray(data[pos:min(n, pos + (1 << 20))])
            nl = np.flatnonzero(step == 10)
            if not nl.size:
                pos += step.size
                continue
            pos += int(nl[0]) + 1
            lines += 1
        out.append(min(pos, n))
    out.append(n)
    return out


def owner_ranges(counts, world):
    """Contiguous root-prefix ranges [(lo, hi)] per rank, in rank order, with
    about equal key totals (every rank owns at least one prefix when
    world <= 256).  Deterministic: every rank computes the same ranges from
    the same global counts."""
    counts = np.asarray(counts, np.float64)
    total = counts.sum()
    ranges, lo = [], 0
    for d in range(world):
        left = world - d  # ranks still to place, this one included
        if d == world - 1:
            hi = N_PREFIX
        else:
            goal = total * (d + 1) / world
            hi = lo + 1
            acc = counts[:hi].sum()
            while hi < N_PREFIX - (left - 1) and acc + counts[hi] / 2 <= goal:
                acc += counts[hi]
                hi += 1
        ranges.append((lo, hi))
        lo = hi
    return ranges


def _raise_any(dist, err):
    """Every rank learns every rank's error; raise on all of them if any."""
    world = dist.get_world_size()
    got = [None] * world
    dist.all_gather_object(got, err)
    errs = [e for e in got if e]
    if errs:
        raise RuntimeError("; ".join(errs))


def exchange_and_count(route, count, nw, device, dist):
    """The sharded count on this rank.  route() -> (keys, counts): the
    rank's routed keys as a 1-D int64 tensor on `device` (nw words per key,
    in prefix order) and uint64[256] keys per prefix; count(keys, counts) ->
    the rank's result, given the keys it owns (same layout) and uint64[256]
    per-prefix totals (zero outside its range).  Returns (result, ranges,
    global counts)."""
    import torch
    rank, world = dist.get_rank(), dist.get_world_size()
    keys, counts, err = None, np.zeros(N_PREFIX, np.uint64), None
    try:
        keys, counts = route()
        counts = np.asarray(counts, np.uint64)
    except Exception as e:  # reported to every rank before any exchange
        err = f"rank {rank}: routing: {e}"
    _raise_any(dist, err)
    g = torch.tensor(counts.astype(np.int64), device=device)
    dist.all_reduce(g)
    counts_global = g.cpu().numpy().astype(np.uint64)
    ranges = owner_ranges(counts_global, world)
    send = [int(counts[lo:hi].sum()) * nw for lo, hi in ranges]
    send_t = torch.tensor(send, dtype=torch.int64, device=device)
    recv_t = torch.empty(world, dtype=torch.int64, device=device)
    dist.all_to_all_single(recv_t, send_t)
    recv = [int(x) for x in recv_t.cpu().tolist()]
    owned = torch.empty(sum(recv), dtype=torch.int64, device=device)
    dist.all_to_all_single(owned, keys, recv, send)
    lo, hi = ranges[rank]
    own = np.zeros(N_PREFIX, np.uint64)
    own[lo:hi] = counts_global[lo:hi]
    res, err = None, None
    try:
        res = count(owned, own)
    except Exception as e:
        err = f"rank {rank}: counting: {e}"
    _raise_any(dist, err)
    return res, ranges, counts_global


def merge_outputs(rank_dirs, ranges, out_dir):
    """low.bin = the ranks' low.bin concatenated in rank order; root_p.bin =
    the owner's root_p.bin."""
    os.makedirs(out_dir, exist_ok=True)
    with open(os.path.join(out_dir, "low.bin"), "wb") as f:
        for d in rank_dirs:
            with open(os.path.join(d, "low.bin"), "rb") as g:
                shutil.copyfileobj(g, f, 16 << 20)
    for r, (lo, hi) in enumerate(ranges):
        for p in range(lo, hi):
            shutil.copyfile(os.path.join(rank_dirs[r], f"root_{p}.bin"), os.path.join(out_dir, f"root_{p}.bin"))


class _DeviceWords:
    """A device buffer of int64 words seen by torch without a copy
    (__cuda_array_interface__)."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<i8", "data": (ptr, False), "version": 3,
                                         "strides": None}


def routed_tensor(counter, nw, device):
    """The context's routed keys as an int64 tensor on `device` (no copy;
    valid until the next call on the counter)."""
    import torch
    ptr, n = counter.routed_keys()
    if n == 0:
        return torch.empty(0, dtype=torch.int64, device=device)
    return torch.as_tensor(_DeviceWords(ptr, n * nw), device=device)


def gpu_stages(counter, slice_bytes, device, d_slice=None):
    """route() and count() for exchange_and_count on this rank's GPU: the
    slice (host uint8 array, or d_slice already on the device) is routed by
    kc_route_device, the context's routed keys are the exchange's send buffer
    as they are (kc_routed_keys, no copy), and kc_count_keys_device counts
    the owned keys once the exchange has finished reading them."""
    import torch
    from ._native import KcError  # noqa: F401  (errors surface as KcError)
    nw = 1 if counter.cfg.k <= 32 else (2 if counter.cfg.k <= 64 else 4)

    def route():
        d = d_slice if d_slice is not None else torch.from_numpy(np.ascontiguousarray(slice_bytes)).to(device)
        # the slice was written on torch's stream; the routing kernels run on
        # the context's own stream
        torch.cuda.synchronize(device)
        counts = counter.route_device(d.data_ptr(), d.numel())
        return routed_tensor(counter, nw, device), counts

    def count(owned, own_counts):
        torch.cuda.synchronize(device)  # the exchange has read the send buffer the count overwrites
        n = owned.numel() // nw
        return counter.count_keys_device(owned.data_ptr() if n else 0, n, own_counts)

    return route, count, nw


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--k", type=int, required=True)
    ap.add_argument("--out", required=True, help="merged low.bin + root_{0..255}.bin")
    ap.add_argument("--min-count", type=int, default=1)
    ap.add_argument("--max-count", type=int, default=0xFFFFFFFF)
    ap.add_argument("file")
    a = ap.parse_args()
    import datetime
    import torch
    import torch.distributed as dist
    from ._native import Counter
    rank, world = int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        data = np.memmap(a.file, np.uint8, mode="r")
        msg = [None]  # one scan of the file (rank 0), not one per rank; its failure reaches every rank
        if rank == 0:
            try:
                msg[0] = ("ok", record_starts(data, world))
            except Exception as e:
                msg[0] = ("err", f"rank 0: slicing {a.file}: {e}")
        dist.broadcast_object_list(msg, src=0)
        if msg[0][0] != "ok":
            raise RuntimeError(msg[0][1])
        cuts = msg[0][1]
        t0 = time.perf_counter()
        with Counter(k=a.k, min_count=a.min_count, max_count=a.max_count, device=local) as c:
            route, count, nw = gpu_stages(c, data[cuts[rank]:cuts[rank + 1]], torch.device("cuda", local))
            st, ranges, _ = exchange_and_count(route, count, nw, torch.device("cuda", local), dist)
            part = os.path.join(a.out, f".rank{rank}")
            os.makedirs(part, exist_ok=True)
            c.write_outputs(part)
        dist.barrier()
        wall = time.perf_counter() - t0
        t = torch.tensor([wall, float(st.total_kmers)], dtype=torch.float64, device="cuda")
        dist.all_reduce(t[:1], op=dist.ReduceOp.MAX)
        dist.all_reduce(t[1:], op=dist.ReduceOp.SUM)
        if rank == 0:
            dirs = [os.path.join(a.out, f".rank{r}") for r in range(world)]
            merge_outputs(dirs, ranges, a.out)
            for d in dirs:
                shutil.rmtree(d)
            print(json.dumps({"ranks": world, "wall_s": float(t[0]), "total_kmers": int(t[1]), "ranges": ranges}))
        dist.barrier()
    finally:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
