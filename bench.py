"""Benchmark: FASTQ Gbases/s to exact canonical k-mer counts on B200.

Workload (default): the genome-scale shape -- seeded 100 Mbp genome, 45% GC,
20% repeat families, 30x coverage of 150 bp reads (20M reads, 3 Gbases,
~6.3 GB FASTQ), canonical k=31 with 64-bit keys.  A step counts the whole
FASTQ once: extraction, routing, first-occurrence filter, repeat tables,
low.bin packing and root-record export, all on the device.

  value   FASTQ resident in HBM, outputs left in HBM (kc_count_device)
  e2e     the C ABI on HOST buffers: pinned FASTQ -> H2D -> count -> packed
          low.bin bytes and root records delivered to host memory through the
          streaming call (kc_count_host_stream), copies overlapped with counting

`--impl reference` times the reference's own CPU implementation (the `Tree`
binary built from the reference sources into oracle/_ref, else the oracle
port) on a bounded sample of the same workload, with all host threads.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
Multi-GPU: one process per GPU under torch.distributed.run; the ranks count
ONE copy of the workload together (strong scaling): each routes its slice of
whole records, one NCCL all-to-all sends every rank the keys of its range of
root prefixes, each counts its range (kmertreecounter_b200/shard.py).
`--shard` runs that form on one GPU too.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

WORKLOADS = {
    # name: (synth preset, k, n_buckets)
    "genome_scale": ("genome_scale", 31, 256),
    "plain_small": ("plain_small", 31, 256),
    "large_long": ("large_long", 63, 4096),
}
# device passes per workload (the 21 GB, k=63 input keeps ~44 GB of packed
# first occurrences and ~48 GB of tables on the device; 4 GiB passes keep the
# routed keys at ~18 GB: 383 ms per step against 401 ms in 2 GiB passes,
# 6 and 8 GiB passes run out of device memory)
DEVICE_BATCH = {"large_long": 4 << 30}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="genome_scale", choices=sorted(WORKLOADS))
    ap.add_argument("--scale", type=float, default=1.0, help="shrink genome and reads together")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-peaks", action="store_true", help="skip the atomic/link microbenchmark")
    ap.add_argument("--sample-scale", type=float, default=0.5, help="CPU sample size, fraction of the workload")
    ap.add_argument("--batch-scale", type=float, default=1.0,
                    help="read-set batch comparison: shrink genomes and read counts of the 512 sets")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-sort-record", action="store_true", help="skip the timed root-record sort")
    ap.add_argument("--no-sizing", action="store_true", help="skip the learned-vs-sampled sizing comparison")
    ap.add_argument("--no-large-long", action="store_true",
                    help="skip the long-key record (200 Mbp, 50x, k=63, 4096 buckets) of the default run")
    ap.add_argument("--ll-steps", type=int, default=3, help="timed steps of the long-key record")
    ap.add_argument("--ll-pass-gib", type=float, default=None,
                    help="device pass size of the long-key record in GiB (default: the workload's)")
    ap.add_argument("--no-file-to-file", action="store_true",
                    help="skip the command-line leg (bin/Tree vs the reference's Tree on the same file)")
    ap.add_argument("--no-reference-full", action="store_true",
                    help="in the command-line leg, skip the reference's Tree on the full-size file (about a minute)")
    ap.add_argument("--shard", action="store_true",
                    help="time the sharded count (root-prefix owners, one NCCL all-to-all) even on one GPU; "
                         "it is the default for more than one GPU")
    ap.add_argument("--write-sample", metavar="PATH", help=argparse.SUPPRESS)
    return ap.parse_args()


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


# --------------------------------------------------------------- clocks

class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []  # (arrival time, csv line)
        self.window = (0.0, float("inf"))

    def start(self):
        """Start polling (every 100 ms) and wait for the first sample, so that
        the timed region that follows is covered from its start."""
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            t_end = time.perf_counter() + 10.0
            while not self.lines and time.perf_counter() < t_end and self.proc.poll() is None:
                time.sleep(0.01)
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.perf_counter(), line.strip()))

    def mark(self, t0, t1):
        """Keep only samples taken between t0 and t1 (perf_counter seconds)."""
        self.window = (t0, t1)

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        t0, t1 = self.window
        for ts, ln in self.lines:
            if not (t0 <= ts <= t1):
                continue
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# --------------------------------------------------------------- workload

DESCRIBE = {
    "genome_scale": "genome_scale: 100 Mbp genome 45% GC 20% repeats, 30x 150 bp (20M reads), k=31",
    "large_long": "large_long: 200 Mbp genome 40% GC 30% repeats, 50x 150 bp (66.7M reads), k=63, 4096 buckets",
    "plain_small": "plain_small: 5 Mbp genome, 100k x 150 bp, k=31",
}


def make_workload(name, scale):
    from kmertreecounter_b200 import synth
    preset, k, buckets = WORKLOADS[name]
    p = getattr(synth, preset)(scale=scale)
    bases = int(p.n_reads) * int(p.read_len_min) if p.read_len_min == p.read_len_max else None
    return p, k, buckets, bases


def sharded(args, world):
    return world > 1 or args.shard


def workload_config(args, world, fastq_bytes, bases, reads):
    """The `config` object of both arms' lines (the reference arm reports our
    arm's config: its steps are bounded samples of this workload)."""
    k, buckets = WORKLOADS[args.workload][1:]
    name = DESCRIBE[args.workload] if args.scale == 1.0 else f"{args.workload} scale={args.scale}"
    par = (f"sharded x{world}: root-prefix owners, one NCCL all-to-all of routed keys" if sharded(args, world)
           else "one GPU")
    return {"workload": name, "k": k, "n_buckets": buckets, "fastq_bytes": int(fastq_bytes), "bases": int(bases),
            "reads": int(reads), "l2": "inputs larger than L2 (FASTQ %.1f GB)" % (fastq_bytes / 1e9),
            "parallelism": par}


def write_sample(name, scale, path):
    """Child-process mode (`bench.py --write-sample`): write a bounded sample
    of the workload (same shape, genome and reads shrunk together) to `path`
    and print the sample's and the full workload's sizes as JSON.  Run in a
    short-lived child so that the process timing the reference maps none of
    the counter's libraries."""
    from kmertreecounter_b200 import synth
    preset, k, _ = WORKLOADS[name]
    p = getattr(synth, preset)(scale=scale)
    data = synth.fastq(p)
    data.tofile(path)
    full = getattr(synth, preset)(scale=1.0)
    print(json.dumps({"path": path, "k": k, "bytes": int(data.size), "bases": int(p.n_reads) * int(p.read_len_min),
                      "reads": int(p.n_reads), "genome_len": int(p.genome_len),
                      "full": {"fastq_bytes": synth.fastq_bytes(full),
                               "bases": int(full.n_reads) * int(full.read_len_min), "reads": int(full.n_reads)}}))


def cpu_sample(name, sample_scale, workdir):
    """Bounded sample of the workload on disk, written by a child process:
    (path, the sample bytes, k, sample bases, description dict)."""
    path = os.path.join(workdir, "sample.fastq")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--write-sample", path,
                          "--workload", name, "--sample-scale", str(sample_scale)],
                         capture_output=True, text=True, check=True)
    info = json.loads(out.stdout.strip().splitlines()[-1])
    data = np.fromfile(path, dtype=np.uint8)
    return path, data, info["k"], info["bases"], info


def host_facts():
    """Host cores, memory and CPU model, for the CPU lines."""
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    try:
        ram = os.sysconf("SC_PAGE_SIZE") * os.sysconf("SC_PHYS_PAGES")
    except (ValueError, OSError):
        ram = None
    return {"cores": len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count(),
            "cpu_model": model, "ram_gb": round(ram / 2**30, 1) if ram else None}


def time_reference(path, data, k, bases, runs, workdir):
    """Reference `Tree` (or the oracle port) on the sample: list of
    (Gbases/s, seconds), kind, cores."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    cores = host_facts()["cores"] or 1
    K_expected = oracle.total_kmers(data, k)
    out = []
    if os.path.exists(oracle.REF_TREE):
        kind = "reference"
        mem = max(4, int(os.sysconf("SC_PAGE_SIZE") * os.sysconf("SC_PHYS_PAGES") / 2**30 * 0.7))
        for _ in range(runs):
            for attempt in range(3):
                t = time.perf_counter()
                stdout, rc = oracle.run_reference(path, k, workdir, threads=max(6, cores), mem_gb=mem)
                dt = time.perf_counter() - t
                if rc == 0 and oracle.reference_total(stdout) == K_expected:
                    out.append((bases / dt / 1e9, dt))
                    break
        if not out:
            kind = "port"
    else:
        kind = "port"
    if kind == "port":
        cores = 1
        for _ in range(runs):
            t = time.perf_counter()
            oracle.count(data, k)
            dt = time.perf_counter() - t
            out.append((bases / dt / 1e9, dt))
    return out, kind, cores


# DRAM traffic (dram__bytes_read.sum + dram__bytes_write.sum) per step of
# each stage of the genome-scale workload, from one ncu capture of the
# 10% case's first count (the kernels of kernel sources whose sha256 is
# given; profiles/launches_genome_scale.md gives the command) scaled to the
# full step by the units each stage processes: k-mers for extraction,
# sub-routing and count (x 10.000), first occurrences for packing
# (x 10.022), table cells for export and initialisation (x 9.781), FASTQ
# bytes for the line scan (x 10.032).  Reported only while the kernel
# sources are unchanged since that capture.
_CAPTURE_SHA = "cbcf5f8cf3571f44171df3491c10b6a6f761db93203f4e2bd6bd49d0ac3a22c3"
PROFILED_TRAFFIC = {
    # workload: {stage: {"sources_sha256": ..., "bytes_per_step": ...}}
    "genome_scale": {
        "extract_scatter": {"sources_sha256": _CAPTURE_SHA, "bytes_per_step": int(2433598976 * 10.000)},
        "subroute": {"sources_sha256": _CAPTURE_SHA, "bytes_per_step": int(3826577408 * 10.000)},
        "count": {"sources_sha256": _CAPTURE_SHA, "bytes_per_step": int(4611119104 * 10.000)},
        "pack_low": {"sources_sha256": _CAPTURE_SHA, "bytes_per_step": int(1245003008 * 10.022)},
        "export": {"sources_sha256": _CAPTURE_SHA, "bytes_per_step": int(1920347904 * 9.781)},
        "lines": {"sources_sha256": _CAPTURE_SHA, "bytes_per_step": int(627610880 * 10.032)},
        "init": {"sources_sha256": _CAPTURE_SHA, "bytes_per_step": int(916590336 * 9.781)},
    },
}
KERNEL_SOURCES = ("kmertreecounter_b200/csrc/kc_kernels.cuh", "kmertreecounter_b200/csrc/kc_window.cuh",
                  "kmertreecounter_b200/csrc/kc_engine.cu")


def kernel_sources_sha256():
    import hashlib
    h = hashlib.sha256()
    for rel in KERNEL_SOURCES:
        with open(os.path.join(ROOT, rel), "rb") as f:
            h.update(f.read())
    return h.hexdigest()


def profile_traffic(args, stage):
    """(traffic bytes per step of `stage` or None, note)."""
    e = PROFILED_TRAFFIC.get(args.workload, {}).get(stage)
    if not e or args.scale != 1.0 or not e["bytes_per_step"]:
        return None, "no capture of this stage on this workload"
    if e["sources_sha256"] != kernel_sources_sha256():
        return None, "kernel sources changed since the last capture"
    return e["bytes_per_step"], "ncu capture of these kernel sources"


STAGE_KERNELS = {
    "extract_scatter": "extract_kernel<SCATTER> + fill_region_gaps",
    "subroute": "subroute_count (1 chunk in 16) + window_caps + scan + subroute_scatter",
    "count": "count_window (x2 phases) + count_routed on the spill area",
    "pack_low": "pack_low",
    "export": "export_count + export_write_bits",
    "lines": "lines_per_tile",
    "init": "init_slots (+ zero16)",
}


def stage_rooflines(stage_ms, stats, F, k, hbm_gbs, P, rec, traffic=None):
    """Algorithmic bytes per step of every timed stage (the bytes its job has
    to move, counted once) over its device time, against the HBM peak:

      extract_scatter  F + 8N K          the FASTQ read once, every key written
      subroute         2 x 8N K          every key read and written again, window-grouped
      count            8N K + 8N L + 2 x 16 x cells x 9/8
                                         (windowed count) every key read, first occurrences
                                         written back, every table cell (16 B: key, count,
                                         filter word) and its window's halo read and written;
                       64 K + 64 (K - L) (global count, no windows) one 32 B filter sector read
                                         + write per k-mer and one table sector per repeat
      pack_low         8N L + P L        first occurrences read, packed low.bin written
      export           S cells + rec R   table read, root records written
      lines            F
      init             S cells + 8 W     table cells (and, for keys over 64 bits,
                                         the separate filter's W words) written
    with S = the table slot's bytes (16, 32, 48 for 64-, 128-, 256-bit keys)."""
    nw = 1 if k <= 32 else (2 if k <= 64 else 4)
    K, L, R = stats["total_kmers"], stats["low_records"], stats["root_records"]
    cells = stats["table_slots"]
    S = {1: 16, 2: 32, 4: 48}[nw]
    W = stats.get("filter_words", 0) if nw > 1 else 0  # 64-bit keys keep the filter in the cells
    windowed = stage_ms.get("subroute", 0.0) > 0
    rules = {
        "extract_scatter": (F + 8 * nw * K, "F + 8N K"),
        "subroute": (2 * 8 * nw * K, "2 x 8N K"),
        "count": ((8 * nw * K + 8 * nw * L + int(2 * 16 * cells * 9 / 8), "8N K + 8N L + 2 x 16 x cells x 9/8")
                  if windowed else (64 * K + 64 * (K - L), "64 K + 64 (K - L)")),
        "pack_low": (8 * nw * L + P * L, "8N L + P L"),
        "export": (S * cells + rec * R, f"{S} cells + rec R"),
        "lines": (F, "F"),
        "init": (S * cells + 8 * W, f"{S} cells" + (" + 8 filter words" if W else "")),
    }
    out = {}
    for s_, (b, rule) in rules.items():
        ms = stage_ms.get(s_, 0.0)
        if ms <= 0:
            continue
        gbs = b / (ms / 1e3) / 1e9
        out[s_] = {"ms": ms, "alg_bytes": b, "rule": rule, "gbs": gbs, "frac": gbs / hbm_gbs,
                   "kernels": STAGE_KERNELS[s_]}
        if traffic and traffic.get(s_) is not None:  # measured DRAM bytes (profiled, scaled)
            out[s_]["traffic"] = traffic[s_]
            out[s_]["traffic_over_alg"] = traffic[s_] / b
    return out


def pipeline_roofline(dev_peaks, pk, F, K, L, R, P, rec, ms_step, count_ms):
    """The workload's fixed roofline: t_roof = max(bytes_alg / HBM, atomics /
    atomic rate[, F / H2D for the host path]), with
    bytes_alg = F + 64 K + 64 (K - L) + L P + R rec (FASTQ read once, one
    filter sector read + write per k-mer and one table sector read + write per
    repeat occurrence, low.bin and root records written once) and one filter
    atomicOr (old value used) per k-mer plus one count atomicAdd (reduction)
    per repeat occurrence, each at its own measured rate.

    Two atomic rates are measured: on a 4 GiB random footprint (every atomic
    misses L2) and on a 32 MiB footprint (L2-resident).  Routing keys into
    buckets before counting keeps one bucket's filter and table words in L2
    while its keys are counted, so the L2-resident rate is the ceiling this
    design runs against; `frac` uses it, `frac_random_4gib` the 4 GiB rate."""
    if not dev_peaks:
        return {}
    hbm = pk["hbm_gbs"] * 1e9

    def t_atom(or_rate, add_rate):
        return K / (or_rate * 1e9) + (K - L) / (add_rate * 1e9)

    t_dram_atom = t_atom(dev_peaks["or_return_gops"], dev_peaks["red_add_gops"])
    t_l2_atom = t_atom(dev_peaks["l2_or_return_gops"], dev_peaks["l2_red_add_gops"])
    bytes_alg = F + 64 * K + 64 * (K - L) + L * P + R * rec
    t_hbm = bytes_alg / hbm
    t_roof = max(t_hbm, t_l2_atom)
    t_link = F / (dev_peaks["h2d_gbs"] * 1e9)
    out = {"pipeline": {
        "bytes_alg": bytes_alg, "atomics_alg": 2 * K - L, "t_hbm_ms": t_hbm * 1e3,
        "t_atomic_l2_ms": t_l2_atom * 1e3, "t_atomic_random_4gib_ms": t_dram_atom * 1e3,
        "t_h2d_ms": t_link * 1e3, "t_roof_ms": t_roof * 1e3, "t_roof_e2e_ms": max(t_roof, t_link) * 1e3,
        "bound": "hbm" if t_hbm >= t_l2_atom else "atomic", "frac": t_roof * 1e3 / ms_step,
        "frac_random_4gib": max(t_hbm, t_dram_atom) * 1e3 / ms_step,
        "peaks": {"hbm_gbs": pk["hbm_gbs"], "hbm_source": pk["source"],
                  "hbm_copy_gbs_this_gpu": dev_peaks["hbm_copy_gbs"],
                  "or_return_gops": dev_peaks["or_return_gops"], "red_add_gops": dev_peaks["red_add_gops"],
                  "l2_or_return_gops": dev_peaks["l2_or_return_gops"],
                  "l2_red_add_gops": dev_peaks["l2_red_add_gops"], "h2d_gbs": dev_peaks["h2d_gbs"],
                  "atomic_footprint_bytes": dev_peaks["footprint_bytes"],
                  "l2_footprint_bytes": dev_peaks["l2_footprint_bytes"], "source": "kc_measure_peaks on this GPU"}}}
    if count_ms > 0:
        out["count_routed_atomic"] = {"atomics_alg_per_step": 2 * K - L, "t_atomic_l2_ms": t_l2_atom * 1e3,
                                      "frac": t_l2_atom * 1e3 / count_ms,
                                      "t_atomic_random_4gib_ms": t_dram_atom * 1e3,
                                      "frac_random_4gib": t_dram_atom * 1e3 / count_ms}
    return out


def compare_batched(args, kc, torch):
    """512 independent read sets (genomes 1-20 Mbp, GC 30-70%, reads
    log-uniform 10k-2M per set, length 50-300, substitution 0.5-2%, k 21 or 31;
    genomes and read counts scaled by --batch-scale), FASTQ resident in HBM.
    plain: one kc_count_device call per set (per-set launches and host syncs);
    batched: kc_count_sets over autotuned groups of sets, one launch per stage
    per group.  Both wall-clock on the host around device-synchronous calls."""
    from concurrent.futures import ThreadPoolExecutor
    from kmertreecounter_b200 import autotune, synth
    specs = synth.batched_sets(n_sets=512, seed=3, scale=args.batch_scale)
    ks = [k for _, k in specs]
    sizes = [synth.fastq_bytes(p) for p, _ in specs]
    offs, pos = [], 0
    for nb in sizes:
        offs.append(pos)
        pos += (nb + 15) // 16 * 16
    buf = np.full(pos, ord("\n"), np.uint8)
    with ThreadPoolExecutor(max_workers=min(32, os.cpu_count() or 1)) as ex:  # the generator releases the GIL
        list(ex.map(lambda i: synth.fastq(specs[i][0], out=buf.ctypes.data + offs[i]), range(len(specs))))
    bases = int(sum(int(p.n_reads) * int(p.read_len_min) for p, _ in specs))
    dev = torch.from_numpy(buf).cuda()
    torch.cuda.synchronize()
    del buf
    sets = [(o, nb, k) for o, nb, k in zip(offs, sizes, ks)]
    base = dev.data_ptr()
    # a pass's keys, segments, filters and tables take up to about 8 bytes
    # per FASTQ byte: passes hold what fits 40% of the memory left
    free, _ = torch.cuda.mem_get_info()
    max_bytes = int(free * 0.4 / 8)
    # plain: one context per k, one call per set
    ctx = {k: kc.Counter(k=k) for k in sorted(set(ks))}
    for o, nb, k in sets[:8]:
        ctx[k].count_device(base + o, nb)
    torch.cuda.synchronize()
    t = time.perf_counter()
    for o, nb, k in sets:
        ctx[k].count_device(base + o, nb)
    torch.cuda.synchronize()
    plain_ms = (time.perf_counter() - t) * 1e3
    for c in ctx.values():
        c.close()
    # batched: autotuned knobs and sets per pass
    best = autotune.tune(base, sets, 31, use_cache=False, max_bytes=max_bytes)
    knobs = {k: v for k, v in best.items() if k in ("table_load", "repeat_ratio", "bloom_bits")}
    per_pass = best["sets_per_pass"]
    groups = autotune.passes(sets, per_pass, max_bytes)
    with kc.Counter(k=31, **knobs) as c:
        autotune.count_in_passes(c, base, sets, per_pass, max_bytes=max_bytes)
        torch.cuda.synchronize()
        t = time.perf_counter()
        grown, slots = [], []
        _, res = autotune.count_in_passes(c, base, sets, per_pass, grown, max_bytes=max_bytes, table_slots=slots)
        torch.cuda.synchronize()
        batched_ms = (time.perf_counter() - t) * 1e3
        stages = {}
        c.set_profiling(True)  # one more run, with stage events, for the breakdown
        autotune.count_in_passes(c, base, sets, per_pass, max_bytes=max_bytes, stages=stages)
        c.set_profiling(False)
        sums_batched = set_checksums(c, base, sets, groups, torch)
    out = {"sets": len(sets), "bases": bases, "fastq_bytes": int(pos), "scale": args.batch_scale,
           "passes": len(groups), "max_pass_fastq_bytes": max_bytes,
           "plain": {"ms": plain_ms, "gbases_s": bases / plain_ms / 1e6},
           "batched": {"ms": batched_ms, "gbases_s": bases / batched_ms / 1e6,
                       "rehashes": sum(grown), "table_slots_largest_pass": max(slots, default=0),
                       "tuned": {k: v for k, v in best.items() if k != "trials"},
                       "stages_ms": {s_: round(v, 3) for s_, v in stages.items() if v}},
           "speedup": plain_ms / batched_ms, "kmers": int(sum(r.total_kmers for r in res))}
    # batched + learned sizing: every pass first predicts its sets' loads (a
    # batched count of their first 1% and one network pass), then counts
    from kmertreecounter_b200 import sizing
    if os.path.exists(sizing.MODEL_PATH):
        model = sizing.MLP.load(max_batch=64)
        read_lens = [int(p.read_len_min) for p, _ in specs]

        def learned_passes(c, split):
            st_all = []
            for i, j in groups:
                t0 = time.perf_counter()
                sizing.predict_sets(c, model, base, sets[i:j], read_lens[i:j])
                torch.cuda.synchronize()
                t1 = time.perf_counter()
                st_all += c.count_sets(base, sets[i:j])
                torch.cuda.synchronize()
                split[0] += (t1 - t0) * 1e3
                split[1] += (time.perf_counter() - t1) * 1e3
                split[2] += int(c.stats.rehashes)
                split[3] = max(split[3], int(c.stats.table_slots))
            return st_all

        with kc.Counter(k=31, sizing=kc.KC_SIZING_LEARNED, **knobs) as c:
            learned_passes(c, [0.0, 0.0, 0, 0])
            torch.cuda.synchronize()
            split = [0.0, 0.0, 0, 0]
            t = time.perf_counter()
            res_l = learned_passes(c, split)
            torch.cuda.synchronize()
            learned_ms = (time.perf_counter() - t) * 1e3
            sums_learned = set_checksums(c, base, sets, groups, torch, learned=(model, read_lens))
        out["batched_learned"] = {"ms": learned_ms, "gbases_s": bases / learned_ms / 1e6,
                                  "speedup_vs_plain": plain_ms / learned_ms,
                                  "speedup_vs_batched": batched_ms / learned_ms,
                                  "predict_ms": split[0], "count_ms": split[1], "rehashes": split[2],
                                  "table_slots_largest_pass": split[3],
                                  "identical_counts": sums_learned == sums_batched,
                                  "kmers": int(sum(r.total_kmers for r in res_l))}
    del dev
    return out


def set_checksums(c, base, sets, groups, torch, learned=None):
    """Per set, a checksum of the exact (k-mer, count) multiset that does not
    depend on how the first-occurrence filter split it between low.bin and
    the root files: sum over low.bin keys of h(key) + sum over root records of
    h(key) x count (mod 2^64), h = a 64-bit mixer, computed on the device."""
    from kmertreecounter_b200 import sizing
    sums = []
    for i, j in groups:
        part = sets[i:j]
        if learned:
            sizing.predict_sets(c, learned[0], base, part, learned[1][i:j])
        res = c.count_sets(base, part)
        d_low, low_bytes, d_roots, n_roots = c.device_results()
        # the context's own buffers, seen by torch without a copy
        low = torch.as_tensor(_DeviceBytes(d_low, low_bytes), device="cuda") if low_bytes else \
            torch.empty(0, dtype=torch.uint8, device="cuda")
        roots = torch.as_tensor(_DeviceBytes(d_roots, n_roots * 16), device="cuda") if n_roots else \
            torch.empty(0, dtype=torch.uint8, device="cuda")
        rr = roots.view(torch.int64).view(-1, 2)
        for (o, b, k), r in zip(part, res):
            P = kc_packed(k)
            lk = low[r.low_offset:r.low_offset + r.low_records * P].view(-1, P)
            w = torch.zeros(lk.shape[0], dtype=torch.int64, device="cuda")
            for q in range(P):  # the packed tail bytes sit at the top of the word
                w |= lk[:, q].to(torch.int64) << (8 * (q + 8 - P))
            rec = rr[r.root_offset:r.root_offset + r.root_records]
            sums.append(int((_mix(w).sum() + (_mix(rec[:, 0]) * (rec[:, 1] & 0xFFFFFFFF)).sum()).item()) % (1 << 64))
    return sums


def sort_record(kc, torch, dev, n, k, merged, hbm_gbs):
    """The optional root-record sort (sort_output=1; the reference's
    export_record_radix_sort) on the workload's root records: one count with
    the sort on after one that sizes its buffers, the sort stage's device
    time from the library's stage events, and the sorted records checked on
    the device: keys strictly ascending as unsigned words (so every root
    file's records stay together, in key order), and the merged result
    (count histogram, distinct keys) equal to the unsorted count's `merged`.
    Algorithmic bytes: every record read and written once per 8-bit digit of
    the 2k-bit key."""
    with kc.Counter(k=k, sort_output=1) as c:
        c.count_device(dev.data_ptr(), n)
        c.set_profiling(True)
        c.count_device(dev.data_ptr(), n)
        ms, launches = c.stage_times().get("sort", (0.0, 0))
        c.set_profiling(False)
        _, _, d_roots, n_roots = c.device_results()
        asc = True
        if n_roots > 1:
            rr = torch.as_tensor(_DeviceBytes(d_roots, n_roots * 16), device="cuda").view(torch.int64).view(-1, 2)
            sign = -(1 << 63)
            asc = bool(((rr[1:, 0] ^ sign) > (rr[:-1, 0] ^ sign)).all().item())
        h, d = c.histogram(1, 10000)
    digits = (2 * k + 7) // 8
    alg = n_roots * 16 * 2 * digits
    gbs = alg / ms / 1e6 if ms else None
    return {"ms": ms, "launches": launches, "records": n_roots, "digit_passes": digits, "alg_bytes": alg,
            "rule": "R x 16 x 2 x digits", "gbs": gbs, "frac": gbs / hbm_gbs if gbs else None,
            "ascending": asc, "same_merged_counts": d == merged[1] and h.tolist() == merged[0].tolist()}


class _DeviceBytes:
    """n bytes of device memory at ptr, for torch.as_tensor without a copy."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "|u1", "data": (ptr, False), "version": 3,
                                         "strides": None}


def kc_packed(k):
    return (k // 32) * 8 + (2 * (k % 32) + 7) // 8


def _mix(x):
    """64-bit mixer in int64 arithmetic (wrapping), for set_checksums."""
    x = x ^ ((x >> 31) & 0x1FFFFFFFF)
    x = x * -7046029254386353131
    x = x ^ ((x >> 29) & 0x7FFFFFFFF)
    return x * -4658895280553007687


def compare_sizing(args, kc, torch, dev, n, k, buckets, device_batch=None, steps=None):
    """Learned vs sampled sizing on the same resident FASTQ, each timed end to
    end per step by wall clock on its own context (every count call returns
    synchronised).  A learned step counts the whole input with predicted
    sizes; the prediction (the first 1% of the reads counted with the plain
    rule on a helper context, the sizing MLP on the library's kernels) is
    made inside the step, at its sizing point, beside its k-mer extraction; a
    sampled step only counts.  Rehashes and
    structure memory for both rules; counts are identical by construction
    (checked by histogram)."""
    from kmertreecounter_b200 import sizing
    if not os.path.exists(sizing.MODEL_PATH):
        return None
    model = sizing.MLP.load()
    out = {}
    hist = {}
    for rule in ("sampled", "learned"):
        mode = kc.KC_SIZING_LEARNED if rule == "learned" else kc.KC_SIZING_SAMPLED
        cfg = kc.default_config(k=k, n_buckets=buckets, sizing=mode)
        if device_batch:
            cfg.device_batch_bytes = device_batch
        elif args.workload in DEVICE_BATCH:
            cfg.device_batch_bytes = DEVICE_BATCH[args.workload]
        with kc.Counter(cfg) as c:
            split = []
            # learned: the prediction (the first 1% counted on a helper
            # context, the network's forward pass) runs inside every step,
            # beside the count's k-mer extraction (sizing.BesideSizing)
            beside = sizing.BesideSizing(c, model, k, 150) if rule == "learned" else None
            if beside:
                beside.target = (dev.data_ptr(), n)

            def step():
                st_ = c.count_device(dev.data_ptr(), n)
                split.append((beside.last_ms if beside else 0.0, st_.device_ms))
                return st_
            step()
            times = []
            split.clear()
            for _ in range(max(steps or args.steps, 1)):
                torch.cuda.synchronize()
                t = time.perf_counter()
                st = step()
                times.append((time.perf_counter() - t) * 1e3)
            hist[rule] = c.histogram(1, 1000)
            out[rule] = dict(ms_per_step=statistics.median(times), rehashes=st.rehashes, table_slots=st.table_slots,
                             filter_words=st.filter_words, table_keys=st.table_keys,
                             predict_beside_ms=statistics.median(x[0] for x in split),
                             count_device_ms=statistics.median(x[1] for x in split))
            if beside:
                if beside.error:
                    raise beside.error
                beside.close()
    out["identical_counts"] = bool(np.array_equal(hist["sampled"][0], hist["learned"][0])
                                   and hist["sampled"][1] == hist["learned"][1])
    out["margin"] = model.margin
    return out


def large_long_record(args, kc, torch, dev_peaks, pk):
    """The long-key shape at full size (seeded 200 Mbp genome, 40% GC, 30%
    repeat families, 50x of 150 bp = 66.7M reads, 10 Gbases, 21 GB FASTQ,
    1% substitution; canonical k=63, 128-bit keys, 4096 buckets), FASTQ
    resident in HBM and counted in 4 GiB device passes: Gbases/s over
    --ll-steps steps timed with CUDA events on the library's stream, stage
    times, the count kernel's roofline in the same units as the main line,
    and learned vs sampled sizing on the same input."""
    from kmertreecounter_b200 import synth
    torch.cuda.empty_cache()
    p = synth.large_long()
    bases = int(p.n_reads) * int(p.read_len_min)
    data = synth.fastq(p)
    n = int(data.size)
    dev = torch.from_numpy(data).cuda()
    del data
    torch.cuda.synchronize()
    k, buckets = 63, 4096
    pass_bytes = int(args.ll_pass_gib * (1 << 30)) if args.ll_pass_gib else DEVICE_BATCH["large_long"]
    cfg = kc.default_config(k=k, n_buckets=buckets, device_batch_bytes=pass_bytes)
    steps = max(1, args.ll_steps)
    stage_ms = {}
    with kc.Counter(cfg) as c:
        stream = torch.cuda.ExternalStream(c.stream)
        c.count_device(dev.data_ptr(), n)  # warm-up, sizes every buffer
        c.set_profiling(True)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            st = c.count_device(dev.data_ptr(), n)
            for name, (ms, _) in c.stage_times().items():
                stage_ms[name] = stage_ms.get(name, 0.0) + ms
        e1.record(stream)
        torch.cuda.synchronize()
        ms_step = e0.elapsed_time(e1) / steps
        _, distinct = c.histogram(1, 2)
        stats = st.as_dict()
        stats.pop("root_counts", None)
    K, L = stats["total_kmers"], stats["low_records"]
    count_ms = stage_ms.get("count", 0.0) / steps
    roof = pipeline_roofline(dev_peaks, pk, n, K, L, stats["root_records"], kc.packed_bytes(k), kc.record_bytes(k),
                             ms_step, count_ms)
    out = {"config": {"workload": DESCRIBE["large_long"], "k": k, "n_buckets": buckets, "fastq_bytes": n,
                      "bases": bases, "reads": int(p.n_reads), "device_pass_bytes": pass_bytes},
           "value": bases / (ms_step / 1e3) / 1e9, "unit": "Gbases/s", "ms_per_step": ms_step, "steps": steps,
           "distinct_kmers": distinct, "distinct_kmers_per_s": distinct / (ms_step / 1e3), "stats": stats,
           "stages_ms_per_step": {s_: v / steps for s_, v in stage_ms.items()},
           "stage_rooflines": stage_rooflines({s_: v / steps for s_, v in stage_ms.items()}, stats, n, k,
                                              pk["hbm_gbs"], kc.packed_bytes(k), kc.record_bytes(k)),
           "pipeline_roofline": roof.get("pipeline")}
    if not args.no_sizing:
        out["sizing"] = compare_sizing(args, kc, torch, dev, n, k, buckets, pass_bytes, steps)
    del dev
    torch.cuda.empty_cache()
    return out


def file_to_file(args, sample_path, sample_bases, k, ref_sample_gbs, full_path, full_bases, full_kmers=None):
    """This build's drop-in command line (`bin/Tree <fastq> <k> <n_thread>
    <mem_gb>`) timed like the reference's `Tree`: wall clock of the whole
    process, from reading the FASTQ file to low.bin and root_0..255.bin
    written under ./tmp/, device set-up included.  On the reference's own
    sample file (beside the reference's time on it) and on the full workload's
    file, where the reference's `Tree` is also run once (all host threads;
    accepted only when the k-mer total it prints equals `full_kmers`)."""
    tree = os.path.join(ROOT, "kmertreecounter_b200", "bin", "Tree")
    threads = str(max(6, host_facts()["cores"] or 6))

    def run(path, bases, runs):
        best = None
        for _ in range(runs):
            with tempfile.TemporaryDirectory(dir=os.path.dirname(path)) as wd:
                t = time.perf_counter()
                r = subprocess.run([tree, path, str(k), threads, "16"], cwd=wd, capture_output=True, text=True)
                dt = time.perf_counter() - t
                if r.returncode:
                    return {"error": f"exit {r.returncode}: {r.stderr.strip()[-200:]}"}
                if best is None or dt < best:
                    best = dt
        return {"seconds": best, "gbases_s": bases / best / 1e9, "runs": runs}

    out = {"method": "wall clock of the process, outputs written to ./tmp/ on local disk, best of the runs"}
    ours = run(sample_path, sample_bases, 2)
    out["sample"] = {"ours": ours, "reference_gbases_s": ref_sample_gbs,
                     "ratio": ours["gbases_s"] / ref_sample_gbs if "gbases_s" in ours and ref_sample_gbs else None}
    if full_path:
        out["full"] = {"ours": run(full_path, full_bases, 2)}
        if ref_sample_gbs and not args.no_reference_full:
            sys.path.insert(0, os.path.join(ROOT, "oracle"))
            import oracle
            cores = host_facts()["cores"] or 1
            mem = max(4, int(os.sysconf("SC_PAGE_SIZE") * os.sysconf("SC_PHYS_PAGES") / 2**30 * 0.7))
            with tempfile.TemporaryDirectory(dir=os.path.dirname(full_path)) as wd:
                t = time.perf_counter()
                stdout, rc = oracle.run_reference(full_path, k, wd, threads=max(6, cores), mem_gb=mem)
                dt = time.perf_counter() - t
            got = oracle.reference_total(stdout) if rc == 0 else None
            ref = {"seconds": dt, "gbases_s": full_bases / dt / 1e9, "threads": max(6, cores), "runs": 1,
                   "kmers_reported": got, "kmers_expected": full_kmers}
            if rc != 0 or (full_kmers is not None and got != full_kmers):
                ref["rejected"] = f"exit {rc}, k-mer total {got} (expected {full_kmers})"
            out["full"]["reference"] = ref
            if "gbases_s" in out["full"]["ours"] and "rejected" not in ref:
                out["full"]["ratio"] = out["full"]["ours"]["gbases_s"] / ref["gbases_s"]
    return out


def postprocess_leg(args, k, scale=0.05):
    """The post-processing row: `bin/Tree` counts a 5% sample of the
    workload to ./tmp/, then this build's `bin/PostProcess` (device merge)
    and the reference's own `PostProcess::merge_all` (oracle/_ref, built from
    its sources; 4 threads as its own main uses) each turn that tmp/ into
    final_root.bin, final_low.bin and freq_hist.txt; wall clock of each
    process, and whether their files are byte-identical."""
    import filecmp
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    tree = os.path.join(ROOT, "kmertreecounter_b200", "bin", "Tree")
    post = os.path.join(ROOT, "kmertreecounter_b200", "bin", "PostProcess")
    nw = 1 if k <= 32 else (2 if k <= 64 else 4)
    out = {"input": f"bin/Tree's tmp/ of the workload at scale {scale}", "method": "wall clock of each process"}
    with tempfile.TemporaryDirectory() as wd:
        path, data, _, _, info = cpu_sample(args.workload, scale, wd)
        r = subprocess.run([tree, path, str(k), "16", "16"], cwd=wd, capture_output=True, text=True,
                           env=dict(os.environ, KC_STAGE0="0"))
        if r.returncode:
            return {"error": f"Tree exit {r.returncode}"}
        tmp = os.path.join(wd, "tmp") + "/"
        out["low_bytes"] = os.path.getsize(tmp + "low.bin")
        dirs = {}
        for name, cmd in (("ours", [post, tmp, None, str(k)]), ("reference", [oracle.REF_POST, tmp, None, str(nw)])):
            if name == "reference" and not os.path.exists(oracle.REF_POST):
                continue
            d = os.path.join(wd, name) + "/"
            os.makedirs(d)
            cmd[2] = d
            t = time.perf_counter()
            r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
            dt = time.perf_counter() - t
            out[name] = {"seconds": dt} if r.returncode == 0 else {"error": f"exit {r.returncode}"}
            dirs[name] = d
        if "seconds" in out.get("ours", {}) and "seconds" in out.get("reference", {}):
            files = ("final_root.bin", "final_low.bin", "freq_hist.txt")
            out["identical"] = all(
                os.path.exists(dirs["ours"] + f) == os.path.exists(dirs["reference"] + f) and
                (not os.path.exists(dirs["ours"] + f) or filecmp.cmp(dirs["ours"] + f, dirs["reference"] + f,
                                                                     shallow=False)) for f in files)
            out["ratio"] = out["reference"]["seconds"] / out["ours"]["seconds"]
    return out


# --------------------------------------------------------------- our arm

def run_ours(args):
    import torch
    import kmertreecounter_b200 as kc
    from kmertreecounter_b200 import synth

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    # roofline denominators of the atomic and link terms, measured on this
    # GPU before the workload is resident (random u32 atomics on a 4 GiB
    # footprint, pinned H2D); the HBM term uses the pool's measured copy
    dev_peaks = None
    if not args.no_peaks:
        try:
            dev_peaks = kc.measure_peaks(local, 4 << 30)
        except kc.KcError as e:  # the pipeline roofline is then left out of the line
            print(f"bench: peak measurement failed: {e}", file=sys.stderr)

    p, k, buckets, bases = make_workload(args.workload, args.scale)
    g = synth.genome(p)
    n = synth.fastq_bytes(p)
    host_ptr = kc.host_alloc(n)  # pinned FASTQ for the e2e leg
    synth.fastq(p, g, out=host_ptr)
    del g
    host = np.ctypeslib.as_array((ctypes.c_uint8 * n).from_address(host_ptr))
    dev = torch.empty(n, dtype=torch.uint8, device="cuda")
    dev.copy_(torch.from_numpy(host))
    torch.cuda.synchronize()

    cfg = kc.default_config(k=k, n_buckets=buckets, device=local)
    if args.workload in DEVICE_BATCH:
        cfg.device_batch_bytes = DEVICE_BATCH[args.workload]
    counter = kc.Counter(cfg)
    stream = torch.cuda.ExternalStream(counter.stream)

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    # warm-up (also sizes every buffer)
    for _ in range(max(args.warmup, 0)):
        counter.count_device(dev.data_ptr(), n)

    # --- device-resident timed region
    counter.set_profiling(True)
    stage_ms, stage_launch = {}, {}
    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    torch.cuda.synchronize()
    t_clk0 = time.perf_counter()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        st = counter.count_device(dev.data_ptr(), n)
        for name, (ms, ln) in counter.stage_times().items():
            stage_ms[name] = stage_ms.get(name, 0.0) + ms
            stage_launch[name] = stage_launch.get(name, 0) + ln
    e1.record(stream)
    torch.cuda.synchronize()
    clocks.mark(t_clk0, time.perf_counter())
    barrier()
    clk = clocks.stop()
    total_ms = e0.elapsed_time(e1)
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([total_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    ms_step = total_ms / args.steps
    _, distinct = counter.histogram(1, 2)  # exact distinct keys (outside the timed region)
    # the merged count histogram of the device-held result (histogram_tool
    # precise's output, counts 1..10000), timed on its own after the steps
    t_h = time.perf_counter()
    merged = counter.histogram(1, 10000)
    histogram_ms = (time.perf_counter() - t_h) * 1e3
    stats = st.as_dict()
    stats.pop("root_counts", None)
    gpu_launches = int(sum(stage_launch.values()))

    # --- end to end through the C ABI with host buffers: pinned FASTQ in,
    # packed low.bin bytes and root records delivered to host memory by the
    # streaming call (kc_count_host_stream), copies overlapped with counting
    rec = kc.record_bytes(k)
    e2e_ms = []
    got = {"low": 0, "root": 0}

    def sink(kind, root, addr, nbytes):
        got["low" if kind == kc.KC_SINK_LOW else "root"] += nbytes
        return 0

    counter.set_profiling(False)
    for i in range(max(1, args.e2e_steps) + 1):
        torch.cuda.synchronize()
        barrier()
        got["low"] = got["root"] = 0
        t_a = time.perf_counter()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        counter.count_host_stream(host_ptr, n, sink)
        b.record(stream)
        torch.cuda.synchronize()
        wall = (time.perf_counter() - t_a) * 1e3
        if i > 0:  # first call is a warm-up of the host path
            e2e_ms.append(max(a.elapsed_time(b), wall))
    lb, nr = got["low"], got["root"] // rec
    e2e_step = statistics.median(e2e_ms)
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([e2e_step], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_step = float(t.item())

    # --- rooflines: every stage's algorithmic bytes per step over its time
    # (stage_rooflines), the dominant stage as the line's `roofline`, and the
    # workload's fixed whole-step roofline (pipeline_roofline)
    from measured import peaks
    pk = peaks()
    K, L = stats["total_kmers"], stats["low_records"]
    count_ms = stage_ms.get("count", 0.0) / args.steps
    per_stage = stage_rooflines({s_: v / args.steps for s_, v in stage_ms.items()}, stats, n, k, pk["hbm_gbs"],
                                kc.packed_bytes(k), kc.record_bytes(k),
                                {s_: profile_traffic(args, s_)[0] for s_ in STAGE_KERNELS})
    dominant = max(per_stage, key=lambda s_: per_stage[s_]["ms"]) if per_stage else None
    roof = pipeline_roofline(dev_peaks, pk, n, K, L, stats["root_records"], kc.packed_bytes(k), kc.record_bytes(k),
                             ms_step, count_ms)
    traffic, traffic_note = profile_traffic(args, dominant)

    line = {
        "metric": "FASTQ Gbases/s to exact k-mer counts on 1 B200",
        "value": bases * world / (ms_step / 1e3) / 1e9,
        "unit": "Gbases/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u64",
        "data": "synthetic (seeded generator, reference benchmark shape)",
        "config": workload_config(args, world, n, bases, p.n_reads),
        "distinct_kmers": distinct,
        "distinct_kmers_per_s": distinct * world / (ms_step / 1e3),
        "histogram_ms": histogram_ms,
        "stats": stats,
        "stages_ms_per_step": {s: v / args.steps for s, v in stage_ms.items()},
        "gpu_launches": gpu_launches,
        "e2e": {"value": bases * world / (e2e_step / 1e3) / 1e9, "unit": "Gbases/s", "ms_per_step": e2e_step,
                "h2d_bytes_per_step": n, "d2h_bytes_per_step": lb + nr * rec,
                "roofline_frac": (roof["pipeline"]["t_roof_e2e_ms"] / e2e_step) if roof.get("pipeline") else None},
        "roofline": dict({"bound": "hbm", "kernel": per_stage[dominant]["kernels"], "stage": dominant,
                          "achieved": per_stage[dominant]["gbs"], "peak": pk["hbm_gbs"], "unit": "GB/s",
                          "frac": per_stage[dominant]["frac"], "peak_source": pk["source"],
                          "alg_bytes_per_launch": per_stage[dominant]["alg_bytes"],
                          "alg_bytes_rule": per_stage[dominant]["rule"],
                          "per": "step (all launches of the stage in one count)",
                          "traffic": traffic, "traffic_source": traffic_note}) if dominant else None,
        "stage_rooflines": per_stage,
        "count_atomic_ceiling": roof.get("count_routed_atomic"),
        "pipeline_roofline": roof.get("pipeline"),
        "clocks": clk,
        "sizing": None,
    }
    counter.close()  # its structures go before the sizing comparison builds two more contexts
    if not args.no_sizing:
        try:
            line["sizing"] = compare_sizing(args, kc, torch, dev, n, k, buckets)
        except kc.KcError as e:
            line["sizing"] = {"error": str(e)}
    if rank == 0 and rec == 16 and not args.no_sort_record:
        try:
            line["sorted_roots"] = sort_record(kc, torch, dev, n, k, merged, pk["hbm_gbs"])
        except Exception as e:  # a record beside the line, never the line itself
            line["sorted_roots"] = {"error": f"{type(e).__name__}: {str(e)[:200]}"}
    del dev
    ftf_dir, full_path = None, None
    if rank == 0 and not args.no_file_to_file and not args.no_cpu_baseline:
        import shutil
        ftf_dir = tempfile.TemporaryDirectory()
        if shutil.disk_usage(ftf_dir.name).free > 3 * n:  # the FASTQ plus the outputs of one run
            full_path = os.path.join(ftf_dir.name, "full.fastq")
            host.tofile(full_path)
    kc.host_free(host_ptr)

    if rank == 0 and not args.no_large_long and args.workload == "genome_scale" and args.scale == 1.0:
        try:
            line["large_long"] = large_long_record(args, kc, torch, dev_peaks, pk)
        except kc.KcError as e:
            line["large_long"] = {"error": str(e)}
    if rank == 0 and not args.no_batched and args.workload == "genome_scale":
        line["batched_sets"] = compare_batched(args, kc, torch)
    if rank == 0 and not args.no_cpu_baseline:
        with tempfile.TemporaryDirectory() as wd:
            path, data, kk, sbases, info = cpu_sample(args.workload, args.sample_scale, wd)
            res, kind, cores = time_reference(path, data, kk, sbases, 2, wd)
            best = max(r[0] for r in res)
            line["cpu_baseline"] = {"value": best, "unit": "Gbases/s", "cores": cores, "kind": kind,
                                    "sample": f"{args.workload} at scale {args.sample_scale}: {info['reads']} reads, "
                                              f"{data.size} FASTQ bytes, best of {len(res)} runs",
                                    "host": host_facts()}
            if not args.no_file_to_file:
                line["file_to_file"] = file_to_file(args, path, sbases, kk, best if kind == "reference" else None,
                                                    full_path, bases, stats["total_kmers"])
                try:
                    line["postprocess"] = postprocess_leg(args, kk)
                except (OSError, subprocess.SubprocessError, ValueError) as e:
                    line["postprocess"] = {"error": str(e)[:200]}
    if ftf_dir is not None:
        ftf_dir.cleanup()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_sharded(args):
    """One input over all ranks (strong scaling): every rank generates the
    same seeded FASTQ, takes its slice of whole 4-line records
    (shard.record_starts), and a step is route (kc_route_device on the slice)
    -> one NCCL all-to-all of the routed keys (sent from the context's own
    buffer) -> count of the owned root prefixes (kc_count_keys_device).
    Timed with CUDA events around whole steps, max over ranks; value = the
    input's bases / that time.  e2e adds, per step, the slice's host->device
    copy from pinned memory and the device->host copy of the rank's outputs."""
    import datetime
    import torch
    import torch.distributed as dist
    import kmertreecounter_b200 as kc
    from kmertreecounter_b200 import shard, synth

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        p, k, buckets, bases = make_workload(args.workload, args.scale)
        n = synth.fastq_bytes(p)
        host_ptr = kc.host_alloc(n)
        synth.fastq(p, out=host_ptr)
        host = np.ctypeslib.as_array((ctypes.c_uint8 * n).from_address(host_ptr))
        cuts = shard.record_starts(host, world)
        lo, hi = cuts[rank], cuts[rank + 1]
        d_slice = torch.empty(max(hi - lo, 16), dtype=torch.uint8, device=device)[:hi - lo]
        d_slice.copy_(torch.from_numpy(host[lo:hi]))
        cfg = kc.default_config(k=k, n_buckets=buckets, device=local)
        if args.workload in DEVICE_BATCH:
            cfg.device_batch_bytes = DEVICE_BATCH[args.workload]
        counter = kc.Counter(cfg)

        launches = [0, 0]  # this rank's kernel launches: route, count (the library's counters)

        def step(e2e=False):
            if e2e:
                d_slice.copy_(torch.from_numpy(host[lo:hi]), non_blocking=True)
            route, count, nw = shard.gpu_stages(counter, None, device, d_slice=d_slice)

            def route_counted():
                r = route()
                launches[0] = int(sum(v[1] for v in counter.stage_times().values()))
                return r

            st, ranges, _ = shard.exchange_and_count(route_counted, count, nw, device, dist)
            launches[1] = int(sum(v[1] for v in counter.stage_times().values()))
            out = 0
            if e2e:
                lb, nr, _ = counter.sizes()
                out = lb + nr * kc.record_bytes(k)
                low_h = torch.empty(max(lb, 1), dtype=torch.uint8, pin_memory=True)
                counter.copy_low_into(low_h.data_ptr(), lb)
                roots_h = torch.empty(max(nr * kc.record_bytes(k), 1), dtype=torch.uint8, pin_memory=True)
                counter.copy_roots_into(roots_h.data_ptr(), nr * kc.record_bytes(k))
            return st, out

        def timed(steps, e2e=False):
            dist.barrier()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            out = 0
            for _ in range(steps):
                st, out = step(e2e)
            torch.cuda.synchronize()
            e1.record()
            torch.cuda.synchronize()
            t = torch.tensor([e0.elapsed_time(e1) / steps], device=device)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            return float(t.item()), st, out

        for _ in range(max(args.warmup, 0)):
            step()
        clocks = ClockSampler(local)
        clocks.start()
        t_clk0 = time.perf_counter()
        ms_step, st, _ = timed(args.steps)
        clocks.mark(t_clk0, time.perf_counter())
        clk = clocks.stop()
        e2e_ms, _, out_bytes = timed(max(1, args.e2e_steps), e2e=True)
        totals = torch.tensor([st.total_kmers, st.low_records, st.root_records, out_bytes], dtype=torch.int64,
                              device=device)
        dist.all_reduce(totals)
        K, L, R, out_all = (int(x) for x in totals.tolist())
        counter.close()
        kc.host_free(host_ptr)
        line = {
            "metric": "FASTQ Gbases/s to exact k-mer counts on 1 B200",
            "value": bases / (ms_step / 1e3) / 1e9, "unit": "Gbases/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "u64", "data": "synthetic (seeded generator, reference benchmark shape)",
            "config": workload_config(args, world, n, bases, p.n_reads),
            "stats": {"total_kmers": K, "low_records": L, "root_records": R},
            "gpu_launches": (launches[0] + launches[1]) * args.steps,
            "gpu_launches_note": "rank 0's kernel launches in the timed steps (route + count, all-to-all excluded)",
            "e2e": {"value": bases / (e2e_ms / 1e3) / 1e9, "unit": "Gbases/s", "ms_per_step": e2e_ms,
                    "h2d_bytes_per_step": n, "d2h_bytes_per_step": out_all},
            "clocks": clk,
        }
        dist.barrier()
        if rank == 0:
            print(json.dumps(line), flush=True)
    finally:
        dist.destroy_process_group()


# --------------------------------------------------------------- reference arm

def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    with tempfile.TemporaryDirectory() as wd:
        path, data, k, bases, info = cpu_sample(args.workload, args.sample_scale, wd)
        res, kind, cores = time_reference(path, data, k, bases, max(args.warmup, 0) + args.steps, wd)
        timed = res[max(args.warmup, 0):] or res
        secs = sum(r[1] for r in timed)
        value = bases * len(timed) / secs / 1e9
        line = {
            "metric": "FASTQ Gbases/s to exact k-mer counts on 1 B200",
            "impl": "reference",
            "value": value,
            "unit": "Gbases/s",
            "n_gpus": world,
            "steps": len(timed),
            "warmup": args.warmup,
            "ms_per_step": secs / len(timed) * 1e3,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "u64",
            "data": "synthetic (seeded generator, reference benchmark shape)",
            "config": workload_config(args, world, info["full"]["fastq_bytes"], info["full"]["bases"],
                                      info["full"]["reads"]),
            "cpu_baseline": {"value": value, "unit": "Gbases/s", "cores": cores, "kind": kind,
                             "sample": f"each step one run of the reference's Tree ({cores} threads) on a bounded "
                                       f"sample of this workload: the same generator at scale {args.sample_scale} "
                                       f"(genome {info['genome_len']} bp, {info['reads']} reads, {data.size} FASTQ "
                                       f"bytes, same coverage and error model); runs whose k-mer total differs "
                                       f"from the oracle's are rejected and repeated",
                             "host": host_facts()},
            "e2e": {"value": value, "unit": "Gbases/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.write_sample:
        write_sample(args.workload, args.sample_scale, args.write_sample)
        return
    if args.impl == "reference":
        run_reference(args)
    elif sharded(args, dist_env()[1]):
        run_sharded(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
