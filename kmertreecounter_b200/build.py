"""Build recipe for the native parts of kmertreecounter_b200.

Produces, in-tree:
  kmertreecounter_b200/libkmertree_b200.so   sm_100a kernels + C ABI (include/kmer_count.h)
  kmertreecounter_b200/libkc_synth.so        seeded workload generator (include/kmer_synth.h)
  kmertreecounter_b200/bin/Tree              reference-compatible command line
  kmertreecounter_b200/bin/PostProcess       tool/PostProcess.h's merge on the device
nvcc cross-compiles sm_100a without a GPU.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

LIB = os.path.join(HERE, "libkmertree_b200.so")
SYNTH = os.path.join(HERE, "libkc_synth.so")
TREE = os.path.join(HERE, "bin", "Tree")
POST = os.path.join(HERE, "bin", "PostProcess")


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _deps(*names):
    out = [os.path.join(CSRC, n) for n in names]
    out += [os.path.join(ROOT, "include", h) for h in ("kmer_count.h", "kmer_synth.h", "kmer_sizing.h", "kmer_peaks.h")]
    return out


def build(force=False, verbose_ptxas=False):
    os.makedirs(os.path.join(HERE, "bin"), exist_ok=True)
    srcs = ["kc_engine.cu", "kc_sort.cu", "kc_post.cu", "kc_io.cpp", "kc_stage0.cpp", "kc_noalloc.cu", "kc_mlp.cu",
            "kc_peaks.cu"]
    hdrs = ["kc_kernels.cuh", "kc_scan.cuh", "kc_window.cuh", "kc_internal.h"]
    if force or _stale(LIB, _deps(*srcs, *hdrs)):
        cmd = [NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++20", "-Xcompiler", "-fPIC", "-shared",
               "--expt-relaxed-constexpr", "-o", LIB]
        if verbose_ptxas:
            cmd += ["-Xptxas", "-v"]
        cmd += [os.path.join(CSRC, s) for s in srcs] + ["-lz"]
        _run(cmd)
    if force or _stale(SYNTH, _deps("synth.cpp")):
        _run(["g++", "-O3", "-std=c++20", "-fPIC", "-shared", "-o", SYNTH, os.path.join(CSRC, "synth.cpp"),
              "-lpthread"])
    if force or _stale(TREE, _deps("tree_main.cpp") + [LIB]):
        _run(["g++", "-O2", "-std=c++20", "-pthread", "-o", TREE, os.path.join(CSRC, "tree_main.cpp"), "-L" + HERE,
              "-lkmertree_b200", "-Wl,-rpath,$ORIGIN/.."])
    if force or _stale(POST, _deps("post_main.cpp") + [LIB]):
        _run(["g++", "-O2", "-std=c++20", "-o", POST, os.path.join(CSRC, "post_main.cpp"), "-L" + HERE,
              "-lkmertree_b200", "-Wl,-rpath,$ORIGIN/.."])
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose_ptxas="-v" in sys.argv)
