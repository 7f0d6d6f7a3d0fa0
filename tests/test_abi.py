"""The C-ABI library loads, exports every symbol include/*.h declares, and
validates arguments before touching a device.  No compute calls here."""
import ctypes as C
import os
import re
import subprocess

import pytest

from conftest import ROOT, has_cuda
import kmertreecounter_b200 as kc
from kmertreecounter_b200 import _native, synth

HEADERS = {"kmer_count.h": _native.LIB_PATH, "kmer_synth.h": _native.SYNTH_PATH,
           "kmer_sizing.h": _native.LIB_PATH, "kmer_peaks.h": _native.LIB_PATH}


def declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(kc_\w+)\s*\(", text)))


@pytest.mark.parametrize("header", sorted(HEADERS))
def test_every_declared_symbol_is_exported(header):
    names = declared(header)
    assert names, header
    lib = C.CDLL(HEADERS[header])
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    if header == "kmer_count.h":
        assert set(names) == set(kc.ABI_SYMBOLS)


def test_sizes():
    assert [kc.packed_bytes(k) for k in (21, 31, 32, 33, 63, 64)] == [6, 8, 8, 9, 16, 16]
    assert [kc.record_bytes(k) for k in (21, 32, 33, 64)] == [16, 16, 24, 24]
    assert kc.record_dtype(31).itemsize == 16 and kc.record_dtype(63).itemsize == 24


@pytest.mark.parametrize("field,value", [("k", 0), ("k", 129), ("canonical", 0), ("n_buckets", 100),
                                         ("table_load", 0.99), ("batch_bytes", 1000),
                                         ("device_batch_bytes", 4096)])
def test_invalid_config_rejected_before_device(field, value):
    with pytest.raises(kc.KcError) as e:
        kc.Counter(kc.default_config(**{field: value}))
    assert e.value.code == kc.KC_ERR_INVALID


def test_struct_layout_matches_header(tmp_path):
    """Every ctypes mirror of a header struct has the C compiler's size and
    field offsets."""
    structs = {"kc_config": _native.KcConfig, "kc_stats": _native.KcStats,
               "kc_set_desc": _native.KcSetDesc, "kc_set_result": _native.KcSetResult, "kc_peaks": _native.KcPeaks,
               "kc_stage0": _native.KcStage0, "kc_post_stats": _native.KcPostStats}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "kmer_count.h"', '#include "kmer_peaks.h"',
             "int main(void) {"]
    for cname, py in structs.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for f in py._fields_:
            lines.append(f'printf("{cname} {f[0]} %zu\\n", offsetof({cname}, {f[0]}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.check_call(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), "-o", str(exe), str(src)])
    got = {}
    for line in subprocess.check_output([str(exe)], text=True).splitlines():
        s, f, v = line.split()
        got[(s, f)] = int(v)
    for cname, py in structs.items():
        assert got[(cname, "size")] == C.sizeof(py), cname
        for f in py._fields_:
            assert got[(cname, f[0])] == getattr(py, f[0]).offset, (cname, f[0])


@pytest.mark.parametrize("footprint", [0, 128 << 20, (4 << 30) + 4096, 64 << 30])
def test_peaks_footprint_rejected_before_device(footprint):
    with pytest.raises(kc.KcError) as e:
        kc.measure_peaks(0, footprint)
    assert e.value.code == kc.KC_ERR_INVALID


def test_min_max_order_rejected():
    with pytest.raises(kc.KcError) as e:
        kc.Counter(kc.default_config(min_count=5, max_count=2))
    assert e.value.code == kc.KC_ERR_INVALID


@pytest.mark.skipif(has_cuda(), reason="checks the no-device error path")
def test_no_device_is_a_loud_error():
    with pytest.raises(kc.KcError) as e:
        kc.Counter(kc.default_config())
    assert e.value.code == kc.KC_ERR_DEVICE


TREE = os.path.join(ROOT, "kmertreecounter_b200", "bin", "Tree")


@pytest.mark.parametrize("args,code", [([], 1), (["x.fq", "31", "8"], 1), (["x.fq", "31", "4", "4"], 255),
                                       (["x.fq", "31", "8", "4", "1"], 1), (["x.fq", "31", "8", "4", "1024", "5", "2"], 1),
                                       (["x.fq", "abc", "8", "4"], 1), (["x.fq", "200", "8", "4"], 1)])
def test_cli_argument_errors_match_reference(args, code):
    # src/main.cpp:316-374 and :579-595: usage errors exit 1, n_thread < 6 exits -1 (255)
    p = subprocess.run([TREE, *args], capture_output=True, text=True)
    assert p.returncode == code, p.stderr


def test_synth_is_deterministic():
    p = synth.plain_small(seed=3, scale=0.01)
    a, b = synth.fastq(p), synth.fastq(p)
    assert a.size == synth.fastq_bytes(p) and (a == b).all()
    p.threads = 1
    assert (synth.fastq(p) == a).all()
