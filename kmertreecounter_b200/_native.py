"""ctypes binding of libkmertree_b200.so (C ABI in include/kmer_count.h).

The shared library is the product; this module only marshals arguments.  It
raises on import when the library is missing -- there is no CPU fallback.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libkmertree_b200.so")
SYNTH_PATH = os.path.join(HERE, "libkc_synth.so")

KC_OK = 0
KC_ERR_INVALID = -1
KC_ERR_IO = -2
KC_ERR_OVERFLOW = -3
KC_ERR_DEVICE = -4
KC_ERR_NOMEM = -5
KC_ERR_STATE = -6

KC_SIZING_SAMPLED = 0
KC_SIZING_LEARNED = 1

# Every extern "C" symbol include/kmer_count.h declares.
ABI_SYMBOLS = (
    "kc_config_default", "kc_last_error", "kc_packed_bytes", "kc_record_bytes", "kc_count_fastq",
    "kc_create", "kc_destroy", "kc_count_host", "kc_count_device", "kc_result_sizes", "kc_copy_low",
    "kc_copy_roots", "kc_write_outputs", "kc_device_results", "kc_host_alloc", "kc_host_free", "kc_stream",
    "kc_set_profiling", "kc_stage_times", "kc_stage_name", "kc_count_device_noalloc", "kc_count_host_stream",
    "kc_histogram", "kc_count_sets", "kc_route_device", "kc_copy_routed", "kc_count_keys_device",
    "kc_stage0_rule", "kc_stage0_file", "kc_post_process", "kc_post_process_dir", "kc_routed_keys",
    "kc_sets_graph_instantiations",
)
KC_SINK_LOW = 0
KC_SINK_ROOT = 1
SINK_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int, C.c_uint32, C.c_void_p, C.c_uint64)
NOALLOC_SCRATCH_BYTES = 64 << 20
NOALLOC_MAX_FASTQ_BYTES = 1 << 20
STAGE_COUNT = 11


class KcConfig(C.Structure):
    _fields_ = [
        ("k", C.c_uint32), ("canonical", C.c_uint32), ("min_count", C.c_uint32), ("max_count", C.c_uint32),
        ("n_buckets", C.c_uint32), ("sizing", C.c_uint32), ("device", C.c_int32), ("sort_output", C.c_uint32),
        ("chunk_bytes", C.c_uint64), ("batch_bytes", C.c_uint64), ("bloom_bits", C.c_double),
        ("table_load", C.c_double), ("repeat_ratio", C.c_double), ("device_batch_bytes", C.c_uint64),
        ("priority", C.c_int32),
    ]


class KcStats(C.Structure):
    _fields_ = [
        ("input_bytes", C.c_uint64), ("total_kmers", C.c_uint64), ("low_records", C.c_uint64),
        ("root_records", C.c_uint64), ("table_keys", C.c_uint64), ("rehashes", C.c_uint64),
        ("batches", C.c_uint64), ("root_counts", C.c_uint64 * 256), ("device_ms", C.c_double),
        ("wall_ms", C.c_double), ("table_slots", C.c_uint64), ("filter_words", C.c_uint64),
        ("overflow_keys", C.c_uint64), ("reroutes", C.c_uint64),
        ("max_bucket_filter_words", C.c_uint64), ("max_bucket_table_slots", C.c_uint64),
    ]

    def as_dict(self):
        d = {f: getattr(self, f) for f, _ in self._fields_ if f != "root_counts"}
        d["root_counts"] = list(self.root_counts)
        return d


class KcSetDesc(C.Structure):
    _fields_ = [("offset", C.c_uint64), ("bytes", C.c_uint64), ("k", C.c_uint32), ("reserved", C.c_uint32)]


class KcSetResult(C.Structure):
    _fields_ = [("total_kmers", C.c_uint64), ("low_records", C.c_uint64), ("low_offset", C.c_uint64),
                ("low_bytes", C.c_uint64), ("root_records", C.c_uint64), ("root_offset", C.c_uint64),
                ("root_counts", C.c_uint64 * 256)]


class KcPeaks(C.Structure):
    _fields_ = [("hbm_copy_gbs", C.c_double), ("red_add_gops", C.c_double), ("or_return_gops", C.c_double),
                ("h2d_gbs", C.c_double), ("footprint_bytes", C.c_uint64), ("ops", C.c_uint64),
                ("l2_red_add_gops", C.c_double), ("l2_or_return_gops", C.c_double),
                ("l2_footprint_bytes", C.c_uint64)]


class KcStage0(C.Structure):
    _fields_ = [("estimated_file_size", C.c_uint64), ("sample_bytes", C.c_uint64), ("sampled_kmers", C.c_uint64),
                ("average_prefix_count", C.c_uint64), ("max_bloom_filter_capacity", C.c_uint64),
                ("classifier_num", C.c_uint32), ("reserved", C.c_uint32), ("prefix_count", C.c_uint64 * 256),
                ("bloom_filter_capacity", C.c_uint64 * 256), ("prefix_owner", C.c_uint32 * 256),
                ("load_order", C.c_uint32 * 256), ("classifier_load", C.c_uint64 * 256)]

    def loads_in_print_order(self):
        """(classifier, load) in the order the reference prints its
        "Classifier i total prefix count: c" lines."""
        return [(int(self.load_order[i]), int(self.classifier_load[self.load_order[i]]))
                for i in range(self.classifier_num)]


class KcPostStats(C.Structure):
    _fields_ = [("root_records", C.c_uint64), ("low_in", C.c_uint64), ("low_in_roots", C.c_uint64),
                ("final_low", C.c_uint64), ("hist_lines", C.c_uint64)]


class KcError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"kc error {code}: {msg}")
        self.code = code


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: run `python -m kmertreecounter_b200.build` "
                          "(the CUDA extension is required; there is no CPU fallback)")
    lib = C.CDLL(LIB_PATH)
    vp, u64, u32, i32 = C.c_void_p, C.c_uint64, C.c_uint32, C.c_int
    cfgp, stp = C.POINTER(KcConfig), C.POINTER(KcStats)
    sig = {
        "kc_config_default": (None, [cfgp]),
        "kc_last_error": (C.c_char_p, []),
        "kc_packed_bytes": (u64, [u32]),
        "kc_record_bytes": (u64, [u32]),
        "kc_count_fastq": (i32, [cfgp, C.c_char_p, C.c_char_p, stp]),
        "kc_create": (i32, [cfgp, C.POINTER(vp)]),
        "kc_destroy": (None, [vp]),
        "kc_count_host": (i32, [vp, vp, u64, stp]),
        "kc_count_device": (i32, [vp, vp, u64, stp]),
        "kc_result_sizes": (i32, [vp, C.POINTER(u64), C.POINTER(u64), C.POINTER(u64)]),
        "kc_copy_low": (i32, [vp, vp, u64]),
        "kc_copy_roots": (i32, [vp, vp, u64]),
        "kc_write_outputs": (i32, [vp, C.c_char_p]),
        "kc_device_results": (i32, [vp, C.POINTER(vp), C.POINTER(u64), C.POINTER(vp), C.POINTER(u64)]),
        "kc_host_alloc": (vp, [u64]),
        "kc_host_free": (None, [vp]),
        "kc_stream": (vp, [vp]),
        "kc_set_profiling": (i32, [vp, i32]),
        "kc_stage_times": (i32, [vp, C.POINTER(C.c_double), C.POINTER(u64), i32]),
        "kc_stage_name": (C.c_char_p, [i32]),
        "kc_count_device_noalloc": (i32, [cfgp, vp, u64, vp, u64, vp, u64, vp, stp]),
        "kc_count_host_stream": (i32, [vp, vp, u64, SINK_FN, vp, stp]),
        "kc_histogram": (i32, [vp, u32, u32, C.POINTER(u64), C.POINTER(u64)]),
        "kc_count_sets": (i32, [vp, vp, C.POINTER(KcSetDesc), u32, C.POINTER(KcSetResult), stp]),
        "kc_sets_graph_instantiations": (u64, [vp]),
        "kc_route_device": (i32, [vp, vp, u64, C.POINTER(u64)]),
        "kc_copy_routed": (i32, [vp, vp, u64]),
        "kc_routed_keys": (i32, [vp, C.POINTER(vp), C.POINTER(u64)]),
        "kc_count_keys_device": (i32, [vp, vp, u64, C.POINTER(u64), stp]),
        "kc_measure_peaks": (i32, [i32, u64, C.POINTER(KcPeaks)]),
        "kc_stage0_rule": (i32, [C.POINTER(u64), u64, u32, C.POINTER(KcStage0)]),
        "kc_stage0_file": (i32, [cfgp, C.c_char_p, u32, C.POINTER(KcStage0)]),
        "kc_post_process": (i32, [vp, C.c_char_p, C.POINTER(KcPostStats)]),
        "kc_post_process_dir": (i32, [cfgp, C.c_char_p, C.c_char_p, C.POINTER(KcPostStats)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def last_error():
    m = lib.kc_last_error()
    return m.decode() if m else ""


def check(rc):
    if rc != KC_OK:
        raise KcError(rc, last_error())
    return rc


def default_config(**kw):
    cfg = KcConfig()
    lib.kc_config_default(C.byref(cfg))
    for k, v in kw.items():
        if not hasattr(cfg, k):
            raise AttributeError(f"kc_config has no field {k}")
        setattr(cfg, k, v)
    return cfg


def packed_bytes(k):
    return int(lib.kc_packed_bytes(k))


def record_bytes(k):
    return int(lib.kc_record_bytes(k))


def record_dtype(k):
    """numpy dtype of ExportRecord<N> (src/definition.h:159-163)."""
    nw = 1 if k <= 32 else (2 if k <= 64 else 4)
    return np.dtype([("key", "<u8", (nw,)), ("count", "<u4"), ("pad", "<u4")])


class Counter:
    """One counting context (a CUDA stream and its device buffers)."""

    def __init__(self, cfg=None, **kw):
        self.cfg = cfg if cfg is not None else default_config(**kw)
        self._ctx = C.c_void_p()
        check(lib.kc_create(C.byref(self.cfg), C.byref(self._ctx)))
        self.stats = KcStats()

    def close(self):
        if self._ctx:
            lib.kc_destroy(self._ctx)
            self._ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def stream(self):
        return lib.kc_stream(self._ctx)

    def count_host(self, data):
        """Count FASTQ bytes in host memory (bytes, bytearray or uint8 ndarray)."""
        if isinstance(data, (bytes, bytearray)):
            buf = np.frombuffer(data, dtype=np.uint8)
        else:
            buf = np.ascontiguousarray(data, dtype=np.uint8)
        ptr = buf.ctypes.data if buf.size else None
        check(lib.kc_count_host(self._ctx, ptr, buf.size, C.byref(self.stats)))
        return self.stats

    def count_host_ptr(self, ptr, n):
        check(lib.kc_count_host(self._ctx, C.c_void_p(ptr), n, C.byref(self.stats)))
        return self.stats

    def count_host_stream(self, ptr, n, sink):
        """Streamed count of host bytes at address `ptr`; sink(kind, root,
        data_address, nbytes) -> int is called as results reach host memory."""
        cb = SINK_FN(lambda u, kind, root, data, nbytes: sink(kind, root, data, nbytes))
        check(lib.kc_count_host_stream(self._ctx, C.c_void_p(ptr), n, cb, None, C.byref(self.stats)))
        return self.stats

    def count_device(self, dptr, n):
        """Count FASTQ bytes already in device memory (an integer device pointer)."""
        check(lib.kc_count_device(self._ctx, C.c_void_p(dptr), n, C.byref(self.stats)))
        return self.stats

    # -- one input over several GPUs (include/kmer_count.h, bucket owners)
    def route_device(self, dptr, n):
        """Extract and route whole FASTQ records in device memory; returns the
        keys per root prefix (uint64[256]); the keys stay in the context."""
        counts = np.zeros(256, np.uint64)
        check(lib.kc_route_device(self._ctx, C.c_void_p(dptr), n, counts.ctypes.data_as(C.POINTER(C.c_uint64))))
        return counts

    def copy_routed(self, addr, cap):
        """Copy the routed keys (prefix order) to addr (device or host)."""
        check(lib.kc_copy_routed(self._ctx, C.c_void_p(addr), cap))

    def routed_keys(self):
        """(device address, key count) of the routed keys inside the context
        (valid until the next call on this context)."""
        p, n = C.c_void_p(), C.c_uint64()
        check(lib.kc_routed_keys(self._ctx, C.byref(p), C.byref(n)))
        return p.value or 0, n.value

    def count_keys_device(self, dptr, n_keys, counts):
        """Count n_keys routed canonical keys in device memory as one input."""
        counts = np.ascontiguousarray(counts, np.uint64)
        check(lib.kc_count_keys_device(self._ctx, C.c_void_p(dptr), n_keys,
                                       counts.ctypes.data_as(C.POINTER(C.c_uint64)), C.byref(self.stats)))
        return self.stats

    def sizes(self):
        lb, nr = C.c_uint64(), C.c_uint64()
        rc = (C.c_uint64 * 256)()
        check(lib.kc_result_sizes(self._ctx, C.byref(lb), C.byref(nr), rc))
        return lb.value, nr.value, list(rc)

    def low_bytes(self):
        lb, _, _ = self.sizes()
        out = np.empty(lb, dtype=np.uint8)
        check(lib.kc_copy_low(self._ctx, out.ctypes.data if lb else None, lb))
        return out

    def root_records(self):
        _, nr, counts = self.sizes()
        dt = record_dtype(self.cfg.k)
        out = np.empty(nr, dtype=dt)
        check(lib.kc_copy_roots(self._ctx, out.ctypes.data if nr else None, nr * dt.itemsize))
        return out, counts

    def sets_graph_instantiations(self):
        """Graph instantiations kc_count_sets has made on this context."""
        return int(lib.kc_sets_graph_instantiations(self._ctx))

    def count_sets(self, dptr, sets):
        """Count many read sets in one device buffer in one pass.  `sets` is a
        list of (offset, bytes, k); returns one KcSetResult per set."""
        n = len(sets)
        desc = (KcSetDesc * n)(*[KcSetDesc(o, b, k, 0) for o, b, k in sets])
        res = (KcSetResult * n)()
        check(lib.kc_count_sets(self._ctx, C.c_void_p(dptr), desc, n, res, C.byref(self.stats)))
        return list(res)

    def histogram(self, min_freq=1, max_freq=10000):
        """(hist array for freq min..max, distinct keys) of the last result."""
        n = max_freq - min_freq + 1
        h = (C.c_uint64 * n)()
        d = C.c_uint64()
        check(lib.kc_histogram(self._ctx, min_freq, max_freq, h, C.byref(d)))
        return np.array(h, dtype=np.uint64), d.value

    def set_profiling(self, on=True):
        check(lib.kc_set_profiling(self._ctx, 1 if on else 0))

    def stage_times(self):
        """{stage: (device ms, kernel launches)} of the last count."""
        ms = (C.c_double * STAGE_COUNT)()
        ln = (C.c_uint64 * STAGE_COUNT)()
        n = lib.kc_stage_times(self._ctx, ms, ln, STAGE_COUNT)
        return {lib.kc_stage_name(i).decode(): (ms[i], ln[i]) for i in range(n)}

    def copy_low_into(self, addr, cap):
        check(lib.kc_copy_low(self._ctx, C.c_void_p(addr), cap))

    def copy_roots_into(self, addr, cap):
        check(lib.kc_copy_roots(self._ctx, C.c_void_p(addr), cap))

    def write_outputs(self, out_dir):
        check(lib.kc_write_outputs(self._ctx, str(out_dir).encode()))

    def post_process(self, out_dir):
        """final_root.bin, final_low.bin and freq_hist.txt of the last result
        (tool/PostProcess.h merge_all) into out_dir; returns KcPostStats."""
        st = KcPostStats()
        check(lib.kc_post_process(self._ctx, str(out_dir).encode(), C.byref(st)))
        return st

    def device_results(self):
        dl, lb, dr, nr = C.c_void_p(), C.c_uint64(), C.c_void_p(), C.c_uint64()
        check(lib.kc_device_results(self._ctx, C.byref(dl), C.byref(lb), C.byref(dr), C.byref(nr)))
        return dl.value, lb.value, dr.value, nr.value


def count_fastq(path, out_dir, **kw):
    """File API: count `path`, write low.bin + root_{0..255}.bin into out_dir."""
    cfg = default_config(**kw)
    st = KcStats()
    check(lib.kc_count_fastq(C.byref(cfg), str(path).encode(), str(out_dir).encode(), C.byref(st)))
    return st


def post_process_dir(temp_dir, out_dir, k, device=0):
    """tool/PostProcess.h merge_all on the low.bin and root files in temp_dir."""
    cfg = default_config(k=k, device=device)
    st = KcPostStats()
    check(lib.kc_post_process_dir(C.byref(cfg), str(temp_dir).encode(), str(out_dir).encode(), C.byref(st)))
    return st


def stage0_rule(prefix_counts, estimated_file_size, n_thread=8):
    """The reference's Stage-0 rules on per-prefix sampled counts (KcStage0)."""
    counts = np.ascontiguousarray(prefix_counts, np.uint64)
    assert counts.size == 256
    out = KcStage0()
    check(lib.kc_stage0_rule(counts.ctypes.data_as(C.POINTER(C.c_uint64)), estimated_file_size, n_thread,
                             C.byref(out)))
    return out


def stage0_file(path, k=31, n_thread=8, device=0):
    """The reference's Stage-0 sample of the FASTQ at `path`, its per-prefix
    k-mer counts (counted on `device`) and rules (KcStage0)."""
    cfg = default_config(k=k, device=device)
    out = KcStage0()
    check(lib.kc_stage0_file(C.byref(cfg), str(path).encode(), n_thread, C.byref(out)))
    return out


def measure_peaks(device=0, footprint_bytes=4 << 30):
    """Roofline denominators measured on `device` (include/kmer_peaks.h):
    HBM copy GB/s, random u32 atomic rates (10^9 ops/s) on a footprint far
    above L2, and the pinned host->device link."""
    out = KcPeaks()
    check(lib.kc_measure_peaks(int(device), int(footprint_bytes), C.byref(out)))
    return {f: getattr(out, f) for f, _ in KcPeaks._fields_}


def host_alloc(nbytes):
    p = lib.kc_host_alloc(nbytes)
    if not p:
        raise KcError(KC_ERR_NOMEM, last_error())
    return p


def host_free(p):
    lib.kc_host_free(p)
