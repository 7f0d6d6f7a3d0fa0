"""Learned sizing of the filter and repeat tables (include/kmer_sizing.h).

The reference sizes its per-prefix Bloom filters from a Stage-0 sample of up
to 256 MB (src/main.cpp:88-108) and never sizes its tree, which grows from a
memory pool.  Here the open-addressing tables must be sized up front; the
plain rule (`KC_SIZING_SAMPLED`) takes each bucket's k-mer total and a fixed
ratio of table keys per k-mer, and grows a table x4 (rehash) when it
overflows.  The learned rule predicts, per model bucket (4096 = the top six
bases of the canonical key), the ratios that the plain rule fixes:

  input  (4104) the 6-mer-prefix histogram of the first 1% of the reads,
         log1p(4096 x bucket share) / 4; k/64, read length/300, ln(FASTQ
         bytes)/25, ln(1 + prefix k-mers)/25; and three rates of the prefix
         counted exactly on the GPU: distinct keys per k-mer, table keys per
         k-mer and its square root; ln(bytes / prefix bytes)/10
  hidden 512 -> 512, ReLU, BF16 weights, FP32 accumulation
  output (8192) per bucket, ln(ratio + 1e-4)/10 + 1 of distinct keys per
         k-mer and of table keys per k-mer

so that predicted loads are ratio x the bucket's k-mer total (the prefix's
total scaled by the file size).  Every input and output is a rate, not a
size: a 100 Mbp genome looks like the small training genomes of the same
coverage, error and repeat structure.  Table keys are multiplied by a margin
calibrated on held-out training sets (a quantile of measured / predicted),
so that few tables overflow; a table that does is grown exactly as under the
plain rule, so counts stay exact either way, and kc_stats reports the
rehashes avoided or incurred.

It is trained by the library's own kernels (kc_mlp_train_step) on exact
loads that the counter itself measures (kc_bucket_loads) on seeded synthetic
genomes.
"""
import ctypes as C
import math
import os

import numpy as np

from . import _native
from ._native import check, lib

MODEL_BUCKETS = 4096
N_IN = MODEL_BUCKETS + 8
N_HID = 512
N_OUT = 2 * MODEL_BUCKETS
IN_SCALE = 25.0
RATIO_FLOOR = 1e-4
RATIO_LOG = 10.0
PREFIX_FRACTION = 0.01
MODEL_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "sizing_mlp.npz")

_f = C.POINTER(C.c_float)
_u64 = C.POINTER(C.c_uint64)
_d = C.POINTER(C.c_double)
_SIG = {
    "kc_bucket_loads": (C.c_int, [C.c_void_p, _u64, _u64, _u64]),
    "kc_set_predicted_loads": (C.c_int, [C.c_void_p, _d, _d]),
    "kc_mlp_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_uint64, C.POINTER(C.c_void_p)]),
    "kc_mlp_destroy": (None, [C.c_void_p]),
    "kc_mlp_set_layer": (C.c_int, [C.c_void_p, C.c_int, _f, _f]),
    "kc_mlp_get_layer": (C.c_int, [C.c_void_p, C.c_int, _f, _f]),
    "kc_mlp_forward": (C.c_int, [C.c_void_p, _f, C.c_int, _f]),
    "kc_mlp_gradients": (C.c_int, [C.c_void_p, _f, _f, C.c_int, C.c_int, _f, _f, _f]),
    "kc_mlp_train_step": (C.c_int, [C.c_void_p, _f, _f, C.c_int, C.c_float, _f]),
    "kc_mlp_last_error": (C.c_char_p, []),
    "kc_mlp_set_under_weight": (C.c_int, [C.c_void_p, C.c_float]),
    "kc_set_prefix_kmers": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(_native.KcSetDesc), C.c_uint32, _u64]),
    "kc_set_predicted_set_rates": (C.c_int, [C.c_void_p, C.c_uint32, _d, _d]),
    "kc_set_sizing_callback": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
}
for _n, (_r, _a) in _SIG.items():
    getattr(lib, _n).restype = _r
    getattr(lib, _n).argtypes = _a


def _fp(a):
    return a.ctypes.data_as(_f)


def _mcheck(rc):
    if rc != 0:
        raise _native.KcError(rc, (lib.kc_mlp_last_error() or b"").decode())


class MLP:
    """The sizing network on the GPU (kc_mlp_*)."""

    def __init__(self, n_in=N_IN, n_hid=N_HID, n_out=N_OUT, max_batch=64, seed=1):
        self.dims = (n_in, n_hid, n_hid, n_out)
        self.max_batch = max_batch
        self._m = C.c_void_p()
        _mcheck(lib.kc_mlp_create(n_in, n_hid, n_out, max_batch, seed, C.byref(self._m)))

    def close(self):
        if self._m:
            lib.kc_mlp_destroy(self._m)
            self._m = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_under_weight(self, w):
        _mcheck(lib.kc_mlp_set_under_weight(self._m, w))

    def set_layer(self, l, w, b):
        w = np.ascontiguousarray(w, np.float32)
        b = np.ascontiguousarray(b, np.float32)
        assert w.shape == (self.dims[l], self.dims[l + 1]) and b.shape == (self.dims[l + 1],)
        _mcheck(lib.kc_mlp_set_layer(self._m, l, _fp(w), _fp(b)))

    def get_layer(self, l):
        w = np.empty((self.dims[l], self.dims[l + 1]), np.float32)
        b = np.empty(self.dims[l + 1], np.float32)
        _mcheck(lib.kc_mlp_get_layer(self._m, l, _fp(w), _fp(b)))
        return w, b

    def forward(self, x):
        x = np.ascontiguousarray(x, np.float32)
        out = np.empty((x.shape[0], self.dims[3]), np.float32)
        for i in range(0, x.shape[0], self.max_batch):
            xb = np.ascontiguousarray(x[i:i + self.max_batch])
            yb = np.empty((xb.shape[0], self.dims[3]), np.float32)
            _mcheck(lib.kc_mlp_forward(self._m, _fp(xb), xb.shape[0], _fp(yb)))
            out[i:i + xb.shape[0]] = yb
        return out

    def gradients(self, x, t, layer):
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        gw = np.empty((self.dims[layer], self.dims[layer + 1]), np.float32)
        gb = np.empty(self.dims[layer + 1], np.float32)
        loss = C.c_float()
        _mcheck(lib.kc_mlp_gradients(self._m, _fp(x), _fp(t), x.shape[0], layer, _fp(gw), _fp(gb), C.byref(loss)))
        return gw, gb, loss.value

    def train_step(self, x, t, lr):
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        loss = C.c_float()
        _mcheck(lib.kc_mlp_train_step(self._m, _fp(x), _fp(t), x.shape[0], lr, C.byref(loss)))
        return loss.value

    margin = 1.0  # table-key multiplier applied by predict (calibrated after training)

    def save(self, path=MODEL_PATH, meta=None):
        """Weights as float16 (the forward pass runs in BF16 anyway), biases
        fp32, the calibrated margin, and a free-form report."""
        arrs = {}
        for l in range(3):
            w, b = self.get_layer(l)
            arrs[f"w{l}"] = w.astype(np.float16)
            arrs[f"b{l}"] = b
        np.savez_compressed(path, **arrs, margin=np.float64(self.margin), meta=np.array(str(meta or {})))

    @classmethod
    def load(cls, path=MODEL_PATH, max_batch=8):
        z = np.load(path, allow_pickle=False)
        if z["w0"].shape[0] != N_IN:
            raise ValueError(f"{path}: model input width {z['w0'].shape[0]} != {N_IN} (features changed; retrain)")
        m = cls(n_in=z["w0"].shape[0], n_hid=z["w0"].shape[1], n_out=z["w2"].shape[1], max_batch=max_batch)
        for l in range(3):
            m.set_layer(l, z[f"w{l}"].astype(np.float32), z[f"b{l}"].astype(np.float32))
        m.margin = float(z["margin"]) if "margin" in z.files else 1.0
        return m


# ------------------------------------------------------------------ features

def bucket_loads(counter):
    """(distinct, table keys, k-mer occurrences) per model bucket of the
    counter's last device-held result."""
    d = np.zeros(MODEL_BUCKETS, np.uint64)
    t = np.zeros(MODEL_BUCKETS, np.uint64)
    km = np.zeros(MODEL_BUCKETS, np.uint64)
    check(lib.kc_bucket_loads(counter._ctx, d.ctypes.data_as(_u64), t.ctypes.data_as(_u64),
                              km.ctypes.data_as(_u64)))
    return d, t, km


def prefix_len(n, fraction=PREFIX_FRACTION):
    return max(1, int(n * fraction))


def prefix_bytes(data, fraction=PREFIX_FRACTION):
    return data[:prefix_len(len(data), fraction)]


def features(prefix_loads, k, read_len, fastq_bytes, prefix_nbytes):
    """Model input from the prefix's per-bucket loads (distinct, table, kmers)."""
    d, t, km = (np.asarray(a, np.float64) for a in prefix_loads)
    return features_batch(km[None, :], [d.sum()], [t.sum()], [k], [read_len], [fastq_bytes], [prefix_nbytes])[0]


def features_batch(km, Dp, Tp, k, read_len, fastq_bytes, prefix_nbytes):
    """features() for many inputs at once: km (n, MODEL_BUCKETS) prefix
    k-mers per model bucket; the others per input (prefix distinct and table
    keys, k, read length, file bytes, prefix bytes)."""
    km = np.asarray(km, np.float64)
    n = km.shape[0]
    Dp, Tp, k, rl, fb, pb = (np.asarray(a, np.float64).reshape(n) for a in (Dp, Tp, k, read_len, fastq_bytes,
                                                                         prefix_nbytes))
    Kp = km.sum(axis=1)
    has = Kp > 0
    Ks = np.where(has, Kp, 1.0)
    x = np.zeros((n, N_IN), np.float32)
    x[:, :MODEL_BUCKETS] = np.where(has[:, None], np.log1p(MODEL_BUCKETS * km / Ks[:, None]) / 4.0, 0.0)
    x[:, MODEL_BUCKETS + 0] = k / 64.0
    x[:, MODEL_BUCKETS + 1] = rl / 300.0
    x[:, MODEL_BUCKETS + 2] = np.log(np.maximum(fb, 1)) / IN_SCALE
    x[:, MODEL_BUCKETS + 3] = np.log1p(Kp) / IN_SCALE
    x[:, MODEL_BUCKETS + 4] = np.where(has, Dp / Ks, 1.0)
    x[:, MODEL_BUCKETS + 5] = np.where(has, Tp / Ks, 0.0)
    x[:, MODEL_BUCKETS + 6] = np.where(has, np.sqrt(np.maximum(Tp / Ks, 0.0)), 0.0)
    x[:, MODEL_BUCKETS + 7] = np.log(np.maximum(fb, 1) / np.maximum(pb, 1)) / 10.0
    return x


def _to_y(ratio):
    return np.log(np.asarray(ratio, np.float64) + RATIO_FLOOR) / RATIO_LOG + 1.0


def _from_y(y):
    return np.clip(np.exp((np.clip(y, 0.0, 1.2) - 1.0) * RATIO_LOG) - RATIO_FLOOR, 0.0, 1.0)


def targets(full_loads):
    """Per bucket: distinct keys per k-mer and table keys per k-mer, encoded."""
    d, t, km = (np.asarray(a, np.float64) for a in full_loads)
    den = np.maximum(km, 1.0)
    y = np.empty(N_OUT, np.float32)
    y[:MODEL_BUCKETS] = _to_y(d / den)
    y[MODEL_BUCKETS:] = _to_y(t / den)
    return y


def decode(y, kmers_est):
    """Model output + estimated k-mers per bucket -> (distinct, table keys)."""
    y = np.asarray(y, np.float64)
    kest = np.asarray(kmers_est, np.float64)
    return _from_y(y[:MODEL_BUCKETS]) * kest, _from_y(y[MODEL_BUCKETS:]) * kest


def predict_on(counter, model, k, read_len, total_bytes, run_prefix, target=None):
    """Profile a prefix on `counter` (plain rule), predict the full run's
    per-bucket loads, hand them to `target` (default: `counter`; it must use
    KC_SIZING_LEARNED) for its next count.  run_prefix() counts the prefix
    and returns its byte length.  Returns (distinct, table keys) as handed
    over (margin applied)."""
    target = counter if target is None else target
    check(lib.kc_set_predicted_loads(target._ctx, None, None))
    pbytes = run_prefix()
    loads = bucket_loads(counter)
    x = features(loads, k, read_len, total_bytes, pbytes)
    scale = total_bytes / max(pbytes, 1)
    d, t = decode(model.forward(x[None, :])[0], loads[2].astype(np.float64) * scale)
    t = t * model.margin
    apply(target, (d, t))
    return d, t


_SIZING_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p)


class BesideSizing:
    """Learned sizing run beside the count (kc_set_sizing_callback): every
    count of device-resident FASTQ on `counter` (KC_SIZING_LEARNED) calls
    back at its sizing point, after its k-mer extraction is enqueued; the
    callback counts the first 1% of the same FASTQ on a helper context (plain
    rule), runs the network and hands the predictions to `counter`, while the
    extraction runs.  Set `target = (device pointer, bytes)` before each
    count; `last_ms` is the callback's own wall time."""

    def __init__(self, counter, model, k, read_len, device=0):
        from ._native import Counter
        self.counter, self.model, self.k, self.read_len = counter, model, k, read_len
        # the helper's kernels go ahead of the count's queued extraction
        self.helper = Counter(k=k, device=device, priority=1)
        self.target = None
        self.last_ms = 0.0
        self.error = None
        self._cb = _SIZING_FN(self._call)  # kept alive as long as the registration
        check(lib.kc_set_sizing_callback(counter._ctx, C.cast(self._cb, C.c_void_p), None))

    def _call(self, user, ctx):
        import time
        t0 = time.perf_counter()
        try:
            dptr, n = self.target
            pn = prefix_len(n)

            def run():
                self.helper.count_device(dptr, pn)
                return pn
            predict_on(self.helper, self.model, self.k, self.read_len, n, run, target=self.counter)
        except Exception as e:  # reported by the count as KC_ERR_INVALID
            self.error = e
            return 1
        self.last_ms = (time.perf_counter() - t0) * 1e3
        return 0

    def close(self):
        check(lib.kc_set_sizing_callback(self.counter._ctx, None, None))
        self.helper.close()


def predict_host(counter, model, data, k, read_len):
    """predict_on for host FASTQ bytes (the prefix is copied and counted)."""
    def run():
        p = prefix_bytes(data)
        counter.count_host(p)
        return len(p)
    return predict_on(counter, model, k, read_len, len(data), run)


def predict_device(counter, model, dptr, n, k, read_len):
    """predict_on for FASTQ already in device memory."""
    def run():
        pn = prefix_len(n)
        counter.count_device(dptr, pn)
        return pn
    return predict_on(counter, model, k, read_len, n, run)


MIN_SET_PREFIX = 128 << 10  # smallest prefix (bytes) a set's learned sizing is made from


def predict_sets(counter, model, dptr, sets, read_lens, min_prefix_bytes=MIN_SET_PREFIX):
    """Learned sizing of a batch of read sets (kc_count_sets): the first 1%
    of every set is counted in one batched call (its k-mers, first
    occurrences and table keys per set) and histogrammed per model bucket
    (kc_set_prefix_kmers); the network runs on all sets at once and its
    per-set, per-root-bucket rates (distinct and table keys per k-mer, the
    table's with the model's margin) go to the counter for its next
    kc_count_sets of these sets (the counter must use KC_SIZING_LEARNED),
    which multiplies them by each bucket's exact k-mer total.  A set whose
    1% is under `min_prefix_bytes` keeps the sampled rule (rate -1): a few
    hundred reads say too little.  `sets` is a list of (offset, bytes, k),
    `read_lens` the sets' read lengths.  Returns the rates (distinct, table
    keys), each (n_sets, 256)."""
    n = len(sets)
    check(lib.kc_set_predicted_set_rates(counter._ctx, 0, None, None))
    dist = np.full((n, 256), -1.0)
    tab = np.full((n, 256), -1.0)
    use = [i for i, (_, b, _) in enumerate(sets) if prefix_len(b) >= min_prefix_bytes]
    if use:
        m = len(use)
        pre = [(sets[i][0], prefix_len(sets[i][1]), sets[i][2]) for i in use]
        res = counter.count_sets(dptr, pre)
        desc = (_native.KcSetDesc * m)(*[_native.KcSetDesc(o, b, k, 0) for o, b, k in pre])
        km = np.zeros(m * MODEL_BUCKETS, np.uint64)
        check(lib.kc_set_prefix_kmers(counter._ctx, C.c_void_p(dptr), desc, m, km.ctypes.data_as(_u64)))
        km = km.reshape(m, MODEL_BUCKETS).astype(np.float64)
        # the prefix's distinct keys are its first occurrences (a filter
        # false positive moves a few into the table), its table keys its
        # root records
        x = features_batch(km, [r.low_records for r in res], [r.root_records for r in res], [p[2] for p in pre],
                           [read_lens[i] for i in use], [sets[i][1] for i in use], [p[1] for p in pre])
        y = np.asarray(model.forward(x), np.float64)
        rd = _from_y(y[:, :MODEL_BUCKETS])
        rt = _from_y(y[:, MODEL_BUCKETS:]) * model.margin
        # a root bucket's rate: its model buckets' rates weighted by their
        # prefix k-mers (plain mean where the prefix has none)
        per = MODEL_BUCKETS // 256
        w = (km + 1e-3).reshape(m, 256, per)
        ws = w.sum(axis=2)
        dist[use] = (rd.reshape(m, 256, per) * w).sum(axis=2) / ws
        tab[use] = (rt.reshape(m, 256, per) * w).sum(axis=2) / ws
    dd, tt = np.ascontiguousarray(dist.ravel()), np.ascontiguousarray(tab.ravel())
    check(lib.kc_set_predicted_set_rates(counter._ctx, n, dd.ctypes.data_as(_d), tt.ctypes.data_as(_d)))
    return dist, tab


def apply(counter, pred):
    """Hand predicted loads to a counter configured with KC_SIZING_LEARNED."""
    d, t = (np.ascontiguousarray(a, np.float64) for a in pred)
    check(lib.kc_set_predicted_loads(counter._ctx, d.ctypes.data_as(_d), t.ctypes.data_as(_d)))


def sampled_table_prediction(full_kmers, repeat_ratio=0.125):
    """What the plain rule assumes per bucket: k-mers x repeat_ratio."""
    return np.asarray(full_kmers, np.float64) * repeat_ratio


def relative_error(pred, true):
    true = np.asarray(true, np.float64)
    pred = np.asarray(pred, np.float64)
    m = true > 0
    return np.abs(pred[m] - true[m]) / true[m]


# ------------------------------------------------------------------ Stage-0 side by side

def stage0_report(path, k, n_thread=8, model=None, device=0, read_len=150, bloom_bits=5.0):
    """Per root prefix (key word 0 >> 56), the first-occurrence filter each
    sizing rule gives for the FASTQ at `path`, in 64-bit words:

      reference   the reference's Stage 0: its own 256 MB sample and
                  calculate_bloom_filter_capacity (src/main.cpp:88-108),
                  with its classifier owner (src/main.cpp:38-86)
      sampled     this build's plain rule on the exact k-mer totals of the
                  whole input: bit_ceil(k-mers x bloom_bits / 64), >= 256
      learned     the sizing model's rule: bit_ceil(predicted distinct keys
                  x 12 / 64), >= 256 (the model run on the first 1% of reads)
      distinct    the exact number of distinct keys (the quantity both the
                  reference's 4.81 bits and the learned 12 bits are per)

    Returns a dict of numpy arrays of length 256 plus the KcStage0 record."""
    from ._native import Counter
    s0 = _native.stage0_file(path, k=k, n_thread=n_thread, device=device)
    data = np.fromfile(path, np.uint8)
    with Counter(k=k, device=device) as c:
        c.count_host(data)
        dist, _, km = bucket_loads(c)
    per = MODEL_BUCKETS // 256
    km256 = km.reshape(256, per).sum(axis=1).astype(np.float64)
    d256 = dist.reshape(256, per).sum(axis=1).astype(np.float64)

    def ceil2(x):
        x = np.maximum(x.astype(np.float64), 256.0)
        return (2.0 ** np.ceil(np.log2(x))).astype(np.int64)

    out = {"prefix": np.arange(256), "reference": np.array(s0.bloom_filter_capacity, np.int64),
           "owner": np.array(s0.prefix_owner, np.int64), "sampled": ceil2(km256 * bloom_bits / 64.0),
           "distinct": d256.astype(np.int64), "kmers": km256.astype(np.int64), "stage0": s0}
    if model is not None:
        with Counter(k=k, device=device) as c:
            d_pred, _ = predict_host(c, model, data, k, read_len)
        out["learned"] = ceil2(np.asarray(d_pred, np.float64).reshape(256, per).sum(axis=1) * 12.0 / 64.0)
    return out


def _main(argv):
    import argparse
    ap = argparse.ArgumentParser(prog="python -m kmertreecounter_b200.sizing")
    sub = ap.add_subparsers(dest="cmd", required=True)
    st = sub.add_parser("stage0", help="the reference's Stage-0 filter sizes beside this build's rules")
    st.add_argument("fastq")
    st.add_argument("k", type=int)
    st.add_argument("--threads", type=int, default=8)
    st.add_argument("--read-len", type=int, default=150)
    a = ap.parse_args(argv)
    model = MLP.load() if os.path.exists(MODEL_PATH) else None
    r = stage0_report(a.fastq, a.k, a.threads, model, read_len=a.read_len)
    s0 = r["stage0"]
    print(f"Average prefix count: {s0.average_prefix_count}")
    for i, load in s0.loads_in_print_order():
        print(f"Classifier {i} total prefix count: {load}")
    print(f"Max Bloom Filter capacity: {s0.max_bloom_filter_capacity}")
    cols = ["prefix", "owner", "kmers", "distinct", "reference", "sampled"] + (["learned"] if "learned" in r else [])
    print("\t".join(cols))
    for p in range(256):
        print("\t".join(str(int(r[c][p])) for c in cols))


if __name__ == "__main__":
    import sys
    _main(sys.argv[1:])
