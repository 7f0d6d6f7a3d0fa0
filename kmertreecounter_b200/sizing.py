"""Learned sizing of the filter and repeat tables (include/kmer_sizing.h).

The reference sizes its per-prefix Bloom filters from a Stage-0 sample of up
to 256 MB (src/main.cpp:88-108) and never sizes its tree, which grows from a
memory pool.  Here the open-addressing tables must be sized up front; the
plain rule (`KC_SIZING_SAMPLED`) takes each bucket's exact k-mer total of the
first batch and a fixed ratio of table keys per k-mer, and grows a table x4
(rehash) when it overflows.  The learned rule predicts each bucket's distinct
keys and table keys from a 1% read prefix with a small MLP:

  input  (4102) log1p 6-mer-prefix histogram of the prefix's k-mers (4096
         buckets = top six bases of the canonical key) / 16, k/64, read
         length/300, ln(FASTQ bytes)/25, and three totals of the prefix counted
         exactly on the GPU: ln(1+k-mers), ln(1+distinct), ln(1+table keys), /25
  hidden 512 -> 512, ReLU, BF16 weights, FP32 accumulation
  output (8192) ln(1+distinct keys)/20 and ln(1+table keys)/20 per bucket

It is trained by the library's own kernels (kc_mlp_train_step) on exact loads
that the counter itself measures (kc_bucket_loads) on seeded synthetic
genomes.  The plain rule stays the fallback: a table that overflows under a
learned size is grown exactly as under the plain rule, so counts stay exact
either way; rehashes avoided or incurred are reported by kc_stats.
"""
import ctypes as C
import math
import os

import numpy as np

from . import _native
from ._native import check, lib

MODEL_BUCKETS = 4096
N_IN = MODEL_BUCKETS + 6
N_HID = 512
N_OUT = 2 * MODEL_BUCKETS
IN_SCALE = 25.0
OUT_SCALE = 20.0
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

    def save(self, path=MODEL_PATH, meta=None):
        """Weights as float16 (the forward pass runs in BF16 anyway), biases fp32."""
        arrs = {}
        for l in range(3):
            w, b = self.get_layer(l)
            arrs[f"w{l}"] = w.astype(np.float16)
            arrs[f"b{l}"] = b
        np.savez_compressed(path, **arrs, meta=np.array(str(meta or {})))

    @classmethod
    def load(cls, path=MODEL_PATH, max_batch=8):
        z = np.load(path, allow_pickle=False)
        m = cls(n_in=z["w0"].shape[0], n_hid=z["w0"].shape[1], n_out=z["w2"].shape[1], max_batch=max_batch)
        for l in range(3):
            m.set_layer(l, z[f"w{l}"].astype(np.float32), z[f"b{l}"].astype(np.float32))
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


def prefix_bytes(data, fraction=PREFIX_FRACTION):
    n = max(1, int(len(data) * fraction))
    return data[:n]


def features(prefix_loads, k, read_len, fastq_bytes):
    """Model input from the prefix's per-bucket loads (distinct, table, kmers)."""
    d, t, km = prefix_loads
    x = np.empty(N_IN, np.float32)
    x[:MODEL_BUCKETS] = np.log1p(km.astype(np.float64)) / 16.0
    x[MODEL_BUCKETS + 0] = k / 64.0
    x[MODEL_BUCKETS + 1] = read_len / 300.0
    x[MODEL_BUCKETS + 2] = math.log(max(fastq_bytes, 1)) / IN_SCALE
    x[MODEL_BUCKETS + 3] = math.log1p(float(km.sum())) / IN_SCALE
    x[MODEL_BUCKETS + 4] = math.log1p(float(d.sum())) / IN_SCALE
    x[MODEL_BUCKETS + 5] = math.log1p(float(t.sum())) / IN_SCALE
    return x


def targets(full_loads):
    d, t, _ = full_loads
    y = np.empty(N_OUT, np.float32)
    y[:MODEL_BUCKETS] = np.log1p(d.astype(np.float64)) / OUT_SCALE
    y[MODEL_BUCKETS:] = np.log1p(t.astype(np.float64)) / OUT_SCALE
    return y


def decode(y):
    """Model output -> (predicted distinct, predicted table keys) per bucket."""
    y = np.clip(np.asarray(y, np.float64), 0.0, 1.6)
    return np.expm1(y[:MODEL_BUCKETS] * OUT_SCALE), np.expm1(y[MODEL_BUCKETS:] * OUT_SCALE)


def profile_prefix(data, k, device=0):
    """Count the first 1% of the FASTQ exactly; return its per-bucket loads."""
    from ._native import Counter
    with Counter(k=k, n_buckets=256, device=device) as c:
        c.count_host(prefix_bytes(data))
        return bucket_loads(c)


def predict_loads(model, data, k, read_len, device=0):
    """Predicted (distinct, table keys) per model bucket for FASTQ bytes."""
    x = features(profile_prefix(data, k, device), k, read_len, len(data))
    return decode(model.forward(x[None, :])[0])


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
