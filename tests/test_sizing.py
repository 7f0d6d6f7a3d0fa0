"""Learned sizing: the MLP kernels against the CPU oracle, the measured
per-bucket loads, and what the trained network gains over the plain rule.

The model is trained by the library's own kernels (kc_mlp_train_step) on
loads the counter measures; counts stay exact under any sizing, because an
undersized table is grown (rehash) exactly as under the plain rule."""
import os

import numpy as np
import pytest

import mlp_oracle
import oracle

pytestmark = pytest.mark.gpu

kc = pytest.importorskip("kmertreecounter_b200")
from kmertreecounter_b200 import sizing, synth  # noqa: E402


def small_mlp(seed=3, n_in=72, n_hid=48, n_out=40, batch=24):
    rng = np.random.default_rng(seed)
    layers = [(rng.normal(0, (2 / a) ** 0.5, (a, b)).astype(np.float32), rng.normal(0, 0.1, b).astype(np.float32))
              for a, b in [(n_in, n_hid), (n_hid, n_hid), (n_hid, n_out)]]
    m = sizing.MLP(n_in, n_hid, n_out, max_batch=batch)
    for l, (w, b) in enumerate(layers):
        m.set_layer(l, w, b)
    x = rng.normal(0, 1, (batch, n_in)).astype(np.float32)
    t = rng.normal(0, 1, (batch, n_out)).astype(np.float32)
    return m, layers, x, t


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30))


def test_forward_matches_oracle():
    m, layers, x, t = small_mlp()
    y = m.forward(x)
    y_bf, _, _ = mlp_oracle.forward_backward(x, t, layers, bf16=True)
    y_32, _, _ = mlp_oracle.forward_backward(x, t, layers, bf16=False)
    assert rel(y, y_bf) < 5e-3      # same rounding points, FP32 vs FP64 accumulation
    assert rel(y, y_32) < 3e-2      # BF16 operands vs the FP32 network


@pytest.mark.parametrize("layer", [0, 1, 2])
def test_gradients_match_oracle(layer):
    m, layers, x, t = small_mlp(seed=10 + layer)
    gw, gb, loss = m.gradients(x, t, layer)
    _, loss_bf, g_bf = mlp_oracle.forward_backward(x, t, layers, bf16=True)
    _, loss_32, g_32 = mlp_oracle.forward_backward(x, t, layers, bf16=False)
    assert abs(loss - loss_bf) / loss_bf < 5e-3
    assert rel(gw, g_bf[layer][0]) < 2e-2 and rel(gb, g_bf[layer][1]) < 2e-2
    assert rel(gw, g_32[layer][0]) < 6e-2 and rel(gb, g_32[layer][1]) < 6e-2


def test_weighted_loss_gradients_match_oracle():
    m, layers, x, t = small_mlp(seed=21)
    m.set_under_weight(4.0)
    gw, gb, loss = m.gradients(x, t, 2)
    _, loss_bf, g_bf = mlp_oracle.forward_backward(x, t, layers, bf16=True, under=4.0)
    assert abs(loss - loss_bf) / loss_bf < 5e-3
    assert rel(gw, g_bf[2][0]) < 2e-2 and rel(gb, g_bf[2][1]) < 2e-2


def test_training_reduces_loss():
    rng = np.random.default_rng(5)
    m = sizing.MLP(64, 64, 32, max_batch=32, seed=3)
    A = rng.normal(0, 0.3, (64, 32)).astype(np.float32)
    x = rng.normal(0, 1, (32, 64)).astype(np.float32)
    t = np.tanh(x @ A).astype(np.float32)
    first = m.train_step(x, t, 3e-3)
    for _ in range(300):
        last = m.train_step(x, t, 3e-3)
    assert last < 0.1 * first


def test_bucket_loads_are_consistent():
    p = synth.plain_small(seed=77, scale=0.1)
    data = synth.fastq(p)
    keys, counts, K = oracle.count(data, 31)
    with kc.Counter(k=31, repeat_ratio=0.02) as c:   # forces rehashes: loads must skip stale copies
        st = c.count_host(data)
        d, t, km = sizing.bucket_loads(c)
    assert int(km.sum()) == K and int(d.sum()) == keys.shape[0] and int(t.sum()) == st.table_keys
    b = (keys[:, 0] >> np.uint64(52)).astype(np.int64)
    assert np.array_equal(d, np.bincount(b, minlength=4096).astype(np.uint64))
    assert np.array_equal(km, np.bincount(b, weights=counts, minlength=4096).astype(np.uint64))


def test_underestimated_sizes_fall_back_exactly():
    """Absurdly small predictions: tables overflow, grow, counts stay exact."""
    p = synth.plain_small(seed=78, scale=0.1)
    data = synth.fastq(p)
    with kc.Counter(k=31, sizing=kc.KC_SIZING_LEARNED) as c:
        sizing.apply(c, (np.ones(4096), np.ones(4096)))
        st = c.count_host(data)
        assert st.rehashes > 0
        h, distinct = c.histogram(1, 200)
    keys, counts, _ = oracle.count(data, 31)
    assert distinct == keys.shape[0]
    assert [int(v) for v in h] == [int(v) for v in oracle.histogram(counts, 1, 200)]


@pytest.mark.skipif(not os.path.exists(sizing.MODEL_PATH), reason="trained sizing model not present")
def test_trained_model_beats_plain_rule():
    """Held-out seeds (never used in training): per bucket, the learned table
    sizes are closer to the loads the counter measures than the plain rule's
    (k-mers x 0.125), and the counts under both rules are identical (the
    fallback grows any table a prediction left too small)."""
    from kmertreecounter_b200.train_sizing import evaluate, summarise
    model = sizing.MLP.load()
    s = summarise(evaluate(model, range(990000, 990008), gmin=3e5, gmax=1.2e7))
    assert s["all_exact"]
    assert s["median_rel_err_table_learned"] < s["median_rel_err_table_sampled"]


@pytest.mark.skipif(not os.path.exists(sizing.MODEL_PATH), reason="trained sizing model not present")
def test_learned_sizing_avoids_rehashes_beyond_training_scale():
    """Held-out 53 Mbp genome at 5.3x coverage (training genomes stop at
    12 Mbp): the plain rule's fixed 0.125 table keys per k-mer is too small at
    this coverage and its tables overflow and grow; the rate-based prediction
    sizes them big enough the first time (here it over-predicts: its median
    per-bucket error is not the point of this case, the overflow is).  Counts
    identical under both rules."""
    from kmertreecounter_b200.train_sizing import evaluate
    model = sizing.MLP.load()
    (r,) = evaluate(model, [950001], 1e7, 1e8, max_bytes=4e9)
    print(r)
    assert r["exact_match"]
    assert r["rehash_sampled"] > 0 and r["rehash_learned"] == 0


@pytest.mark.skipif(not os.path.exists(sizing.MODEL_PATH), reason="trained sizing model not present")
def test_sizing_beside_the_count():
    """kc_set_sizing_callback (sizing.BesideSizing): the count calls back at
    its sizing point with its extraction already enqueued; the prefix is
    counted on a helper context and the predictions size this count's
    structures (the same sizes as predicting first); counts are the oracle's;
    a failing callback fails the count and the context stays usable."""
    import torch
    p = synth.plain_small(seed=81, scale=0.3)
    data = synth.fastq(p)
    d = torch.from_numpy(data).cuda()
    model = sizing.MLP.load()
    keys, counts, _ = oracle.count(data, 31)
    want = [int(v) for v in oracle.histogram(counts, 1, 200)]
    with kc.Counter(k=31, sizing=kc.KC_SIZING_LEARNED) as first:
        sizing.predict_device(first, model, d.data_ptr(), data.size, 31, 150)
        st_first = first.count_device(d.data_ptr(), data.size)
    with kc.Counter(k=31, sizing=kc.KC_SIZING_LEARNED) as c:
        beside = sizing.BesideSizing(c, model, 31, 150)
        beside.target = (d.data_ptr(), data.size)
        for _ in range(2):
            beside.last_ms = 0.0
            st = c.count_device(d.data_ptr(), data.size)
            assert beside.error is None and beside.last_ms > 0
            assert st.table_slots == st_first.table_slots and st.filter_words == st_first.filter_words
            h, distinct = c.histogram(1, 200)
            assert distinct == keys.shape[0] and [int(v) for v in h] == want
        beside.target = None  # the callback raises: the count fails
        with pytest.raises(kc.KcError) as e:
            c.count_device(d.data_ptr(), data.size)
        assert e.value.code == kc.KC_ERR_INVALID
        beside.close()
        c.count_device(d.data_ptr(), data.size)  # no callback: the last predictions handed over
        h, distinct = c.histogram(1, 200)
        assert distinct == keys.shape[0] and [int(v) for v in h] == want
