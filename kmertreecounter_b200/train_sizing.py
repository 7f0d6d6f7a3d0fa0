"""Train and evaluate the sizing MLP on loads measured by the counter itself.

    python -m kmertreecounter_b200.train_sizing --train 2000 --test 100 --out sizing_mlp.npz --report r.json

For each seeded synthetic read set (genome length log-uniform in
--genome-min..--genome-max, GC uniform 30-70%, repeat fraction uniform
0-50%, coverage log-uniform 5-100x, substitution 0.2-2%, 150 bp reads, k in
{21, 31, 63}) the GPU counter runs on the first 1% of the FASTQ (model input)
and on the whole file (targets: per-bucket ratios of kc_bucket_loads).
Training is Adam on the under-weighted squared error of the encoded ratios,
by kc_mlp_train_step, on 90% of the sets; the other 10% calibrate the
table-key margin (a quantile of measured / predicted table keys per engine
bucket).  Held-out sets are then counted with the plain sampled rule and with
the learned rule, each timed end to end (the learned time includes counting
the prefix and the network's forward pass), reporting per-bucket relative
error, rehashes, structure memory and time; both counts must agree exactly.
--scale-test adds held-out sets at 10-100 Mbp, larger than any training
genome, to check that the rate-based model carries over.

Training genomes are scaled down from the benchmark's 10-200 Mbp to
0.3-12 Mbp by default so that 2000 read sets fit in minutes of GPU time;
coverage, error and repeat structure keep the benchmark's ranges.
"""
import argparse
import json
import math
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from kmertreecounter_b200 import KC_SIZING_LEARNED, KC_SIZING_SAMPLED, Counter, synth  # noqa: E402
from kmertreecounter_b200 import sizing  # noqa: E402

ENGINE_BUCKETS = 256


def draw_params(seed, gmin=3e5, gmax=1.2e7, max_bytes=None):
    rng = np.random.default_rng(seed)
    G = int(math.exp(rng.uniform(math.log(gmin), math.log(gmax))))
    cov = math.exp(rng.uniform(math.log(5), math.log(100)))
    k = int(rng.choice([21, 31, 31, 63]))
    n_reads = max(100, int(cov * G / 150))
    if max_bytes:
        n_reads = min(n_reads, int(max_bytes / 320))
        cov = n_reads * 150 / G
    p = synth.params(seed=seed * 7919 + 13, genome_len=G, gc=float(rng.uniform(0.3, 0.7)),
                     repeat_frac=float(rng.uniform(0.0, 0.5)), rep_len=(1000, min(10000, max(1000, G // 20))),
                     n_reads=n_reads, read_len=(150, 150),
                     sub_rate=float(rng.uniform(0.002, 0.02)), sub_profile=int(rng.integers(0, 2)), n_rate=0.001)
    return p, k, cov


def sample(seed, gmin, gmax):
    """(input, target, full loads, meta) of one synthetic read set."""
    p, k, cov = draw_params(seed, gmin, gmax)
    data = synth.fastq(p)
    pre = sizing.prefix_bytes(data)
    with Counter(k=k, n_buckets=ENGINE_BUCKETS) as c:
        c.count_host(pre)
        lp = sizing.bucket_loads(c)
        c.count_host(data)
        full = sizing.bucket_loads(c)
    x = sizing.features(lp, k, 150, data.size, pre.size)
    meta = dict(seed=seed, k=k, genome=int(p.genome_len), coverage=round(cov, 2), bytes=int(data.size))
    kest = lp[2].astype(np.float64) * (data.size / max(pre.size, 1))
    return x, sizing.targets(full), full, kest, meta


def engine_sum(a):
    """Per model bucket (4096) -> per engine bucket (256)."""
    return np.asarray(a, np.float64).reshape(ENGINE_BUCKETS, -1).sum(axis=1)


def calibrate_margin(model, X, kest, fulls, q=0.95, min_keys=1000):
    """Quantile of measured / predicted table keys over engine buckets with
    at least min_keys measured keys."""
    y = model.forward(X)
    ratios = []
    for i in range(X.shape[0]):
        _, t_pred = sizing.decode(y[i], kest[i])
        t_true = engine_sum(fulls[i][1])
        tp = engine_sum(t_pred)
        m = t_true >= min_keys
        ratios.append(t_true[m] / np.maximum(tp[m], 1.0))
    r = np.concatenate(ratios) if ratios else np.ones(1)
    return max(1.0, float(np.quantile(r, q)))


def _timed(fn):
    t = time.perf_counter()
    out = fn()
    return out, (time.perf_counter() - t) * 1e3


def evaluate(model, seeds, gmin=3e5, gmax=1.2e7, max_bytes=None):
    """Held-out comparison of the learned and sampled rules (GPU), end to end
    from host FASTQ bytes."""
    rows = []
    for seed in seeds:
        p, k, cov = draw_params(seed, gmin, gmax, max_bytes)
        data = synth.fastq(p)
        # each rule counts twice on its own context; the second (warm) run is
        # timed, so both pay for their structures but not for first-use setup
        with Counter(k=k, sizing=KC_SIZING_SAMPLED) as c:
            c.count_host(data)
            st, s_ms = _timed(lambda: c.count_host(data))
            s_rehash, s_slots, s_words = st.rehashes, st.table_slots, st.filter_words
            s_hist, s_distinct = c.histogram(1, 64)
            d_true, t_true, km_true = sizing.bucket_loads(c)
        with Counter(k=k, sizing=KC_SIZING_LEARNED) as c:
            sizing.predict_host(c, model, data, k, 150)
            c.count_host(data)

            def learned():
                pred = sizing.predict_host(c, model, data, k, 150)
                return pred, c.count_host(data)
            (pred, st), l_ms = _timed(learned)
            l_rehash, l_slots, l_words = st.rehashes, st.table_slots, st.filter_words
            l_hist, l_distinct = c.histogram(1, 64)
        raw_t = pred[1] / model.margin
        rows.append(dict(
            seed=seed, k=k, genome=int(p.genome_len), coverage=round(cov, 2), bytes=int(data.size),
            exact_match=bool(np.array_equal(s_hist, l_hist) and s_distinct == l_distinct),
            rel_err_table_learned=float(np.median(sizing.relative_error(raw_t, t_true))),
            rel_err_table_sampled=float(np.median(sizing.relative_error(
                sizing.sampled_table_prediction(km_true), t_true))),
            rel_err_distinct_learned=float(np.median(sizing.relative_error(pred[0], d_true))),
            table_keys=int(t_true.sum()), predicted_table_keys=float(raw_t.sum()),
            rehash_sampled=int(s_rehash), rehash_learned=int(l_rehash),
            table_slots_sampled=int(s_slots), table_slots_learned=int(l_slots),
            filter_words_sampled=int(s_words), filter_words_learned=int(l_words),
            ms_sampled=round(s_ms, 3), ms_learned=round(l_ms, 3)))
    return rows


def summarise(rows):
    def med(key):
        return float(np.median([r[key] for r in rows]))

    def tot(key):
        return float(sum(r[key] for r in rows))
    return {
        "sets": len(rows),
        "all_exact": all(r["exact_match"] for r in rows),
        "median_rel_err_table_learned": med("rel_err_table_learned"),
        "median_rel_err_table_sampled": med("rel_err_table_sampled"),
        "median_rel_err_distinct_learned": med("rel_err_distinct_learned"),
        "rehashes_sampled": int(tot("rehash_sampled")),
        "rehashes_learned": int(tot("rehash_learned")),
        "table_slots_sampled": int(tot("table_slots_sampled")),
        "table_slots_learned": int(tot("table_slots_learned")),
        "ms_sampled": tot("ms_sampled"),
        "ms_learned": tot("ms_learned"),
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=2000)
    ap.add_argument("--test", type=int, default=100)
    ap.add_argument("--scale-test", type=int, default=0, help="held-out sets at 10-100 Mbp")
    ap.add_argument("--epochs", type=int, default=120)
    ap.add_argument("--batch", type=int, default=32)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--under-weight", type=float, default=4.0,
                    help="loss weight of under-predictions (a table that is too small costs a rehash)")
    ap.add_argument("--margin-quantile", type=float, default=0.95)
    ap.add_argument("--genome-min", type=float, default=3e5)
    ap.add_argument("--genome-max", type=float, default=1.2e7)
    ap.add_argument("--out", default=sizing.MODEL_PATH)
    ap.add_argument("--report", default=None)
    a = ap.parse_args()

    t0 = time.time()
    X, Y, F, KE, info = [], [], [], [], []
    for s in range(a.train):
        x, y, full, kest, meta = sample(1000 + s, a.genome_min, a.genome_max)
        X.append(x)
        Y.append(y)
        F.append(full)
        KE.append(kest)
        info.append(meta)
    X, Y, KE = np.stack(X), np.stack(Y), np.stack(KE)
    t_data = time.time() - t0

    n_val = max(1, a.train // 10)
    tr = np.arange(a.train - n_val)
    va = np.arange(a.train - n_val, a.train)
    model = sizing.MLP(max_batch=a.batch, seed=7)
    model.set_under_weight(a.under_weight)
    rng = np.random.default_rng(0)
    t1 = time.time()
    losses = []
    steps = 0
    for ep in range(a.epochs):
        order = rng.permutation(tr)
        lr = a.lr * 0.5 * (1 + math.cos(math.pi * ep / a.epochs))
        el = []
        for i in range(0, len(order) - a.batch + 1, a.batch):
            idx = order[i:i + a.batch]
            el.append(model.train_step(X[idx], Y[idx], lr))
            steps += 1
        losses.append(float(np.mean(el)))
    t_train = time.time() - t1
    model.margin = calibrate_margin(model, X[va], KE[va], [F[i] for i in va], q=a.margin_quantile)

    rows = evaluate(model, range(900000, 900000 + a.test), a.genome_min, a.genome_max)
    report = dict(train_sets=int(len(tr)), validation_sets=int(n_val), epochs=a.epochs, under_weight=a.under_weight,
                  margin=model.margin, margin_quantile=a.margin_quantile, steps=steps,
                  data_seconds=round(t_data, 1), train_seconds=round(t_train, 1),
                  loss_first_epoch=losses[0], loss_last_epoch=losses[-1],
                  genome_range=[a.genome_min, a.genome_max], heldout=summarise(rows))
    scale_rows = []
    if a.scale_test:
        scale_rows = evaluate(model, range(950000, 950000 + a.scale_test), 1e7, 1e8, max_bytes=4e9)
        report["heldout_10_100_mbp"] = summarise(scale_rows)
    model.save(a.out, meta=report)
    print(json.dumps(report))
    if a.report:
        with open(a.report, "w") as f:
            json.dump({"report": report, "losses": losses, "heldout_rows": rows, "scale_rows": scale_rows,
                       "train_info": info}, f, indent=1)


if __name__ == "__main__":
    main()
