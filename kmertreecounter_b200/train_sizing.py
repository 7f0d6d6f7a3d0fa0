"""Train and evaluate the sizing MLP on loads measured by the counter itself.

    python -m kmertreecounter_b200.train_sizing --train 480 --test 48 --out sizing_mlp.npz --report r.json

For each seeded synthetic read set (genome length log-uniform in
--genome-min..--genome-max, GC uniform 30-70%, repeat fraction uniform
0-50%, coverage log-uniform 5-100x, substitution 0.2-2%, 150 bp reads, k in
{21, 31, 63}) the GPU counter runs on the first 1% of the FASTQ (model input)
and on the whole file (targets: kc_bucket_loads).  Training is Adam on the
batch-mean squared error of the log loads, by kc_mlp_train_step.  The
held-out sets are then counted twice, with the plain sampled rule and with the
learned sizes, reporting per-bucket relative error of the table-size
prediction, rehashes, table memory and device time; both counts must agree
exactly.

Genomes are scaled down from the benchmark's 10-200 Mbp to 0.2-4 Mbp by
default so that several hundred read sets fit in minutes of GPU time;
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


def draw_params(seed, gmin=2e5, gmax=4e6):
    rng = np.random.default_rng(seed)
    G = int(math.exp(rng.uniform(math.log(gmin), math.log(gmax))))
    cov = math.exp(rng.uniform(math.log(5), math.log(100)))
    k = int(rng.choice([21, 31, 31, 63]))
    p = synth.params(seed=seed * 7919 + 13, genome_len=G, gc=float(rng.uniform(0.3, 0.7)),
                     repeat_frac=float(rng.uniform(0.0, 0.5)), rep_len=(1000, min(10000, max(1000, G // 20))),
                     n_reads=max(100, int(cov * G / 150)), read_len=(150, 150),
                     sub_rate=float(rng.uniform(0.002, 0.02)), sub_profile=int(rng.integers(0, 2)), n_rate=0.001)
    return p, k, cov


def sample(seed, gmin, gmax):
    p, k, cov = draw_params(seed, gmin, gmax)
    data = synth.fastq(p)
    x = sizing.features(sizing.profile_prefix(data, k), k, 150, data.size)
    with Counter(k=k, n_buckets=256) as c:
        c.count_host(data)
        full = sizing.bucket_loads(c)
    meta = dict(seed=seed, k=k, genome=int(p.genome_len), coverage=round(cov, 2), bytes=int(data.size))
    return x, sizing.targets(full), full, meta


def evaluate(model, seeds, gmin=2e5, gmax=4e6):
    """Held-out comparison of the learned and sampled rules (GPU)."""
    rows = []
    for seed in seeds:
        p, k, cov = draw_params(seed, gmin, gmax)
        data = synth.fastq(p)
        # each mode counts twice on its own context; the second (warm) run is
        # timed, so both pay for their structures but not for first-use setup
        with Counter(k=k, sizing=KC_SIZING_SAMPLED) as c:
            c.count_host(data)
            st = c.count_host(data)
            s_ms, s_rehash = st.device_ms, st.rehashes
            s_hist, s_distinct = c.histogram(1, 64)
            d_true, t_true, km_true = sizing.bucket_loads(c)
        t0 = time.perf_counter()
        pred = sizing.predict_loads(model, data, k, 150)
        predict_ms = (time.perf_counter() - t0) * 1e3
        with Counter(k=k, sizing=KC_SIZING_LEARNED) as c:
            sizing.apply(c, pred)
            c.count_host(data)
            st = c.count_host(data)
            l_ms, l_rehash = st.device_ms, st.rehashes
            l_hist, l_distinct = c.histogram(1, 64)
        rows.append(dict(
            seed=seed, k=k, genome=int(p.genome_len), coverage=round(cov, 2),
            exact_match=bool(np.array_equal(s_hist, l_hist) and s_distinct == l_distinct),
            rel_err_table_learned=float(np.median(sizing.relative_error(pred[1], t_true))),
            rel_err_table_sampled=float(np.median(sizing.relative_error(
                sizing.sampled_table_prediction(km_true), t_true))),
            rel_err_distinct_learned=float(np.median(sizing.relative_error(pred[0], d_true))),
            table_keys=int(t_true.sum()), predicted_table_keys=float(pred[1].sum()),
            sampled_table_keys=float(sizing.sampled_table_prediction(km_true).sum()),
            rehash_sampled=int(s_rehash), rehash_learned=int(l_rehash),
            device_ms_sampled=round(s_ms, 3), device_ms_learned=round(l_ms, 3), predict_ms=round(predict_ms, 2)))
    return rows


def summarise(rows):
    def med(key):
        return float(np.median([r[key] for r in rows]))
    return {
        "sets": len(rows),
        "all_exact": all(r["exact_match"] for r in rows),
        "median_rel_err_table_learned": med("rel_err_table_learned"),
        "median_rel_err_table_sampled": med("rel_err_table_sampled"),
        "median_rel_err_distinct_learned": med("rel_err_distinct_learned"),
        "rehashes_sampled": int(sum(r["rehash_sampled"] for r in rows)),
        "rehashes_learned": int(sum(r["rehash_learned"] for r in rows)),
        "device_ms_sampled": float(sum(r["device_ms_sampled"] for r in rows)),
        "device_ms_learned": float(sum(r["device_ms_learned"] for r in rows)),
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=2000)
    ap.add_argument("--test", type=int, default=100)
    ap.add_argument("--epochs", type=int, default=120)
    ap.add_argument("--batch", type=int, default=32)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--under-weight", type=float, default=6.0,
                    help="loss weight of under-predictions (a table that is too small costs a rehash)")
    ap.add_argument("--genome-min", type=float, default=2e5)
    ap.add_argument("--genome-max", type=float, default=4e6)
    ap.add_argument("--out", default=sizing.MODEL_PATH)
    ap.add_argument("--report", default=None)
    a = ap.parse_args()

    t0 = time.time()
    X, Y, info = [], [], []
    for s in range(a.train):
        x, y, _, meta = sample(1000 + s, a.genome_min, a.genome_max)
        X.append(x)
        Y.append(y)
        info.append(meta)
    X, Y = np.stack(X), np.stack(Y)
    t_data = time.time() - t0

    model = sizing.MLP(max_batch=a.batch, seed=7)
    model.set_under_weight(a.under_weight)
    rng = np.random.default_rng(0)
    t1 = time.time()
    losses = []
    steps = 0
    for ep in range(a.epochs):
        order = rng.permutation(a.train)
        lr = a.lr * 0.5 * (1 + math.cos(math.pi * ep / a.epochs))
        el = []
        for i in range(0, a.train - a.batch + 1, a.batch):
            idx = order[i:i + a.batch]
            el.append(model.train_step(X[idx], Y[idx], lr))
            steps += 1
        losses.append(float(np.mean(el)))
    t_train = time.time() - t1

    rows = evaluate(model, range(900000, 900000 + a.test), a.genome_min, a.genome_max)
    report = dict(train_sets=a.train, epochs=a.epochs, under_weight=a.under_weight, steps=steps, data_seconds=round(t_data, 1),
                  train_seconds=round(t_train, 1), loss_first_epoch=losses[0], loss_last_epoch=losses[-1],
                  genome_range=[a.genome_min, a.genome_max], heldout=summarise(rows))
    model.save(a.out, meta=report)
    print(json.dumps(report))
    if a.report:
        with open(a.report, "w") as f:
            json.dump({"report": report, "losses": losses, "heldout_rows": rows, "train_info": info}, f, indent=1)


if __name__ == "__main__":
    main()
