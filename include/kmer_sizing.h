/* kmer_sizing.h -- learned sizing of the first-occurrence filter and repeat
 * tables (libkmertree_b200.so).
 *
 * The reference sizes its per-prefix Bloom filters from a Stage-0 sample
 * (src/main.cpp:88-108, src/FastqPreReader.h) and assigns prefixes to
 * classifier threads by LPT (src/main.cpp:38-86).  Here a small MLP (BF16
 * weights, FP32 accumulation, trained and run by the library's own tensor-core
 * kernels) predicts per-bucket loads from a 1% read prefix; the counter uses
 * them to size its structures, and falls back to growing a table (rehash) if a
 * prediction was too small.  Model buckets are the 4096 six-base prefixes of
 * the canonical key (key word 0 >> 52).
 */
#ifndef KMER_SIZING_H
#define KMER_SIZING_H

#include <stdint.h>

#include "kmer_count.h"

#ifdef __cplusplus
extern "C" {
#endif

#define KC_MODEL_BUCKETS 4096

/* Per model bucket of the last device-held count (kc_count_host /
 * kc_count_device): distinct keys, keys held by the repeat tables (the table
 * load) and k-mer occurrences.  The exact loads the model is trained on and
 * whose error it is measured against; on a 1% read prefix, `kmers` is the
 * model's input histogram.
 * Any pointer may be NULL. */
int kc_bucket_loads(kc_context* ctx, uint64_t* distinct, uint64_t* table_keys, uint64_t* kmers);

/* Predicted distinct keys and table keys per model bucket for the NEXT count
 * on this context with cfg.sizing = KC_SIZING_LEARNED (NULL clears). */
int kc_set_predicted_loads(kc_context* ctx, const double* distinct, const double* table_keys);

/* A callback for learned sizing beside the count: with cfg.sizing =
 * KC_SIZING_LEARNED, every count on this context calls fn(user, ctx) at its
 * sizing point -- after the first batch's k-mer extraction has been enqueued
 * and before any filter or table is laid out -- so that work the callback
 * does (a prefix count on ANOTHER context, the network's forward pass) runs
 * while that extraction does.  The callback hands its predictions with
 * kc_set_predicted_loads(ctx, ...) and returns 0; a non-zero return fails the
 * count with KC_ERR_INVALID; no prediction keeps the sampled rule.  It must
 * not start a count on ctx.  fn = NULL removes it.  No reference
 * counterpart. */
typedef int (*kc_sizing_fn)(void* user, kc_context* ctx);
int kc_set_sizing_callback(kc_context* ctx, kc_sizing_fn fn, void* user);

/* ---- learned sizing of many read sets (kc_count_sets) -------------------
 * Per set s, k-mers per model bucket (top 12 bits of the canonical key) of
 * bytes [offset, offset + bytes) of each set descriptor (typically each set's
 * first 1%): counts[s * KC_MODEL_BUCKETS + b].  No reference counterpart
 * (the reference counts one file per process). */
int kc_set_prefix_kmers(kc_context* ctx, const uint8_t* d_fastq, const kc_set_desc* sets, uint32_t n_sets,
                        uint64_t* counts);

/* Predicted distinct keys and table keys PER K-MER of each (set, root
 * bucket) -- n_sets x 256 entries each, set-major -- for the NEXT
 * kc_count_sets of n_sets sets on this context with cfg.sizing =
 * KC_SIZING_LEARNED (NULL clears).  kc_count_sets multiplies them by the
 * bucket's exact k-mer total (from its extraction histogram); a negative
 * entry keeps the sampled rule for that bucket.  A table a prediction left
 * too small grows exactly as under the sampled rule. */
int kc_set_predicted_set_rates(kc_context* ctx, uint32_t n_sets, const double* distinct_per_kmer,
                               const double* table_keys_per_kmer);

/* ---- the MLP ---------------------------------------------------------- */
typedef struct kc_mlp kc_mlp;
int kc_mlp_create(int in, int hidden, int out, int max_batch, uint64_t seed, kc_mlp** m);
void kc_mlp_destroy(kc_mlp* m);
/* layer l in 0..2: weights row-major (fan_in x fan_out), bias (fan_out) */
int kc_mlp_set_layer(kc_mlp* m, int l, const float* w, const float* bias);
int kc_mlp_get_layer(kc_mlp* m, int l, float* w, float* bias);
/* y (B x out) = f(x (B x in)), FP32 host arrays */
int kc_mlp_forward(kc_mlp* m, const float* x, int batch, float* y);
/* loss weight for outputs below their target (default 1 = plain squared
 * error); > 1 makes the network lean towards over- rather than under-sizing */
int kc_mlp_set_under_weight(kc_mlp* m, float under);
/* gradients of the batch-mean (weighted) squared error w.r.t. layer l */
int kc_mlp_gradients(kc_mlp* m, const float* x, const float* target, int batch, int l, float* grad_w,
                     float* grad_b, float* loss);
/* one Adam step (beta 0.9/0.999) on a batch; *loss = the pre-update loss */
int kc_mlp_train_step(kc_mlp* m, const float* x, const float* target, int batch, float lr, float* loss);
const char* kc_mlp_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* KMER_SIZING_H */
