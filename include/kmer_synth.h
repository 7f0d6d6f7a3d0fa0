/* Seeded synthetic genomes and FASTQ read sets (libkc_synth.so).
 *
 * Not part of the counting path: a workload generator for benchmarks and
 * tests.  The reference publishes no dataset; its benchmark shapes are given
 * as genome length, GC content, repeat families, coverage, read length and
 * error rates, which these parameters describe.  Output is a pure function of
 * the parameters (thread count included or not).
 */
#ifndef KMER_SYNTH_H
#define KMER_SYNTH_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct kc_synth_params {
    uint64_t seed;
    uint64_t genome_len;      /* bases */
    double gc;                /* GC fraction; 0.5 gives i.i.d. uniform ACGT */
    double repeat_frac;       /* fraction of the genome overwritten by repeat-family copies */
    uint32_t rep_min_len;     /* template length range, bases */
    uint32_t rep_max_len;
    uint32_t rep_min_copies;  /* copies per family */
    uint32_t rep_max_copies;
    double rep_divergence;    /* per-base substitution probability of each copy */
    uint64_t n_reads;
    uint32_t read_len_min;
    uint32_t read_len_max;
    double sub_rate;          /* mean per-base substitution probability */
    uint32_t sub_profile;     /* 0 uniform; 1 rising linearly toward the 3' end, same mean */
    double n_rate;            /* per-base probability of 'N' */
    uint32_t threads;         /* 0 = hardware concurrency (capped at 64) */
} kc_synth_params;

/* Fill genome[0..genome_len) with 'A','C','G','T'. Returns 0 on success. */
int kc_synth_genome(const kc_synth_params* p, uint8_t* genome);

/* Exact FASTQ size in bytes for these parameters. */
uint64_t kc_synth_fastq_bytes(const kc_synth_params* p);

/* Write the FASTQ records into out[0..cap). Returns bytes written, or
 * -(bytes needed) when cap is too small, or -1 on bad arguments. */
int64_t kc_synth_fastq(const kc_synth_params* p, const uint8_t* genome, uint8_t* out, uint64_t cap);

#ifdef __cplusplus
}
#endif

#endif /* KMER_SYNTH_H */
