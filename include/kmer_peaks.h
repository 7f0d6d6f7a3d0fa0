/* kmer_peaks.h -- roofline denominators measured on the device the counter
 * runs on (libkmertree_b200.so).
 *
 * The counting path is bound by HBM bandwidth and by the rate of random
 * 32-bit atomics that miss L2: one first-occurrence filter atomicOr per k-mer
 * and one table atomicAdd per repeat occurrence (the reference's per-k-mer
 * ConcurrentBloomFilter::insert fetch_or, src/BloomFilter.h:207-234, and its
 * ConcurrentMap count add, src/ConcurrentMap.h:112-160).  These figures are
 * the denominators of those two roofline terms, plus the pinned host->device
 * link for streamed inputs.
 */
#ifndef KMER_PEAKS_H
#define KMER_PEAKS_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct kc_peaks {
    double hbm_copy_gbs;     /* device-to-device copy: bytes read + written per second / 1e9 */
    double red_add_gops;     /* random u32 atomicAdd, result unused (reduction), 1e9 ops/s */
    double or_return_gops;   /* random u32 atomicOr whose old value is used, 1e9 ops/s */
    double h2d_gbs;          /* pinned host -> device copy, 1e9 bytes/s */
    uint64_t footprint_bytes; /* the random atomics' footprint */
    uint64_t ops;            /* atomics per timed launch */
    /* the same two atomic forms on an L2-resident footprint (32 MiB, about a
     * quarter of L2): the rate when routing keeps the working set in L2 */
    double l2_red_add_gops;
    double l2_or_return_gops;
    uint64_t l2_footprint_bytes;
} kc_peaks;

/* Measure on `device` (best of three launches each).  `footprint_bytes` is
 * the random-atomic footprint: a power of two from 256 MiB to 32 GiB (4 GiB
 * is the usual figure, well above the 126 MB L2); the copy moves half of it
 * each way, the link test copies min(footprint, 1 GiB).  Returns KC_OK or a
 * negative KC_ERR_* code (kmer_count.h) with kc_last_error() set. */
int kc_measure_peaks(int device, uint64_t footprint_bytes, kc_peaks* out);

#ifdef __cplusplus
}
#endif

#endif
