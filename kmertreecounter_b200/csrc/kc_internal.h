// Internal (non-ABI) declarations shared by the engine's translation units.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/kmer_count.h"

struct kc_context;

// Device scratch of the root-record sort (sizes from kc_sort_scratch_bytes).
struct KcSortScratch {
    void* tmp;
    void* hist;
    void* offs;
    void* sums;
};
void kc_sort_scratch_bytes(uint64_t n, uint64_t record_bytes, uint64_t* tmp, uint64_t* hist, uint64_t* offs,
                           uint64_t* sums);

// Sort root records (ExportRecord<N>, record_bytes each, grouped by root id)
// by key, keeping the grouping, in place on `stream` (asynchronous).
// Returns 0 or a negative KC_ERR_* code.
int kc_sort_roots(void* records, uint64_t n, uint64_t record_bytes, uint32_t k, const KcSortScratch& w,
                  cudaStream_t stream);
const char* kc_sort_error();
// The same over bare keys of nw 64-bit words (scratch sizes from
// kc_sort_scratch_bytes with record_bytes = 8 nw).
int kc_sort_keys(void* keys, uint64_t n, uint32_t nw, uint32_t k, const KcSortScratch& w, cudaStream_t stream);

int kc_internal_set_error(int code, const char* msg);
uint64_t kc_internal_record_bytes(const kc_context* c);
uint32_t kc_internal_k(const kc_context* c);

// Canonical k-mers per root prefix (key word 0 >> 56, 256 counts) of FASTQ
// bytes in host memory, counted on the context's device.
int kc_internal_prefix_counts(kc_context* c, const uint8_t* host, uint64_t n, uint64_t* counts);

// The streamed count (kc_count_host_stream) of a plain FASTQ file's n bytes
// read from fd in pieces (parallel preads into a small pinned ring).
int kc_internal_count_fd_stream(kc_context* c, int fd, uint64_t n, kc_sink_fn sink, void* user, kc_stats* stats);
