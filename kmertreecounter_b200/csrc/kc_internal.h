// Internal (non-ABI) declarations shared by the engine's translation units.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

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

int kc_internal_set_error(int code, const char* msg);
uint64_t kc_internal_record_bytes(const kc_context* c);
