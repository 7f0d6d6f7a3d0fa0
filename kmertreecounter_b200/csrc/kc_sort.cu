// Root-record ordering.  Placeholder until the radix sort lands: reports that
// sorted output is unavailable so callers fail loudly instead of silently
// writing unsorted files.
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/kmer_count.h"
#include "kc_internal.h"

int kc_sort_roots(void*, uint64_t, uint64_t, uint32_t, const uint64_t*, cudaStream_t) { return KC_ERR_INVALID; }
const char* kc_sort_error() { return "sorted root output is not available in this build"; }
