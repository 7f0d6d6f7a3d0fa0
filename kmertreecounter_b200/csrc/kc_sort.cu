// Root-record radix sort (replaces sort/ExportRecordRadixSort.h:19-269), and
// the same sort over bare keys (post-processing's sorted low keys).
//
// The reference's LSD radix sort orders ExportRecord<N> by key with 8-bit
// digits, skipping bits shared by a leaf; here the records of all 256 root
// files sit in one array grouped by root id = top 8 key bits, so one stable
// LSD sort over the key's 2k significant bits orders every root file by key
// and keeps the grouping (the last pass is over the most significant bits).
//
// One pass = upsweep (per-tile digit histogram, digit-major) -> exclusive
// scan -> downsweep (stable rank inside the tile, scatter).  Stable ranking:
// a tile of 256 threads x ITEMS records is processed in ITEMS rounds of 256
// consecutive records; inside a round, __match_any_sync ranks equal digits
// within a warp and per-warp digit counts in shared memory order the warps.

#include <algorithm>
#include <cstdint>
#include <string>

#include <cuda_runtime.h>

#include "../../include/kmer_count.h"
#include "kc_internal.h"
#include "kc_scan.cuh"

namespace {

constexpr int SORT_THREADS = 256;
constexpr int SORT_ITEMS = 8;
constexpr int SORT_TILE = SORT_THREADS * SORT_ITEMS;
constexpr int RADIX = 256;

thread_local std::string g_sort_err;

// Digit `pass` of a record: bits [lowbit + 8*pass, +8) of the key taken as
// one (64*NW)-bit number (word 0 most significant).
template <int NW>
__device__ __forceinline__ uint32_t digit_of(const uint64_t* rec, uint32_t bit) {
    if constexpr (NW == 1) {
        return (uint32_t)(rec[0] >> bit) & 0xFFu;
    } else if constexpr (NW == 2) {
        // 128-bit key: w0 = rec[0] (high), w1 = rec[1] (low)
        if (bit >= 64) return (uint32_t)(rec[0] >> (bit - 64)) & 0xFFu;
        if (bit + 8 <= 64) return (uint32_t)(rec[1] >> bit) & 0xFFu;
        return (uint32_t)((rec[1] >> bit) | (rec[0] << (64 - bit))) & 0xFFu;
    } else {
        // 256-bit key: rec[0] high .. rec[3] low; a digit may straddle two words
        const uint32_t wi = 3 - (bit >> 6), sh = bit & 63;
        uint64_t v = rec[wi] >> sh;
        if (sh > 56 && wi > 0) v |= rec[wi - 1] << (64 - sh);
        return (uint32_t)v & 0xFFu;
    }
}

// A record of W 64-bit words whose first NW words are the key: an
// ExportRecord<NW> (W = NW + 1: key words, then count|pad) or a bare key
// (W = NW).
template <int W>
struct Rec {
    uint64_t w[W];
};

template <int NW, int W>
__global__ void __launch_bounds__(SORT_THREADS) upsweep(const Rec<W>* __restrict__ in, uint64_t n, uint32_t bit,
                                                         uint32_t* __restrict__ hist, uint64_t n_tiles) {
    __shared__ uint32_t h[RADIX];
    h[threadIdx.x] = 0;
    __syncthreads();
    const uint64_t t0 = (uint64_t)blockIdx.x * SORT_TILE;
#pragma unroll
    for (int r = 0; r < SORT_ITEMS; ++r) {
        const uint64_t i = t0 + (uint64_t)r * SORT_THREADS + threadIdx.x;
        if (i < n) atomicAdd(&h[digit_of<NW>(in[i].w, bit)], 1u);
    }
    __syncthreads();
    hist[(uint64_t)threadIdx.x * n_tiles + blockIdx.x] = h[threadIdx.x];
}

template <int NW, int W>
__global__ void __launch_bounds__(SORT_THREADS) downsweep(const Rec<W>* __restrict__ in, Rec<W>* __restrict__ out,
                                                           uint64_t n, uint32_t bit, const uint64_t* __restrict__ offs,
                                                           uint64_t n_tiles) {
    __shared__ uint32_t base[RADIX];                        // running count per digit inside the tile
    __shared__ uint32_t wcnt[SORT_THREADS / 32][RADIX];     // per-warp digit counts of the round
    __shared__ unsigned long long goff[RADIX];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    base[tid] = 0;
    goff[tid] = offs[(uint64_t)tid * n_tiles + blockIdx.x];
    const uint64_t t0 = (uint64_t)blockIdx.x * SORT_TILE;
    const uint32_t lt = (1u << lane) - 1u;
    for (int r = 0; r < SORT_ITEMS; ++r) {
#pragma unroll
        for (int w = 0; w < SORT_THREADS / 32; ++w) wcnt[w][tid] = 0;
        __syncthreads();
        const uint64_t i = t0 + (uint64_t)r * SORT_THREADS + tid;
        const bool valid = i < n;
        Rec<W> rec;
        uint32_t d = 0, rank_in_warp = 0;
        const uint32_t active = __ballot_sync(0xffffffffu, valid);
        if (valid) {
            rec = in[i];
            d = digit_of<NW>(rec.w, bit);
            const uint32_t same = __match_any_sync(active, d);
            rank_in_warp = __popc(same & lt);
            if (rank_in_warp == 0) wcnt[warp][d] = __popc(same);
        }
        __syncthreads();
        // thread `tid` owns digit tid: exclusive prefix over warps
        uint32_t run = 0;
#pragma unroll
        for (int w = 0; w < SORT_THREADS / 32; ++w) {
            const uint32_t c = wcnt[w][tid];
            wcnt[w][tid] = run;
            run += c;
        }
        __syncthreads();
        if (valid) out[goff[d] + base[d] + wcnt[warp][d] + rank_in_warp] = rec;
        __syncthreads();
        base[tid] += run;
    }
}

template <int NW, int W>
int sort_impl(void* records, uint64_t n, uint32_t k, const KcSortScratch& w, cudaStream_t st) {
    using R = Rec<W>;
    const uint32_t key_bits = 2 * k;
    const uint32_t lowbit = 64 * NW - key_bits;
    const uint32_t passes = (key_bits + 7) / 8;
    const uint64_t n_tiles = (n + SORT_TILE - 1) / SORT_TILE;
    const uint64_t hn = (uint64_t)RADIX * n_tiles;
    R* a = static_cast<R*>(records);
    R* src = a;
    R* dst = static_cast<R*>(w.tmp);
    uint32_t* hist = static_cast<uint32_t*>(w.hist);
    uint64_t* offs = static_cast<uint64_t*>(w.offs);
    uint64_t* sums = static_cast<uint64_t*>(w.sums);
    for (uint32_t p = 0; p < passes; ++p) {
        const uint32_t bit = lowbit + 8 * p;
        upsweep<NW, W><<<n_tiles, SORT_THREADS, 0, st>>>(src, n, bit, hist, n_tiles);
        const uint64_t nb = (hn + kc::SCAN_TILE - 1) / kc::SCAN_TILE;
        kc::scan_reduce<uint32_t><<<nb, kc::SCAN_BLOCK, 0, st>>>(hist, hn, sums);
        kc::scan_sums<<<1, kc::SCAN_BLOCK, 0, st>>>(sums, nb, 0, nullptr);
        kc::scan_apply<uint32_t, uint64_t><<<nb, kc::SCAN_BLOCK, 0, st>>>(hist, hn, sums, offs);
        downsweep<NW, W><<<n_tiles, SORT_THREADS, 0, st>>>(src, dst, n, bit, offs, n_tiles);
        std::swap(src, dst);
    }
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess && src != a) e = cudaMemcpyAsync(a, src, n * sizeof(R), cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) {
        g_sort_err = cudaGetErrorString(e);
        return KC_ERR_DEVICE;
    }
    return KC_OK;
}

}  // namespace

void kc_sort_scratch_bytes(uint64_t n, uint64_t record_bytes, uint64_t* tmp, uint64_t* hist, uint64_t* offs,
                           uint64_t* sums) {
    const uint64_t n_tiles = (n + SORT_TILE - 1) / SORT_TILE;
    const uint64_t hn = (uint64_t)RADIX * n_tiles;
    *tmp = n * record_bytes;
    *hist = hn * sizeof(uint32_t);
    *offs = hn * sizeof(uint64_t);
    *sums = ((hn + kc::SCAN_TILE - 1) / kc::SCAN_TILE + 1) * sizeof(uint64_t);
}

int kc_sort_roots(void* records, uint64_t n, uint64_t record_bytes, uint32_t k, const KcSortScratch& w,
                  cudaStream_t stream) {
    if (n < 2) return KC_OK;
    if (record_bytes == 16 && k <= 32) return sort_impl<1, 2>(records, n, k, w, stream);
    if (record_bytes == 24 && k <= 64) return sort_impl<2, 3>(records, n, k, w, stream);
    if (record_bytes == 40 && k <= 128) return sort_impl<4, 5>(records, n, k, w, stream);
    g_sort_err = "unsupported record layout";
    return KC_ERR_INVALID;
}

int kc_sort_keys(void* keys, uint64_t n, uint32_t nw, uint32_t k, const KcSortScratch& w, cudaStream_t stream) {
    if (n < 2) return KC_OK;
    if (nw == 1 && k <= 32) return sort_impl<1, 1>(keys, n, k, w, stream);
    if (nw == 2 && k <= 64) return sort_impl<2, 2>(keys, n, k, w, stream);
    if (nw == 4 && k <= 128) return sort_impl<4, 4>(keys, n, k, w, stream);
    g_sort_err = "unsupported key width";
    return KC_ERR_INVALID;
}

const char* kc_sort_error() { return g_sort_err.c_str(); }
