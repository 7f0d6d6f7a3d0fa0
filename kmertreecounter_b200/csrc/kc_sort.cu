// Root-record radix sort (replaces sort/ExportRecordRadixSort.h:19-269), and
// the same sort over bare keys (post-processing's sorted low keys).
//
// The reference's LSD radix sort orders ExportRecord<N> by key with 8-bit
// digits, skipping bits shared by a leaf; here the records of all 256 root
// files sit in one array grouped by root id = top 8 key bits, so one stable
// LSD sort over the key's 2k significant bits orders every root file by key
// and keeps the grouping (the last pass is over the most significant bits).
//
// Onesweep form: one read of the input counts every digit of every pass at
// once (`hist_all`, then `scan_digits` turns the counts into each digit's
// first output position), and each pass is ONE kernel (`onesweep_pass`):
//   * a CTA takes the next tile in start order from a per-pass counter, so a
//     tile only ever waits on tiles whose CTAs are already running;
//   * it ranks its records stably (warp-striped items in input order,
//     __match_any_sync ranks equal digits inside a warp, per-warp digit
//     counts order the warps);
//   * it publishes its per-digit counts, then looks back over its
//     predecessors' published words (a count, or an inclusive prefix that
//     ends the walk) to find how many records of each digit come before it;
//   * it sorts the tile by digit in shared memory and writes it out as runs,
//     one per digit, at their global positions.
// Traffic per pass: one read and one write of every record; the look-back
// words are 2 KiB per tile.  Each look-back word carries the pass number, so
// the array is cleared once per sort, not once per pass.  Every wait on a
// predecessor is bounded: past the bound the CTA flags the error, writes
// nothing, and the call reports a device error.

#include <algorithm>
#include <cstdint>
#include <string>

#include <cuda_runtime.h>

#include "../../include/kmer_count.h"
#include "kc_internal.h"

namespace {

constexpr int SORT_THREADS = 256;
constexpr int NWARP = SORT_THREADS / 32;
constexpr int RADIX = 256;
constexpr uint32_t MAX_PASSES = 32;                 // 256-bit keys, 8-bit digits
constexpr int MIN_TILE = SORT_THREADS * 4;          // the smallest tile of any record width
constexpr uint32_t LOOK_SPINS = 1u << 20;           // polls of one predecessor's word before giving up
constexpr unsigned long long PREFIX_BIT = 1ull << 57;
constexpr unsigned long long VALUE_MASK = PREFIX_BIT - 1;

thread_local std::string g_sort_err;

// Records per thread of a tile, by record width in 64-bit words.
template <int W>
__host__ __device__ constexpr int items_of() {
    return W <= 2 ? 8 : 4;
}

// Dynamic shared memory of one pass: the tile's records (aliased with the
// per-warp digit counts, which are dead before the records are staged), the
// tile-local start of each digit and each digit's global destination base.
template <int W>
constexpr size_t pass_smem() {
    const size_t recs = (size_t)SORT_THREADS * items_of<W>() * 8 * W;
    const size_t cnts = (size_t)NWARP * RADIX * 4;
    return (recs > cnts ? recs : cnts) + RADIX * 4 + RADIX * 8;
}

// Digit at bit `bit` of a record's key taken as one (64*NW)-bit number
// (word 0 most significant).
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
        // (word picked by selects, not by a runtime index, so the record
        // stays in registers)
        const uint32_t wi = 3 - (bit >> 6), sh = bit & 63;
        const uint64_t lo = wi == 3 ? rec[3] : (wi == 2 ? rec[2] : (wi == 1 ? rec[1] : rec[0]));
        const uint64_t hi = wi == 3 ? rec[2] : (wi == 2 ? rec[1] : rec[0]);
        uint64_t v = lo >> sh;
        if (sh > 56 && wi > 0) v |= hi << (64 - sh);
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

__device__ __forceinline__ void st_relaxed(unsigned long long* p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_relaxed(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ uint32_t ld_relaxed(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Counts of every digit of every pass (hist[pass * 256 + digit]) in one read
// of the input.  A digit that is the same across the warp (the high digits of
// records grouped by root id) is added once by one lane.
template <int NW, int W>
__global__ void __launch_bounds__(SORT_THREADS) hist_all(const Rec<W>* __restrict__ in, uint64_t n, uint32_t lowbit,
                                                         uint32_t passes, unsigned long long* __restrict__ hist) {
    __shared__ uint32_t h[MAX_PASSES * RADIX];
    for (uint32_t i = threadIdx.x; i < passes * RADIX; i += SORT_THREADS) h[i] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const uint64_t stride = (uint64_t)gridDim.x * SORT_THREADS;
    for (uint64_t base = (uint64_t)blockIdx.x * SORT_THREADS; base < n; base += stride) {
        const uint64_t i = base + threadIdx.x;
        const uint32_t active = __ballot_sync(0xffffffffu, i < n);
        if (i >= n) continue;
        const Rec<W> r = in[i];
        const int first = __ffs(active) - 1;
        for (uint32_t p = 0; p < passes; ++p) {
            const uint32_t d = digit_of<NW>(r.w, lowbit + 8 * p);
            if (__all_sync(active, d == __shfl_sync(active, d, first))) {
                if (lane == first) atomicAdd(&h[p * RADIX + d], (uint32_t)__popc(active));
            } else {
                atomicAdd(&h[p * RADIX + d], 1u);
            }
        }
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < passes * RADIX; i += SORT_THREADS)
        if (h[i]) atomicAdd(&hist[i], (unsigned long long)h[i]);
}

// Digit counts -> first output position of each digit, one block per pass.
__global__ void __launch_bounds__(RADIX) scan_digits(unsigned long long* hist) {
    __shared__ unsigned long long wsum[RADIX / 32];
    unsigned long long* h = hist + (uint64_t)blockIdx.x * RADIX;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const unsigned long long v = h[tid];
    unsigned long long x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    unsigned long long add = 0;
    for (int w = 0; w < warp; ++w) add += wsum[w];
    h[tid] = add + x - v;
}

// One LSD pass over the digit at `bit`.  `digit_base` = this pass's first
// output position per digit; `look` = n_tiles x 256 look-back words (bits
// 63..58 the pass's epoch, bit 57 set for an inclusive prefix, bits 56..0
// the value); `tile_ctr` = this pass's tile counter (0 at launch).
template <int NW, int W>
__global__ void __launch_bounds__(SORT_THREADS) onesweep_pass(const Rec<W>* __restrict__ in, Rec<W>* __restrict__ out,
                                                              uint64_t n, uint32_t bit, uint32_t epoch,
                                                              const unsigned long long* __restrict__ digit_base,
                                                              unsigned long long* look, uint32_t* tile_ctr,
                                                              uint32_t* err) {
    constexpr int IT = items_of<W>();
    constexpr int TILE = SORT_THREADS * IT;
    constexpr size_t RECS = (size_t)TILE * sizeof(Rec<W>);
    constexpr size_t CNTS = (size_t)NWARP * RADIX * 4;
    constexpr size_t BODY = RECS > CNTS ? RECS : CNTS;
    extern __shared__ __align__(16) unsigned char smem[];
    Rec<W>* s_rec = reinterpret_cast<Rec<W>*>(smem);
    uint32_t* s_cnt = reinterpret_cast<uint32_t*>(smem);
    uint32_t* s_start = reinterpret_cast<uint32_t*>(smem + BODY);
    unsigned long long* s_dst = reinterpret_cast<unsigned long long*>(smem + BODY + RADIX * 4);
    __shared__ uint32_t s_tile, s_bad, s_wsum[NWARP];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) {
        s_tile = atomicAdd(tile_ctr, 1u);
        s_bad = 0;
    }
#pragma unroll
    for (int w = 0; w < NWARP; ++w) s_cnt[w * RADIX + tid] = 0;
    __syncthreads();
    const uint64_t tile = s_tile;
    const uint64_t t0 = tile * TILE;
    const uint64_t wb = t0 + (uint64_t)warp * 32 * IT;
    const uint32_t lt = (1u << lane) - 1u;
    uint32_t* wc = s_cnt + warp * RADIX;

    // warp-striped items: item `it` of lane l is record wb + 32 it + l, so a
    // warp's items in (it, lane) order are in input order
    Rec<W> r[IT];
    uint32_t rk[IT];
#pragma unroll
    for (int it = 0; it < IT; ++it) {
        const uint64_t i = wb + (uint64_t)it * 32 + lane;
        if (i < n) r[it] = in[i];
        rk[it] = 0;
    }
#pragma unroll
    for (int it = 0; it < IT; ++it) {
        const bool valid = wb + (uint64_t)it * 32 + lane < n;
        const uint32_t active = __ballot_sync(0xffffffffu, valid);
        uint32_t d = 0, same = 0, prev = 0;
        if (valid) {
            d = digit_of<NW>(r[it].w, bit);
            same = __match_any_sync(active, d);
            prev = wc[d];
        }
        __syncwarp();
        if (valid) {
            rk[it] = prev + __popc(same & lt);
            if ((same & lt) == 0) wc[d] = prev + __popc(same);
        }
        __syncwarp();
    }
    __syncthreads();

    // thread tid owns digit tid: exclusive prefix over the warps, tile count
    uint32_t run = 0;
#pragma unroll
    for (int w = 0; w < NWARP; ++w) {
        const uint32_t c = s_cnt[w * RADIX + tid];
        s_cnt[w * RADIX + tid] = run;
        run += c;
    }
    unsigned long long* mine = look + tile * RADIX + tid;
    const unsigned long long tag = (unsigned long long)epoch << 58;
    st_relaxed(mine, tag | (tile == 0 ? PREFIX_BIT : 0ull) | run);

    // tile-local start of each digit (exclusive scan over the digits)
    uint32_t x = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_wsum[warp] = x;

    // records of digit tid in earlier tiles
    unsigned long long before = 0;
    if (tile > 0) {
        uint64_t j = tile - 1;
        uint32_t spins = 0;
        for (;;) {
            const unsigned long long v = ld_relaxed(look + j * RADIX + tid);
            if ((v >> 58) != epoch) {
                ++spins;
                if (spins >= LOOK_SPINS || ((spins & 63) == 0 && ld_relaxed(err) != 0)) {
                    atomicOr(err, 1u);
                    s_bad = 1;
                    break;
                }
                if (spins > 8) __nanosleep(64);
                continue;
            }
            before += v & VALUE_MASK;
            if ((v & PREFIX_BIT) || j == 0) break;
            --j;
            spins = 0;
        }
        st_relaxed(mine, tag | PREFIX_BIT | (before + run));
    }
    __syncthreads();
    uint32_t start = 0;
    for (int w = 0; w < warp; ++w) start += s_wsum[w];
    start += x - run;
    s_start[tid] = start;
    s_dst[tid] = digit_base[tid] + before - start;
    __syncthreads();

    // stage the tile sorted by digit, then write each digit's run
#pragma unroll
    for (int it = 0; it < IT; ++it)
        if (wb + (uint64_t)it * 32 + lane < n) {
            const uint32_t d = digit_of<NW>(r[it].w, bit);
            rk[it] += s_start[d] + wc[d];
        }
    __syncthreads();  // the per-warp counts are overwritten by the staged records
#pragma unroll
    for (int it = 0; it < IT; ++it)
        if (wb + (uint64_t)it * 32 + lane < n) s_rec[rk[it]] = r[it];
    __syncthreads();
    if (s_bad) return;
    const uint32_t cnt = (uint32_t)(n - t0 < (uint64_t)TILE ? n - t0 : (uint64_t)TILE);
    for (uint32_t s = tid; s < cnt; s += SORT_THREADS) {
        const Rec<W> v = s_rec[s];
        const unsigned long long dst = s_dst[digit_of<NW>(v.w, bit)] + s;
        if (dst < n) out[dst] = v;
        else atomicOr(err, 2u);
    }
}

template <int NW, int W>
int sort_impl(void* records, uint64_t n, uint32_t k, const KcSortScratch& w, cudaStream_t st) {
    using R = Rec<W>;
    constexpr int TILE = SORT_THREADS * items_of<W>();
    const uint32_t key_bits = 2 * k;
    const uint32_t lowbit = 64 * NW - key_bits;
    const uint32_t passes = (key_bits + 7) / 8;
    const uint64_t n_tiles = (n + TILE - 1) / TILE;
    R* a = static_cast<R*>(records);
    R* src = a;
    R* dst = static_cast<R*>(w.tmp);
    auto* look = static_cast<unsigned long long*>(w.hist);
    auto* hist = static_cast<unsigned long long*>(w.offs);
    auto* ctr = static_cast<uint32_t*>(w.sums);
    uint32_t* err = ctr + MAX_PASSES;
    int dev = 0, sms = 148;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaMemsetAsync(look, 0, n_tiles * RADIX * sizeof(unsigned long long), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(hist, 0, (uint64_t)passes * RADIX * sizeof(unsigned long long), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(ctr, 0, (MAX_PASSES + 1) * sizeof(uint32_t), st);
    if (e == cudaSuccess) {
        const uint64_t hgrid = std::min<uint64_t>((n + SORT_THREADS - 1) / SORT_THREADS, (uint64_t)sms * 4);
        hist_all<NW, W><<<(unsigned)hgrid, SORT_THREADS, 0, st>>>(src, n, lowbit, passes, hist);
        scan_digits<<<passes, RADIX, 0, st>>>(hist);
        for (uint32_t p = 0; p < passes; ++p) {
            onesweep_pass<NW, W><<<n_tiles, SORT_THREADS, pass_smem<W>(), st>>>(
                src, dst, n, lowbit + 8 * p, p + 1, hist + (uint64_t)p * RADIX, look, ctr + p, err);
            std::swap(src, dst);
        }
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && src != a) e = cudaMemcpyAsync(a, src, n * sizeof(R), cudaMemcpyDeviceToDevice, st);
    uint32_t h_err = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h_err, err, sizeof h_err, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        g_sort_err = cudaGetErrorString(e);
        return KC_ERR_DEVICE;
    }
    if (h_err) {
        g_sort_err = (h_err & 1u) ? "look-back wait on an earlier tile exceeded its bound"
                                  : "record destination outside the array";
        return KC_ERR_DEVICE;
    }
    return KC_OK;
}

}  // namespace

void kc_sort_scratch_bytes(uint64_t n, uint64_t record_bytes, uint64_t* tmp, uint64_t* hist, uint64_t* offs,
                           uint64_t* sums) {
    const uint64_t n_tiles = (n + MIN_TILE - 1) / MIN_TILE;
    *tmp = n * record_bytes;
    *hist = n_tiles * RADIX * sizeof(unsigned long long);         // look-back words
    *offs = (uint64_t)MAX_PASSES * RADIX * sizeof(unsigned long long);  // digit counts, then first positions
    *sums = 256;                                                  // tile counter per pass + error word
}

uint32_t kc_sort_launches(uint32_t k) { return 2 + (2 * k + 7) / 8; }

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
