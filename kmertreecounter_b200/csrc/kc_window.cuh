// Windowed count of 64-bit keys: first-occurrence filter and repeat table in
// shared memory.
//
// The count_routed kernel works on a bucket-sorted key array against the
// bucket's filter + table cells in global memory: every key costs a cell
// read and one or two atomics at L2 round-trip latency.  Here the keys of a
// bucket are grouped once more, by the slice of the bucket's table where
// their probe sequence starts (a window of WIN_Z cells), and one CTA per
// window stages the window's cells in shared memory, runs the filter test
// and the table insert of all its keys there, and writes the cells back:
// global traffic is the keys (read once, first occurrences written back in
// place) and each table cell read and written once per batch.
//
// The table layout and its probing rule are unchanged (one linear-probing
// table per bucket, the filter word of a key in the pad field of its first
// probe cell; src/BloomFilter.h:207-234 and src/ConcurrentMap.h:112-160 are
// the reference operations it replaces), so every other kernel (rehash,
// retry, export, histogram) reads the tables as before.  A probe sequence
// can run past its window into the next one; it never runs further than
// PROBE_LIMIT cells before the key counts as an overflow, so each window
// also stages the PROBE_LIMIT cells after it (the halo), and windows run in
// two phases (even, then odd windows of a bucket): no two CTAs of one phase
// stage the same cell.  A bucket table of at most WIN_Z cells is one window
// holding the whole table (probing wraps inside it).
//
//   subroute_count    keys per window, of every 16th chunk     (reads 8K/16)
//   window_caps, scan window ranges: estimate x 1.1 + 4 sigma + 64, in
//                     whole 64-key segments, then a spill area
//   subroute_scatter  keys into their window's range, staged    (reads 8K, writes 8K)
//                     in shared memory and written as runs; what
//                     a window cannot hold goes to the spill area
//   count_window x 2  filter + table in shared memory, per      (reads 8K + cells,
//                     64-key segment: first occurrences at the   writes L keys +
//                     front (seg_low), overflowed keys at the    cells)
//                     back (seg_fail), as count_routed leaves them
//   count_routed      the spill area's keys, in global memory
// Small batches, and a batch whose spill area overflows, take exact window
// counts (every chunk) instead: exact ranges, no spill.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "kc_kernels.cuh"

namespace kc {

constexpr int WIN_Z = 4096;                        // cells owned by one window
constexpr int WIN_HALO = PROBE_LIMIT;              // cells staged after it
constexpr int WIN_CELLS = WIN_Z + WIN_HALO;        // staged per CTA (16 B each: 73.7 KB)
constexpr uint32_t WIN_ZSHIFT = 12;                // log2(WIN_Z)
constexpr uint32_t WIN_SINGLE = 63;                // zshift of a one-window bucket
constexpr int WIN_THREADS = 512;
constexpr int WIN_SEG = 64;                        // count_seg<1>(): output segment of 64 keys
constexpr int WIN_GROUP = 1;                       // segments a warp loads at once
constexpr int SUB_THREADS = 256;
constexpr int SUB_ITEMS = 16;
constexpr int SUB_CHUNK = SUB_THREADS * SUB_ITEMS; // keys per subroute CTA
constexpr int SUB_BINS = 2048;                     // windows a chunk counts in shared memory

// Windows of one bucket: global window ids [range_base, range_base + S), the
// window of a key = ((hash >> 17) & tab_mask) >> zshift (WIN_SINGLE: 0).
struct BucketWin {
    uint32_t range_base;
    uint32_t zshift;
};
struct WinInfo {
    uint32_t bucket;
    uint32_t sub;
};

// Window of a key, with the chunk's first bucket's entries held in registers
// (a chunk's keys lie in that bucket but for a few at its edges).
struct WinCache {
    uint32_t bucket;
    BucketWin w;
    uint64_t mask;
};
__device__ __forceinline__ uint32_t window_of(uint64_t key, uint32_t bucket_shift, const WinCache& c,
                                              const BucketMeta* __restrict__ meta, const BucketWin* __restrict__ bw) {
    const uint32_t b = (uint32_t)(key >> bucket_shift);
    BucketWin w = c.w;
    uint64_t m = c.mask;
    if (b != c.bucket) {
        w = bw[b];
        m = __ldg(&meta[b].tab_mask);
    }
    const uint64_t cell = (hash_key(key) >> 17) & m;
    return w.range_base + (w.zshift >= WIN_SINGLE ? 0u : (uint32_t)(cell >> w.zshift));
}

// Smallest bucket of the chunk's keys (EMPTY keys skipped); 0xFFFFFFFF if none.
__device__ __forceinline__ uint32_t chunk_min_bucket(const uint64_t (&k)[SUB_ITEMS], uint32_t bucket_shift,
                                                     uint32_t* s_min) {
    uint32_t m = 0xFFFFFFFFu;
#pragma unroll
    for (int j = 0; j < SUB_ITEMS; ++j)
        if (k[j] != EMPTY) m = min(m, (uint32_t)(k[j] >> bucket_shift));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = min(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMin(s_min, m);
    __syncthreads();
    return *s_min;
}

// Keys per window.  A chunk's keys lie in one or a few buckets (the input is
// bucket-routed), so they are counted in shared memory relative to the first
// window of the chunk's smallest bucket; windows out of that span (keys of
// the extraction's overflow area, or a chunk spanning many tiny buckets) go
// to global atomics.
__global__ void __launch_bounds__(SUB_THREADS) subroute_count(const uint64_t* __restrict__ keys, uint64_t n,
                                                             const BucketMeta* __restrict__ meta,
                                                             const BucketWin* __restrict__ bw, uint32_t bucket_shift,
                                                             uint32_t chunk_stride, uint32_t* __restrict__ win_count) {
    __shared__ uint32_t hist[SUB_BINS];
    __shared__ uint32_t s_min;
    const uint64_t c0 = (uint64_t)blockIdx.x * chunk_stride * SUB_CHUNK;
    for (int i = threadIdx.x; i < SUB_BINS; i += SUB_THREADS) hist[i] = 0;
    if (threadIdx.x == 0) s_min = 0xFFFFFFFFu;
    uint64_t k[SUB_ITEMS];
#pragma unroll
    for (int j = 0; j < SUB_ITEMS; ++j) {
        const uint64_t i = c0 + (uint64_t)j * SUB_THREADS + threadIdx.x;
        k[j] = i < n ? __ldcs(keys + i) : EMPTY;
    }
    __syncthreads();
    const uint32_t bmin = chunk_min_bucket(k, bucket_shift, &s_min);
    if (bmin == 0xFFFFFFFFu) return;  // block-uniform: no key in this chunk
    const WinCache wc{bmin, bw[bmin], __ldg(&meta[bmin].tab_mask)};
    const uint32_t r0 = wc.w.range_base;
#pragma unroll
    for (int j = 0; j < SUB_ITEMS; ++j) {
        if (k[j] == EMPTY) continue;
        const uint32_t r = window_of(k[j], bucket_shift, wc, meta, bw);
        if (r - r0 < (uint32_t)SUB_BINS) atomicAdd(&hist[r - r0], 1u);
        else atomicAdd(&win_count[r], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < SUB_BINS; i += SUB_THREADS)
        if (hist[i]) atomicAdd(&win_count[r0 + i], hist[i]);
}

// Window capacities (keys, whole 64-key output segments).  Exact: the
// window's key count.  Estimated from every chunk_stride-th chunk of keys:
// est = sampled x stride, capacity = est x 1.1 + 4 sqrt(est) + 64; the keys a
// window receives beyond it go to the spill area.
__global__ void window_caps(const uint32_t* __restrict__ cnt, uint64_t n, uint32_t chunk_stride,
                            uint32_t* __restrict__ cap) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t c = cnt[i];
        if (chunk_stride > 1) {
            const double est = (double)c * (double)chunk_stride;
            c = (uint64_t)(est * 1.1 + 4.0 * sqrt(est) + 64.0);
        }
        cap[i] = (uint32_t)min((c + (WIN_SEG - 1)) & ~(uint64_t)(WIN_SEG - 1), (uint64_t)0xFFFFFFC0u);
    }
}

// cursor = start; end = start + cap, for every window.
__global__ void window_bounds(const uint64_t* __restrict__ start, const uint32_t* __restrict__ cap, uint64_t n,
                              uint64_t* __restrict__ cursor, uint64_t* __restrict__ end) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        cursor[i] = start[i];
        end[i] = start[i] + cap[i];
    }
}

constexpr int SCAT_THREADS = 512;
constexpr int SCAT_ITEMS = 8;
constexpr int SCAT_CHUNK = SCAT_THREADS * SCAT_ITEMS;  // 4096 keys
constexpr int SCAT_BINS = 1024;                         // windows staged in shared memory
// dynamic shared memory of subroute_scatter
constexpr size_t scatter_smem_bytes() {
    return (size_t)SCAT_CHUNK * 8 + (size_t)SCAT_CHUNK * 2 + (size_t)SCAT_BINS * (4 + 4 + 4 + 8 + 8) + 128;
}

struct ScatterArgs {
    const uint64_t* keys;
    uint64_t n;
    const BucketMeta* meta;
    const BucketWin* bw;
    uint32_t bucket_shift;
    unsigned long long* win_cursor;  // next free place of each window
    const uint64_t* win_end;         // end of each window's range
    unsigned long long* spill_cursor;
    uint64_t spill_end;
    uint32_t* spill_full;            // set when the spill area overflowed
    uint64_t* out;
};

// Keys into their window's range.  A chunk of 8192 keys is counted per
// window in shared memory, reserves one block per window it holds keys of
// (one global atomic per window and chunk; the part of a block past the
// window's capacity is reserved in the spill area instead), is staged in
// shared memory in window order, and leaves as contiguous runs.  Keys of
// windows outside the chunk's staged span are placed one by one.
__global__ void __launch_bounds__(SCAT_THREADS, 3) subroute_scatter(ScatterArgs a) {
    extern __shared__ __align__(16) uint8_t sc_smem[];
    uint64_t* stage = reinterpret_cast<uint64_t*>(sc_smem);
    uint16_t* stage_bin = reinterpret_cast<uint16_t*>(sc_smem + (size_t)SCAT_CHUNK * 8);
    uint32_t* hist = reinterpret_cast<uint32_t*>(sc_smem + (size_t)SCAT_CHUNK * 10);
    uint32_t* offs = hist + SCAT_BINS;
    uint32_t* avail = offs + SCAT_BINS;
    unsigned long long* gbase = reinterpret_cast<unsigned long long*>(avail + SCAT_BINS);
    unsigned long long* sbase = gbase + SCAT_BINS;
    uint32_t* misc = reinterpret_cast<uint32_t*>(sbase + SCAT_BINS);  // [0] min bucket, [1] staged total, [2..] scan
    const uint64_t c0 = (uint64_t)blockIdx.x * SCAT_CHUNK;
    for (int i = threadIdx.x; i < SCAT_BINS; i += SCAT_THREADS) hist[i] = 0;
    if (threadIdx.x == 0) misc[0] = 0xFFFFFFFFu;
    uint64_t k[SCAT_ITEMS];
#pragma unroll
    for (int j = 0; j < SCAT_ITEMS; ++j) {
        const uint64_t i = c0 + (uint64_t)j * SCAT_THREADS + threadIdx.x;
        k[j] = i < a.n ? __ldcs(a.keys + i) : EMPTY;
    }
    __syncthreads();
    {
        uint32_t m = 0xFFFFFFFFu;
#pragma unroll
        for (int j = 0; j < SCAT_ITEMS; ++j)
            if (k[j] != EMPTY) m = min(m, (uint32_t)(k[j] >> a.bucket_shift));
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = min(m, __shfl_xor_sync(0xffffffffu, m, o));
        if ((threadIdx.x & 31) == 0) atomicMin(&misc[0], m);
    }
    __syncthreads();
    const uint32_t bmin = misc[0];
    if (bmin == 0xFFFFFFFFu) return;  // block-uniform: no key in this chunk
    // the first bucket's entries in shared memory (registers are short here)
    __shared__ WinCache s_wc;
    if (threadIdx.x == 0) s_wc = WinCache{bmin, a.bw[bmin], a.meta[bmin].tab_mask};
    __syncthreads();
    const WinCache& wc = s_wc;
    const uint32_t r0 = wc.w.range_base;
    // per key: staged bin (high 16 bits) and place inside it (low 16), or
    // FAR for a window outside the staged span (placed one by one later)
    constexpr uint32_t FAR = 0xFFFFFFFFu;
    uint32_t slot[SCAT_ITEMS];
#pragma unroll
    for (int j = 0; j < SCAT_ITEMS; ++j) {
        slot[j] = FAR;
        if (k[j] == EMPTY) continue;
        const uint32_t l = window_of(k[j], a.bucket_shift, wc, a.meta, a.bw) - r0;
        if (l < (uint32_t)SCAT_BINS) slot[j] = (l << 16) | atomicAdd(&hist[l], 1u);
    }
    __syncthreads();
    // exclusive scan of the bins (2 per thread) -> staging offsets
    {
        const int t = threadIdx.x;
        const uint32_t h0 = hist[2 * t], h1 = hist[2 * t + 1];
        uint32_t v = h0 + h1, x = v;
        const int lane = t & 31, warp = t >> 5;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) misc[2 + warp] = x;
        __syncthreads();
        if (warp == 0) {
            uint32_t w = lane < SCAT_THREADS / 32 ? misc[2 + lane] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += y;
            }
            if (lane < SCAT_THREADS / 32) misc[2 + lane] = w;
        }
        __syncthreads();
        const uint32_t ex = (warp ? misc[2 + warp - 1] : 0) + x - v;
        offs[2 * t] = ex;
        offs[2 * t + 1] = ex + h0;
        if (t == SCAT_THREADS - 1) misc[1] = ex + v;
    }
    // reservations: the window's block, and the spill block for what does not fit
    for (int l = threadIdx.x; l < SCAT_BINS; l += SCAT_THREADS) {
        const uint32_t h = hist[l];
        avail[l] = 0;
        if (!h) continue;
        const unsigned long long g = atomicAdd(&a.win_cursor[r0 + l], (unsigned long long)h);
        const uint64_t end = a.win_end[r0 + l];
        const uint32_t fit = g >= end ? 0u : (uint32_t)min((uint64_t)h, (uint64_t)(end - g));
        gbase[l] = g;
        avail[l] = fit;
        if (fit < h) {
            const unsigned long long sp = atomicAdd(a.spill_cursor, (unsigned long long)(h - fit));
            sbase[l] = sp;
            if (sp + (h - fit) > a.spill_end) atomicOr(a.spill_full, 1u);
        }
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < SCAT_ITEMS; ++j) {
        if (k[j] == EMPTY) continue;
        if (slot[j] != FAR) {
            const uint32_t l = slot[j] >> 16;
            const uint32_t pos = offs[l] + (slot[j] & 0xFFFFu);
            stage[pos] = k[j];
            stage_bin[pos] = (uint16_t)l;
        } else {  // far window: one key at a time
            const uint32_t w = window_of(k[j], a.bucket_shift, wc, a.meta, a.bw);
            const unsigned long long g = atomicAdd(&a.win_cursor[w], 1ull);
            if (g < a.win_end[w]) {
                a.out[g] = k[j];
            } else {
                const unsigned long long sp = atomicAdd(a.spill_cursor, 1ull);
                if (sp < a.spill_end) a.out[sp] = k[j];
                else atomicOr(a.spill_full, 1u);
            }
        }
    }
    __syncthreads();
    const uint32_t staged = misc[1];
    for (uint32_t i = threadIdx.x; i < staged; i += SCAT_THREADS) {
        const uint32_t l = stage_bin[i];
        const uint32_t r = i - offs[l];
        if (r < avail[l]) {
            a.out[gbase[l] + r] = stage[i];
        } else {
            const uint64_t sp = sbase[l] + (r - avail[l]);
            if (sp < a.spill_end) a.out[sp] = stage[i];
        }
    }
}

struct WindowArgs {
    uint64_t* keys;                  // window-grouped keys (subroute_scatter's output)
    const uint64_t* win_start;       // first key of each window (multiple of WIN_SEG)
    const unsigned long long* win_fill;  // place after the last key the scatter put there
    const uint32_t* win_cap;         // capacity (multiple of WIN_SEG) of each window
    const WinInfo* wins;
    const uint32_t* order;           // windows in launch order (phase 0's, then phase 1's)
    uint32_t order_base;             // this launch's first entry of `order`
    const BucketWin* bw;
    const BucketMeta* meta;
    Slot1* table;                    // filter words in the cells' pad fields
    uint32_t* seg_low;               // per 64-key segment, as count_routed
    uint32_t* seg_fail;
    uint32_t* bucket_overflow;
    uint32_t phase;                  // 0: one-window buckets and even windows; 1: odd windows
};

// Asynchronous global -> shared copies (cp.async, L1-allocating for the
// 4- and 8-byte sizes) and the wait for all of this thread's copies.
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
    const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// One CTA per window of the current phase (the launch's list of windows).
__global__ void __launch_bounds__(WIN_THREADS, 3) count_window(WindowArgs a) {
    extern __shared__ __align__(16) uint8_t win_smem[];
    unsigned long long* s_key = reinterpret_cast<unsigned long long*>(win_smem);
    uint32_t* s_cnt = reinterpret_cast<uint32_t*>(win_smem + (size_t)WIN_CELLS * 8);
    uint32_t* s_pad = s_cnt + WIN_CELLS;

    const uint32_t r = a.order[a.order_base + blockIdx.x];
    const WinInfo wi = a.wins[r];
    const BucketWin bw = a.bw[wi.bucket];
    const bool single = bw.zshift >= WIN_SINGLE;
    if ((single ? 0u : (wi.sub & 1u)) != a.phase) return;  // never: the launch lists this phase's windows
    const uint64_t k0 = a.win_start[r];
    const uint32_t capk = a.win_cap[r];
    const uint32_t cnt = (uint32_t)min((unsigned long long)capk, a.win_fill[r] - k0);
    const uint32_t nseg = (cnt + WIN_SEG - 1) / WIN_SEG;
    // output segments of the window's range that hold no key (estimated
    // capacity beyond what arrived) report nothing
    for (uint32_t sg = nseg + threadIdx.x; sg < capk / WIN_SEG; sg += WIN_THREADS) {
        a.seg_low[k0 / WIN_SEG + sg] = 0;
        a.seg_fail[k0 / WIN_SEG + sg] = 0;
    }
    if (cnt == 0) return;  // block-uniform; the window's cells are left as they are
    const uint64_t M = a.meta[wi.bucket].tab_mask;
    Slot1* tab = a.table + a.meta[wi.bucket].tab_off;
    const uint64_t base = single ? 0 : ((uint64_t)wi.sub << bw.zshift);
    const uint32_t W = single ? (uint32_t)(M + 1) : (uint32_t)WIN_CELLS;

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int ITEMS = 2 * WIN_GROUP;  // keys per lane: 2 per segment
    constexpr uint32_t GSTEP = (WIN_THREADS / 32) * WIN_GROUP;
    // a warp's keys of segment group g (EMPTY past the window's keys); the
    // loads of the next group are issued before the current one is counted,
    // the first group's before the window's cells are staged
    auto load_group = [&](uint32_t g, uint64_t (&dst)[ITEMS]) {
#pragma unroll
        for (int j = 0; j < ITEMS; ++j) {
            const uint32_t idx = (g + j / 2) * WIN_SEG + (j & 1) * 32 + lane;
            dst[j] = (g < nseg && idx < cnt) ? __ldcs(a.keys + k0 + idx) : EMPTY;
        }
    };
    uint64_t nxt[ITEMS];
    load_group((uint32_t)warp * WIN_GROUP, nxt);

    // stage the window (wrapping at the table's end: the last window's
    // halo) with asynchronous copies straight into the shared-memory arrays,
    // every cell's copies in flight at once
    for (uint32_t i = threadIdx.x; i < W; i += WIN_THREADS) {
        const Slot1* src = tab + ((base + i) & M);
        cp_async8(&s_key[i], &src->key);
        cp_async4(&s_cnt[i], &src->count);
        cp_async4(&s_pad[i], &src->pad);
    }
    cp_async_wait_all();
    __syncthreads();

    const uint32_t lt = (1u << lane) - 1u;
    const uint32_t limit = (uint32_t)min((uint64_t)PROBE_LIMIT, M + 1);
    for (uint32_t g = (uint32_t)warp * WIN_GROUP; g < nseg; g += GSTEP) {
        uint64_t it[ITEMS];
        uint32_t mult[ITEMS];
#pragma unroll
        for (int j = 0; j < ITEMS; ++j) {
            const uint32_t idx = (g + j / 2) * WIN_SEG + (j & 1) * 32 + lane;
            mult[j] = idx < cnt ? 1u : 0u;
            it[j] = nxt[j];
        }
        load_group(g + GSTEP, nxt);  // other segments: never written below
        __syncwarp();  // every read of these segments precedes the in-place writes
        // hot keys arrive in runs: merge equal neighbours' keys first, so the
        // shared-memory atomics of a run are one per distinct key
#pragma unroll
        for (int j = 0; j < ITEMS; ++j) {
            const uint64_t nx = __shfl_down_sync(0xffffffffu, it[j], 1);
            if (!__any_sync(0xffffffffu, nx == it[j] && lane < 31 && mult[j] != 0)) continue;
            const uint32_t active = __ballot_sync(0xffffffffu, mult[j] != 0);
            if (mult[j]) {
                const uint32_t same = __match_any_sync(active, it[j]);
                mult[j] = ((__ffs(same) - 1) == lane) ? (uint32_t)__popc(same) : 0u;
            }
        }
        uint32_t first_bits = 0, fail_bits = 0;
#pragma unroll
        for (int j = 0; j < ITEMS; ++j) {
            if (!mult[j]) continue;
            const uint64_t h = hash_key(it[j]);
            const uint32_t local = (uint32_t)(((h >> 17) & M) - base);  // < WIN_Z (or < M + 1 for one window)
            const uint32_t bits = bloom_bits32(h);
            const uint32_t old = atomicOr(&s_pad[local], bits);
            uint32_t reps = mult[j];
            if ((old & bits) != bits) {
                first_bits |= 1u << j;
                --reps;
            }
            if (!reps) continue;
            bool done = false;
            for (uint32_t p = 0; p < limit; ++p) {
                const uint32_t c = single ? (uint32_t)((local + p) & M) : local + p;
                unsigned long long cur = *reinterpret_cast<volatile unsigned long long*>(&s_key[c]);
                if (cur == EMPTY) {
                    cur = atomicCAS(&s_key[c], EMPTY, (unsigned long long)it[j]);
                    if (cur == EMPTY) cur = it[j];
                }
                if (cur == it[j]) {
                    atomicAdd(&s_cnt[c], reps);
                    done = true;
                    break;
                }
            }
            if (!done) {
                fail_bits |= 1u << j;
                mult[j] = reps;  // occurrences still to add after the table grows
                a.bucket_overflow[wi.bucket] = 1u;
            }
        }
        // per 64-key segment, as count_routed: first occurrences at the front,
        // keys that met a full probe window at the back (one copy per
        // occurrence still to add)
#pragma unroll
        for (int s = 0; s < WIN_GROUP; ++s) {
            const uint32_t seg = g + s;
            if (seg >= nseg) break;  // warp-uniform
            const uint64_t s0 = k0 + (uint64_t)seg * WIN_SEG;
            const uint64_t s_end = s0 + WIN_SEG;
            uint32_t n_low = 0, n_fail = 0;
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const int j = 2 * s + q;
                const bool first = (first_bits >> j) & 1u;
                const uint32_t lm = __ballot_sync(0xffffffffu, first);
                if (first) a.keys[s0 + n_low + __popc(lm & lt)] = it[j];
                n_low += __popc(lm);
            }
            if (__any_sync(0xffffffffu, ((fail_bits >> (2 * s)) & 3u) != 0)) {
#pragma unroll
                for (int q = 0; q < 2; ++q) {
                    const int j = 2 * s + q;
                    const uint32_t f = ((fail_bits >> j) & 1u) ? mult[j] : 0u;
                    uint32_t fsum = f;
#pragma unroll
                    for (int o = 1; o < 32; o <<= 1) {
                        const uint32_t y = __shfl_up_sync(0xffffffffu, fsum, o);
                        if (lane >= o) fsum += y;
                    }
                    const uint32_t wtot = __shfl_sync(0xffffffffu, fsum, 31);
                    const uint32_t my0 = n_fail + fsum - f;
                    for (uint32_t rr = 0; rr < f; ++rr) a.keys[s_end - 1 - (my0 + rr)] = it[j];
                    n_fail += wtot;
                }
            }
            if (lane == 0) {
                a.seg_low[s0 / WIN_SEG] = n_low;
                a.seg_fail[s0 / WIN_SEG] = n_fail;
            }
        }
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < W; i += WIN_THREADS) {
        const ulonglong2 v = make_ulonglong2(s_key[i], (uint64_t)s_cnt[i] | ((uint64_t)s_pad[i] << 32));
        __stcg(reinterpret_cast<ulonglong2*>(tab + ((base + i) & M)), v);
    }
}

constexpr size_t window_smem_bytes() { return (size_t)WIN_CELLS * 16; }

}  // namespace kc
