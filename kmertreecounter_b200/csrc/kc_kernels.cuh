// Device kernels of the B200 exact canonical k-mer counter (sm_100a).
//
// Data flow of one batch of FASTQ bytes resident in HBM:
//
//   lines_per_tile      '\n' count of every 8 KiB tile            (reads F)
//   scan                line index at each tile start
//   extract<HIST>       canonical windows -> per-bucket totals    (reads F)
//   extract<SCATTER>    canonical windows -> bucket-contiguous    (reads F,
//                       routed key array                           writes 8N*K)
//   count_routed        first-occurrence filter + repeat tables   (reads 8N*K,
//                       on the routed array, bucket by bucket:     filter and
//                       the working set of in-flight CTAs stays    tables stay
//                       within one or two buckets, i.e. in L2      L2-resident)
//   retry_failed        re-insert keys whose table overflowed, after the host
//                       grew that bucket's table (rehash)
//   pack_low            first occurrences -> packed low.bin bytes
//   export_{count,write} table slots -> ExportRecord<N> grouped by root id
//
// Reference semantics are restated in the comments of each kernel with the
// file:line of ScorchShana/KmerTreeCounter they follow.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace kc {

constexpr int EXT_THREADS = 256;                     // extraction CTA
constexpr int EXT_BPT = 32;                          // bytes per thread
constexpr int EXT_TILE = EXT_THREADS * EXT_BPT;      // 8 KiB per CTA
constexpr int HALO = 64;                             // bytes kept before a batch
constexpr int CNT_THREADS = 256;                     // count CTA
constexpr uint64_t EMPTY = ~0ull;                    // never a canonical key
constexpr int PROBE_LIMIT = 512;                     // linear-probe bound before overflow

// One 128-bit key word pair in the reference's kmer<2> order: w0 = data[0]
// (most significant, first bases), w1 = data[1].
struct Key2 {
    uint64_t w0, w1;
};

// Per-bucket placement of the first-occurrence filter and the repeat table.
struct BucketMeta {
    uint64_t bloom_off;   // in 64-bit words
    uint64_t bloom_mask;  // words - 1 (power of two)
    uint64_t tab_off;     // in slots
    uint64_t tab_mask;    // slots - 1 (power of two)
};

// Repeat-table slots.  Slot1 has exactly the ExportRecord<1> layout
// {u64 key; u32 count; u32 pad} (src/definition.h:159-163).
struct __align__(16) Slot1 {
    uint64_t key;
    uint32_t count;
    uint32_t pad;
};
struct __align__(32) Slot2 {
    uint64_t w0, w1;
    uint32_t count;
    uint32_t pad[3];
};

// ---------------------------------------------------------------- helpers

__device__ __forceinline__ uint64_t mix64(uint64_t x) {
    // 64-bit finaliser of MurmurHash3 (Appleby, public domain).
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdull;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ull;
    x ^= x >> 33;
    return x;
}
__device__ __forceinline__ uint64_t hash_key(uint64_t k) { return mix64(k); }
__device__ __forceinline__ uint64_t hash_key(const Key2& k) {
    return mix64(k.w0 ^ mix64(k.w1 + 0x9e3779b97f4a7c15ull));
}

// Reverse the order of the 32 two-bit bases of a word (base p -> 31-p).
__device__ __forceinline__ uint64_t rev_bases(uint64_t x) {
    x = __brevll(x);
    return ((x >> 1) & 0x5555555555555555ull) | ((x & 0x5555555555555555ull) << 1);
}

// 2-bit code of an ASCII base: A/a=0 C/c=1 G/g=2 T/t/U/u=3 (src/GetKmer.h:22-37).
__device__ __forceinline__ uint32_t base_code(uint32_t c) { return ((c >> 1) ^ (c >> 2)) & 3u; }
__device__ __forceinline__ bool is_base(uint32_t c) {
    const uint32_t u = c & 0xDFu;  // fold lowercase, as src/FastqParser.h:211-230
    return u == 'A' || u == 'C' || u == 'G' || u == 'T' || u == 'U';
}

template <int NW>
struct KeyOf;
template <>
struct KeyOf<1> {
    using T = uint64_t;
};
template <>
struct KeyOf<2> {
    using T = Key2;
};

__device__ __forceinline__ uint64_t key_hi(uint64_t k) { return k; }
__device__ __forceinline__ uint64_t key_hi(const Key2& k) { return k.w0; }

// Canonical key of the window W (the last k bases, oldest base in the high
// bits of the 2k-bit value, newest in bits 1..0).
//
// The reference keeps two registers (src/GetKmer.h:58-82):
//   F = the window bases in REVERSE read order, not complemented, left-aligned
//   C = the complemented bases in read order, left-aligned
// and emits min(F, C) compared word by word (src/GetKmer.h:181-207).  With W
// as defined here F = rev_bases(W) (left-aligned by the reversal itself) and
// C = (~W masked to 2k bits) << (64N - 2k).
__device__ __forceinline__ uint64_t canonical1(uint64_t W, uint32_t k) {
    const uint64_t F = rev_bases(W);
    const uint64_t C = (k == 32) ? ~W : ((~W) << (64 - 2 * k));
    return F < C ? F : C;
}
__device__ __forceinline__ Key2 canonical2(uint64_t Whi, uint64_t Wlo, uint32_t k) {
    // F = base-reverse of the 128-bit (Whi:Wlo); the window occupies the low
    // 2k bits so the reversal lands it left-aligned.
    Key2 F{rev_bases(Wlo), rev_bases(Whi)};
    // C = ~W in 2k bits, shifted left by 128 - 2k (k in 33..64 -> 0..62).
    const uint32_t s = 128 - 2 * k;
    const uint64_t nhi = ~Whi, nlo = ~Wlo;
    Key2 C;
    if (s == 0) {
        C.w0 = nhi;
        C.w1 = nlo;
    } else {
        C.w0 = (nhi << s) | (nlo >> (64 - s));
        C.w1 = nlo << s;
    }
    const bool f_less = (F.w0 < C.w0) || (F.w0 == C.w0 && F.w1 < C.w1);
    return f_less ? F : C;
}

// ------------------------------------------------------------ block scans

// Exclusive scan of one uint32 per thread over a CTA of BLOCK threads.
template <int BLOCK>
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* smem_warp, uint32_t* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) smem_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < BLOCK / 32 ? smem_warp[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < BLOCK / 32) smem_warp[lane] = w;
    }
    __syncthreads();
    const uint32_t warp_prefix = warp ? smem_warp[warp - 1] : 0;
    if (total) *total = smem_warp[BLOCK / 32 - 1];
    const uint32_t r = warp_prefix + x - v;
    __syncthreads();
    return r;
}

// ------------------------------------------------------- FASTQ line split

// '\n' count per 8 KiB tile of the batch buf[0..n) (16-byte vector reads,
// byte reads for the ragged end).
__global__ void lines_per_tile(const uint8_t* __restrict__ buf, uint64_t n, uint32_t* __restrict__ tile_nl) {
    __shared__ uint32_t warp_sums[EXT_THREADS / 32];
    const uint64_t tile = blockIdx.x;
    const uint64_t pos = tile * EXT_TILE + (uint64_t)threadIdx.x * EXT_BPT;
    uint32_t cnt = 0;
    if (pos < n) {
        const uint64_t rem = n - pos;
        if (rem >= 32) {
            const uint4* p = reinterpret_cast<const uint4*>(buf + pos);
            const uint4 a = __ldcs(p), b = __ldcs(p + 1);
            const uint32_t w[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
            for (int i = 0; i < 8; ++i) cnt += __popc(__vcmpeq4(w[i], 0x0A0A0A0Au) & 0x01010101u);
        } else {
            for (uint32_t j = 0; j < (uint32_t)rem; ++j) cnt += buf[pos + j] == '\n';
        }
    }
    uint32_t total;
    block_exclusive_scan<EXT_THREADS>(cnt, warp_sums, &total);
    if (threadIdx.x == 0) tile_nl[tile] = total;
}

// ------------------------------------------------------- k-mer extraction

enum ExtractMode { HIST = 0, SCATTER = 1 };

// Classification of one thread's 32 bytes.
struct Seg {
    uint64_t codes;  // 2-bit codes, byte 0 in bits 63..62 (appending order)
    uint32_t bases;  // bit j set: byte j is A/C/G/T/U (either case)
    uint32_t nls;    // bit j set: byte j is '\n'
};

__device__ __forceinline__ Seg classify(const uint32_t (&w)[8], uint64_t valid_bytes) {
    Seg s{0, 0, 0};
#pragma unroll
    for (int i = 0; i < 8; ++i) {
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int j = 4 * i + b;
            const uint32_t c = (w[i] >> (8 * b)) & 0xFFu;
            const bool in = (uint64_t)j < valid_bytes;
            const bool base = in && is_base(c);
            s.codes = (s.codes << 2) | (base ? base_code(c) : 0u);
            s.bases |= (base ? 1u : 0u) << j;
            s.nls |= ((in && c == '\n') ? 1u : 0u) << j;
        }
    }
    return s;
}

// 32 bytes starting at p, of which only the first `avail` may be read (the
// rest read as 0).  Full segments use two 16-byte vector loads.
__device__ __forceinline__ void load32(const uint8_t* p, uint64_t avail, uint32_t (&w)[8]) {
    if (avail >= 32) {
        const uint4* q = reinterpret_cast<const uint4*>(p);
        const uint4 a = __ldcs(q), b = __ldcs(q + 1);
        w[0] = a.x; w[1] = a.y; w[2] = a.z; w[3] = a.w;
        w[4] = b.x; w[5] = b.y; w[6] = b.z; w[7] = b.w;
    } else {
#pragma unroll
        for (int i = 0; i < 8; ++i) w[i] = 0;
        for (uint32_t j = 0; j < (uint32_t)avail; ++j) w[j >> 2] |= (uint32_t)p[j] << (8 * (j & 3));
    }
}

// Length of the run of bases at the END of a 32-byte segment.
__device__ __forceinline__ uint32_t tail_run(uint32_t bases) { return __clz(~bases); }

struct ExtractArgs {
    const uint8_t* buf;      // batch start (16-byte aligned)
    uint64_t n;              // batch bytes
    int has_halo;            // buf[-HALO..-1] are the bytes before the batch
    const uint64_t* tile_line;  // line index at each tile start
    uint32_t k;
    uint32_t bucket_shift;   // 64 - log2(n_buckets)
    uint32_t n_buckets;
    unsigned long long* bucket_count;  // HIST: per-bucket totals (accumulated)
    unsigned long long* bucket_cursor; // SCATTER: next free index per bucket
    void* routed;            // SCATTER: routed key array
};

// Canonical k-mer extraction over one 8 KiB tile per CTA.
//
// Emission rule (reference: src/FastqReader.h:140-308 + src/FastqParser.h:
// 182-455 + src/GetKmer.h:58-131): a window ending at byte p is a k-mer iff
// p lies on a sequence line (line index = 1 mod 4 counted from the start of
// the file) and the k bytes ending at p are all bases.  A window never
// crosses '\n' because '\n' is not a base, so only p's line matters.
//
// Each thread owns 32 consecutive bytes.  The k-1 <= 63 bases before its
// first byte come from the two preceding segments, passed by warp shuffles
// (smem for lanes 0/1, whose predecessors sit in the previous warp or, for
// warp 0, in the 64-byte halo before the tile).
template <int NW, int MODE>
__global__ void __launch_bounds__(EXT_THREADS) extract_kernel(ExtractArgs a) {
    // dynamic smem: u64 base[n_buckets] | u32 hist[n_buckets] | u32 fill[n_buckets]
    extern __shared__ unsigned long long ext_smem[];
    __shared__ uint64_t tail_codes[EXT_THREADS / 32 + 1][2];
    __shared__ uint32_t tail_bases[EXT_THREADS / 32 + 1][2];
    __shared__ uint32_t warp_sums[EXT_THREADS / 32];
    unsigned long long* bbase = ext_smem;
    uint32_t* hist = reinterpret_cast<uint32_t*>(ext_smem + a.n_buckets);
    uint32_t* fill = hist + a.n_buckets;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint64_t tile_start = (uint64_t)blockIdx.x * EXT_TILE;
    const uint64_t seg_start = tile_start + (uint64_t)tid * EXT_BPT;

    for (uint32_t b = tid; b < a.n_buckets; b += EXT_THREADS) {
        hist[b] = 0;
        if (MODE == SCATTER) fill[b] = 0;
    }

    uint32_t w[8];
    const uint64_t valid = seg_start < a.n ? a.n - seg_start : 0;
    load32(a.buf + seg_start, valid, w);
    const Seg s = classify(w, valid);

    // Halo segments before the tile (before a batch start they are
    // buf[-HALO..-1] when has_halo, else no bases); only their bases matter,
    // a window that reaches them cannot contain a '\n'.
    if (warp == 0 && lane < 2) {
        uint32_t hw[8];
        const bool readable = tile_start > 0 || a.has_halo;
        load32(a.buf + (int64_t)tile_start - HALO + 32 * lane, readable ? 32 : 0, hw);
        const Seg h = classify(hw, readable ? 32 : 0);
        tail_codes[0][lane] = h.codes;
        tail_bases[0][lane] = h.bases;
    }
    if (lane >= 30) {
        tail_codes[warp + 1][lane - 30] = s.codes;
        tail_bases[warp + 1][lane - 30] = s.bases;
    }
    // line index at this thread's first byte
    uint32_t nl_total;
    const uint32_t nl_before = block_exclusive_scan<EXT_THREADS>(__popc(s.nls), warp_sums, &nl_total);
    (void)nl_total;  // block_exclusive_scan synchronised: tails are visible
    const uint32_t line0 = (uint32_t)a.tile_line[blockIdx.x] + nl_before;

    uint64_t p1c = __shfl_up_sync(0xffffffffu, s.codes, 1);
    uint64_t p2c = __shfl_up_sync(0xffffffffu, s.codes, 2);
    uint32_t p1b = __shfl_up_sync(0xffffffffu, s.bases, 1);
    uint32_t p2b = __shfl_up_sync(0xffffffffu, s.bases, 2);
    if (lane == 0) {
        p1c = tail_codes[warp][1];
        p1b = tail_bases[warp][1];
        p2c = tail_codes[warp][0];
        p2b = tail_bases[warp][0];
    } else if (lane == 1) {
        p2c = tail_codes[warp][1];
        p2b = tail_bases[warp][1];
    }

    // Does this segment touch a sequence line at all?  Lines inside the
    // segment are line0, line0+1, ...; a sequence line is = 1 (mod 4).
    const uint32_t nls = __popc(s.nls);
    bool any_seq = false;
#pragma unroll
    for (uint32_t d = 0; d < 4; ++d) any_seq |= (d <= nls) && (((line0 + d) & 3u) == 1u);
    any_seq &= (s.bases != 0);

    const uint32_t k = a.k;
    const uint64_t kmask1 = (k >= 32) ? ~0ull : ((1ull << (2 * k)) - 1ull);

    // Two passes in SCATTER mode: histogram, reservation, then placement.
#pragma unroll 1
    for (int pass = 0; pass < (MODE == SCATTER ? 2 : 1); ++pass) {
        if (pass == 1) {
            __syncthreads();
            for (uint32_t b = tid; b < a.n_buckets; b += EXT_THREADS) {
                const uint32_t c = hist[b];
                fill[b] = 0;
                bbase[b] = c ? atomicAdd(a.bucket_cursor + b, (unsigned long long)c) : 0ull;
            }
            __syncthreads();
        }
        if (any_seq) {
            uint64_t win_lo = p1c, win_hi = p2c;  // the 64 bases before byte 0
            uint32_t run = tail_run(p1b);
            if (run == 32) run += tail_run(p2b);
            uint32_t line = line0;
#pragma unroll 4
            for (int j = 0; j < 32; ++j) {
                const uint32_t code = (uint32_t)(s.codes >> (62 - 2 * j)) & 3u;
                const bool base = (s.bases >> j) & 1u;
                win_hi = (win_hi << 2) | (win_lo >> 62);
                win_lo = (win_lo << 2) | code;
                run = base ? run + 1 : 0;
                if (base && run >= k && (line & 3u) == 1u) {
                    uint32_t bucket;
                    typename KeyOf<NW>::T key;
                    if constexpr (NW == 1) {
                        key = canonical1(win_lo & kmask1, k);
                        bucket = (uint32_t)(key >> a.bucket_shift);
                    } else {
                        const uint32_t hb = 2 * k - 64;  // bits of the window in win_hi
                        const uint64_t hmask = hb >= 64 ? ~0ull : ((1ull << hb) - 1ull);
                        key = canonical2(win_hi & hmask, win_lo, k);
                        bucket = (uint32_t)(key.w0 >> a.bucket_shift);
                    }
                    if (MODE == HIST || pass == 0) {
                        atomicAdd(hist + bucket, 1u);
                    } else {
                        const uint32_t r = atomicAdd(fill + bucket, 1u);
                        typename KeyOf<NW>::T* out = reinterpret_cast<typename KeyOf<NW>::T*>(a.routed);
                        out[bbase[bucket] + r] = key;
                    }
                }
                if ((s.nls >> j) & 1u) ++line;
            }
        }
    }
    if (MODE == HIST) {
        __syncthreads();
        for (uint32_t b = tid; b < a.n_buckets; b += EXT_THREADS) {
            const uint32_t c = hist[b];
            if (c) atomicAdd(a.bucket_count + b, (unsigned long long)c);
        }
    }
}

// --------------------------------------------------- first occurrence + repeats

__device__ __forceinline__ uint64_t bloom_bits(uint64_t h) {
    // Three bit positions in one 64-bit word, taken from hash bits 40..57
    // (the word index uses the low bits).  The reference uses XXH3-128 and
    // (lo + i*(hi|1)) & 63 (src/BloomFilter.h:207-258); only the low/root
    // partition depends on this choice, never the merged counts.
    return (1ull << ((h >> 40) & 63)) | (1ull << ((h >> 46) & 63)) | (1ull << ((h >> 52) & 63));
}

// Insert `add` occurrences of key into a bucket table; false = probe limit hit.
__device__ __forceinline__ bool table_add(Slot1* __restrict__ tab, uint64_t mask, uint64_t h, uint64_t key,
                                          uint32_t add) {
    uint64_t i = (h >> 17) & mask;
    const int limit = (int)min((uint64_t)PROBE_LIMIT, mask + 1);
    for (int p = 0; p < limit; ++p) {
        Slot1* s = tab + ((i + p) & mask);
        uint64_t cur = __ldcg(&s->key);
        if (cur == EMPTY) {
            cur = atomicCAS(reinterpret_cast<unsigned long long*>(&s->key), EMPTY, key);
            if (cur == EMPTY) cur = key;
        }
        if (cur == key) {
            atomicAdd(&s->count, add);
            return true;
        }
    }
    return false;
}

__device__ __forceinline__ bool table_add(Slot2* __restrict__ tab, uint64_t mask, uint64_t h, const Key2& key,
                                          uint32_t add) {
    uint64_t i = (h >> 17) & mask;
    const int limit = (int)min((uint64_t)PROBE_LIMIT, mask + 1);
    for (int p = 0; p < limit; ++p) {
        Slot2* s = tab + ((i + p) & mask);
        const ulonglong2 v = __ldcg(reinterpret_cast<const ulonglong2*>(s));
        bool mine = (v.x == key.w0 && v.y == key.w1);
        // A slot goes EMPTY -> key exactly once.  A 16-byte read that shows an
        // EMPTY half may be torn, so ask the CAS for the authoritative value.
        if (!mine && (v.x == EMPTY || v.y == EMPTY)) {
            const unsigned __int128 e = ~(unsigned __int128)0;
            const unsigned __int128 kv = ((unsigned __int128)key.w1 << 64) | key.w0;
            const unsigned __int128 old = atomicCAS(reinterpret_cast<unsigned __int128*>(s), e, kv);
            mine = (old == e) || (old == kv);
        }
        if (mine) {
            atomicAdd(&s->count, add);
            return true;
        }
    }
    return false;
}

__device__ __forceinline__ bool key_eq(uint64_t a, uint64_t b) { return a == b; }
__device__ __forceinline__ bool key_eq(const Key2& a, const Key2& b) { return a.w0 == b.w0 && a.w1 == b.w1; }

template <int NW>
struct SlotOf;
template <>
struct SlotOf<1> {
    using T = Slot1;
};
template <>
struct SlotOf<2> {
    using T = Slot2;
};

template <int NW>
__host__ __device__ constexpr int count_items() {
    return NW == 1 ? 16 : 8;
}
template <int NW>
__host__ __device__ constexpr int count_tile() {
    return CNT_THREADS * count_items<NW>();
}

struct CountArgs {
    void* routed;                 // bucket-contiguous keys of this batch
    uint64_t n_keys;
    const BucketMeta* meta;
    uint64_t* bloom;
    void* table;
    uint32_t* tile_low;           // first occurrences kept at the tile front
    uint32_t* tile_fail;          // overflowed keys kept at the tile back
    uint32_t* bucket_overflow;    // set to 1 for a bucket whose table overflowed
    uint32_t bucket_shift;
    int use_filter;               // 0: retry pass (table only, no filter)
};

// One tile of routed keys per CTA: for each key, the first-occurrence filter
// decides low.bin (first) or the repeat table (seen before), as the
// reference's classifier does with ConcurrentBloomFilter::insert
// (src/FastqClassifier.h:241-349, src/BloomFilter.h:207-234): a relaxed read
// first, then fetch_or; "first" = the old word lacked one of the bits.
// Repeats increment the bucket's open-addressing table (replaces KmerTree +
// ConcurrentMap::increment, src/NewKmerTree.h:383-489,
// src/ConcurrentMap.h:112-160).
//
// Equal keys inside a warp are merged first (__match_any_sync): one filter
// probe and one table add per distinct key per warp.
//
// Outputs are compacted IN PLACE into the tile's own range of the routed
// array, after every key of the tile is in registers: first occurrences at
// the front, keys that met a full table at the back (for the retry pass).
template <int NW>
__global__ void __launch_bounds__(CNT_THREADS) count_routed(CountArgs a) {
    using K = typename KeyOf<NW>::T;
    using S = typename SlotOf<NW>::T;
    constexpr int ITEMS = count_items<NW>();
    constexpr int TILE = count_tile<NW>();
    __shared__ uint32_t s_low, s_fail;

    K* keys = reinterpret_cast<K*>(a.routed);
    const uint64_t t0 = (uint64_t)blockIdx.x * TILE;
    const uint64_t t_end = min(a.n_keys, t0 + TILE);
    uint64_t base = t0;
    uint32_t n_in = (uint32_t)(t_end - t0);
    if (!a.use_filter) {
        // retry pass: only the overflowed keys at the back of the tile
        const uint32_t nf = a.tile_fail[blockIdx.x];
        if (nf == 0) return;
        base = t_end - nf;
        n_in = nf;
    }
    const int tid = threadIdx.x, lane = tid & 31;
    if (tid == 0) {
        s_low = 0;
        s_fail = 0;
    }
    K item[ITEMS];
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        const uint32_t idx = (uint32_t)(j * CNT_THREADS + tid);
        if (idx < n_in) item[j] = keys[base + idx];
    }
    __syncthreads();  // every read of the tile precedes any in-place write

    const uint32_t fail_base_tile = (uint32_t)(t_end - t0);  // fail slots grow down from t_end
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        const uint32_t idx = (uint32_t)(j * CNT_THREADS + tid);
        const bool valid = idx < n_in;
        const uint32_t active = __ballot_sync(0xffffffffu, valid);
        if (!active) break;
        bool first = false;
        uint32_t fails = 0;
        K key = item[j];
        if (valid) {
            uint32_t same;
            if constexpr (NW == 1) {
                same = __match_any_sync(active, key);
            } else {
                same = __match_any_sync(active, key.w0) & __match_any_sync(active, key.w1);
            }
            const bool leader = (__ffs(same) - 1) == lane;
            if (leader) {
                const uint32_t mult = __popc(same);
                const uint32_t b = (uint32_t)(key_hi(key) >> a.bucket_shift);
                const BucketMeta m = a.meta[b];
                const uint64_t h = hash_key(key);
                uint32_t reps = mult;
                if (a.use_filter) {
                    uint64_t* word = a.bloom + m.bloom_off + (h & m.bloom_mask);
                    const uint64_t bits = bloom_bits(h);
                    uint64_t old = __ldcg(word);
                    if ((old & bits) != bits) old = atomicOr(reinterpret_cast<unsigned long long*>(word), bits);
                    first = (old & bits) != bits;
                    reps -= first ? 1u : 0u;
                }
                if (reps) {
                    S* tab = reinterpret_cast<S*>(a.table) + m.tab_off;
                    if (!table_add(tab, m.tab_mask, h, key, reps)) {
                        fails = reps;
                        a.bucket_overflow[b] = 1u;
                    }
                }
            }
        } else {
            // inactive lanes still take part in the warp-wide compaction below
        }
        // warp-aggregated reservations in the tile's low / fail regions
        const uint32_t lowmask = __ballot_sync(0xffffffffu, first);
        uint32_t low_base = 0;
        if (lowmask) {
            if (lane == 0) low_base = atomicAdd(&s_low, __popc(lowmask));
            low_base = __shfl_sync(0xffffffffu, low_base, 0);
            if (first) keys[t0 + low_base + __popc(lowmask & ((1u << lane) - 1u))] = key;
        }
        uint32_t fsum = fails;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, fsum, o);
            if (lane >= o) fsum += y;
        }
        const uint32_t wtotal = __shfl_sync(0xffffffffu, fsum, 31);
        if (wtotal) {
            uint32_t fb = 0;
            if (lane == 0) fb = atomicAdd(&s_fail, wtotal);
            fb = __shfl_sync(0xffffffffu, fb, 0);
            const uint32_t my0 = fb + fsum - fails;
            for (uint32_t r = 0; r < fails; ++r) keys[t0 + fail_base_tile - 1 - (my0 + r)] = key;
        }
    }
    __syncthreads();
    if (tid == 0) {
        if (a.use_filter) a.tile_low[blockIdx.x] = s_low;
        a.tile_fail[blockIdx.x] = s_fail;
    }
}

// Move every occupied slot of one bucket's old table into its new table.
template <int NW>
__global__ void rehash_bucket(const void* old_tab, uint64_t old_slots, void* new_tab, uint64_t new_mask,
                              uint32_t* failed) {
    using S = typename SlotOf<NW>::T;
    const S* src = reinterpret_cast<const S*>(old_tab);
    S* dst = reinterpret_cast<S*>(new_tab);
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < old_slots;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const S s = src[i];
        if constexpr (NW == 1) {
            if (s.key == EMPTY) continue;
            if (!table_add(dst, new_mask, hash_key(s.key), s.key, s.count)) atomicExch(failed, 1u);
        } else {
            if (s.w0 == EMPTY && s.w1 == EMPTY) continue;
            const Key2 k{s.w0, s.w1};
            if (!table_add(dst, new_mask, hash_key(k), k, s.count)) atomicExch(failed, 1u);
        }
    }
}

// Initialise table slots to EMPTY with count 0.
template <int NW>
__global__ void init_slots(void* tab, uint64_t n) {
    using S = typename SlotOf<NW>::T;
    S* t = reinterpret_cast<S*>(tab);
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        S s;
        if constexpr (NW == 1) {
            s.key = EMPTY;
            s.count = 0;
            s.pad = 0;
        } else {
            s.w0 = EMPTY;
            s.w1 = EMPTY;
            s.count = 0;
            s.pad[0] = s.pad[1] = s.pad[2] = 0;
        }
        t[i] = s;
    }
}

// ------------------------------------------------------------------ export

// low.bin packing (src/ExportWriter.h:522-550): k/32 full words as raw
// little-endian u64, then the top ceil(2(k%32)/8) bytes of the tail word
// (masked to its 2(k%32) high bits), in little-endian byte order.
template <int NW>
__global__ void pack_low(const void* routed, const uint32_t* tile_low, const uint64_t* tile_low_prefix,
                         uint64_t n_tiles, uint32_t tile_keys, uint32_t k, uint8_t* out, uint64_t out_base) {
    using K = typename KeyOf<NW>::T;
    const K* keys = reinterpret_cast<const K*>(routed);
    const uint32_t full = k / 32, tail_bits = 2 * (k % 32), tail_bytes = (tail_bits + 7) / 8;
    const uint32_t P = full * 8 + tail_bytes;
    const uint64_t tmask = tail_bits ? (~0ull << (64 - tail_bits)) : 0ull;
    for (uint64_t t = blockIdx.x; t < n_tiles; t += gridDim.x) {
        const uint32_t n = tile_low[t];
        const uint64_t o = out_base + tile_low_prefix[t];
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
            const K key = keys[t * (uint64_t)tile_keys + i];
            uint64_t w[2];
            if constexpr (NW == 1) {
                w[0] = key;
                w[1] = 0;
            } else {
                w[0] = key.w0;
                w[1] = key.w1;
            }
            uint8_t* d = out + (o + i) * P;
            if (P == 8 && full == 0) {
                *reinterpret_cast<uint64_t*>(d) = w[0] & tmask;
            } else if (P == 8) {
                *reinterpret_cast<uint64_t*>(d) = w[0];
            } else if (P == 16) {
                reinterpret_cast<uint64_t*>(d)[0] = w[0];
                reinterpret_cast<uint64_t*>(d)[1] = full == 2 ? w[1] : (w[1] & tmask);
            } else {
                uint32_t q = 0;
                for (uint32_t f = 0; f < full; ++f)
                    for (uint32_t b = 0; b < 8; ++b) d[q++] = (uint8_t)(w[f] >> (8 * b));
                if (tail_bytes) {
                    const uint64_t tw = w[full] & tmask;
                    for (uint32_t b = 8 - tail_bytes; b < 8; ++b) d[q++] = (uint8_t)(tw >> (8 * b));
                }
            }
        }
    }
}

// Work item of the table export: a range of one bucket's slots.
struct ExportChunk {
    uint64_t slot_begin;  // absolute slot index in the table arena
    uint32_t n_slots;
    uint32_t root;        // root file id of the bucket
};

// Count slots passing the filter min <= count <= max per root id
// (src/NewKmerTree.h:1159-1168) and occupied slots overall.
template <int NW>
__global__ void export_count(const void* table, const ExportChunk* chunks, uint64_t n_chunks, uint32_t min_c,
                             uint32_t max_c, unsigned long long* root_count, unsigned long long* occupied) {
    using S = typename SlotOf<NW>::T;
    __shared__ uint32_t s_pass, s_occ;
    const S* tab = reinterpret_cast<const S*>(table);
    for (uint64_t c = blockIdx.x; c < n_chunks; c += gridDim.x) {
        if (threadIdx.x == 0) {
            s_pass = 0;
            s_occ = 0;
        }
        __syncthreads();
        const ExportChunk ch = chunks[c];
        uint32_t pass = 0, occ = 0;
        for (uint32_t i = threadIdx.x; i < ch.n_slots; i += blockDim.x) {
            const S s = tab[ch.slot_begin + i];
            bool used;
            if constexpr (NW == 1) used = s.key != EMPTY;
            else used = !(s.w0 == EMPTY && s.w1 == EMPTY);
            occ += used;
            pass += used && s.count >= min_c && s.count <= max_c;
        }
        for (int o = 16; o; o >>= 1) {
            pass += __shfl_xor_sync(0xffffffffu, pass, o);
            occ += __shfl_xor_sync(0xffffffffu, occ, o);
        }
        if ((threadIdx.x & 31) == 0) {
            atomicAdd(&s_pass, pass);
            atomicAdd(&s_occ, occ);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            if (s_pass) atomicAdd(root_count + ch.root, (unsigned long long)s_pass);
            if (s_occ) atomicAdd(occupied, (unsigned long long)s_occ);
        }
        __syncthreads();
    }
}

// Write ExportRecord<N> {key words, count, pad = 0} into each root's segment.
template <int NW>
__global__ void export_write(const void* table, const ExportChunk* chunks, uint64_t n_chunks, uint32_t min_c,
                             uint32_t max_c, unsigned long long* root_cursor, uint8_t* records) {
    using S = typename SlotOf<NW>::T;
    __shared__ uint32_t s_n;
    __shared__ unsigned long long s_base;
    const S* tab = reinterpret_cast<const S*>(table);
    const int lane = threadIdx.x & 31;
    for (uint64_t c = blockIdx.x; c < n_chunks; c += gridDim.x) {
        const ExportChunk ch = chunks[c];
        // pass 1: count, reserve
        if (threadIdx.x == 0) s_n = 0;
        __syncthreads();
        uint32_t pass = 0;
        for (uint32_t i = threadIdx.x; i < ch.n_slots; i += blockDim.x) {
            const S s = tab[ch.slot_begin + i];
            bool used;
            if constexpr (NW == 1) used = s.key != EMPTY;
            else used = !(s.w0 == EMPTY && s.w1 == EMPTY);
            pass += used && s.count >= min_c && s.count <= max_c;
        }
        for (int o = 16; o; o >>= 1) pass += __shfl_xor_sync(0xffffffffu, pass, o);
        if (lane == 0 && pass) atomicAdd(&s_n, pass);
        __syncthreads();
        if (threadIdx.x == 0) {
            s_base = s_n ? atomicAdd(root_cursor + ch.root, (unsigned long long)s_n) : 0ull;
            s_n = 0;
        }
        __syncthreads();
        // pass 2: place
        for (uint32_t i0 = 0; i0 < ch.n_slots; i0 += blockDim.x) {
            const uint32_t i = i0 + threadIdx.x;
            bool keep = false;
            S s;
            if (i < ch.n_slots) {
                s = tab[ch.slot_begin + i];
                bool used;
                if constexpr (NW == 1) used = s.key != EMPTY;
                else used = !(s.w0 == EMPTY && s.w1 == EMPTY);
                keep = used && s.count >= min_c && s.count <= max_c;
            }
            const uint32_t m = __ballot_sync(0xffffffffu, keep);
            uint32_t wb = 0;
            if (lane == 0 && m) wb = atomicAdd(&s_n, __popc(m));
            wb = __shfl_sync(0xffffffffu, wb, 0);
            if (keep) {
                const unsigned long long r = s_base + wb + __popc(m & ((1u << lane) - 1u));
                if constexpr (NW == 1) {
                    uint4 v;
                    v.x = (uint32_t)s.key;
                    v.y = (uint32_t)(s.key >> 32);
                    v.z = s.count;
                    v.w = 0;
                    reinterpret_cast<uint4*>(records)[r] = v;
                } else {
                    uint64_t* d = reinterpret_cast<uint64_t*>(records + r * 24);
                    d[0] = s.w0;
                    d[1] = s.w1;
                    d[2] = (uint64_t)s.count;
                }
            }
        }
        __syncthreads();
    }
}

}  // namespace kc
