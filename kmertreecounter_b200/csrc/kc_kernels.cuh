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
//   grow_init,          after the host grew the overflowed buckets' tables
//   grow_move,          (all of them in one arena growth): move their keys,
//   count_routed        then re-insert the keys that met a full table
//     (table only)      (rehash_bucket: the same for one bucket)
//   pack_low            first occurrences -> packed low.bin bytes
//   export_count,       table slots -> ExportRecord<N> grouped by root id
//   export_write_bits   (per-chunk counts and a bitmap of passing slots, then
//                       one read of only those slots)
//
// Reference semantics are restated in the comments of each kernel with the
// file:line of ScorchShana/KmerTreeCounter they follow.
#pragma once

#include <cstdint>
#include <type_traits>
#include <cuda_runtime.h>

namespace kc {

#define KC_HD __host__ __device__ __forceinline__

// Bit reversal usable from host code (unit tests) and device code.
KC_HD uint32_t brev32(uint32_t x) {
#ifdef __CUDA_ARCH__
    return __brev(x);
#else
    x = ((x >> 1) & 0x55555555u) | ((x & 0x55555555u) << 1);
    x = ((x >> 2) & 0x33333333u) | ((x & 0x33333333u) << 2);
    x = ((x >> 4) & 0x0F0F0F0Fu) | ((x & 0x0F0F0F0Fu) << 4);
    x = ((x >> 8) & 0x00FF00FFu) | ((x & 0x00FF00FFu) << 8);
    return (x >> 16) | (x << 16);
#endif
}
KC_HD uint64_t brev64(uint64_t x) {
#ifdef __CUDA_ARCH__
    return __brevll(x);
#else
    return ((uint64_t)brev32((uint32_t)x) << 32) | brev32((uint32_t)(x >> 32));
#endif
}
KC_HD uint32_t popc32(uint32_t x) {
#ifdef __CUDA_ARCH__
    return (uint32_t)__popc(x);
#else
    return (uint32_t)__builtin_popcount(x);
#endif
}

// Position of the r-th (0-based) set bit of x, by halving with popcounts;
// always 0..31 (the export's bitmap walk).
KC_HD uint32_t nth_set_bit(uint32_t x, uint32_t r) {
    uint32_t pos = 0, c;
    c = popc32(x & 0xFFFFu);
    if (r >= c) { r -= c; pos += 16; x >>= 16; }
    c = popc32(x & 0xFFu);
    if (r >= c) { r -= c; pos += 8; x >>= 8; }
    c = popc32(x & 0xFu);
    if (r >= c) { r -= c; pos += 4; x >>= 4; }
    c = popc32(x & 0x3u);
    if (r >= c) { r -= c; pos += 2; x >>= 2; }
    if (r >= (x & 1u)) pos += 1;
    return pos;
}

constexpr int EXT_THREADS = 256;                     // extraction CTA
constexpr int EXT_BPT = 32;                          // bytes per thread
constexpr int EXT_TILE = EXT_THREADS * EXT_BPT;      // 8 KiB per CTA
constexpr int HALO = 128;                            // bytes kept before a batch (k - 1 <= 127)
constexpr int HALO_SEGS = HALO / 32;                 // extraction segments of halo
// The 256-bucket scatter staging area holds extraction to 4 CTAs per SM;
// telling the compiler so lets it use up to 64 registers (measured 6% faster
// than its default of 32).
constexpr int EXT_MIN_CTAS = 4;
// Bucket regions of a batch of at least EST_MIN_TILES tiles are sized from a
// histogram of every EST_STRIDE-th tile instead of all of them.
constexpr uint32_t EST_STRIDE = 32;
constexpr uint64_t EST_MIN_TILES = 4096;
constexpr int CNT_THREADS = 256;                     // count CTA
constexpr uint64_t EMPTY = ~0ull;                    // never a canonical key
constexpr int PROBE_LIMIT = 512;                     // linear-probe bound before overflow

// One 128-bit key word pair in the reference's kmer<2> order: w0 = data[0]
// (most significant, first bases), w1 = data[1].
struct Key2 {
    uint64_t w0, w1;
};
// 256-bit key (k = 65..128), kmer<4> order: w0 most significant.
struct Key4 {
    uint64_t w0, w1, w2, w3;
};

// One extraction tile of a multi-set batch: bytes [start, min(start + 8 KiB,
// end)) of read set `set`, whose k-mers are counted with `k` into buckets
// [set * n_buckets, (set + 1) * n_buckets).  first_tile = index of the set's
// first tile (line numbers restart there; no halo before it).
struct SetTile {
    uint64_t start, end;
    uint32_t set, k, first_tile, pad;
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
// 256-bit keys have no CAS of their width: a slot is claimed by a CAS of
// `state` (SLOT_EMPTY -> SLOT_WRITING); the owner writes the key and the first
// count and publishes them with a release of state = SLOT_READY.  A thread
// that meets a SLOT_WRITING slot waits for it (bounded) before comparing.
constexpr uint32_t SLOT_EMPTY = 0, SLOT_WRITING = 1, SLOT_READY = 2;
constexpr uint32_t PUBLISH_WAIT_LIMIT = 1u << 22;  // polls before a wait counts as a device error
struct __align__(16) Slot4 {
    uint64_t w0, w1, w2, w3;
    uint32_t count;
    uint32_t state;
    uint64_t mark;  // merged-histogram mark (hist_* kernels)
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
__device__ __forceinline__ uint64_t hash_key(const Key4& k) {
    return mix64(k.w0 ^ mix64(k.w1 ^ mix64(k.w2 ^ mix64(k.w3 + 0x9e3779b97f4a7c15ull))));
}

// Bit 7 of each byte of the result: that byte of x is zero.  Exact per byte:
// (b & 0x7F) + 0x7F carries into bit 7 unless the low seven bits are zero,
// and never out of the byte.
KC_HD uint32_t zero_bytes(uint32_t x) {
    const uint32_t t = ((x & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | x;
    return ~t & 0x80808080u;
}

// Bit 7 of byte j (j = 0..3) -> bit j of the result: the four flag bits sit
// at 7, 15, 23, 31; times 2^21 + 2^14 + 2^7 + 1 they meet at bits 28..31
// (the other products fall below bit 22 or out of the word).
KC_HD uint32_t gather_bit7(uint32_t f) { return (f * 0x00204081u) >> 28; }

// Reverse the order of the 32 two-bit bases of a word (base p -> 31-p).
KC_HD uint64_t rev_bases(uint64_t x) {
    x = brev64(x);
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
template <>
struct KeyOf<4> {
    using T = Key4;
};

__device__ __forceinline__ uint64_t key_hi(uint64_t k) { return k; }
__device__ __forceinline__ uint64_t key_hi(const Key2& k) { return k.w0; }
__device__ __forceinline__ uint64_t key_hi(const Key4& k) { return k.w0; }

// Canonical key of the window W (the last k bases, oldest base in the high
// bits of the 2k-bit value, newest in bits 1..0).
//
// The reference keeps two registers (src/GetKmer.h:58-82):
//   F = the window bases in REVERSE read order, not complemented, left-aligned
//   C = the complemented bases in read order, left-aligned
// and emits min(F, C) compared word by word (src/GetKmer.h:181-207).  With W
// as defined here F = rev_bases(W) (left-aligned by the reversal itself) and
// C = (~W masked to 2k bits) << (64N - 2k).
KC_HD uint64_t canonical1(uint64_t W, uint32_t k) {
    const uint64_t F = rev_bases(W);
    const uint64_t C = (k == 32) ? ~W : ((~W) << (64 - 2 * k));
    return F < C ? F : C;
}
KC_HD Key2 canonical2(uint64_t Whi, uint64_t Wlo, uint32_t k) {
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

// k = 65..128: the window is the 256-bit W3:W2:W1:W0 (W0 = the newest 32
// bases, oldest base highest), of which the low 2k bits are the k bases.
// F = base-reverse of all 256 bits (left-aligned by the reversal itself);
// C = (~W masked to 2k bits) << (256 - 2k); key = the lexicographic min.
KC_HD Key4 canonical4(uint64_t W0, uint64_t W1, uint64_t W2, uint64_t W3, uint32_t k) {
    const uint32_t kb = 2 * k;  // 130..256
    if (kb <= 192) {
        W3 = 0;
        if (kb < 192) W2 &= (1ull << (kb - 128)) - 1ull;
    } else if (kb < 256) {
        W3 &= (1ull << (kb - 192)) - 1ull;
    }
    const Key4 F{rev_bases(W0), rev_bases(W1), rev_bases(W2), rev_bases(W3)};
    // ~W restricted to the 2k bits
    uint64_t n0 = ~W0, n1 = ~W1, n2 = ~W2, n3 = ~W3;
    if (kb <= 192) {
        n3 = 0;
        if (kb < 192) n2 &= (1ull << (kb - 128)) - 1ull;
    } else if (kb < 256) {
        n3 &= (1ull << (kb - 192)) - 1ull;
    }
    // shift left by sh = 256 - 2k (0..126): whole words first, then bits
    const uint32_t sh = 256 - kb;
    if (sh >= 64) {
        n3 = n2;
        n2 = n1;
        n1 = n0;
        n0 = 0;
    }
    const uint32_t r = sh & 63;
    if (r) {
        n3 = (n3 << r) | (n2 >> (64 - r));
        n2 = (n2 << r) | (n1 >> (64 - r));
        n1 = (n1 << r) | (n0 >> (64 - r));
        n0 = n0 << r;
    }
    const Key4 C{n3, n2, n1, n0};
    bool f_less;
    if (F.w0 != C.w0) f_less = F.w0 < C.w0;
    else if (F.w1 != C.w1) f_less = F.w1 < C.w1;
    else if (F.w2 != C.w2) f_less = F.w2 < C.w2;
    else f_less = F.w3 < C.w3;
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

// ------------------------------------------------ control-path transfers
//
// Counts, cursors and flags move between host and device as kernels that
// read or write mapped pinned memory, and small fills run as kernels: the
// copy engines are kept for the bulk FASTQ and output copies, behind which a
// few-byte copy would otherwise wait.

static __global__ void copy_words(const uint32_t* __restrict__ src, uint32_t* __restrict__ dst, uint64_t n) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        dst[i] = src[i];
}

static __global__ void fill_words(uint32_t* __restrict__ dst, uint64_t n, uint32_t v) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        dst[i] = v;
}

// Zero n 16-byte units (16-byte aligned).
static __global__ void zero16(uint4* __restrict__ dst, uint64_t n) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        dst[i] = make_uint4(0u, 0u, 0u, 0u);
}

// ------------------------------------------------------- FASTQ line split

// '\n' count per 8 KiB tile of the batch buf[0..n) (16-byte vector reads,
// byte reads for the ragged end).
static __global__ void lines_per_tile(const uint8_t* __restrict__ buf, uint64_t n, uint32_t* __restrict__ tile_nl) {
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
            for (int i = 0; i < 8; ++i) cnt += __popc(zero_bytes(w[i] ^ 0x0A0A0A0Au));
        } else {
            for (uint32_t j = 0; j < (uint32_t)rem; ++j) cnt += buf[pos + j] == '\n';
        }
    }
    uint32_t total;
    block_exclusive_scan<EXT_THREADS>(cnt, warp_sums, &total);
    if (threadIdx.x == 0) tile_nl[tile] = total;
}

// '\n' count of each set tile (multi-set batches).
static __global__ void lines_per_set_tile(const uint8_t* __restrict__ buf, const SetTile* __restrict__ tiles,
                                          uint32_t* __restrict__ tile_nl) {
    __shared__ uint32_t warp_sums[EXT_THREADS / 32];
    const SetTile t = tiles[blockIdx.x];
    const uint64_t pos = t.start + (uint64_t)threadIdx.x * EXT_BPT;
    uint32_t cnt = 0;
    if (pos < t.end) {
        const uint64_t rem = t.end - pos;
        if (rem >= 32) {
            const uint4* p = reinterpret_cast<const uint4*>(buf + pos);
            const uint4 a = __ldcs(p), b = __ldcs(p + 1);
            const uint32_t w[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
            for (int i = 0; i < 8; ++i) cnt += __popc(zero_bytes(w[i] ^ 0x0A0A0A0Au));
        } else {
            for (uint32_t j = 0; j < (uint32_t)rem; ++j) cnt += buf[pos + j] == '\n';
        }
    }
    uint32_t total;
    block_exclusive_scan<EXT_THREADS>(cnt, warp_sums, &total);
    if (threadIdx.x == 0) tile_nl[blockIdx.x] = total;
}

// Line index at each tile start, counted from its own set's first byte.
static __global__ void rebase_set_lines(const uint64_t* __restrict__ global_prefix, const SetTile* __restrict__ tiles,
                                        uint64_t n_tiles, uint64_t* __restrict__ tile_line) {
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n_tiles; t += (uint64_t)gridDim.x * blockDim.x)
        tile_line[t] = global_prefix[t] - global_prefix[tiles[t].first_tile];
}

// ------------------------------------------------------- k-mer extraction

enum ExtractMode { HIST = 0, SCATTER = 1 };

// Classification of one thread's 32 bytes.
struct Seg {
    uint64_t codes;  // 2-bit codes, byte 0 in bits 63..62 (appending order)
    uint32_t bases;  // bit j set: byte j is A/C/G/T/U (either case)
    uint32_t nls;    // bit j set: byte j is '\n'
};

// Four bytes at a time: base test (A/C/G/T/U after folding case) by the
// exact zero-byte test of x ^ letter, newline likewise, 2-bit code by the
// ((c >> 1) ^ (c >> 2)) & 3 identity (A=0 C=1 G=2 T/U=3, either case).
KC_HD Seg classify(const uint32_t (&w)[8], uint64_t valid_bytes) {
    Seg s{0, 0, 0};
    uint32_t chi = 0, clo = 0;  // codes of bytes 0..15 (chi) and 16..31 (clo)
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const uint32_t x = w[i];
        const uint32_t u = x & 0xDFDFDFDFu;
        const uint32_t isb = zero_bytes(u ^ 0x41414141u) | zero_bytes(u ^ 0x43434343u) | zero_bytes(u ^ 0x47474747u) |
                             zero_bytes(u ^ 0x54545454u) | zero_bytes(u ^ 0x55555555u);
        const uint32_t isn = zero_bytes(x ^ 0x0A0A0A0Au);
        s.bases |= gather_bit7(isb) << (4 * i);
        s.nls |= gather_bit7(isn) << (4 * i);
        // codes of bytes 4i..4i+3 -> 8 bits, byte 4i in the high pair: the
        // 2-bit fields at 0, 8, 16, 24 times 2^30 + 2^20 + 2^10 + 1 land at
        // 30, 28, 26, 24 (the other products fall below bit 22 or out)
        const uint32_t code4 = ((x >> 1) ^ (x >> 2)) & 0x03030303u;
        const uint32_t c8 = (code4 * 0x40100401u) >> 24;
        if (i < 4) chi |= c8 << (24 - 8 * i);
        else clo |= c8 << (24 - 8 * (i - 4));
    }
    s.codes = ((uint64_t)chi << 32) | clo;
    if (valid_bytes < 32) {
        const uint32_t keep = valid_bytes ? (0xFFFFFFFFu >> (32 - (uint32_t)valid_bytes)) : 0u;
        s.bases &= keep;
        s.nls &= keep;
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

typedef unsigned __int128 u128;

// Bit i of the result: bits [i-k+1, i] of X are all set (bits below 0 read
// as clear).  Shift-AND doubling: R_2m = R_m & (R_m << m), then one
// overlapping step to reach k exactly.
__device__ __forceinline__ u128 runs_at_least(u128 X, uint32_t k) {
    u128 R = X;
    uint32_t have = 1;
    while (2 * have <= k) {
        R &= R << have;
        have *= 2;
    }
    if (have < k) R &= R << (k - have);
    return R;
}

// The same over five segments' base bits (b0 oldest .. b4 current, 160 bits)
// for k = 65..128: bit j of the result = the k bytes ending at byte j of b4
// are all bases.
KC_HD uint32_t runs_at_least5(uint32_t b0, uint32_t b1, uint32_t b2, uint32_t b3, uint32_t b4, uint32_t k) {
    uint64_t x0 = (uint64_t)b0 | ((uint64_t)b1 << 32), x1 = (uint64_t)b2 | ((uint64_t)b3 << 32), x2 = b4;
    auto and_shifted = [&](uint32_t n) {  // X &= X << n, 1 <= n <= 64
        uint64_t y0, y1, y2;
        if (n == 64) {
            y2 = x1;
            y1 = x0;
            y0 = 0;
        } else {
            y2 = (x2 << n) | (x1 >> (64 - n));
            y1 = (x1 << n) | (x0 >> (64 - n));
            y0 = x0 << n;
        }
        x0 &= y0;
        x1 &= y1;
        x2 &= y2;
    };
    uint32_t have = 1;
    while (2 * have <= k) {
        and_shifted(have);
        have *= 2;
    }
    if (have < k) and_shifted(k - have);
    return (uint32_t)x2;
}

// Bits of the 32 bytes that lie on sequence lines (line index = 1 mod 4),
// line0 = line index of byte 0, nls = newline bits.
__device__ __forceinline__ uint32_t sequence_mask(uint32_t line0, uint32_t nls) {
    uint32_t seq = 0, start = 0, line = line0, m = nls;
    for (;;) {
        const uint32_t end = m ? (uint32_t)__ffs(m) : 32u;  // bytes [start, end) share `line`
        if ((line & 3u) == 1u && end > start) {
            const uint32_t hi = end >= 32 ? 0xFFFFFFFFu : ((1u << end) - 1u);
            seq |= hi & ~((1u << start) - 1u);
        }
        if (!m) break;
        start = end;
        m &= m - 1;
        ++line;
    }
    return seq;
}

// Reverse the order of the nb two-bit bases in the low 2*nb bits of x.
KC_HD uint32_t rev_small(uint32_t x, uint32_t nb) {
    uint32_t r = brev32(x);
    r = ((r >> 1) & 0x55555555u) | ((r & 0x55555555u) << 1);
    return r >> (32 - 2 * nb);
}

// Window of the last k bases ending at byte j of segment s2 (segments s0,
// s1 precede it): low 64 bits and, for k > 32, the next 64 bits.
KC_HD void window_at(uint64_t s0, uint64_t s1, uint64_t s2, uint32_t j, uint64_t& lo,
                                          uint64_t& hi) {
    const uint32_t sh = 2 * (31 - j);  // 0..62
    if (sh == 0) {
        lo = s2;
        hi = s1;
    } else {
        lo = (s2 >> sh) | (s1 << (64 - sh));
        hi = (s1 >> sh) | (s0 << (64 - sh));
    }
}

// The 256-bit window of the last 128 bases ending at byte j of segment s4
// (segments s0..s3 precede it): W0 = the newest 32 bases.
KC_HD void window_at4(uint64_t s0, uint64_t s1, uint64_t s2, uint64_t s3, uint64_t s4, uint32_t j, uint64_t& W0,
                      uint64_t& W1, uint64_t& W2, uint64_t& W3) {
    const uint32_t sh = 2 * (31 - j);
    if (sh == 0) {
        W0 = s4;
        W1 = s3;
        W2 = s2;
        W3 = s1;
    } else {
        W0 = (s4 >> sh) | (s3 << (64 - sh));
        W1 = (s3 >> sh) | (s2 << (64 - sh));
        W2 = (s2 >> sh) | (s1 << (64 - sh));
        W3 = (s1 >> sh) | (s0 << (64 - sh));
    }
}

struct ExtractArgs {
    const SetTile* tiles;    // multi-set batch: per-tile descriptor (nullptr: one input)
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
    uint32_t* error;         // bit 0: a key's bucket disagreed with its reservation;
                             // bit 1: the overflow area was full (keys dropped)
    uint32_t tile_stride;    // HIST over every tile_stride-th tile only (0 or 1: all)
    // SCATTER into estimated regions: bucket b owns routed[cursor0[b], region_end[b]).
    // A CTA's run of bucket b that does not fit whole goes whole to the overflow
    // area routed[overflow_start, overflow_end) (cursor *overflow_cursor), and
    // region_fill[b] (atomicMin) records where the region stopped filling.
    // region_end == nullptr: the regions are exact (no overflow).
    const unsigned long long* region_end;
    unsigned long long* region_fill;
    unsigned long long* overflow_cursor;
    uint64_t overflow_start, overflow_end;
    // multi-set batch with estimated regions: per set s an overflow area
    // [set_ovf_start[s], set_ovf_end[s]) with cursor set_ovf_cursor[s]; the
    // region arrays are indexed by set x n_buckets + bucket
    const uint64_t* set_ovf_start;
    const uint64_t* set_ovf_end;
    unsigned long long* set_ovf_cursor;
    // HIST over the listed tiles only (nullptr: every tile_stride-th)
    const uint32_t* tile_list;
};

// Bucket of the canonical key of window (hi:lo) without building the key:
// the top B bits of min(F, C) equal min(top B bits of F, top B bits of C).
// top(F) = the newest B/2 bases reversed; top(C) = the oldest B/2 bases
// complemented.
KC_HD uint32_t bucket_of_window(uint64_t lo, uint64_t hi, uint32_t k, uint32_t B) {
    const uint32_t nb = B / 2;
    const uint32_t mask = (1u << B) - 1u;
    const uint32_t topF = k >= nb ? rev_small((uint32_t)lo & mask, nb) : (rev_small((uint32_t)lo & ((1u << (2 * k)) - 1u), k) << (B - 2 * k));
    uint32_t topC;
    const uint32_t lo_bit = 2 * k >= B ? 2 * k - B : 0;  // lowest bit of the oldest B/2 bases
    if (2 * k < B) {
        topC = ((~(uint32_t)lo) & ((1u << (2 * k)) - 1u)) << (B - 2 * k);
    } else if (lo_bit + B <= 64) {
        topC = (uint32_t)(~lo >> lo_bit) & mask;
    } else if (lo_bit >= 64) {
        topC = (uint32_t)(~hi >> (lo_bit - 64)) & mask;
    } else {
        topC = (uint32_t)(((~lo) >> lo_bit) | ((~hi) << (64 - lo_bit))) & mask;
    }
    return topF < topC ? topF : topC;
}

// Canonical k-mer extraction over one 8 KiB tile per CTA.
//
// Emission rule (reference: src/FastqReader.h:140-308 + src/FastqParser.h:
// 182-455 + src/GetKmer.h:58-131): a window ending at byte p is a k-mer iff
// p lies on a sequence line (line index = 1 mod 4 counted from the start of
// the file) and the k bytes ending at p are all bases.  A window never
// crosses '\n' because '\n' is not a base, so only p's line matters.
//
// Phase A, per thread (32 bytes): classify, then a bit-parallel emit mask:
//   run of >= k bases ending at byte j (shift-AND doubling over the bases
//   of this and the two preceding segments) AND byte j on a sequence line.
// Phase C, per position: round r covers bytes [256r, 256r+256) of the tile,
//   so a warp owns one 32-byte segment per round -- warps over quality and
//   header bytes skip uniformly.  The window comes from the segment's codes
//   and its two predecessors (shared memory; the two before the tile are the
//   64-byte halo).
// HIST: per-bucket totals via the bucket-only path.  SCATTER: bucket-only
// histogram, one reservation per bucket per CTA, then full keys written to
// routed[base[bucket] + rank].
// Keys of one SCATTER tile staged in shared memory (bucket-sorted) before
// they are written out as contiguous runs; keys beyond this go out directly.
// (3840 keys for 64-bit keys: an 8 KiB tile of 150 bp FASTQ holds ~3150, and
// 4 CTAs of the scatter still fit one SM's shared memory)
template <int NW>
__host__ __device__ constexpr int stage_keys() {
    return NW == 1 ? 3840 : (NW == 2 ? 2048 : 1024);
}

// Dynamic shared memory of extract_kernel.
template <int NW, int MODE>
__host__ __device__ constexpr size_t extract_smem_bytes(uint32_t n_buckets) {
    return (size_t)n_buckets * (8 + 4 + 4 + 4) + (MODE == SCATTER ? (size_t)stage_keys<NW>() * (8 * NW + 2 + 2) : 0);
}

template <int NW, int MODE>
__global__ void __launch_bounds__(EXT_THREADS, EXT_MIN_CTAS) extract_kernel(ExtractArgs a) {
    // dynamic smem: u64 base[nb] | u32 hist[nb] | u32 fill[nb] | u32 loff[nb]
    //               | SCATTER: K keys[stage] | u16 rank_or_bucket[stage] | u16 order[stage]
    extern __shared__ unsigned long long ext_smem[];
    // segment t of the tile is seg_*[t + HALO_SEGS]; the HALO_SEGS before it
    // hold the halo bytes (zero where there is nothing to read)
    __shared__ uint64_t seg_codes[EXT_THREADS + HALO_SEGS];
    __shared__ uint32_t seg_bases[EXT_THREADS + HALO_SEGS];
    __shared__ uint32_t seg_emit[EXT_THREADS];
    __shared__ uint32_t seg_first[EXT_THREADS];  // arrival index of the segment's first k-mer
    __shared__ uint32_t warp_sums[EXT_THREADS / 32];
    using K = typename KeyOf<NW>::T;
    constexpr int STAGE = stage_keys<NW>();
    unsigned long long* bbase = ext_smem;
    uint32_t* hist = reinterpret_cast<uint32_t*>(ext_smem + a.n_buckets);
    uint32_t* fill = hist + a.n_buckets;
    uint32_t* loff = fill + a.n_buckets;
    K* skeys = reinterpret_cast<K*>(loff + a.n_buckets + (a.n_buckets & 1));  // 8-byte aligned
    uint16_t* sbkt = reinterpret_cast<uint16_t*>(skeys + STAGE);  // two-pass: bucket; one pass: rank
    uint16_t* sorder = sbkt + STAGE;                               // one pass: arrival index by bucket order

    const int tid = threadIdx.x;
    const uint64_t tile = a.tile_list ? (uint64_t)a.tile_list[blockIdx.x]
                                      : (uint64_t)blockIdx.x * (a.tile_stride > 1 ? a.tile_stride : 1u);
    uint64_t tile_start = tile * EXT_TILE;
    uint64_t n_end = a.n;
    bool halo_ok = tile_start > 0 || a.has_halo;
    uint32_t k = a.k;
    uint64_t bucket_off = 0;
    uint32_t set = 0;
    if (a.tiles) {
        const SetTile t = a.tiles[tile];
        tile_start = t.start;
        n_end = t.end;
        halo_ok = t.first_tile != tile;
        set = t.set;
        k = t.k;
        bucket_off = (uint64_t)t.set * a.n_buckets;
    }
    const uint64_t seg_start = tile_start + (uint64_t)tid * EXT_BPT;
    const uint32_t B = 64 - a.bucket_shift;

    for (uint32_t b = tid; b < a.n_buckets; b += EXT_THREADS) {
        hist[b] = 0;
        fill[b] = 0;
    }

    // ---- phase A: classify own segment (+ the halo segments)
    uint32_t w[8];
    const uint64_t valid = seg_start < n_end ? n_end - seg_start : 0;
    load32(a.buf + seg_start, valid, w);
    const Seg s = classify(w, valid);
    seg_codes[tid + HALO_SEGS] = s.codes;
    seg_bases[tid + HALO_SEGS] = s.bases;
    if (tid < HALO_SEGS) {
        uint32_t hw[8];
        const bool readable = halo_ok;
        load32(a.buf + (int64_t)tile_start - HALO + 32 * tid, readable ? 32 : 0, hw);
        const Seg h = classify(hw, readable ? 32 : 0);
        seg_codes[tid] = h.codes;
        seg_bases[tid] = h.bases;
    }
    uint32_t nl_total;
    const uint32_t nl_before = block_exclusive_scan<EXT_THREADS>(__popc(s.nls), warp_sums, &nl_total);
    (void)nl_total;  // the scan synchronised the block: seg_* are visible
    const uint32_t line0 = (uint32_t)a.tile_line[tile] + nl_before;

    uint32_t emit = 0;
    if (s.bases) {
        const uint32_t seq = sequence_mask(line0, s.nls);
        if (seq & s.bases) {
            const uint32_t* sb = seg_bases + tid + HALO_SEGS;  // sb[0] = this segment
            if constexpr (NW == 4) {
                emit = runs_at_least5(sb[-4], sb[-3], sb[-2], sb[-1], s.bases, k) & seq;
            } else {
                const u128 X = ((u128)s.bases << 64) | ((u128)sb[-1] << 32) | (u128)sb[-2];
                emit = (uint32_t)(runs_at_least(X, k) >> 64) & seq;
            }
        }
    }
    seg_emit[tid] = emit;
    uint32_t n_tile;  // k-mers of the tile; the scan also publishes seg_emit
    seg_first[tid] = block_exclusive_scan<EXT_THREADS>(__popc(emit), warp_sums, &n_tile);
    __syncthreads();  // every segment's seg_first is read by another warp below
    if (!n_tile) {
        return;  // nothing to count in this tile (HIST adds nothing; SCATTER reserves nothing)
    }

    // ---- phase C
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const uint32_t lt = (1u << lane) - 1u;
    // canonical key and routing bucket of the window ending at byte `lane` of segment t
    auto full_key = [&](int t, K& key, uint32_t& bucket) {
        const uint64_t* sc = seg_codes + t + HALO_SEGS;  // sc[0] = segment t
        uint64_t lo, hi, w2 = 0, w3 = 0;
        if constexpr (NW == 4) window_at4(sc[-4], sc[-3], sc[-2], sc[-1], sc[0], (uint32_t)lane, lo, hi, w2, w3);
        else window_at(sc[-2], sc[-1], sc[0], (uint32_t)lane, lo, hi);
        if constexpr (NW == 1) {
            const uint64_t km = k >= 32 ? ~0ull : ((1ull << (2 * k)) - 1ull);
            key = canonical1(lo & km, k);
            bucket = (uint32_t)(key >> a.bucket_shift);
        } else if constexpr (NW == 2) {
            const uint32_t hb = 2 * k - 64;
            const uint64_t hmask = hb >= 64 ? ~0ull : ((1ull << hb) - 1ull);
            key = canonical2(hi & hmask, lo, k);
            bucket = (uint32_t)(key.w0 >> a.bucket_shift);
        } else {
            key = canonical4(lo, hi, w2, w3, k);
            bucket = (uint32_t)(key.w0 >> a.bucket_shift);
        }
    };
    // reserve each bucket's run in the routed array (bbase) and the local
    // offsets of the bucket-sorted staging area (loff), from hist
    auto reserve = [&]() {
        const uint32_t per = (a.n_buckets + EXT_THREADS - 1) / EXT_THREADS;
        uint32_t sum = 0;
        for (uint32_t q = 0; q < per; ++q) {
            const uint32_t b = tid * per + q;
            if (b < a.n_buckets) {
                const uint32_t c = hist[b];
                const uint64_t rb = bucket_off + b;  // the region (of this set)
                unsigned long long base = c ? atomicAdd(a.bucket_cursor + rb, (unsigned long long)c) : 0ull;
                if (a.region_end && c && base + c > a.region_end[rb]) {
                    // the run does not fit the region: it goes whole to the
                    // overflow area.  If that is full too, the batch is routed
                    // again (error bit 1) and the run lands, in bounds, at the
                    // overflow area's start (at least 65536 keys >= one run).
                    atomicMin(a.region_fill + rb, base);
                    // a multi-set batch has an overflow area per set
                    unsigned long long* const ocur = a.set_ovf_cursor ? a.set_ovf_cursor + set : a.overflow_cursor;
                    const uint64_t oend = a.set_ovf_cursor ? a.set_ovf_end[set] : a.overflow_end;
                    const uint64_t ostart = a.set_ovf_cursor ? a.set_ovf_start[set] : a.overflow_start;
                    const unsigned long long ob = atomicAdd(ocur, (unsigned long long)c);
                    if (ob + c <= oend) {
                        base = ob;
                    } else {
                        base = ostart;
                        atomicOr(a.error, 2u);
                    }
                }
                bbase[b] = base;
                sum += c;
            }
        }
        uint32_t run = block_exclusive_scan<EXT_THREADS>(sum, warp_sums, nullptr);
        for (uint32_t q = 0; q < per; ++q) {
            const uint32_t b = tid * per + q;
            if (b < a.n_buckets) {
                loff[b] = run;
                run += hist[b];
            }
        }
        __syncthreads();
    };

    if (MODE == SCATTER && n_tile <= (uint32_t)STAGE) {
        // One extraction pass: the bucket's shared-memory counter gives each
        // key its rank in the bucket and builds the tile histogram at once;
        // keys are staged in arrival order, then indexed in bucket order and
        // written out as contiguous runs.
#pragma unroll 1
        for (int r = 0; r < EXT_BPT; ++r) {
            const int t = r * (EXT_THREADS / 32) + warp;
            const uint32_t em = seg_emit[t];
            if (!em) continue;  // warp-uniform
            if (!((em >> lane) & 1u)) continue;
            K key;
            uint32_t bucket;
            full_key(t, key, bucket);
            const uint32_t arr = seg_first[t] + __popc(em & lt);
            if (arr >= n_tile) {  // cannot happen; reported, never written
                atomicOr(a.error, 1u);
                continue;
            }
            const uint32_t rnk = atomicAdd(hist + bucket, 1u);
            skeys[arr] = key;
            sbkt[arr] = (uint16_t)rnk;
        }
        __syncthreads();
        reserve();
        for (uint32_t i = tid; i < n_tile; i += EXT_THREADS) {
            const uint32_t b = (uint32_t)(key_hi(skeys[i]) >> a.bucket_shift);
            const uint32_t pos = loff[b] + sbkt[i];
            if (sbkt[i] < hist[b] && pos < n_tile) sorder[pos] = (uint16_t)i;
            else atomicOr(a.error, 1u);
        }
        __syncthreads();
        K* out = reinterpret_cast<K*>(a.routed);
        for (uint32_t p = tid; p < n_tile; p += EXT_THREADS) {
            const uint32_t i = sorder[p];
            if (i >= n_tile) {
                atomicOr(a.error, 1u);
                continue;
            }
            const K key = skeys[i];
            const uint32_t b = (uint32_t)(key_hi(key) >> a.bucket_shift);
            if (p - loff[b] < hist[b]) out[bbase[b] + (p - loff[b])] = key;  // inside the bucket's reservation
            else atomicOr(a.error, 1u);
        }
        return;
    }

    // Two passes (histogram, then keys; and the HIST kernel's only pass):
    // tiles with more k-mers than the staging area holds
#pragma unroll 1
    for (int pass = 0; pass < (MODE == SCATTER ? 2 : 1); ++pass) {
        if (pass == 1) reserve();
#pragma unroll 1
        for (int r = 0; r < EXT_BPT; ++r) {
            const int t = r * (EXT_THREADS / 32) + warp;  // segment owned by this warp this round
            const uint32_t em = seg_emit[t];
            if (!em) continue;  // warp-uniform
            if (!((em >> lane) & 1u)) continue;
            const uint64_t* sc = seg_codes + t + HALO_SEGS;  // sc[0] = segment t
            uint64_t lo, hi, w2 = 0, w3 = 0;
            if constexpr (NW == 4) window_at4(sc[-4], sc[-3], sc[-2], sc[-1], sc[0], (uint32_t)lane, lo, hi, w2, w3);
            else window_at(sc[-2], sc[-1], sc[0], (uint32_t)lane, lo, hi);
            if (pass == 0 && NW == 4) {
                // 256-bit keys: the bucket from the full canonical key
                const Key4 key4 = canonical4(lo, hi, w2, w3, k);
                atomicAdd(hist + (uint32_t)(key4.w0 >> a.bucket_shift), 1u);
            } else if (pass == 0) {
                if (NW == 1) {
                    const uint64_t km = k >= 32 ? ~0ull : ((1ull << (2 * k)) - 1ull);
                    lo &= km;
                } else {
                    const uint32_t hb = 2 * k - 64;
                    hi &= hb >= 64 ? ~0ull : ((1ull << hb) - 1ull);
                }
                atomicAdd(hist + bucket_of_window(lo, hi, k, B), 1u);
            } else {
                K key;
                uint32_t bucket;
                full_key(t, key, bucket);
                const uint32_t rnk = atomicAdd(fill + bucket, 1u);
                if (rnk < hist[bucket]) {
                    const uint32_t sidx = loff[bucket] + rnk;
                    if (sidx < (uint32_t)STAGE) {
                        skeys[sidx] = key;
                        sbkt[sidx] = (uint16_t)bucket;
                    } else {
                        reinterpret_cast<K*>(a.routed)[bbase[bucket] + rnk] = key;
                    }
                } else {
                    atomicOr(a.error, 1u);  // never write outside the reservation
                }
            }
        }
        __syncthreads();
        if (MODE == SCATTER && pass == 1) {
            // staged keys out as contiguous runs: consecutive slots of one
            // bucket go to consecutive routed positions
            uint32_t total = 0;
            for (uint32_t b = tid; b < a.n_buckets; b += EXT_THREADS) total += hist[b];
            for (int o = 16; o; o >>= 1) total += __shfl_xor_sync(0xffffffffu, total, o);
            if ((tid & 31) == 0) warp_sums[tid >> 5] = total;
            __syncthreads();
            total = 0;
            for (int w = 0; w < EXT_THREADS / 32; ++w) total += warp_sums[w];
            const uint32_t staged = min(total, (uint32_t)STAGE);
            K* out = reinterpret_cast<K*>(a.routed);
            for (uint32_t i = tid; i < staged; i += EXT_THREADS) {
                const uint32_t b = sbkt[i];
                out[bbase[b] + (i - loff[b])] = skeys[i];
            }
        }
    }
    if (MODE == HIST) {
        for (uint32_t b = tid; b < a.n_buckets; b += EXT_THREADS) {
            const uint32_t c = hist[b];
            if (c) atomicAdd(a.bucket_count + bucket_off + b, (unsigned long long)c);
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
// Three bit positions in a 32-bit filter word kept in a table cell (64-bit
// keys); hash bits 0..14, while the cell index uses bits 17 and up.
__device__ __forceinline__ uint32_t bloom_bits32(uint64_t h) {
    return (1u << (h & 31)) | (1u << ((h >> 5) & 31)) | (1u << ((h >> 10) & 31));
}

// Insert `add` occurrences of key into a bucket table starting at slot
// (h >> 17) & mask; false = probe limit hit.  Linear probing; a slot goes
// EMPTY -> key exactly once (CAS), counts only grow (atomicAdd).
static __device__ __noinline__ bool table_add_slow(Slot1* __restrict__ tab, uint64_t mask, uint64_t h, uint64_t key,
                                            uint32_t add, int first_p) {
    const uint64_t i = (h >> 17) & mask;
    const int limit = (int)min((uint64_t)PROBE_LIMIT, mask + 1);
    for (int p = first_p; p < limit; ++p) {
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

static __device__ __noinline__ bool table_add_slow(Slot2* __restrict__ tab, uint64_t mask, uint64_t h, const Key2 key,
                                            uint32_t add, int first_p) {
    const uint64_t i = (h >> 17) & mask;
    const int limit = (int)min((uint64_t)PROBE_LIMIT, mask + 1);
    for (int p = first_p; p < limit; ++p) {
        Slot2* s = tab + ((i + p) & mask);
        const ulonglong2 v = __ldcg(reinterpret_cast<const ulonglong2*>(s));
        bool mine = (v.x == key.w0 && v.y == key.w1);
        // A 16-byte read that shows an EMPTY half may be torn, so ask the CAS
        // for the authoritative value.
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

// Insert `add` occurrences of a 256-bit key, probing from (h >> 17) & mask.
// Returns 1 when added, 0 when the probe limit was hit (the bucket
// overflows), -1 when a slot stayed SLOT_WRITING for PUBLISH_WAIT_LIMIT polls.
static __device__ __noinline__ int table_add4(Slot4* __restrict__ tab, uint64_t mask, uint64_t h, const Key4& key,
                                              uint32_t add) {
    const uint64_t i = (h >> 17) & mask;
    const int limit = (int)min((uint64_t)PROBE_LIMIT, mask + 1);
    for (int p = 0; p < limit; ++p) {
        Slot4* s = tab + ((i + p) & mask);
        volatile uint32_t* state = &s->state;
        uint32_t st = *state;
        if (st == SLOT_EMPTY) {
            st = atomicCAS(&s->state, SLOT_EMPTY, SLOT_WRITING);
            if (st == SLOT_EMPTY) {  // claimed: key and first count, then publish
                s->w0 = key.w0;
                s->w1 = key.w1;
                s->w2 = key.w2;
                s->w3 = key.w3;
                s->count = add;
                __threadfence();
                atomicExch(&s->state, SLOT_READY);
                return 1;
            }
        }
        for (uint32_t n = 0; st == SLOT_WRITING; ++n) {
            if (n >= PUBLISH_WAIT_LIMIT) return -1;
            st = *state;
        }
        __threadfence();  // pairs with the owner's fence: its key words are visible
        const Key4 have{__ldcg(&s->w0), __ldcg(&s->w1), __ldcg(&s->w2), __ldcg(&s->w3)};
        if (have.w0 == key.w0 && have.w1 == key.w1 && have.w2 == key.w2 && have.w3 == key.w3) {
            atomicAdd(&s->count, add);
            return 1;
        }
    }
    return 0;
}

// Full insert (used by the table rehash).
__device__ __forceinline__ bool table_add(Slot1* tab, uint64_t mask, uint64_t h, uint64_t key, uint32_t add) {
    return table_add_slow(tab, mask, h, key, add, 0);
}
__device__ __forceinline__ bool table_add(Slot2* tab, uint64_t mask, uint64_t h, const Key2& key, uint32_t add) {
    return table_add_slow(tab, mask, h, key, add, 0);
}
__device__ __forceinline__ bool table_add(Slot4* tab, uint64_t mask, uint64_t h, const Key4& key, uint32_t add) {
    return table_add4(tab, mask, h, key, add) > 0;
}

// Probe-round helpers of count_routed (64- and 128-bit keys): a cell's key
// as read (16-byte reads of a 128-bit cell may be torn while it is claimed:
// any EMPTY half counts as empty and is settled by the CAS), the claim of a
// cell read empty (returns the cell's key after the CAS: `key` when this
// thread claimed it), and the match test.
__device__ __forceinline__ bool cell_empty(uint64_t v) { return v == EMPTY; }
__device__ __forceinline__ bool cell_empty(const ulonglong2& v) { return v.x == EMPTY || v.y == EMPTY; }
__device__ __forceinline__ bool cell_holds(uint64_t v, uint64_t key) { return v == key; }
__device__ __forceinline__ bool cell_holds(const ulonglong2& v, const Key2& key) {
    return v.x == key.w0 && v.y == key.w1;
}
__device__ __forceinline__ uint64_t read_cell(const Slot1* s) { return __ldcg(&s->key); }
__device__ __forceinline__ ulonglong2 read_cell(const Slot2* s) {
    return __ldcg(reinterpret_cast<const ulonglong2*>(s));
}
__device__ __forceinline__ uint64_t claim_cell(Slot1* s, uint64_t key) {
    const uint64_t old = atomicCAS(reinterpret_cast<unsigned long long*>(&s->key), EMPTY, key);
    return old == EMPTY ? key : old;
}
__device__ __forceinline__ ulonglong2 claim_cell(Slot2* s, const Key2& key) {
    const unsigned __int128 e = ~(unsigned __int128)0;
    const unsigned __int128 kv = ((unsigned __int128)key.w1 << 64) | key.w0;
    const unsigned __int128 old = atomicCAS(reinterpret_cast<unsigned __int128*>(s), e, kv);
    const unsigned __int128 now = old == e ? kv : old;
    return make_ulonglong2((uint64_t)now, (uint64_t)(now >> 64));
}

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
template <>
struct SlotOf<4> {
    using T = Slot4;
};

// Keys per lane of the count kernel and its CTAs per SM (the register budget
// is 65536 / (256 x CTAs)).  The kernel waits on L2 round trips, so resident
// warps hide more than items per lane: for 64-bit keys 2 items at 6 CTAs/SM
// (40 registers) ran 42.7 ms where 4 items at 4 CTAs ran 47.4 and 6 at 3 ran
// 58.3 (genome-scale step, same counts); for 128-bit keys 2 items at 4 CTAs
// ran 233 ms where 5 CTAs (48 registers) ran 246 (the full k=63 shape, ten
// passes over 48 GB of tables; at a tenth of that size 5 CTAs were ahead).
template <int NW>
__host__ __device__ constexpr int count_items() {
    return NW == 1 ? 2 : (NW == 2 ? 2 : 1);
}
template <int NW>
__host__ __device__ constexpr int count_min_ctas() {
    return NW == 1 ? 6 : (NW == 2 ? 4 : 4);
}
// Keys owned by one warp of the count kernel (a contiguous segment).
template <int NW>
__host__ __device__ constexpr int count_seg() {
    return 32 * count_items<NW>();
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
    uint32_t* seg_low;            // per warp segment: first occurrences kept at its front
    uint32_t* seg_fail;           // per warp segment: overflowed keys kept at its back
    uint32_t* bucket_overflow;    // set to 1 for a bucket whose table overflowed
    uint32_t* error;              // 256-bit keys: set when a slot was never published
    uint32_t bucket_shift;
    uint32_t n_buckets;
    int use_filter;               // 0: retry pass (table only, no filter)
    // 64-bit keys: the filter words are the pad fields of table cells
    // (bloom_off / bloom_mask count cells of the table arena)
    uint32_t filter_in_table;
    // multi-set batch: set s owns segments [set_seg_start[s], set_seg_start[s+1])
    // and buckets [s * set_buckets, (s + 1) * set_buckets); EMPTY keys are gaps
    const uint64_t* set_seg_start;
    uint32_t n_sets;
    uint32_t set_buckets;
};

// Bucket placement as read by the count kernel (shared memory copy).
struct MetaS {
    uint64_t bloom_off, tab_off;
    uint32_t bloom_mask, tab_mask;
};
constexpr int META_SMEM_BUCKETS = 256;
constexpr int CNT_SEGS_PER_WARP = 8;

// For each routed key: the first-occurrence filter decides low.bin (first)
// or the repeat table (seen before), as the reference's classifier does with
// ConcurrentBloomFilter::insert (src/FastqClassifier.h:241-349,
// src/BloomFilter.h:207-234): a relaxed read first, then fetch_or; "first" =
// the old word lacked one of the bits.  Repeats increment the bucket's
// open-addressing table (replaces KmerTree + ConcurrentMap::increment,
// src/NewKmerTree.h:383-489, src/ConcurrentMap.h:112-160).
//
// Persistent CTAs; each warp walks contiguous segments of count_seg<NW>()
// keys.  Per segment: equal keys inside the warp are merged
// (__match_any_sync); every item's filter word and first table slot are read
// together (one round trip settles most repeats); filter atomics and table
// adds follow.  Outputs are compacted IN PLACE into the warp's own segment
// (only this warp reads it; __syncwarp orders reads before writes): first
// occurrences at the front, keys that met a full table at the back.
template <int NW>
__global__ void __launch_bounds__(CNT_THREADS, count_min_ctas<NW>()) count_routed(CountArgs a) {
    using K = typename KeyOf<NW>::T;
    using S = typename SlotOf<NW>::T;
    // first table slot read ahead of the filter result (not for 256-bit keys,
    // whose slots are read under the publish protocol of table_add4)
    using Seen = typename std::conditional<NW == 1, uint64_t,
                                           typename std::conditional<NW == 2, ulonglong2, uint32_t>::type>::type;
    constexpr int ITEMS = count_items<NW>();
    constexpr int SEG = count_seg<NW>();
    __shared__ MetaS sm[META_SMEM_BUCKETS];
    const bool meta_in_smem = a.n_buckets <= META_SMEM_BUCKETS;
    if (meta_in_smem) {
        for (uint32_t b = threadIdx.x; b < a.n_buckets; b += blockDim.x) {
            const BucketMeta m = a.meta[b];
            sm[b] = MetaS{m.bloom_off, m.tab_off, (uint32_t)m.bloom_mask, (uint32_t)m.tab_mask};
        }
        __syncthreads();
    }
    auto meta_of = [&](uint32_t b) -> MetaS {
        if (meta_in_smem) return sm[b];
        const BucketMeta* m = a.meta + b;
        return MetaS{__ldg(&m->bloom_off), __ldg(&m->tab_off), (uint32_t)__ldg(&m->bloom_mask),
                     (uint32_t)__ldg(&m->tab_mask)};
    };

    K* keys = reinterpret_cast<K*>(a.routed);
    S* table = reinterpret_cast<S*>(a.table);
    const int lane = threadIdx.x & 31;
    const uint32_t lt = (1u << lane) - 1u;
    const uint64_t n_segs = (a.n_keys + SEG - 1) / SEG;
    // Each CTA owns CNT_SEGS_PER_WARP consecutive segments per warp; CTAs are
    // dispatched in blockIdx order, so the keys in flight stay within a narrow
    // window of the bucket-sorted array (one or two buckets' filter and table
    // lines live in L2 at a time).
    const uint64_t cta_seg0 = (uint64_t)blockIdx.x * (CNT_THREADS / 32) * CNT_SEGS_PER_WARP;
    const uint64_t cta_seg1 = min(n_segs, cta_seg0 + (uint64_t)(CNT_THREADS / 32) * CNT_SEGS_PER_WARP);
    for (uint64_t gw = cta_seg0 + (threadIdx.x >> 5); gw < cta_seg1; gw += CNT_THREADS / 32) {
        const uint64_t s0 = gw * SEG;
        const uint64_t s_end = min(a.n_keys, s0 + SEG);
        uint64_t base = s0;
        uint32_t n_in = (uint32_t)(s_end - s0);
        if (!a.use_filter) {
            const uint32_t nf = a.seg_fail[gw];
            if (nf == 0) continue;  // warp-uniform
            base = s_end - nf;
            n_in = nf;
        }

        uint32_t set_bucket0 = 0;
        if (a.n_sets) {
            uint32_t lo = 0, hi = a.n_sets;  // last set whose first segment <= gw
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) / 2;
                if (a.set_seg_start[mid] <= gw) lo = mid;
                else hi = mid;
            }
            set_bucket0 = lo * a.set_buckets;
        }
        K it[ITEMS];
        uint32_t mult[ITEMS];
#pragma unroll
        for (int j = 0; j < ITEMS; ++j) {
            const uint32_t idx = (uint32_t)(j * 32 + lane);
            mult[j] = idx < n_in ? 1u : 0u;
            if constexpr (NW == 1) it[j] = EMPTY;
            else if constexpr (NW == 2) it[j] = Key2{EMPTY, EMPTY};
            else it[j] = Key4{EMPTY, EMPTY, EMPTY, EMPTY};
            if (mult[j]) {
                it[j] = keys[base + idx];
                if constexpr (NW == 1) mult[j] = it[j] != EMPTY;
                else if constexpr (NW == 2) mult[j] = !(it[j].w0 == EMPTY && it[j].w1 == EMPTY);
                else mult[j] = !(it[j].w0 == EMPTY && it[j].w1 == EMPTY && it[j].w2 == EMPTY && it[j].w3 == EMPTY);
            }
        }
        __syncwarp();  // every read of the segment precedes any in-place write

        // merge equal keys: the lowest lane of a group carries the multiplicity.
        // Equal keys inside one segment arrive in runs (a hot k-mer repeated
        // along a read lands in consecutive routed slots), so the full match
        // runs only when some lane's key equals its neighbour's; otherwise the
        // warp goes on with one atomic per key, which is exact either way.
#pragma unroll
        for (int j = 0; j < ITEMS; ++j) {
            bool eq_next;
            if constexpr (NW == 1) {
                const uint64_t nx = __shfl_down_sync(0xffffffffu, it[j], 1);
                eq_next = nx == it[j];
            } else if constexpr (NW == 2) {
                const uint64_t n0 = __shfl_down_sync(0xffffffffu, it[j].w0, 1);
                const uint64_t n1 = __shfl_down_sync(0xffffffffu, it[j].w1, 1);
                eq_next = n0 == it[j].w0 && n1 == it[j].w1;
            } else {
                const uint64_t n0 = __shfl_down_sync(0xffffffffu, it[j].w0, 1);
                const uint64_t n1 = __shfl_down_sync(0xffffffffu, it[j].w1, 1);
                const uint64_t n2 = __shfl_down_sync(0xffffffffu, it[j].w2, 1);
                const uint64_t n3 = __shfl_down_sync(0xffffffffu, it[j].w3, 1);
                eq_next = n0 == it[j].w0 && n1 == it[j].w1 && n2 == it[j].w2 && n3 == it[j].w3;
            }
            if (!__any_sync(0xffffffffu, eq_next && lane < 31 && mult[j] != 0)) continue;  // warp-uniform
            const uint32_t active = __ballot_sync(0xffffffffu, mult[j] != 0);
            if (mult[j]) {
                uint32_t same;
                if constexpr (NW == 1) same = __match_any_sync(active, it[j]);
                else if constexpr (NW == 2) same = __match_any_sync(active, it[j].w0) & __match_any_sync(active, it[j].w1);
                else
                    same = __match_any_sync(active, it[j].w0) & __match_any_sync(active, it[j].w1) &
                           __match_any_sync(active, it[j].w2) & __match_any_sync(active, it[j].w3);
                mult[j] = ((__ffs(same) - 1) == lane) ? (uint32_t)__popc(same) : 0u;
            }
        }

        // one round trip: filter word + first table slot of every item
        uint64_t h[ITEMS];
        uint64_t old[ITEMS];
        Seen seen[ITEMS];
#pragma unroll
        for (int j = 0; j < ITEMS; ++j) {
            if (mult[j]) {
                h[j] = hash_key(it[j]);
                const MetaS m = meta_of(set_bucket0 + (uint32_t)(key_hi(it[j]) >> a.bucket_shift));
                const S* slot = table + m.tab_off + ((h[j] >> 17) & m.tab_mask);
                if constexpr (NW == 1) {
                    if (a.filter_in_table) {
                        // the filter word is the cell's pad field, at the index
                        // of the first table probe: one 16-byte read gives key,
                        // count and filter bits unless the bucket's table has
                        // moved to a grown region (then the cells are filter only)
                        const ulonglong2 cv = __ldcg(reinterpret_cast<const ulonglong2*>(
                            table + m.bloom_off + ((h[j] >> 17) & m.bloom_mask)));
                        old[j] = cv.y >> 32;
                        seen[j] = m.bloom_off == m.tab_off ? cv.x : __ldcg(&slot->key);
                    } else {
                        if (a.use_filter) old[j] = __ldcg(a.bloom + m.bloom_off + (h[j] & m.bloom_mask));
                        seen[j] = __ldcg(&slot->key);
                    }
                } else {
                    if (a.use_filter) old[j] = __ldcg(a.bloom + m.bloom_off + (h[j] & m.bloom_mask));
                    if constexpr (NW == 2) seen[j] = __ldcg(reinterpret_cast<const ulonglong2*>(slot));
                    else seen[j] = 0;
                }
            }
        }
        uint32_t first_bits = 0;  // bit j: item j is a first occurrence
        if (a.use_filter) {
            // every item's filter atomic is issued before any old value is
            // tested (old[j] is replaced by the atomic's return value; an item
            // whose bits were all set already keeps its read value)
            bool in_table = false;
            if constexpr (NW == 1) in_table = a.filter_in_table != 0;
            uint32_t issued = 0;
#pragma unroll
            for (int j = 0; j < ITEMS; ++j) {
                if (mult[j]) {
                    const uint64_t bits = in_table ? (uint64_t)bloom_bits32(h[j]) : bloom_bits(h[j]);
                    if ((old[j] & bits) != bits) {
                        const MetaS m = meta_of(set_bucket0 + (uint32_t)(key_hi(it[j]) >> a.bucket_shift));
                        if constexpr (NW == 1) {
                            if (in_table)
                                old[j] = atomicOr(&(table + m.bloom_off + ((h[j] >> 17) & m.bloom_mask))->pad,
                                                  (uint32_t)bits);
                            else
                                old[j] = atomicOr(reinterpret_cast<unsigned long long*>(a.bloom + m.bloom_off +
                                                                                        (h[j] & m.bloom_mask)),
                                                  bits);
                        } else {
                            old[j] = atomicOr(
                                reinterpret_cast<unsigned long long*>(a.bloom + m.bloom_off + (h[j] & m.bloom_mask)), bits);
                        }
                        issued |= 1u << j;
                    }
                }
            }
#pragma unroll
            for (int j = 0; j < ITEMS; ++j) {
                if ((issued >> j) & 1u) {
                    const uint64_t bits = in_table ? (uint64_t)bloom_bits32(h[j]) : bloom_bits(h[j]);
                    if ((old[j] & bits) != bits) first_bits |= 1u << j;
                }
            }
        }
        uint32_t fail_bits = 0;
        if constexpr (NW == 4) {
#pragma unroll
            for (int j = 0; j < ITEMS; ++j) {
                const uint32_t reps = mult[j] - ((first_bits >> j) & 1u);
                if (mult[j] && reps) {
                    const uint32_t b = set_bucket0 + (uint32_t)(key_hi(it[j]) >> a.bucket_shift);
                    const MetaS m = meta_of(b);
                    const int r = table_add4(table + m.tab_off, m.tab_mask, h[j], it[j], reps);
                    if (r < 0) atomicOr(a.error, 1u);  // a slot was never published: reported, not retried
                    if (r == 0) {
                        fail_bits |= 1u << j;
                        mult[j] = reps;  // keep the count that still has to be added
                        a.bucket_overflow[b] = 1u;
                    }
                }
            }
        } else {
            // Repeats into the table by linear probing in lockstep rounds.
            // Round p settles every item whose probe cell p it has read
            // (`seen`; round 0 is the cell read with the filter word): the
            // claims of all items (CAS on a cell read EMPTY, or with an EMPTY
            // half for 128-bit keys) are issued before any result is used,
            // then items whose cell holds their key add their count, and items
            // that met another key read their next cell together.  A collision
            // in one lane costs the warp one more round for all its items,
            // not one more dependent chain per item.
            uint32_t todo = 0;
#pragma unroll
            for (int j = 0; j < ITEMS; ++j) {
                mult[j] = mult[j] ? mult[j] - ((first_bits >> j) & 1u) : 0u;  // occurrences left to add
                if (mult[j]) todo |= 1u << j;
            }
            for (uint32_t p = 0;; ++p) {
#pragma unroll
                for (int j = 0; j < ITEMS; ++j) {
                    if (((todo >> j) & 1u) && cell_empty(seen[j])) {
                        const MetaS m = meta_of(set_bucket0 + (uint32_t)(key_hi(it[j]) >> a.bucket_shift));
                        seen[j] = claim_cell(table + m.tab_off + (((h[j] >> 17) + p) & m.tab_mask), it[j]);
                    }
                }
#pragma unroll
                for (int j = 0; j < ITEMS; ++j) {
                    if (!((todo >> j) & 1u)) continue;
                    const uint32_t b = set_bucket0 + (uint32_t)(key_hi(it[j]) >> a.bucket_shift);
                    const MetaS m = meta_of(b);
                    if (cell_holds(seen[j], it[j])) {
                        atomicAdd(&table[m.tab_off + (((h[j] >> 17) + p) & m.tab_mask)].count, mult[j]);
                        todo &= ~(1u << j);
                    } else if ((uint64_t)p + 1 >= min((uint64_t)PROBE_LIMIT, (uint64_t)m.tab_mask + 1)) {
                        fail_bits |= 1u << j;  // mult[j] keeps the count that still has to be added
                        todo &= ~(1u << j);
                        a.bucket_overflow[b] = 1u;
                    }
                }
                if (!__any_sync(0xffffffffu, todo != 0)) break;  // warp-uniform
#pragma unroll
                for (int j = 0; j < ITEMS; ++j) {
                    if ((todo >> j) & 1u) {
                        const MetaS m = meta_of(set_bucket0 + (uint32_t)(key_hi(it[j]) >> a.bucket_shift));
                        seen[j] = read_cell(table + m.tab_off + (((h[j] >> 17) + p + 1) & m.tab_mask));
                    }
                }
            }
        }

        // in-place compaction inside the warp's segment
        uint32_t n_low = 0, n_fail = 0;
#pragma unroll
        for (int j = 0; j < ITEMS; ++j) {
            const bool first = (first_bits >> j) & 1u;
            const uint32_t lm = __ballot_sync(0xffffffffu, first);
            if (first) keys[s0 + n_low + __popc(lm & lt)] = it[j];
            n_low += __popc(lm);
        }
        if (__any_sync(0xffffffffu, fail_bits != 0)) {
#pragma unroll
            for (int j = 0; j < ITEMS; ++j) {
                const uint32_t f = ((fail_bits >> j) & 1u) ? mult[j] : 0u;
                uint32_t fsum = f;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const uint32_t y = __shfl_up_sync(0xffffffffu, fsum, o);
                    if (lane >= o) fsum += y;
                }
                const uint32_t wtot = __shfl_sync(0xffffffffu, fsum, 31);
                const uint32_t my0 = n_fail + fsum - f;
                for (uint32_t r = 0; r < f; ++r) keys[s_end - 1 - (my0 + r)] = it[j];
                n_fail += wtot;
            }
        }
        if (lane == 0) {
            if (a.use_filter) a.seg_low[gw] = n_low;
            a.seg_fail[gw] = n_fail;
        }
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
        } else if constexpr (NW == 2) {
            if (s.w0 == EMPTY && s.w1 == EMPTY) continue;
            const Key2 k{s.w0, s.w1};
            if (!table_add(dst, new_mask, hash_key(k), k, s.count)) atomicExch(failed, 1u);
        } else {
            if (s.state != SLOT_READY) continue;
            const Key4 k{s.w0, s.w1, s.w2, s.w3};
            if (!table_add(dst, new_mask, hash_key(k), k, s.count)) atomicExch(failed, 1u);
        }
    }
}

// One bucket's table growth: its old table (old_off, old_slots slots) moves
// into a new table of new_mask + 1 slots at new_off (slot offsets in the
// table arena).
struct GrowJob {
    uint64_t old_off, old_slots, new_off, new_mask;
};

template <int NW>
__device__ __forceinline__ void init_slot(typename SlotOf<NW>::T& s) {
    if constexpr (NW == 1) {
        s.key = EMPTY;
        s.count = 0;
        s.pad = 0;
    } else if constexpr (NW == 2) {
        s.w0 = EMPTY;
        s.w1 = EMPTY;
        s.count = 0;
        s.pad[0] = s.pad[1] = s.pad[2] = 0;
    } else {
        s.w0 = s.w1 = s.w2 = s.w3 = 0;
        s.count = 0;
        s.state = SLOT_EMPTY;
        s.mark = 0;
    }
}

// Many growths at once: blockIdx.y = job; the new tables are initialised by
// grow_init, then grow_move moves every occupied old slot (failed[job] = 1
// when a key met a full probe window of the new table).
template <int NW>
__global__ void grow_init(void* table, const GrowJob* __restrict__ jobs) {
    using S = typename SlotOf<NW>::T;
    const GrowJob j = jobs[blockIdx.y];
    S* t = reinterpret_cast<S*>(table) + j.new_off;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= j.new_mask;
         i += (uint64_t)gridDim.x * blockDim.x) {
        S s;
        init_slot<NW>(s);
        t[i] = s;
    }
}

template <int NW>
__global__ void grow_move(void* table, const GrowJob* __restrict__ jobs, uint32_t* __restrict__ failed) {
    using S = typename SlotOf<NW>::T;
    const GrowJob j = jobs[blockIdx.y];
    const S* src = reinterpret_cast<const S*>(table) + j.old_off;
    S* dst = reinterpret_cast<S*>(table) + j.new_off;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < j.old_slots;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const S s = src[i];
        if constexpr (NW == 1) {
            if (s.key == EMPTY) continue;
            if (!table_add(dst, j.new_mask, hash_key(s.key), s.key, s.count)) failed[blockIdx.y] = 1u;
        } else if constexpr (NW == 2) {
            if (s.w0 == EMPTY && s.w1 == EMPTY) continue;
            const Key2 k{s.w0, s.w1};
            if (!table_add(dst, j.new_mask, hash_key(k), k, s.count)) failed[blockIdx.y] = 1u;
        } else {
            if (s.state != SLOT_READY) continue;
            const Key4 k{s.w0, s.w1, s.w2, s.w3};
            if (!table_add(dst, j.new_mask, hash_key(k), k, s.count)) failed[blockIdx.y] = 1u;
        }
    }
}

// Initialise table slots to EMPTY with count 0.
template <int NW>
__global__ void init_slots(void* tab, uint64_t n) {
    // the table as 16-byte words, each lane one coalesced word per step: a
    // slot is 1, 2 or 3 words, EMPTY keys are all ones, counts, padding,
    // the 256-bit slot's state (SLOT_EMPTY = 0) and mark are zeros
    using S = typename SlotOf<NW>::T;
    constexpr uint64_t Q = sizeof(S) / 16;
    static_assert(sizeof(S) % 16 == 0, "slots are whole 16-byte words");
    uint4* t = reinterpret_cast<uint4*>(tab);
    const uint64_t n16 = n * Q;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n16; i += (uint64_t)gridDim.x * blockDim.x) {
        uint4 v = make_uint4(0u, 0u, 0u, 0u);
        if constexpr (NW == 1) v = make_uint4(~0u, ~0u, 0u, 0u);           // {key = EMPTY, count, pad}
        else if constexpr (NW == 2) if ((i & 1) == 0) v = make_uint4(~0u, ~0u, ~0u, ~0u);  // {w0, w1} = EMPTY
        t[i] = v;
    }
}

// ------------------------------------------------------------------ export

// Bytes of one low.bin record for k.
KC_HD uint32_t kc_packed(uint32_t k) { return (k / 32) * 8 + (2 * (k % 32) + 7) / 8; }

// low.bin packing (src/ExportWriter.h:522-550): k/32 full words as raw
// little-endian u64, then the top ceil(2(k%32)/8) bytes of the tail word
// (masked to its 2(k%32) high bits), in little-endian byte order.
// One key packed at d (P bytes; full = k/32 whole words, tail_bytes of the
// masked tail word).
template <int NW>
KC_HD void pack_key(const typename KeyOf<NW>::T& key, uint8_t* d, uint32_t full,
                                         uint32_t tail_bytes, uint32_t P, uint64_t tmask) {
    // word f of the key (f < 4; words past the key's width read 0)
    auto word = [&](uint32_t f) -> uint64_t {
        if constexpr (NW == 1) {
            return f == 0 ? key : 0ull;
        } else if constexpr (NW == 2) {
            return f == 0 ? key.w0 : (f == 1 ? key.w1 : 0ull);
        } else {
            return f == 0 ? key.w0 : (f == 1 ? key.w1 : (f == 2 ? key.w2 : key.w3));
        }
    };
    if (P == 8) {
        *reinterpret_cast<uint64_t*>(d) = full ? word(0) : (word(0) & tmask);
    } else if (P == 16) {
        reinterpret_cast<uint64_t*>(d)[0] = word(0);
        reinterpret_cast<uint64_t*>(d)[1] = full == 2 ? word(1) : (word(1) & tmask);
    } else {
        // k/32 whole words little-endian, then the top tail_bytes bytes
        // of the masked tail word (src/ExportWriter.h:522-550): the record is
        // the little-endian byte string of the words w_0..w_{full-1}, t with
        // t = the masked tail word's top tail_bytes bytes.  d is a multiple
        // of P from an 8-byte aligned base, so it is aligned to P's lowest
        // set bit: stores of that width (1, 2 or 4 bytes) never straddle a
        // word of the string.
        const uint64_t t = tail_bytes ? (((full < 4 ? word(full) : 0ull) & tmask) >> (8 * (8 - tail_bytes))) : 0ull;
        auto sw = [&](uint32_t f) -> uint64_t { return f < full ? word(f) : t; };
        const uint32_t W = P & (0u - P);
        if (W >= 4) {
            for (uint32_t q = 0; q < P; q += 4)
                *reinterpret_cast<uint32_t*>(d + q) = (uint32_t)(sw(q >> 3) >> (8 * (q & 7)));
        } else if (W == 2) {
            for (uint32_t q = 0; q < P; q += 2)
                *reinterpret_cast<uint16_t*>(d + q) = (uint16_t)(sw(q >> 3) >> (8 * (q & 7)));
        } else {
            for (uint32_t q = 0; q < P; ++q) d[q] = (uint8_t)(sw(q >> 3) >> (8 * (q & 7)));
        }
    }
}

// A warp packs 32 segments at a time: lane l loads segment l's count and
// output index (one coalesced load each), then the warp walks the segments
// that have first occurrences, B at a time, every lane loading all of its
// keys of those segments before storing any, so that 4 loads per lane are in
// flight.
template <int NW>
__global__ void pack_low(const void* routed, const uint32_t* seg_low, const uint64_t* seg_low_prefix, uint64_t n_segs,
                         uint32_t k, uint8_t* out, uint64_t out_base) {
    using K = typename KeyOf<NW>::T;
    constexpr int SEG = count_seg<NW>();
    constexpr int PER = SEG / 32;                  // keys per lane per segment
    constexpr int B = PER >= 4 ? 1 : 4 / PER;      // segments per round: 4 keys per lane in flight
    const K* __restrict__ keys = reinterpret_cast<const K*>(routed);
    const uint32_t full = k / 32, tail_bits = 2 * (k % 32), tail_bytes = (tail_bits + 7) / 8;
    const uint32_t P = full * 8 + tail_bytes;
    const uint64_t tmask = tail_bits ? (~0ull << (64 - tail_bits)) : 0ull;
    const int lane = threadIdx.x & 31;
    const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
    for (uint64_t g = ((uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 32; g < n_segs;
         g += warps * 32) {
        const uint64_t my = g + lane;
        const uint32_t n_l = my < n_segs ? seg_low[my] : 0u;
        const uint64_t o_l = my < n_segs ? seg_low_prefix[my] : 0ull;
        uint32_t todo = __ballot_sync(0xffffffffu, n_l != 0);
        while (todo) {
            // B segments per round (warp-uniform picks from `todo`)
            uint32_t n[B];
            uint64_t o[B], s0[B];
#pragma unroll
            for (int b = 0; b < B; ++b) {
                const int q = todo ? __ffs(todo) - 1 : -1;
                todo &= todo - 1;
                const int src = q >= 0 ? q : 0;
                const uint32_t nq = __shfl_sync(0xffffffffu, n_l, src);
                const uint64_t oq = __shfl_sync(0xffffffffu, o_l, src);
                n[b] = q >= 0 ? nq : 0u;
                o[b] = out_base + oq;
                s0[b] = (g + (uint64_t)src) * (uint64_t)SEG;
            }
            K v[B][PER];
#pragma unroll
            for (int b = 0; b < B; ++b)
#pragma unroll
                for (int j = 0; j < PER; ++j) {
                    const uint32_t i = j * 32 + lane;
                    if (i < n[b]) v[b][j] = keys[s0[b] + i];
                }
#pragma unroll
            for (int b = 0; b < B; ++b)
#pragma unroll
                for (int j = 0; j < PER; ++j) {
                    const uint32_t i = j * 32 + lane;
                    if (i < n[b]) pack_key<NW>(v[b][j], out + (o[b] + i) * P, full, tail_bytes, P, tmask);
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

template <int NW>
__device__ __forceinline__ bool slot_used(const typename SlotOf<NW>::T& s) {
    if constexpr (NW == 1) return s.key != EMPTY;
    else if constexpr (NW == 2) return !(s.w0 == EMPTY && s.w1 == EMPTY);
    else return s.state == SLOT_READY;
}

constexpr int EXP_THREADS = 256;
constexpr int EXP_ITEMS = 4;  // slots per thread per round (strided by EXP_THREADS)

// One ExportRecord<N> {key words, count, pad = 0} at index r.
template <int NW>
__device__ __forceinline__ void write_record(uint8_t* records, uint64_t r, const typename SlotOf<NW>::T& v) {
    if constexpr (NW == 1) {
        uint4 w;
        w.x = (uint32_t)v.key;
        w.y = (uint32_t)(v.key >> 32);
        w.z = v.count;
        w.w = 0;
        reinterpret_cast<uint4*>(records)[r] = w;
    } else if constexpr (NW == 2) {
        uint64_t* d = reinterpret_cast<uint64_t*>(records + r * 24);
        d[0] = v.w0;
        d[1] = v.w1;
        d[2] = (uint64_t)v.count;
    } else {
        uint64_t* d = reinterpret_cast<uint64_t*>(records + r * 40);
        d[0] = v.w0;
        d[1] = v.w1;
        d[2] = v.w2;
        d[3] = v.w3;
        d[4] = (uint64_t)v.count;
    }
}

// Count slots passing the filter min <= count <= max per export chunk and per
// root id (src/NewKmerTree.h:1159-1168), and occupied slots overall.  The
// per-chunk counts, scanned in chunk order, are the chunks' output offsets:
// chunks are listed root by root, so each root's records are contiguous.
// With `pass_bits` (chunks start at and span multiples of 32 slots), bit i of
// word w is set when arena slot 32w + i passes: a warp reads 32 consecutive
// slots, so one ballot is one word, and export_write_bits then reads only the
// passing slots.
template <int NW>
__global__ void __launch_bounds__(EXP_THREADS) export_count(const void* table, const ExportChunk* chunks,
                                                            uint64_t n_chunks, uint32_t min_c, uint32_t max_c,
                                                            uint32_t* chunk_pass, unsigned long long* root_count,
                                                            unsigned long long* occupied, uint32_t* pass_bits) {
    using S = typename SlotOf<NW>::T;
    __shared__ uint32_t s_pass[EXP_THREADS / 32], s_occ[EXP_THREADS / 32];
    const S* tab = reinterpret_cast<const S*>(table);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint64_t c = blockIdx.x; c < n_chunks; c += gridDim.x) {
        const ExportChunk ch = chunks[c];
        uint32_t pass = 0, occ = 0;
        for (uint32_t i0 = 0; i0 < ch.n_slots; i0 += EXP_THREADS * EXP_ITEMS) {
            S v[EXP_ITEMS];
#pragma unroll
            for (int j = 0; j < EXP_ITEMS; ++j) {
                const uint32_t i = i0 + j * EXP_THREADS + threadIdx.x;
                if (i < ch.n_slots) v[j] = tab[ch.slot_begin + i];
            }
#pragma unroll
            for (int j = 0; j < EXP_ITEMS; ++j) {
                const uint32_t i = i0 + j * EXP_THREADS + threadIdx.x;
                bool ok = false;
                if (i < ch.n_slots && slot_used<NW>(v[j])) {
                    ++occ;
                    ok = v[j].count >= min_c && v[j].count <= max_c;
                    pass += ok;
                }
                if (pass_bits) {
                    const uint32_t word = __ballot_sync(0xffffffffu, ok);
                    const uint32_t i_lane0 = i - (uint32_t)lane;
                    if (lane == 0 && i_lane0 < ch.n_slots) pass_bits[(ch.slot_begin + i_lane0) >> 5] = word;
                }
            }
        }
        for (int o = 16; o; o >>= 1) {
            pass += __shfl_xor_sync(0xffffffffu, pass, o);
            occ += __shfl_xor_sync(0xffffffffu, occ, o);
        }
        if (lane == 0) {
            s_pass[warp] = pass;
            s_occ[warp] = occ;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t tp = 0, to = 0;
            for (int w = 0; w < EXP_THREADS / 32; ++w) {
                tp += s_pass[w];
                to += s_occ[w];
            }
            chunk_pass[c] = tp;
            if (tp) atomicAdd(root_count + ch.root, (unsigned long long)tp);
            if (to) atomicAdd(occupied, (unsigned long long)to);
        }
        __syncthreads();
    }
}

// Write ExportRecord<N> {key words, count, pad = 0} of every passing slot,
// one read of the table: chunk c's records start at chunk_off[c] and follow
// table order (rounds of EXP_THREADS x EXP_ITEMS slots; inside a round, by
// thread, then item).  No atomics decide positions, so the record order is a
// function of the table alone.
template <int NW>
__global__ void __launch_bounds__(EXP_THREADS) export_write(const void* table, const ExportChunk* chunks,
                                                            uint64_t n_chunks, uint32_t min_c, uint32_t max_c,
                                                            const uint64_t* chunk_off, uint8_t* records) {
    using S = typename SlotOf<NW>::T;
    __shared__ uint32_t s_warp[EXP_THREADS / 32];
    const S* tab = reinterpret_cast<const S*>(table);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint64_t c = blockIdx.x; c < n_chunks; c += gridDim.x) {
        const ExportChunk ch = chunks[c];
        uint64_t out = chunk_off[c];
        for (uint32_t i0 = 0; i0 < ch.n_slots; i0 += EXP_THREADS * EXP_ITEMS) {
            S v[EXP_ITEMS];
            uint32_t keep = 0;
#pragma unroll
            for (int j = 0; j < EXP_ITEMS; ++j) {
                const uint32_t i = i0 + j * EXP_THREADS + threadIdx.x;
                if (i < ch.n_slots) {
                    v[j] = tab[ch.slot_begin + i];
                    if (slot_used<NW>(v[j]) && v[j].count >= min_c && v[j].count <= max_c) keep |= 1u << j;
                }
            }
            // block-wide exclusive scan of the per-thread keep counts
            const uint32_t mine = __popc(keep);
            uint32_t incl = mine;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            if (lane == 31) s_warp[warp] = incl;
            __syncthreads();
            uint32_t before = 0, total = 0;
#pragma unroll
            for (int w = 0; w < EXP_THREADS / 32; ++w) {
                const uint32_t t = s_warp[w];
                before += w < warp ? t : 0u;
                total += t;
            }
            __syncthreads();  // s_warp is rewritten next round
            uint64_t r = out + before + incl - mine;
#pragma unroll
            for (int j = 0; j < EXP_ITEMS; ++j)
                if ((keep >> j) & 1u) write_record<NW>(records, r++, v[j]);
            out += total;
        }
    }
}

// export_write over the passing-slot bitmap of export_count.  Per round a
// warp covers 32 bitmap words (1024 slots) and lane l of each pass takes the
// warp's l-th passing slot: the owning word by a binary search over the
// lanes' running popcounts, the bit by nth_set_bit.  Every lane reads one slot per
// pass and consecutive lanes write consecutive records, in table order (the
// order export_write produces).
template <int NW>
__global__ void __launch_bounds__(EXP_THREADS) export_write_bits(const void* table, const uint32_t* pass_bits,
                                                                 const ExportChunk* chunks, uint64_t n_chunks,
                                                                 const uint64_t* chunk_off, uint8_t* records) {
    using S = typename SlotOf<NW>::T;
    __shared__ uint32_t s_warp[EXP_THREADS / 32];
    const S* tab = reinterpret_cast<const S*>(table);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint64_t c = blockIdx.x; c < n_chunks; c += gridDim.x) {
        const ExportChunk ch = chunks[c];
        const uint64_t w0 = ch.slot_begin >> 5;
        const uint32_t nw = ch.n_slots >> 5;
        uint64_t out = chunk_off[c];
        for (uint32_t r0 = 0; r0 < nw; r0 += EXP_THREADS) {
            const uint32_t wi = r0 + threadIdx.x;
            const uint32_t m = wi < nw ? __ldcg(pass_bits + w0 + wi) : 0u;
            uint32_t incl = __popc(m);  // warp-inclusive running count
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            const uint32_t wtot = __shfl_sync(0xffffffffu, incl, 31);
            if (lane == 31) s_warp[warp] = wtot;
            __syncthreads();
            uint32_t before = 0, total = 0;
#pragma unroll
            for (int w = 0; w < EXP_THREADS / 32; ++w) {
                const uint32_t t = s_warp[w];
                before += w < warp ? t : 0u;
                total += t;
            }
            __syncthreads();  // s_warp is rewritten next round
            const uint64_t base = out + before;
            const uint64_t cell_w = (w0 + r0 + (uint32_t)warp * 32) << 5;  // first slot of lane 0's word
            for (uint32_t n0 = 0; n0 < wtot; n0 += 32) {
                const uint32_t n = n0 + lane;
                // owner lane q: the first lane whose running count exceeds n
                uint32_t lo = 0, hi = 31;
#pragma unroll
                for (int step = 0; step < 5; ++step) {
                    const uint32_t mid = (lo + hi) >> 1;
                    const uint32_t v = __shfl_sync(0xffffffffu, incl, mid);
                    if (v > n) hi = mid;
                    else lo = mid + 1;
                }
                const uint32_t q = lo;
                const uint32_t mq = __shfl_sync(0xffffffffu, m, q);
                const uint32_t eq = __shfl_sync(0xffffffffu, incl, q) - __popc(mq);  // passing slots before word q
                if (n < wtot) {
                    const uint32_t bit = nth_set_bit(mq, n - eq);
                    const S v = tab[cell_w + ((uint64_t)q << 5) + bit];
                    write_record<NW>(records, base + n, v);
                }
            }
            out += total;
        }
    }
}

// ------------------------------------------------------ merged histogram
//
// Device form of tool/histogram_tool.cpp "precise"
// (tool/HighFrequencyInsertThreadPool.h:150-177,
// tool/LowFrequencyQueryThreadPool.h:375-432): exact count of a key = its
// table count + [key in low.bin].  Pass 1 walks the packed low.bin keys,
// looks each up in its bucket's table, marks the slot (pad field) and adds
// count+1 (or 1) to the histogram; pass 2 adds every unmarked table key with
// its table count.  Histogram bins are aggregated per CTA in shared memory
// (HIST_SMEM bins; larger counts go straight to global atomics).

constexpr int HIST_SMEM = 1024;

// Key of low.bin record r (layout of src/ExportWriter.h:522-550, read back as
// tool/ExportReader.h:355-391 does).  Records of a multiple of 8 bytes
// (k = 29..32, 61..64, 93..96, 125..128) are read as aligned words.
template <int NW>
__device__ __forceinline__ typename KeyOf<NW>::T unpack_low(const uint8_t* low, uint64_t r, uint32_t P, uint32_t full,
                                                            uint32_t tail_bytes) {
    const uint8_t* p = low + r * P;
    uint64_t w[4] = {0, 0, 0, 0};
    if ((P & 7u) == 0) {
        const uint64_t* q = reinterpret_cast<const uint64_t*>(p);
        for (uint32_t f = 0; f < P / 8 && f < (uint32_t)NW; ++f) w[f] = q[f];
    } else {
        for (uint32_t f = 0; f < full; ++f)
            for (uint32_t b = 0; b < 8; ++b) w[f] |= (uint64_t)p[8 * f + b] << (8 * b);
        for (uint32_t b = 0; b < tail_bytes; ++b) w[full] |= (uint64_t)p[8 * full + b] << (8 * (8 - tail_bytes + b));
    }
    typename KeyOf<NW>::T key;
    if constexpr (NW == 1) key = w[0];
    else if constexpr (NW == 2) key = Key2{w[0], w[1]};
    else key = Key4{w[0], w[1], w[2], w[3]};
    return key;
}

template <int NW>
__device__ __forceinline__ bool table_find(const typename SlotOf<NW>::T* tab, uint64_t mask, uint64_t h,
                                           const typename KeyOf<NW>::T& key, uint64_t* where) {
    const uint64_t i0 = (h >> 17) & mask;
    for (uint64_t p = 0; p <= mask; ++p) {
        const uint64_t i = (i0 + p) & mask;
        const typename SlotOf<NW>::T& s = tab[i];
        bool empty, eq;
        if constexpr (NW == 1) {
            empty = s.key == EMPTY;
            eq = s.key == key;
        } else if constexpr (NW == 2) {
            empty = s.w0 == EMPTY && s.w1 == EMPTY;
            eq = s.w0 == key.w0 && s.w1 == key.w1;
        } else {
            empty = s.state != SLOT_READY;  // after the count every used slot is ready
            eq = !empty && s.w0 == key.w0 && s.w1 == key.w1 && s.w2 == key.w2 && s.w3 == key.w3;
        }
        if (eq) {
            *where = i;
            return true;
        }
        if (empty) return false;
    }
    return false;
}

__device__ __forceinline__ void hist_add(uint32_t* sh, unsigned long long* gh, uint64_t merged, uint32_t lo,
                                         uint32_t hi) {
    // the active lanes of the warp that share a shared-memory bin add once
    // (nearly every low.bin key lands in the bin of count 1, and shared-memory
    // atomics on one address are serialised)
    const bool in = merged >= lo && merged <= hi;
    const uint64_t bin = merged - lo;
    const uint32_t key = in && bin < HIST_SMEM ? (uint32_t)bin : 0xFFFFFFFFu;
    const uint32_t same = __match_any_sync(__activemask(), key);
    if (key != 0xFFFFFFFFu) {
        if ((int)(__ffs(same) - 1) == (int)(threadIdx.x & 31)) atomicAdd(sh + key, (uint32_t)__popc(same));
    } else if (in) {
        atomicAdd(gh + bin, 1ull);
    }
}

template <int NW>
__global__ void hist_clear_marks(void* table, uint64_t n_slots) {
    using S = typename SlotOf<NW>::T;
    S* t = reinterpret_cast<S*>(table);
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_slots; i += (uint64_t)gridDim.x * blockDim.x) {
        if constexpr (NW == 1) t[i].pad = 0;
        else if constexpr (NW == 2) t[i].pad[0] = 0;
        else t[i].mark = 0;
    }
}

template <int NW>
__global__ void hist_low_pass(const uint8_t* low, uint64_t n_low, uint32_t k, const BucketMeta* meta,
                              uint32_t bucket_shift, void* table, uint32_t lo, uint32_t hi,
                              unsigned long long* gh) {
    using K = typename KeyOf<NW>::T;
    using S = typename SlotOf<NW>::T;
    __shared__ uint32_t sh[HIST_SMEM];
    for (int i = threadIdx.x; i < HIST_SMEM; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    const uint32_t full = k / 32, tail_bits = 2 * (k % 32), tail_bytes = (tail_bits + 7) / 8;
    const uint32_t P = full * 8 + tail_bytes;
    for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n_low; r += (uint64_t)gridDim.x * blockDim.x) {
        const K key = unpack_low<NW>(low, r, P, full, tail_bytes);
        const BucketMeta m = meta[key_hi(key) >> bucket_shift];
        S* tab = reinterpret_cast<S*>(table) + m.tab_off;
        uint64_t at;
        uint64_t merged = 1;
        if (table_find<NW>(tab, m.tab_mask, hash_key(key), key, &at)) {
            merged = (uint64_t)tab[at].count + 1;
            if constexpr (NW == 1) tab[at].pad = 1;
            else if constexpr (NW == 2) tab[at].pad[0] = 1;
            else tab[at].mark = 1;
        }
        hist_add(sh, gh, merged, lo, hi);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < HIST_SMEM; i += blockDim.x)
        if (sh[i]) atomicAdd(gh + i, (unsigned long long)sh[i]);
}

template <int NW>
__global__ void hist_table_pass(const void* table, const ExportChunk* chunks, uint64_t n_chunks, uint32_t lo, uint32_t hi,
                                unsigned long long* gh, unsigned long long* unmarked) {
    using S = typename SlotOf<NW>::T;
    __shared__ uint32_t sh[HIST_SMEM];
    __shared__ unsigned long long s_un;
    for (int i = threadIdx.x; i < HIST_SMEM; i += blockDim.x) sh[i] = 0;
    if (threadIdx.x == 0) s_un = 0;
    __syncthreads();
    uint32_t un = 0;
    for (uint64_t c = blockIdx.x; c < n_chunks; c += gridDim.x)
    for (uint32_t q = threadIdx.x; q < chunks[c].n_slots; q += blockDim.x) {
        const S s = reinterpret_cast<const S*>(table)[chunks[c].slot_begin + q];
        bool used, marked;
        if constexpr (NW == 1) {
            used = s.key != EMPTY;
            marked = s.pad != 0;
        } else if constexpr (NW == 2) {
            used = !(s.w0 == EMPTY && s.w1 == EMPTY);
            marked = s.pad[0] != 0;
        } else {
            used = s.state == SLOT_READY;
            marked = s.mark != 0;
        }
        if (used && !marked) {
            ++un;
            hist_add(sh, gh, s.count, lo, hi);
        }
    }
    for (int o = 16; o; o >>= 1) un += __shfl_xor_sync(0xffffffffu, un, o);
    if ((threadIdx.x & 31) == 0 && un) atomicAdd(&s_un, (unsigned long long)un);
    __syncthreads();
    for (int i = threadIdx.x; i < HIST_SMEM; i += blockDim.x)
        if (sh[i]) atomicAdd(gh + i, (unsigned long long)sh[i]);
    if (threadIdx.x == 0 && s_un) atomicAdd(unmarked, s_un);
}

// Per model bucket (key word 0 >> 52) loads of the last result: low keys,
// looked up in their table (marked as in hist_low_pass), then every table
// key.  distinct = low keys + unmarked table keys; kmers = occurrences.
// model buckets of the sizing loads (the top 12 bits of the key)
constexpr uint32_t KC_LOADS_BINS = 4096;
// dynamic shared memory of loads_low_pass / loads_table_pass
constexpr size_t loads_low_smem() { return KC_LOADS_BINS * (8 + 4); }
constexpr size_t loads_table_smem() { return KC_LOADS_BINS * (8 + 4 + 4); }

template <int NW>
__global__ void loads_low_pass(const uint8_t* low, uint64_t n_low, uint32_t k, const BucketMeta* meta,
                               uint32_t bucket_shift, void* table, unsigned long long* distinct,
                               unsigned long long* kmers) {
    // per-CTA totals per model bucket in shared memory (consecutive low keys
    // share their model bucket, so global atomics would serialise on it),
    // added to the global totals once per CTA
    extern __shared__ unsigned long long ld_smem[];
    unsigned long long* s_kmers = ld_smem;                                        // [KC_LOADS_BINS]
    uint32_t* s_distinct = reinterpret_cast<uint32_t*>(ld_smem + KC_LOADS_BINS);  // [KC_LOADS_BINS]
    for (uint32_t i = threadIdx.x; i < KC_LOADS_BINS; i += blockDim.x) {
        s_kmers[i] = 0;
        s_distinct[i] = 0;
    }
    __syncthreads();
    using K = typename KeyOf<NW>::T;
    using S = typename SlotOf<NW>::T;
    const uint32_t full = k / 32, tail_bits = 2 * (k % 32), tail_bytes = (tail_bits + 7) / 8;
    const uint32_t P = full * 8 + tail_bytes;
    for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n_low; r += (uint64_t)gridDim.x * blockDim.x) {
        const K key = unpack_low<NW>(low, r, P, full, tail_bytes);
        const BucketMeta m = meta[key_hi(key) >> bucket_shift];
        S* tab = reinterpret_cast<S*>(table) + m.tab_off;
        uint64_t at;
        unsigned long long occ = 1;
        if (table_find<NW>(tab, m.tab_mask, hash_key(key), key, &at)) {
            occ += tab[at].count;
            if constexpr (NW == 1) tab[at].pad = 1;
            else if constexpr (NW == 2) tab[at].pad[0] = 1;
            else tab[at].mark = 1;
        }
        const uint32_t bin = (uint32_t)(key_hi(key) >> 52);
        atomicAdd(s_distinct + bin, 1u);
        atomicAdd(s_kmers + bin, occ);
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < KC_LOADS_BINS; i += blockDim.x) {
        if (s_distinct[i]) atomicAdd(distinct + i, (unsigned long long)s_distinct[i]);
        if (s_kmers[i]) atomicAdd(kmers + i, s_kmers[i]);
    }
}

template <int NW>
__global__ void loads_table_pass(const void* table, const ExportChunk* chunks, uint64_t n_chunks,
                                 unsigned long long* distinct, unsigned long long* tkeys, unsigned long long* kmers) {
    extern __shared__ unsigned long long ld_smem[];
    unsigned long long* s_kmers = ld_smem;                                        // [KC_LOADS_BINS]
    uint32_t* s_distinct = reinterpret_cast<uint32_t*>(ld_smem + KC_LOADS_BINS);  // [KC_LOADS_BINS]
    uint32_t* s_tkeys = s_distinct + KC_LOADS_BINS;                               // [KC_LOADS_BINS]
    for (uint32_t i = threadIdx.x; i < KC_LOADS_BINS; i += blockDim.x) {
        s_kmers[i] = 0;
        s_distinct[i] = 0;
        s_tkeys[i] = 0;
    }
    __syncthreads();
    using S = typename SlotOf<NW>::T;
    for (uint64_t c = blockIdx.x; c < n_chunks; c += gridDim.x)
    for (uint32_t q = threadIdx.x; q < chunks[c].n_slots; q += blockDim.x) {
        const S s = reinterpret_cast<const S*>(table)[chunks[c].slot_begin + q];
        uint64_t hi;
        bool used, marked;
        if constexpr (NW == 1) {
            used = s.key != EMPTY;
            marked = s.pad != 0;
            hi = s.key;
        } else if constexpr (NW == 2) {
            used = !(s.w0 == EMPTY && s.w1 == EMPTY);
            marked = s.pad[0] != 0;
            hi = s.w0;
        } else {
            used = s.state == SLOT_READY;
            marked = s.mark != 0;
            hi = s.w0;
        }
        if (!used) continue;
        const uint32_t bin = (uint32_t)(hi >> 52);
        atomicAdd(s_tkeys + bin, 1u);
        if (!marked) {
            atomicAdd(s_distinct + bin, 1u);
            atomicAdd(s_kmers + bin, (unsigned long long)s.count);
        }
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < KC_LOADS_BINS; i += blockDim.x) {
        if (s_tkeys[i]) atomicAdd(tkeys + i, (unsigned long long)s_tkeys[i]);
        if (s_distinct[i]) atomicAdd(distinct + i, (unsigned long long)s_distinct[i]);
        if (s_kmers[i]) atomicAdd(kmers + i, s_kmers[i]);
    }
}

// EMPTY keys into the unfilled tail of each estimated bucket region:
// routed[min(cursor[b], region_fill[b], region_end[b]), region_end[b]).
template <int NW>
__global__ void fill_region_gaps(void* routed, const unsigned long long* cursor, const unsigned long long* region_fill,
                                 const unsigned long long* region_end, uint32_t n_buckets) {
    using K = typename KeyOf<NW>::T;
    K* keys = reinterpret_cast<K*>(routed);
    const uint32_t b = blockIdx.x;
    if (b >= n_buckets) return;
    const unsigned long long end = region_end[b];
    for (unsigned long long i = min(min(cursor[b], region_fill[b]), end) + threadIdx.x; i < end; i += blockDim.x) {
        if constexpr (NW == 1) keys[i] = EMPTY;
        else if constexpr (NW == 2) keys[i] = Key2{EMPTY, EMPTY};
        else keys[i] = Key4{EMPTY, EMPTY, EMPTY, EMPTY};
    }
}

// ------------------------------------------------------- multi-set batches

// EMPTY keys into the alignment gap after each set's routed region.
template <int NW>
__global__ void fill_set_gaps(void* routed, const uint64_t* set_end_key, const uint64_t* set_next_key, uint32_t n_sets) {
    using K = typename KeyOf<NW>::T;
    K* keys = reinterpret_cast<K*>(routed);
    const uint32_t s = blockIdx.x;
    if (s >= n_sets) return;
    for (uint64_t i = set_end_key[s] + threadIdx.x; i < set_next_key[s]; i += blockDim.x) {
        if constexpr (NW == 1) keys[i] = EMPTY;
        else if constexpr (NW == 2) keys[i] = Key2{EMPTY, EMPTY};
        else keys[i] = Key4{EMPTY, EMPTY, EMPTY, EMPTY};
    }
}

// Pack first occurrences of a multi-set batch: segment sg of set s writes at
// low_byte_base[s] (a multiple of 16) + (prefix[sg] - prefix[first segment
// of s]) * P(k_s).  A warp takes 32 segments at a time (each lane finds its
// segment's set and output place), then packs the segments that have first
// occurrences one after another, every lane a key.
template <int NW>
__global__ void pack_low_sets(const void* routed, const uint32_t* seg_low, const uint64_t* seg_low_prefix, uint64_t n_segs,
                              const uint64_t* set_seg_start, const uint32_t* set_k, const uint64_t* low_byte_base,
                              uint32_t n_sets, uint8_t* out) {
    using K = typename KeyOf<NW>::T;
    constexpr int SEG = count_seg<NW>();
    constexpr int PER = SEG / 32;  // keys per lane per segment
    const K* __restrict__ keys = reinterpret_cast<const K*>(routed);
    const int lane = threadIdx.x & 31;
    const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
    for (uint64_t g = ((uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 32; g < n_segs;
         g += warps * 32) {
        const uint64_t my = g + lane;
        uint32_t n_l = 0, k_l = 1;
        uint64_t dst_l = 0;
        if (my < n_segs && (n_l = seg_low[my]) != 0) {
            uint32_t lo = 0, hi = n_sets;
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) / 2;
                if (set_seg_start[mid] <= my) lo = mid;
                else hi = mid;
            }
            k_l = set_k[lo];
            dst_l = low_byte_base[lo] + (seg_low_prefix[my] - seg_low_prefix[set_seg_start[lo]]) * kc_packed(k_l);
        }
        uint32_t todo = __ballot_sync(0xffffffffu, n_l != 0);
        while (todo) {
            const int q = __ffs(todo) - 1;
            todo &= todo - 1;
            const uint32_t n = __shfl_sync(0xffffffffu, n_l, q);
            const uint32_t k = __shfl_sync(0xffffffffu, k_l, q);
            const uint64_t dst = __shfl_sync(0xffffffffu, dst_l, q);
            const uint32_t full = k / 32, tail_bits = 2 * (k % 32), tail_bytes = (tail_bits + 7) / 8;
            const uint32_t P = full * 8 + tail_bytes;
            const uint64_t tmask = tail_bits ? (~0ull << (64 - tail_bits)) : 0ull;
            const uint64_t s0 = (g + (uint64_t)q) * (uint64_t)SEG;
            K v[PER];
#pragma unroll
            for (int j = 0; j < PER; ++j) {
                const uint32_t i = j * 32 + lane;
                if (i < n) v[j] = keys[s0 + i];
            }
#pragma unroll
            for (int j = 0; j < PER; ++j) {
                const uint32_t i = j * 32 + lane;
                if (i < n) pack_key<NW>(v[j], out + dst + (uint64_t)i * P, full, tail_bytes, P, tmask);
            }
        }
    }
}

}  // namespace kc
