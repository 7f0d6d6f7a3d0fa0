// CPU oracle for the exact canonical k-mer counting path.
//
// TEST INFRASTRUCTURE ONLY.  Nothing in the product links, loads or runs this
// file: the tests, the smoke check and the CPU-baseline leg of bench.py use it
// as the checker.  It is a deliberately plain, single-threaded restatement of
// the reference's semantics, written in a different formulation from the GPU
// kernels (a rolling register pair here, a windowed bit-reverse there), so the
// two agreeing is evidence rather than an echo.
//
// Semantics restated (reference files of ScorchShana/KmerTreeCounter):
//  * Line state machine, every '\n' advances Header -> Sequence -> Plus ->
//    Quality -> Header; only Sequence-line bytes are k-mer input, and the
//    newline itself ends the run.  (src/FastqReader.h:293-308, the block
//    overlap at :338-365 only guarantees that block splits neither lose nor
//    duplicate windows, so the whole file behaves as one stream.)
//  * Base table: A/a=0, C/c=1, G/g=2, T/t/U/u=3, anything else clears the
//    rolling state.  (src/GetKmer.h:22-37, clear at :51-56; the AVX2/SSE
//    classification at src/FastqParser.h:211-300 is equivalent because
//    x & 0xDF only folds lowercase.)
//  * Forward register F: shift right one base, new base into the top two
//    bits of word 0, last word masked to the k-th base.  Reverse register C:
//    shift left one base, complement inserted at the k-th base slot.
//    (src/GetKmer.h:58-82, masks at :38-47)
//  * Canonical key = lexicographic min(F, C) over words 0..N-1.
//    (src/GetKmer.h:181-207, kmer<=> at src/kmer.h:21)
//  * A key is emitted once at least k consecutive bases were seen.
//    (src/GetKmer.h:81 / :105)
//  * N = 1 for k<=32, 2 for k<=64, 4 for k<=128.  (src/main.cpp:579-595)
//  * low.bin packing: k/32 full words as raw little-endian u64, then the
//    top ceil(2(k%32)/8) bytes of the masked tail word, in LE byte order.
//    (src/ExportWriter.h:339-342, :522-550)
//
// Build: make -C oracle oracle  ->  oracle/_build/libkmer_oracle.so

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

inline uint32_t words_for_k(uint32_t k) { return k <= 32 ? 1u : (k <= 64 ? 2u : 4u); }

struct Roll {
    uint32_t k, nw, last, have = 0;
    uint64_t back_mask, rev_shift;
    uint64_t F[4], C[4];
    explicit Roll(uint32_t kk) : k(kk), nw(words_for_k(kk)), last((kk - 1) / 32) {
        const uint32_t rem = k % 32;
        if (rem) {
            back_mask = ((1ULL << (2 * rem)) - 1ULL) << (64 - 2 * rem);
            rev_shift = 2 * (32 - rem);
        } else {
            back_mask = ~0ULL;
            rev_shift = 0;
        }
        reset();
    }
    void reset() {
        std::memset(F, 0, sizeof F);
        std::memset(C, 0, sizeof C);
        have = 0;
    }
    // returns true when a full window is available in key[]
    bool push(uint32_t code, uint64_t* key) {
        for (int i = (int)nw - 1; i > 0; --i) F[i] = (F[i] >> 2) | (F[i - 1] << 62);
        F[0] = (F[0] >> 2) | ((uint64_t)code << 62);
        F[last] &= back_mask;
        for (uint32_t i = 0; i + 1 < nw; ++i) C[i] = (C[i] << 2) | (C[i + 1] >> 62);
        C[nw - 1] <<= 2;
        C[last] |= (uint64_t)(code ^ 3u) << rev_shift;
        if (++have < k) return false;
        bool f_less = false;
        for (uint32_t i = 0; i < nw; ++i) {
            if (F[i] != C[i]) { f_less = F[i] < C[i]; break; }
        }
        const uint64_t* src = f_less ? F : C;
        for (uint32_t i = 0; i < nw; ++i) key[i] = src[i];
        return true;
    }
};

inline int code_of(uint8_t c) {
    switch (c) {
        case 'A': case 'a': return 0;
        case 'C': case 'c': return 1;
        case 'G': case 'g': return 2;
        case 'T': case 't': case 'U': case 'u': return 3;
        default: return -1;
    }
}

// Runs the FASTQ state machine and calls emit(key) for every canonical window.
template <class F>
uint64_t scan(const uint8_t* data, uint64_t n, uint32_t k, F&& emit) {
    Roll r(k);
    uint32_t line_state = 0;  // 0 header, 1 sequence, 2 plus, 3 quality
    uint64_t key[4];
    uint64_t count = 0;
    for (uint64_t i = 0; i < n; ++i) {
        const uint8_t c = data[i];
        if (c == '\n') {
            line_state = (line_state + 1) & 3u;
            r.reset();
            continue;
        }
        if (line_state != 1) continue;
        const int code = code_of(c);
        if (code < 0) { r.reset(); continue; }
        if (r.push((uint32_t)code, key)) {
            emit(key);
            ++count;
        }
    }
    return count;
}

template <uint32_t NW>
struct Key { uint64_t w[NW]; };
template <uint32_t NW>
inline bool key_less(const Key<NW>& a, const Key<NW>& b) {
    for (uint32_t i = 0; i < NW; ++i)
        if (a.w[i] != b.w[i]) return a.w[i] < b.w[i];
    return false;
}

template <uint32_t NW>
int64_t count_impl(const uint8_t* data, uint64_t n, uint32_t k, uint64_t* keys_out, uint32_t* counts_out,
                   uint64_t cap, uint64_t* total) {
    std::vector<Key<NW>> all;
    all.reserve(n / 2 + 16);
    const uint64_t K = scan(data, n, k, [&](const uint64_t* key) {
        Key<NW> x;
        for (uint32_t i = 0; i < NW; ++i) x.w[i] = key[i];
        all.push_back(x);
    });
    if (total) *total = K;
    std::sort(all.begin(), all.end(), key_less<NW>);
    uint64_t d = 0;
    for (uint64_t i = 0; i < all.size();) {
        uint64_t j = i + 1;
        while (j < all.size() && std::memcmp(all[j].w, all[i].w, sizeof(all[i].w)) == 0) ++j;
        if (d < cap && keys_out) {
            for (uint32_t w = 0; w < NW; ++w) keys_out[d * NW + w] = all[i].w[w];
            counts_out[d] = (uint32_t)(j - i);
        }
        ++d;
        i = j;
    }
    return (int64_t)d;
}

}  // namespace

extern "C" {

uint32_t kor_words(uint32_t k) { return words_for_k(k); }

// Number of canonical k-mers in a FASTQ byte stream; if keys != nullptr the
// first `cap` keys are written in emission order (N words each).
uint64_t kor_extract(const uint8_t* data, uint64_t n, uint32_t k, uint64_t* keys, uint64_t cap) {
    const uint32_t nw = words_for_k(k);
    uint64_t idx = 0;
    return scan(data, n, k, [&](const uint64_t* key) {
        if (keys && idx < cap)
            for (uint32_t i = 0; i < nw; ++i) keys[idx * nw + i] = key[i];
        ++idx;
    });
}

// Exact (key, count) table sorted by key.  Returns the number of distinct
// keys; only the first `cap` are written.  *total receives K.
int64_t kor_count(const uint8_t* data, uint64_t n, uint32_t k, uint64_t* keys, uint32_t* counts, uint64_t cap,
                  uint64_t* total) {
    if (k == 0 || k > 128) return -1;
    switch (words_for_k(k)) {
        case 1: return count_impl<1>(data, n, k, keys, counts, cap, total);
        case 2: return count_impl<2>(data, n, k, keys, counts, cap, total);
        default: return count_impl<4>(data, n, k, keys, counts, cap, total);
    }
}

// Bytes per packed low.bin record for k.
uint64_t kor_packed_bytes(uint32_t k) {
    const uint32_t full = k / 32, tail_bits = 2 * (k % 32);
    return full * 8ull + (tail_bits + 7) / 8;
}

// Pack n keys (N words each) into the low.bin byte layout.
void kor_pack(const uint64_t* keys, uint64_t n, uint32_t k, uint8_t* out) {
    const uint32_t nw = words_for_k(k), full = k / 32, tail_bits = 2 * (k % 32), tail_bytes = (tail_bits + 7) / 8;
    const uint64_t mask = tail_bits ? (~0ULL << (64 - tail_bits)) : 0;
    uint8_t* p = out;
    for (uint64_t i = 0; i < n; ++i) {
        const uint64_t* key = keys + i * nw;
        for (uint32_t w = 0; w < full; ++w) {
            for (uint32_t b = 0; b < 8; ++b) *p++ = (uint8_t)(key[w] >> (8 * b));
        }
        if (tail_bytes) {
            const uint64_t t = key[full] & mask;
            for (uint32_t b = 8 - tail_bytes; b < 8; ++b) *p++ = (uint8_t)(t >> (8 * b));
        }
    }
}

// Inverse of kor_pack (tool/ExportReader.h:355-391 restated).
void kor_unpack(const uint8_t* in, uint64_t n, uint32_t k, uint64_t* keys) {
    const uint32_t nw = words_for_k(k), full = k / 32, tail_bits = 2 * (k % 32), tail_bytes = (tail_bits + 7) / 8;
    const uint8_t* p = in;
    for (uint64_t i = 0; i < n; ++i) {
        uint64_t* key = keys + i * nw;
        for (uint32_t w = 0; w < nw; ++w) key[w] = 0;
        for (uint32_t w = 0; w < full; ++w) {
            uint64_t v = 0;
            for (uint32_t b = 0; b < 8; ++b) v |= (uint64_t)(*p++) << (8 * b);
            key[w] = v;
        }
        if (tail_bytes) {
            uint64_t v = 0;
            for (uint32_t b = 8 - tail_bytes; b < 8; ++b) v |= (uint64_t)(*p++) << (8 * b);
            key[full] = v;
        }
    }
}

}  // extern "C"
