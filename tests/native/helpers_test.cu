// Host-side unit test of the extraction helpers in kc_kernels.cuh
// (compiled by tests/test_kernel_helpers.py; runs on the CPU).
//
// For random base strings and every k in 1..128 and bucket widths 8/12 bits:
//   * window_at() returns exactly the last k bases ending at byte j,
//   * canonical1/canonical2 equal min(F, C) built from the definition in the
//     reference (src/GetKmer.h:58-82, :181-207): F = bases in reverse order,
//     C = complemented bases in read order, both left-aligned,
//   * bucket_of_window() equals the top bits of that canonical key (k <= 64),
//   * for k = 65..128: window_at4() and canonical4() the same way, and
//     runs_at_least5() marks exactly the bytes that end k consecutive bases,
//   * pack_key() writes every k's low.bin record layout,
//   * classify() flags bases and newlines and codes every byte,
//   * nth_set_bit() finds every set bit of random words in order.
#include <cstdio>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <random>
#include <vector>

#include "../../kmertreecounter_b200/csrc/kc_kernels.cuh"

using namespace kc;

static void pack_left(const std::vector<int>& b, uint64_t out[2]) {
    out[0] = out[1] = 0;
    for (size_t i = 0; i < b.size(); ++i) {
        const int w = (int)(i / 32), pos = 62 - 2 * (int)(i % 32);
        out[w] |= (uint64_t)b[i] << pos;
    }
}

static void pack_left4(const std::vector<int>& b, uint64_t out[4]) {
    out[0] = out[1] = out[2] = out[3] = 0;
    for (size_t i = 0; i < b.size(); ++i) {
        const int w = (int)(i / 32), pos = 62 - 2 * (int)(i % 32);
        out[w] |= (uint64_t)b[i] << pos;
    }
}

// k = 65..128 over five segments (160 bytes); returns the number of checks
static long check_long_keys(std::mt19937_64& rng) {
    long checks = 0;
    for (int iter = 0; iter < 4000; ++iter) {
        std::vector<int> bases(160);
        for (auto& x : bases) x = (int)(rng() & 3);
        uint64_t seg[5] = {0, 0, 0, 0, 0};
        for (int s = 0; s < 5; ++s)
            for (int j = 0; j < 32; ++j) seg[s] |= (uint64_t)bases[32 * s + j] << (62 - 2 * j);
        const uint32_t j = (uint32_t)(rng() % 32);
        uint64_t W[4];
        window_at4(seg[0], seg[1], seg[2], seg[3], seg[4], j, W[0], W[1], W[2], W[3]);
        for (uint32_t k = 65; k <= 128; ++k) {
            const int end = 128 + (int)j;
            std::vector<int> win(bases.begin() + end - k + 1, bases.begin() + end + 1);
            for (uint32_t i = 0; i < k; ++i) {
                const uint32_t bit = 2 * (k - 1 - i);
                if ((int)((W[bit / 64] >> (bit % 64)) & 3) != win[i]) {
                    std::printf("window4 mismatch k=%u j=%u\n", k, j);
                    std::exit(1);
                }
            }
            std::vector<int> rf(win.rbegin(), win.rend()), cc(win.size());
            for (size_t i = 0; i < win.size(); ++i) cc[i] = 3 - win[i];
            uint64_t F[4], C[4];
            pack_left4(rf, F);
            pack_left4(cc, C);
            int cmp = 0;
            for (int w = 0; w < 4 && !cmp; ++w) cmp = F[w] < C[w] ? -1 : (F[w] > C[w] ? 1 : 0);
            const uint64_t* want = cmp <= 0 ? F : C;
            // bits above the window (from bit 2k up) must not matter
            uint64_t g2 = W[2], g3 = W[3];
            const uint32_t kb = 2 * k;
            if (kb < 192) {
                g2 |= rng() << (kb - 128);
                g3 = rng();
            } else if (kb == 192) {
                g3 = rng();
            } else if (kb < 256) {
                g3 |= rng() << (kb - 192);
            }
            const Key4 got = canonical4(W[0], W[1], g2, g3, k);
            if (got.w0 != want[0] || got.w1 != want[1] || got.w2 != want[2] || got.w3 != want[3]) {
                std::printf("canonical4 mismatch k=%u\n", k);
                std::exit(1);
            }
            ++checks;
        }
        // run mask: random base/non-base bytes
        uint32_t fl[5];
        for (auto& f : fl) f = (uint32_t)rng() | (uint32_t)rng() | (uint32_t)rng();  // mostly bases
        if (iter % 3 == 0) fl[0] = fl[1] = fl[2] = fl[3] = fl[4] = 0xFFFFFFFFu;
        for (uint32_t k = 65; k <= 128; ++k) {
            const uint32_t got = runs_at_least5(fl[0], fl[1], fl[2], fl[3], fl[4], k);
            for (int b = 0; b < 32; ++b) {
                bool all = true;
                for (uint32_t q = 0; q < k && all; ++q) {
                    const int pos = 128 + b - (int)q;
                    all = (fl[pos / 32] >> (pos % 32)) & 1u;
                }
                if (all != (bool)((got >> b) & 1u)) {
                    std::printf("runs_at_least5 mismatch k=%u byte %d\n", k, b);
                    std::exit(1);
                }
            }
            ++checks;
        }
    }
    return checks;
}

// classify (bases, newlines and 2-bit codes of 32 bytes) against the
// per-byte definition, for random bytes (all 256 values, and runs of the
// letters that matter) and every valid length.
static long check_classify(std::mt19937_64& rng) {
    long checks = 0;
    const char* alpha = "ACGTUacgtuNn\n\r@+IJ";
    for (int iter = 0; iter < 200000; ++iter) {
        uint8_t b[32];
        for (int j = 0; j < 32; ++j)
            b[j] = (iter & 1) ? (uint8_t)alpha[rng() % 20] : (uint8_t)rng();
        uint32_t w[8];
        for (int i = 0; i < 8; ++i)
            w[i] = (uint32_t)b[4 * i] | ((uint32_t)b[4 * i + 1] << 8) | ((uint32_t)b[4 * i + 2] << 16) |
                   ((uint32_t)b[4 * i + 3] << 24);
        const uint64_t valid = iter % 7 == 0 ? rng() % 33 : 32;
        const Seg s = classify(w, valid);
        uint32_t bases = 0, nls = 0;
        uint64_t codes = 0;
        for (int j = 0; j < 32; ++j) {
            const uint32_t c = b[j], u = c & 0xDF;
            const bool base = u == 'A' || u == 'C' || u == 'G' || u == 'T' || u == 'U';
            if (base && (uint64_t)j < valid) bases |= 1u << j;
            if (c == '\n' && (uint64_t)j < valid) nls |= 1u << j;
            codes |= (uint64_t)(((c >> 1) ^ (c >> 2)) & 3u) << (62 - 2 * j);
        }
        if (s.bases != bases || s.nls != nls || s.codes != codes) {
            std::printf("classify mismatch at iteration %d\n", iter);
            std::exit(1);
        }
        ++checks;
    }
    return checks;
}

// pack_key (low.bin records, widest aligned stores) against the record
// layout written byte by byte: k/32 whole words little-endian, then the top
// ceil(2(k%32)/8) bytes of the masked tail word, for every k and records
// packed back to back from an aligned base.
static long check_pack_key(std::mt19937_64& rng) {
    long checks = 0;
    alignas(16) uint8_t got[40 * 8], want[40 * 8];
    for (uint32_t k = 1; k <= 128; ++k) {
        const uint32_t full = k / 32, tail_bits = 2 * (k % 32), tail_bytes = (tail_bits + 7) / 8;
        const uint32_t P = full * 8 + tail_bytes;
        const uint64_t tmask = tail_bits ? (~0ull << (64 - tail_bits)) : 0ull;
        for (int rep = 0; rep < 50; ++rep) {
            std::memset(got, 0xAB, sizeof got);
            std::memset(want, 0xAB, sizeof want);
            for (uint32_t i = 0; i < 8; ++i) {
                const uint64_t w[4] = {rng(), rng(), rng(), rng()};
                uint8_t* d = want + i * P;
                uint32_t q = 0;
                for (uint32_t f = 0; f < full; ++f)
                    for (uint32_t b = 0; b < 8; ++b) d[q++] = (uint8_t)(w[f] >> (8 * b));
                if (tail_bytes) {
                    const uint64_t tw = (full < 4 ? w[full] : 0ull) & tmask;
                    for (uint32_t b = 8 - tail_bytes; b < 8; ++b) d[q++] = (uint8_t)(tw >> (8 * b));
                }
                if (k <= 32) pack_key<1>(w[0], got + i * P, full, tail_bytes, P, tmask);
                else if (k <= 64) pack_key<2>(Key2{w[0], w[1]}, got + i * P, full, tail_bytes, P, tmask);
                else pack_key<4>(Key4{w[0], w[1], w[2], w[3]}, got + i * P, full, tail_bytes, P, tmask);
            }
            if (std::memcmp(got, want, sizeof got) != 0) {
                std::printf("pack_key mismatch k=%u\n", k);
                std::exit(1);
            }
            ++checks;
        }
    }
    return checks;
}

// nth_set_bit (the export's bitmap walk) against a plain enumeration.
static long check_nth_set_bit(std::mt19937_64& rng) {
    long checks = 0;
    for (int t = 0; t < 100000; ++t) {
        uint32_t x = (uint32_t)rng();
        if (t % 3 == 0) x &= (uint32_t)rng();
        if (t % 7 == 0) x = t % 14 ? 0xFFFFFFFFu : 0u;
        uint32_t r = 0;
        for (uint32_t b = 0; b < 32; ++b) {
            if (!((x >> b) & 1u)) continue;
            if (nth_set_bit(x, r) != b) {
                std::printf("nth_set_bit mismatch x=%08x r=%u\n", x, r);
                std::exit(1);
            }
            ++r;
            ++checks;
        }
    }
    return checks;
}

int main() {
    std::mt19937_64 rng(12345);
    long checks = 0;
    checks += check_nth_set_bit(rng);
    checks += check_pack_key(rng);
    checks += check_classify(rng);
    for (int iter = 0; iter < 20000; ++iter) {
        // three 32-byte segments of codes, byte 0 of each in bits 63..62
        std::vector<int> bases(96);
        for (auto& x : bases) x = (int)(rng() & 3);
        uint64_t seg[3] = {0, 0, 0};
        for (int s = 0; s < 3; ++s)
            for (int j = 0; j < 32; ++j) seg[s] |= (uint64_t)bases[32 * s + j] << (62 - 2 * j);
        const uint32_t j = (uint32_t)(rng() % 32);
        uint64_t lo, hi;
        window_at(seg[0], seg[1], seg[2], j, lo, hi);
        for (uint32_t k = 1; k <= 64; ++k) {
            const int end = 64 + (int)j;  // stream index of the newest base
            std::vector<int> win(bases.begin() + end - k + 1, bases.begin() + end + 1);
            // window value check (oldest base highest)
            for (uint32_t i = 0; i < k; ++i) {
                const uint32_t bit = 2 * (k - 1 - i);
                const uint64_t v = bit < 64 ? (lo >> bit) & 3 : (hi >> (bit - 64)) & 3;
                if ((int)v != win[i]) { std::printf("window mismatch k=%u j=%u\n", k, j); return 1; }
            }
            std::vector<int> rf(win.rbegin(), win.rend()), cc(win.size());
            for (size_t i = 0; i < win.size(); ++i) cc[i] = 3 - win[i];
            uint64_t F[2], C[2];
            pack_left(rf, F);
            pack_left(cc, C);
            const bool f_less = F[0] != C[0] ? F[0] < C[0] : F[1] < C[1];
            const uint64_t* want = f_less ? F : C;
            uint64_t got0, got1 = 0;
            if (k <= 32) {
                const uint64_t km = k >= 32 ? ~0ull : ((1ull << (2 * k)) - 1ull);
                got0 = canonical1(lo & km, k);
            } else {
                const uint32_t hb = 2 * k - 64;
                const uint64_t hm = hb >= 64 ? ~0ull : ((1ull << hb) - 1ull);
                const Key2 key = canonical2(hi & hm, lo, k);
                got0 = key.w0;
                got1 = key.w1;
            }
            if (got0 != want[0] || got1 != (k <= 32 ? 0 : want[1])) {
                std::printf("canonical mismatch k=%u\n", k);
                return 1;
            }
            for (uint32_t B : {8u, 12u}) {
                uint64_t l2 = lo, h2 = hi;
                if (k <= 32) l2 &= k >= 32 ? ~0ull : ((1ull << (2 * k)) - 1ull);
                else h2 &= (2 * k - 64) >= 64 ? ~0ull : ((1ull << (2 * k - 64)) - 1ull);
                const uint32_t b = bucket_of_window(l2, h2, k, B);
                if (b != (uint32_t)(want[0] >> (64 - B))) {
                    std::printf("bucket mismatch k=%u B=%u got %u want %u\n", k, B, b, (unsigned)(want[0] >> (64 - B)));
                    return 1;
                }
                // garbage above the window must not matter either
                const uint32_t b2 = bucket_of_window(lo, k <= 32 ? rng() : h2, k, B);
                if (k <= 32 && b2 != b) { std::printf("bucket depends on bits above the window k=%u\n", k); return 1; }
            }
            ++checks;
        }
    }
    checks += check_long_keys(rng);
    std::printf("ok %ld\n", checks);
    return 0;
}
