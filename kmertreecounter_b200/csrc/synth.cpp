// Seeded synthetic genomes and FASTQ read sets.
//
// The reference has no public dataset; its benchmark shapes are described by
// genome length, GC content, repeat-family structure, coverage, read length,
// substitution and N rates.  This generator produces FASTQ bytes of those
// shapes deterministically from a 64-bit seed: every read is a pure function
// of (seed, read index), so the same file comes out on any thread count.
//
// Record layout (strict 4-line FASTQ, as the reference reader expects,
// src/FastqReader.h:293-308):
//     @r<index>\n<bases>\n+\n<qualities Phred+33 uniform 20..40>\n

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "../../include/kmer_synth.h"

namespace {

inline uint64_t splitmix(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

struct Rng {
    uint64_t s;
    explicit Rng(uint64_t seed) : s(seed) {}
    uint64_t next() { return splitmix(s); }
    double uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
    uint64_t below(uint64_t n) { return n ? (uint64_t)(((unsigned __int128)next() * n) >> 64) : 0; }
};

const char kBases[4] = {'A', 'C', 'G', 'T'};

inline char gc_base(Rng& r, double gc) {
    const double u = r.uniform();
    if (u < gc) return (u < gc * 0.5) ? 'C' : 'G';
    return (u < gc + (1.0 - gc) * 0.5) ? 'A' : 'T';
}

inline char substitute(Rng& r, char b) {
    static const char others[4][3] = {{'C', 'G', 'T'}, {'A', 'G', 'T'}, {'A', 'C', 'T'}, {'A', 'C', 'G'}};
    const int idx = b == 'A' ? 0 : b == 'C' ? 1 : b == 'G' ? 2 : 3;
    return others[idx][r.below(3)];
}

inline char complement(char b) {
    switch (b) {
        case 'A': return 'T';
        case 'C': return 'G';
        case 'G': return 'C';
        default: return 'A';
    }
}

inline uint64_t read_seed(uint64_t seed, uint64_t i) {
    uint64_t s = seed ^ (i * 0xD1B54A32D192ED03ULL + 0x8CB92BA72F3D8DD7ULL);
    splitmix(s);
    return s;
}

inline uint32_t read_length(const kc_synth_params* p, Rng& r) {
    if (p->read_len_max <= p->read_len_min) return p->read_len_min;
    return p->read_len_min + (uint32_t)r.below(p->read_len_max - p->read_len_min + 1);
}

inline uint32_t digits(uint64_t v) {
    uint32_t d = 1;
    while (v >= 10) { v /= 10; ++d; }
    return d;
}

// Bytes of record i: '@' 'r' digits '\n' L '\n' '+' '\n' L '\n'
inline uint64_t record_bytes(uint64_t i, uint32_t L) { return 2 + digits(i) + 1 + L + 3 + L + 1; }

void write_record(const kc_synth_params* p, const uint8_t* genome, uint64_t i, uint8_t* out) {
    Rng r(read_seed(p->seed, i));
    const uint32_t L = read_length(p, r);
    const uint64_t G = p->genome_len;
    const uint64_t span = G > L ? G - L + 1 : 1;
    const uint64_t pos = r.below(span);
    const bool rc = (r.next() >> 63) != 0;
    uint8_t* o = out;
    *o++ = '@';
    *o++ = 'r';
    {
        char tmp[24];
        uint32_t n = 0;
        uint64_t v = i;
        do { tmp[n++] = (char)('0' + v % 10); v /= 10; } while (v);
        while (n) *o++ = (uint8_t)tmp[--n];
    }
    *o++ = '\n';
    for (uint32_t j = 0; j < L; ++j) {
        char b;
        const uint64_t gi = pos + j;
        if (gi >= G) b = 'A';
        else if (!rc) b = (char)genome[gi];
        else b = complement((char)genome[pos + (L - 1 - j) < G ? pos + (L - 1 - j) : G - 1]);
        double rate = p->sub_rate;
        if (p->sub_profile == 1 && L > 1) rate = 2.0 * p->sub_rate * (j + 0.5) / (double)L;
        if (r.uniform() < rate) b = substitute(r, b);
        if (r.uniform() < p->n_rate) b = 'N';
        *o++ = (uint8_t)b;
    }
    *o++ = '\n';
    *o++ = '+';
    *o++ = '\n';
    for (uint32_t j = 0; j < L; ++j) *o++ = (uint8_t)(33 + 20 + r.below(21));
    *o++ = '\n';
}

// Splits [0, n) into `threads` contiguous ranges, one std::thread each.
template <class F>
void parallel_for(uint64_t n, uint32_t threads, F&& f) {
    if (threads <= 1 || n <= 1) { f(0, n); return; }
    std::vector<std::thread> pool;
    const uint64_t step = (n + threads - 1) / threads;
    for (uint32_t t = 0; t < threads; ++t) {
        const uint64_t a = t * step, b = std::min(n, a + step);
        if (a >= b) break;
        pool.emplace_back([=, &f] { f(a, b); });
    }
    for (auto& th : pool) th.join();
}

uint32_t default_threads(uint32_t t) {
    if (t) return t;
    const unsigned hc = std::thread::hardware_concurrency();
    return hc ? std::min(hc, 64u) : 1u;
}

}  // namespace

extern "C" {

int kc_synth_genome(const kc_synth_params* p, uint8_t* genome) {
    if (!p || !genome || p->genome_len == 0) return -1;
    const uint64_t G = p->genome_len;
    const uint32_t threads = default_threads(p->threads);
    // i.i.d. background, generated in independent 1 Mbp slabs so that it is
    // thread-count independent.
    const uint64_t slab = 1ull << 20;
    const uint64_t nslab = (G + slab - 1) / slab;
    parallel_for(nslab, threads, [&](uint64_t a, uint64_t b) {
        for (uint64_t s = a; s < b; ++s) {
            Rng r(read_seed(p->seed ^ 0x5bd1e995ULL, s));
            const uint64_t lo = s * slab, hi = std::min(G, lo + slab);
            if (p->gc == 0.5) {
                for (uint64_t i = lo; i < hi;) {
                    uint64_t w = r.next();
                    for (int j = 0; j < 32 && i < hi; ++j, ++i, w >>= 2) genome[i] = (uint8_t)kBases[w & 3];
                }
            } else {
                for (uint64_t i = lo; i < hi; ++i) genome[i] = (uint8_t)gc_base(r, p->gc);
            }
        }
    });
    // Repeat families: a template of rep_min_len..rep_max_len bases copied
    // rep_min_copies..rep_max_copies times at uniform positions, each copy
    // diverged by rep_divergence, until repeat_frac of the genome is covered.
    if (p->repeat_frac > 0.0 && p->rep_max_len > 0 && G > p->rep_max_len) {
        Rng r(p->seed ^ 0xC2B2AE3D27D4EB4FULL);
        const double target = p->repeat_frac * (double)G;
        double covered = 0.0;
        std::vector<char> tmpl;
        while (covered < target) {
            const uint32_t lo = std::max<uint32_t>(1, p->rep_min_len), hi = std::max(lo, p->rep_max_len);
            const uint32_t L = lo + (uint32_t)r.below(hi - lo + 1);
            const uint32_t clo = std::max<uint32_t>(2, p->rep_min_copies), chi = std::max(clo, p->rep_max_copies);
            const uint32_t copies = clo + (uint32_t)r.below(chi - clo + 1);
            tmpl.resize(L);
            for (uint32_t i = 0; i < L; ++i) tmpl[i] = gc_base(r, p->gc);
            for (uint32_t c = 0; c < copies; ++c) {
                const uint64_t pos = r.below(G - L + 1);
                for (uint32_t i = 0; i < L; ++i) {
                    char b = tmpl[i];
                    if (r.uniform() < p->rep_divergence) b = substitute(r, b);
                    genome[pos + i] = (uint8_t)b;
                }
                covered += L;
            }
        }
    }
    return 0;
}

uint64_t kc_synth_fastq_bytes(const kc_synth_params* p) {
    if (!p) return 0;
    const uint32_t threads = default_threads(p->threads);
    std::vector<uint64_t> sums(threads, 0);
    const uint64_t step = (p->n_reads + threads - 1) / (threads ? threads : 1);
    parallel_for(threads, threads, [&](uint64_t a, uint64_t b) {
        for (uint64_t t = a; t < b; ++t) {
            uint64_t s = 0;
            const uint64_t lo = t * step, hi = std::min(p->n_reads, lo + step);
            for (uint64_t i = lo; i < hi; ++i) {
                Rng r(read_seed(p->seed, i));
                s += record_bytes(i, read_length(p, r));
            }
            sums[t] = s;
        }
    });
    uint64_t total = 0;
    for (uint64_t s : sums) total += s;
    return total;
}

int64_t kc_synth_fastq(const kc_synth_params* p, const uint8_t* genome, uint8_t* out, uint64_t cap) {
    if (!p || !genome || !out) return -1;
    const uint32_t threads = default_threads(p->threads);
    const uint64_t n = p->n_reads;
    const uint64_t step = (n + threads - 1) / threads;
    std::vector<uint64_t> sums(threads + 1, 0);
    parallel_for(threads, threads, [&](uint64_t a, uint64_t b) {
        for (uint64_t t = a; t < b; ++t) {
            uint64_t s = 0;
            const uint64_t lo = t * step, hi = std::min(n, lo + step);
            for (uint64_t i = lo; i < hi; ++i) {
                Rng r(read_seed(p->seed, i));
                s += record_bytes(i, read_length(p, r));
            }
            sums[t + 1] = s;
        }
    });
    for (uint32_t t = 0; t < threads; ++t) sums[t + 1] += sums[t];
    if (sums[threads] > cap) return -(int64_t)sums[threads];
    parallel_for(threads, threads, [&](uint64_t a, uint64_t b) {
        for (uint64_t t = a; t < b; ++t) {
            uint64_t off = sums[t];
            const uint64_t lo = t * step, hi = std::min(n, lo + step);
            for (uint64_t i = lo; i < hi; ++i) {
                Rng r(read_seed(p->seed, i));
                const uint32_t L = read_length(p, r);
                write_record(p, genome, i, out + off);
                off += record_bytes(i, L);
            }
        }
    });
    return (int64_t)sums[threads];
}

}  // extern "C"
