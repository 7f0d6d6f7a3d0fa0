// kc_count_device_noalloc: the whole count of a SMALL FASTQ held in device
// memory, with every piece of scratch memory taken from one file-scope
// device array instead of cudaMalloc.
//
// Who needs this: callers that must not allocate device memory on this path
// -- a framework whose caching allocator owns the whole device budget and
// forbids raw cudaMalloc, or a latency-sensitive service thread that cannot
// afford cudaMalloc/cudaFree (cudaFree synchronises the whole device, and a
// first-time cudaMalloc can stall).  They pass inputs and outputs as device
// pointers and a stream; this entry point allocates nothing (no cudaMalloc,
// cudaFree, cudaHostAlloc, stream or event creation, no library allocator).
//
// Limits and sharing rules:
//   * scratch = KC_NOALLOC_SCRATCH_BYTES (64 MiB) per device, held by every
//     GPU that loads this library until the process exits;
//   * input at most KC_NOALLOC_MAX_FASTQ_BYTES (1 MiB), 256 buckets, k 1..64,
//     canonical only; other requests are rejected with KC_ERR_INVALID before
//     any work;
//   * the first call on a device resolves the array's device address
//     (cudaGetSymbolAddress) with that device current.  Under CUDA's lazy
//     module loading (the default since CUDA 12.2) this is also when the
//     64 MiB are reserved, so make that first call before the caller's
//     allocator claims the device budget (or set CUDA_MODULE_LOADING=EAGER),
//     and before any stream capture;
//   * every call reuses the same array and clears what must start at zero;
//     calls that overlap on the GPU (two streams, two host threads) race on
//     it and must be serialised by the caller.
//
// The kernels are the same ones kc_count_device runs.

#include <algorithm>
#include <bit>
#include <cstring>

#include <cuda_runtime.h>

#include "../../include/kmer_count.h"
#include "kc_internal.h"
#include "kc_kernels.cuh"
#include "kc_scan.cuh"

namespace {

static __device__ __align__(256) uint8_t g_noalloc_scratch[KC_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
uint8_t* g_scratch_ptr[kMaxDevices] = {};

int err(int code, const char* msg) { return kc_internal_set_error(code, msg); }

#define NK(x)                                                                 \
    do {                                                                      \
        cudaError_t e_ = (x);                                                 \
        if (e_ != cudaSuccess) return err(KC_ERR_DEVICE, cudaGetErrorString(e_)); \
    } while (0)

// Inside a count: on a CUDA error, wait for the work already queued on the
// caller's stream first, so that no kernel of this call still reads the
// shared array or writes the caller's buffers after the call returned.
#define NKS(x)                                                                \
    do {                                                                      \
        cudaError_t e_ = (x);                                                 \
        if (e_ != cudaSuccess) {                                              \
            cudaStreamSynchronize(st);                                        \
            return err(KC_ERR_DEVICE, cudaGetErrorString(e_));                \
        }                                                                     \
    } while (0)

// Bump allocator over the static array (host-side offsets only).
struct Carve {
    uint8_t* base;
    uint64_t used = 0;
    bool ok = true;
    template <class T>
    T* take(uint64_t count) {
        const uint64_t off = (used + 255) & ~255ull;
        const uint64_t bytes = count * sizeof(T);
        if (off + bytes > KC_NOALLOC_SCRATCH_BYTES) {
            ok = false;
            return nullptr;
        }
        used = off + bytes;
        return reinterpret_cast<T*>(base + off);
    }
};

inline uint64_t cdiv(uint64_t a, uint64_t b) { return (a + b - 1) / b; }

template <class TI, class TO>
void scan(const TI* in, uint64_t n, TO* out, uint64_t base, uint64_t* sums, uint64_t* total, cudaStream_t st) {
    const uint64_t nb = std::max<uint64_t>(1, cdiv(n, kc::SCAN_TILE));
    if (n) kc::scan_reduce<TI><<<nb, kc::SCAN_BLOCK, 0, st>>>(in, n, sums);
    else cudaMemsetAsync(sums, 0, sizeof(uint64_t), st);
    kc::scan_sums<<<1, kc::SCAN_BLOCK, 0, st>>>(sums, n ? nb : 1, base, total);
    if (n) kc::scan_apply<TI, TO><<<nb, kc::SCAN_BLOCK, 0, st>>>(in, n, sums, out);
}

template <int NW>
int run(const kc_config* g, const uint8_t* d_fastq, uint64_t n, uint8_t* d_low, uint64_t low_cap, uint8_t* d_roots,
        uint64_t roots_cap, cudaStream_t st, uint8_t* scratch, kc_stats* stats) {
    constexpr int NB = 256, BITS = 8, SHIFT = 56;
    const uint32_t k = g->k;
    Carve cv{scratch};
    uint64_t* scal = cv.take<uint64_t>(16);
    const uint64_t tiles = cdiv(n, kc::EXT_TILE);
    uint32_t* tile_nl = cv.take<uint32_t>(std::max<uint64_t>(tiles, 1));
    uint64_t* tile_line = cv.take<uint64_t>(std::max<uint64_t>(tiles, 1));
    uint64_t* sums = cv.take<uint64_t>(4096);
    unsigned long long* bcount = cv.take<unsigned long long>(NB);
    unsigned long long* bcursor = cv.take<unsigned long long>(NB);
    uint32_t* overflow = cv.take<uint32_t>(NB);
    kc::BucketMeta* meta = cv.take<kc::BucketMeta>(NB);
    unsigned long long* rcount = cv.take<unsigned long long>(257);
    constexpr uint64_t MAX_CHUNKS = 1024;
    uint32_t* chunk_pass = cv.take<uint32_t>(MAX_CHUNKS);
    uint64_t* chunk_off = cv.take<uint64_t>(MAX_CHUNKS);
    if (!cv.ok) return err(KC_ERR_OVERFLOW, "no-alloc scratch exhausted (fixed part)");
    NKS(cudaMemsetAsync(scal, 0, 16 * sizeof(uint64_t), st));

    // line index per tile, then per-bucket k-mer totals
    if (tiles) kc::lines_per_tile<<<tiles, kc::EXT_THREADS, 0, st>>>(d_fastq, n, tile_nl);
    scan<uint32_t, uint64_t>(tile_nl, tiles, tile_line, 0, sums, scal + 0, st);
    NKS(cudaMemsetAsync(bcount, 0, NB * sizeof(uint64_t), st));
    kc::ExtractArgs ea{};
    ea.buf = d_fastq;
    ea.n = n;
    ea.has_halo = 0;
    ea.tile_line = tile_line;
    ea.k = k;
    ea.bucket_shift = SHIFT;
    ea.n_buckets = NB;
    ea.bucket_count = bcount;
    ea.bucket_cursor = bcursor;
    ea.error = reinterpret_cast<uint32_t*>(scal + 8);
    if (tiles) kc::extract_kernel<NW, kc::HIST><<<tiles, kc::EXT_THREADS, kc::extract_smem_bytes<NW, kc::HIST>(NB), st>>>(ea);
    NKS(cudaGetLastError());
    uint64_t h_count[NB];
    NKS(cudaMemcpyAsync(h_count, bcount, sizeof h_count, cudaMemcpyDeviceToHost, st));
    NKS(cudaStreamSynchronize(st));
    uint64_t start[NB], K = 0;
    for (int b = 0; b < NB; ++b) {
        start[b] = K;
        K += h_count[b];
    }

    // k-mer dependent scratch: routed keys, per-segment counters, filter, tables
    constexpr int CT = kc::count_tile<NW>();
    constexpr int SEG = kc::count_seg<NW>();
    const uint64_t ctiles = cdiv(K, CT), nsegs = cdiv(K, SEG);
    using KeyT = typename kc::KeyOf<NW>::T;
    using SlotT = typename kc::SlotOf<NW>::T;
    KeyT* routed = cv.take<KeyT>(std::max<uint64_t>(ctiles * CT, 1));
    uint32_t* seg_low = cv.take<uint32_t>(std::max<uint64_t>(ctiles * (CT / SEG), 1));
    uint32_t* seg_fail = cv.take<uint32_t>(std::max<uint64_t>(ctiles * (CT / SEG), 1));
    uint64_t* seg_prefix = cv.take<uint64_t>(std::max<uint64_t>(ctiles * (CT / SEG), 1));
    kc::BucketMeta h_meta[NB];
    uint64_t bw = 0, ts = 0;
    for (int b = 0; b < NB; ++b) {
        const double kb = (double)h_count[b];
        const uint64_t words = std::bit_ceil(std::max<uint64_t>((uint64_t)(kb * g->bloom_bits / 64.0), 64));
        const uint64_t slots = std::bit_ceil(std::max<uint64_t>((uint64_t)(kb * g->repeat_ratio / g->table_load), 64));
        h_meta[b] = kc::BucketMeta{bw, words - 1, ts, slots - 1};
        bw += words;
        ts += slots;
    }
    uint64_t* bloom = cv.take<uint64_t>(bw);
    if (!cv.ok) return err(KC_ERR_OVERFLOW, "no-alloc scratch exhausted: input has too many k-mers");
    // the table arena takes the rest; growth after an overflow comes from it
    const uint64_t tab_off = (cv.used + 255) & ~255ull;
    const uint64_t tab_cap = (KC_NOALLOC_SCRATCH_BYTES - tab_off) / sizeof(SlotT);
    SlotT* table = reinterpret_cast<SlotT*>(scratch + tab_off);
    if (ts > tab_cap) return err(KC_ERR_OVERFLOW, "no-alloc scratch exhausted: tables do not fit");

    NKS(cudaMemcpyAsync(meta, h_meta, sizeof h_meta, cudaMemcpyHostToDevice, st));
    NKS(cudaMemsetAsync(bloom, 0, bw * sizeof(uint64_t), st));
    NKS(cudaMemsetAsync(overflow, 0, NB * sizeof(uint32_t), st));
    kc::init_slots<NW><<<256, 256, 0, st>>>(table, ts);
    NKS(cudaMemcpyAsync(bcursor, start, sizeof start, cudaMemcpyHostToDevice, st));
    ea.routed = routed;
    // the scatter's staging area needs more than the default 48 KiB
    const size_t smem_sc = kc::extract_smem_bytes<NW, kc::SCATTER>(NB);
    NKS(cudaFuncSetAttribute(kc::extract_kernel<NW, kc::SCATTER>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_sc));
    if (tiles) kc::extract_kernel<NW, kc::SCATTER><<<tiles, kc::EXT_THREADS, smem_sc, st>>>(ea);

    kc::CountArgs ca{};
    ca.routed = routed;
    ca.n_keys = K;
    ca.meta = meta;
    ca.bloom = bloom;
    ca.table = table;
    ca.seg_low = seg_low;
    ca.seg_fail = seg_fail;
    ca.bucket_overflow = overflow;
    ca.bucket_shift = SHIFT;
    ca.n_buckets = NB;
    ca.use_filter = 1;
    const uint64_t cgrid = cdiv(K, (uint64_t)CT * kc::CNT_SEGS_PER_WARP);
    if (cgrid) kc::count_routed<NW><<<cgrid, kc::CNT_THREADS, 0, st>>>(ca);
    NKS(cudaGetLastError());

    // overflow: grow the bucket's table inside the arena, move, retry
    uint64_t rehashes = 0;
    for (int round = 0;; ++round) {
        uint32_t h_over[NB];
        NKS(cudaMemcpyAsync(h_over, overflow, sizeof h_over, cudaMemcpyDeviceToHost, st));
        NKS(cudaStreamSynchronize(st));
        bool any = false;
        for (int b = 0; b < NB; ++b) any |= h_over[b] != 0;
        if (!any) break;
        if (round > 16) return err(KC_ERR_OVERFLOW, "no-alloc tables kept overflowing");
        NKS(cudaMemsetAsync(overflow, 0, NB * sizeof(uint32_t), st));
        for (int b = 0; b < NB; ++b) {
            if (!h_over[b]) continue;
            // grow x4 into the free end of the arena; a growth whose rehash
            // still meets a full probe window (pathological clustering) is
            // dropped and the table grown x4 again, as the engine does
            const uint64_t old_slots = h_meta[b].tab_mask + 1;
            for (uint64_t new_slots = old_slots * 4;; new_slots *= 4) {
                if (ts + new_slots > tab_cap)
                    return err(KC_ERR_OVERFLOW, "no-alloc scratch exhausted while growing a table");
                kc::init_slots<NW><<<64, 256, 0, st>>>(table + ts, new_slots);
                uint32_t* failed = reinterpret_cast<uint32_t*>(scal + 9);
                NKS(cudaMemsetAsync(failed, 0, sizeof(uint32_t), st));
                kc::rehash_bucket<NW><<<64, 256, 0, st>>>(table + h_meta[b].tab_off, old_slots, table + ts,
                                                          new_slots - 1, failed);
                uint32_t h_failed = 0;
                NKS(cudaMemcpyAsync(&h_failed, failed, sizeof h_failed, cudaMemcpyDeviceToHost, st));
                NKS(cudaStreamSynchronize(st));
                if (!h_failed) {
                    h_meta[b].tab_off = ts;
                    h_meta[b].tab_mask = new_slots - 1;
                    ts += new_slots;
                    break;
                }
            }
            ++rehashes;
        }
        NKS(cudaMemcpyAsync(meta, h_meta, sizeof h_meta, cudaMemcpyHostToDevice, st));
        ca.use_filter = 0;
        kc::count_routed<NW><<<cgrid, kc::CNT_THREADS, 0, st>>>(ca);
        NKS(cudaGetLastError());
    }

    // first occurrences -> packed low.bin bytes in the caller's buffer
    scan<uint32_t, uint64_t>(seg_low, nsegs, seg_prefix, 0, sums, scal + 1, st);
    uint64_t nlow = 0;
    uint32_t ext_err = 0;
    NKS(cudaMemcpyAsync(&nlow, scal + 1, sizeof nlow, cudaMemcpyDeviceToHost, st));
    NKS(cudaMemcpyAsync(&ext_err, scal + 8, sizeof ext_err, cudaMemcpyDeviceToHost, st));
    NKS(cudaStreamSynchronize(st));
    if (ext_err) return err(KC_ERR_DEVICE, "internal error: routing bucket disagreed with its reservation");
    const uint64_t P = kc_packed_bytes(k);
    if (nlow * P > low_cap) return err(KC_ERR_INVALID, "low output buffer too small");

    // export chunk list (root records grouped by root id): checked for room
    // before anything else is launched, so every error return below finds
    // the stream idle
    kc::ExportChunk h_chunks[MAX_CHUNKS];
    uint64_t nch = 0;
    const uint64_t CH = std::max<uint64_t>(16384, cdiv(ts, 700));
    for (int b = 0; b < NB; ++b) {
        const uint64_t slots = h_meta[b].tab_mask + 1;
        for (uint64_t s = 0; s < slots && nch < MAX_CHUNKS; s += CH)
            h_chunks[nch++] = kc::ExportChunk{h_meta[b].tab_off + s, (uint32_t)std::min<uint64_t>(CH, slots - s), (uint32_t)b};
    }
    kc::ExportChunk* chunks = reinterpret_cast<kc::ExportChunk*>(table + ts);
    if ((ts * sizeof(SlotT) + nch * sizeof(kc::ExportChunk) + 256) > tab_cap * sizeof(SlotT))
        return err(KC_ERR_OVERFLOW, "no-alloc scratch exhausted at export");
    if (nsegs)
        kc::pack_low<NW><<<std::min<uint64_t>(cdiv(nsegs, 256), 148 * 4), 256, 0, st>>>(routed, seg_low, seg_prefix,
                                                                                       nsegs, k, d_low, 0);

    // root records grouped by root id
    NKS(cudaMemcpyAsync(chunks, h_chunks, nch * sizeof(kc::ExportChunk), cudaMemcpyHostToDevice, st));
    NKS(cudaMemsetAsync(rcount, 0, 257 * sizeof(uint64_t), st));
    const uint64_t egrid = std::max<uint64_t>(1, std::min<uint64_t>(nch, 148 * 4));
    if (nch)
        kc::export_count<NW><<<egrid, kc::EXP_THREADS, 0, st>>>(table, chunks, nch, g->min_count, g->max_count,
                                                                chunk_pass, rcount, rcount + 256, nullptr);
    uint64_t h_r[257];
    uint32_t h_pass[MAX_CHUNKS];
    NKS(cudaMemcpyAsync(h_r, rcount, sizeof h_r, cudaMemcpyDeviceToHost, st));
    if (nch) NKS(cudaMemcpyAsync(h_pass, chunk_pass, nch * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    NKS(cudaStreamSynchronize(st));
    uint64_t R = 0;
    for (int r = 0; r < 256; ++r) R += h_r[r];
    uint64_t h_off[MAX_CHUNKS];
    for (uint64_t i = 0, o = 0; i < nch; ++i) {
        h_off[i] = o;
        o += h_pass[i];
    }
    const uint64_t rec = kc_record_bytes(k);
    if (R * rec > roots_cap) return err(KC_ERR_INVALID, "root output buffer too small");
    if (nch) NKS(cudaMemcpyAsync(chunk_off, h_off, nch * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
    if (nch && R)
        kc::export_write<NW><<<egrid, kc::EXP_THREADS, 0, st>>>(table, chunks, nch, g->min_count, g->max_count,
                                                                chunk_off, d_roots);
    NKS(cudaGetLastError());
    NKS(cudaStreamSynchronize(st));
    if (stats) {
        std::memset(stats, 0, sizeof *stats);
        stats->input_bytes = n;
        stats->total_kmers = K;
        stats->low_records = nlow;
        stats->root_records = R;
        stats->table_keys = h_r[256];
        stats->rehashes = rehashes;
        stats->batches = 1;
        for (int r = 0; r < 256; ++r) stats->root_counts[r] = h_r[r];
        for (int b = 0; b < NB; ++b) {
            stats->table_slots += h_meta[b].tab_mask + 1;
            stats->max_bucket_table_slots = std::max<uint64_t>(stats->max_bucket_table_slots, h_meta[b].tab_mask + 1);
            stats->max_bucket_filter_words = std::max<uint64_t>(stats->max_bucket_filter_words, h_meta[b].bloom_mask + 1);
            stats->filter_words += h_meta[b].bloom_mask + 1;
        }
    }
    (void)BITS;
    return KC_OK;
}

}  // namespace

extern "C" int kc_count_device_noalloc(const kc_config* cfg, const uint8_t* d_fastq, uint64_t n, uint8_t* d_low,
                                       uint64_t low_cap, uint8_t* d_roots, uint64_t roots_cap, void* stream,
                                       kc_stats* stats) {
    if (!cfg || (!d_fastq && n)) return err(KC_ERR_INVALID, "null argument");
    if (cfg->k < 1 || cfg->k > 64) return err(KC_ERR_INVALID, "k out of range: 1..64");
    if (cfg->canonical != 1) return err(KC_ERR_INVALID, "only canonical counting is supported");
    if (cfg->max_count < cfg->min_count) return err(KC_ERR_INVALID, "max_count < min_count");
    if (cfg->n_buckets != 256) return err(KC_ERR_INVALID, "the no-alloc entry point supports 256 buckets only");
    if (cfg->bloom_bits <= 0.0 || cfg->table_load <= 0.05 || cfg->table_load > 0.95 || cfg->repeat_ratio <= 0.0)
        return err(KC_ERR_INVALID, "bloom_bits, table_load (0.05..0.95) and repeat_ratio must be positive");
    if (n > KC_NOALLOC_MAX_FASTQ_BYTES)
        return err(KC_ERR_INVALID, "input larger than KC_NOALLOC_MAX_FASTQ_BYTES (1 MiB) for the no-alloc entry point");
    if (reinterpret_cast<uintptr_t>(d_fastq) % 16) return err(KC_ERR_INVALID, "device FASTQ must be 16-byte aligned");
    // the packing and export kernels store whole words into the outputs
    if (reinterpret_cast<uintptr_t>(d_low) % 16 || reinterpret_cast<uintptr_t>(d_roots) % 16)
        return err(KC_ERR_INVALID, "output buffers must be 16-byte aligned");
    int dev = 0;
    NK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return err(KC_ERR_DEVICE, "device ordinal out of range for the no-alloc path");
    if (!g_scratch_ptr[dev]) {
        // one-time set-up on this device (the current one): resolve the
        // static array's device address; do this call before any capture
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) return err(KC_ERR_DEVICE, "cudaGetSymbolAddress of the no-alloc scratch failed");
        g_scratch_ptr[dev] = static_cast<uint8_t*>(p);
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    return cfg->k <= 32 ? run<1>(cfg, d_fastq, n, d_low, low_cap, d_roots, roots_cap, st, g_scratch_ptr[dev], stats)
                        : run<2>(cfg, d_fastq, n, d_low, low_cap, d_roots, roots_cap, st, g_scratch_ptr[dev], stats);
}
