// Host engine and C ABI of the B200 exact canonical k-mer counter.
//
// One kc_context = one CUDA stream + the device buffers of the pipeline.  A
// count runs batch by batch over the FASTQ bytes (one batch = up to
// batch_bytes, resident in HBM), then exports the repeat tables:
//
//   per batch   lines_per_tile -> scan -> extract<HIST> -> [size tables on the
//               first batch] -> extract<SCATTER> -> count_routed -> [rehash
//               overflowed buckets + retry] -> scan -> pack_low
//   at the end  export_count -> export_write (ExportRecord<N> grouped by root)
//
// This replaces the reference's reader/parser/classifier/tree thread pipeline
// (src/main.cpp:111-312) as a whole; see the kernel header for the per-kernel
// correspondence.

#include <algorithm>
#include <bit>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <cerrno>
#include <unistd.h>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/kmer_count.h"
#include "../../include/kmer_sizing.h"
#include "kc_internal.h"
#include "kc_kernels.cuh"
#include "kc_scan.cuh"
#include "kc_window.cuh"

namespace {

thread_local std::string g_err;

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

#define CK(x)                                                                                         \
    do {                                                                                              \
        cudaError_t e_ = (x);                                                                         \
        if (e_ != cudaSuccess) return fail(KC_ERR_DEVICE, "%s failed: %s (%s:%d)", #x, cudaGetErrorString(e_), \
                                           __FILE__, __LINE__);                                       \
    } while (0)

struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
    // Grow to at least `bytes` (contents not kept).
    cudaError_t ensure(size_t bytes) {
        if (bytes <= cap && p) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        size_t want = std::max<size_t>(bytes + bytes / 8, 4096);
        cudaError_t e = cudaMalloc(&p, want);
        if (e != cudaSuccess) {
            cudaGetLastError();
            e = cudaMalloc(&p, bytes);
            want = bytes;
        }
        if (e == cudaSuccess) cap = want;
        else p = nullptr;
        return e;
    }
    // Grow keeping the first `keep` bytes.
    cudaError_t grow_keep(size_t bytes, size_t keep, cudaStream_t st) {
        if (bytes <= cap && p) return cudaSuccess;
        void* q = nullptr;
        size_t want = std::max<size_t>(bytes + bytes / 4, 4096);
        cudaError_t e = cudaMalloc(&q, want);
        if (e != cudaSuccess) {
            cudaGetLastError();
            want = bytes;
            e = cudaMalloc(&q, want);
            if (e != cudaSuccess) return e;
        }
        if (p && keep) {
            e = cudaMemcpyAsync(q, p, keep, cudaMemcpyDeviceToDevice, st);
            if (e != cudaSuccess) return e;
            e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) return e;
        }
        if (p) cudaFree(p);
        p = q;
        cap = want;
        return cudaSuccess;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
    template <class T>
    T* as() const {
        return reinterpret_cast<T*>(p);
    }
};

inline uint64_t ceil_div(uint64_t a, uint64_t b) { return (a + b - 1) / b; }
inline uint64_t pow2_at_least(uint64_t x) { return std::bit_ceil(std::max<uint64_t>(x, 1)); }

}  // namespace

struct kc_context {
    kc_config cfg{};
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // table initialisation runs on `side` (high priority) beside the
    // extraction; `stream` waits for ev_init before the table's first use
    cudaStream_t side = nullptr;
    cudaEvent_t ev_side_in = nullptr, ev_init = nullptr;
    bool init_pending = false;
    uint32_t nw = 1, bucket_bits = 8, n_buckets = 256, bucket_shift = 56;
    int sm_count = 148;
    uint64_t slot_bytes = 16, record_bytes = 16, packed_bytes = 8;

    // host-input streaming: copy streams, double-buffered staging, pinned ring
    cudaStream_t h2d = nullptr, d2h = nullptr;
    cudaEvent_t ev_h2d[2] = {}, ev_free[2] = {}, ev_pack = nullptr, ev_lowfree[2] = {};
    DevBuf stage2;       // second [HALO | batch | pad] staging buffer
    DevBuf lowring[2];   // per-batch packed first occurrences (streamed mode)
    int batch_slot = 0;  // staging slot of the batch being counted
    cudaEvent_t after_scatter = nullptr;  // recorded once the batch's FASTQ bytes are no longer read
    bool stream_low = false;
    kc_sink_fn sink = nullptr;
    void* sink_user = nullptr;
    int sink_rc = 0;        // first non-zero sink return (guarded by pin_mu)
    bool deliver_err = false;  // a piece's copy failed (guarded by pin_mu)
    static constexpr uint64_t PIN_BYTES = 128ull << 20;
    static constexpr int PIN_SLOTS = 4;
    // input read from a file descriptor (kc_count_fastq): pieces are read
    // into a small pinned ring by parallel preads, then copied to the device
    int src_fd = -1;
    static constexpr uint64_t RING_BYTES = 64ull << 20;
    static constexpr int RING_SLOTS = 4;
    uint8_t* ring[RING_SLOTS] = {};
    cudaEvent_t ev_ring[RING_SLOTS] = {};
    uint64_t ring_next = 0;
    uint8_t* pin[PIN_SLOTS] = {};
    cudaEvent_t ev_pin[PIN_SLOTS] = {};
    struct Piece {
        int kind;
        uint32_t root;
        uint64_t bytes;
        int slot;
    };
    // FIFO of in-flight device->host pieces, delivered to the sink in order by
    // the `deliverer` thread; slot_busy / pending / flags are guarded by pin_mu
    std::deque<Piece> pending;
    bool slot_busy[PIN_SLOTS] = {};
    bool deliver_stop = false;
    std::mutex pin_mu;
    std::condition_variable pin_cv;
    std::thread deliverer;

    // batch pipeline
    DevBuf stage;        // [HALO | batch | pad] for host input
    DevBuf tile_nl, tile_line;
    DevBuf bucket_count, bucket_cursor, region_end, region_fill;
    DevBuf routed;
    DevBuf tile_low, tile_fail, tile_low_prefix;
    DevBuf scan_sums, scalars;
    DevBuf overflow, meta;
    DevBuf bloom, table;
    DevBuf low_packed;
    DevBuf roots, chunks, chunk_pass, chunk_off, root_count;
    DevBuf pass_bits;  // export: bit per table slot that passes min..max
    DevBuf grow_jobs, grow_failed;  // table growth of many buckets at once
    DevBuf loads;      // kc_bucket_loads: per-model-bucket totals (kept: no cudaMalloc/cudaFree per call)
    uint64_t n_chunks = 0;  // entries of `chunks` (live table regions) of the last export
    // kc_route_device: keys held in `routed` (bucket order) and per routing bucket
    uint64_t routed_keys = 0;
    std::vector<uint64_t> route_counts;
    bool have_route = false;
    DevBuf sort_tmp, sort_hist, sort_offs, sort_sums;
    DevBuf set_tiles, tile_prefix, set_info, hist_tiles;  // multi-set batches
    std::vector<double> set_pred_distinct, set_pred_table;  // learned rates per (set, root bucket)
    // the multi-set scatter/gap/count graphs, replayed: one executable per
    // shape (key width and kernel list; estimated regions add a gap fill)
    static constexpr int SETS_EXECS = 4;
    cudaGraphExec_t sets_exec[SETS_EXECS] = {};
    int sets_exec_key[SETS_EXECS] = {};
    int sets_exec_next = 0;                   // slot a new shape replaces
    uint64_t sets_instantiations = 0;         // times that graph had to be instantiated
    // windowed count of 64-bit keys (kc_window.cuh): window-grouped keys,
    // per-bucket window ids and per-window counts and key ranges
    bool window_count = true;    // KC_WINDOW_COUNT=0 in the environment: count_routed only
    bool win_ready = false;      // windows built for the current table layout
    uint64_t n_wins = 0, n_wins_phase0 = 0;
    std::vector<kc::BucketWin> h_bucket_win;
    std::vector<kc::WinInfo> h_win_info;
    std::vector<uint32_t> h_win_order;  // windows in launch order: phase 0, then phase 1
    DevBuf routed2, bucket_win, win_info, win_order, win_count, win_padded, win_start, win_cursor, win_end;
    uint64_t window_spill = 0;   // keys counted from the spill area (all batches of the run)

    // host mirrors
    std::vector<kc::BucketMeta> h_meta;
    std::vector<uint64_t> h_bucket_count;
    std::vector<uint32_t> h_overflow;
    uint64_t bloom_words = 0, table_slots_used = 0;
    bool sized = false;
    uint64_t expected_total_bytes = 0;

    // run state
    uint64_t line_base = 0;
    uint64_t low_total = 0;
    uint64_t last_batch_low = 0;
    uint64_t K = 0;
    uint64_t rehashes = 0, batches = 0, input_bytes = 0;
    uint64_t overflow_keys = 0, reroutes = 0;  // estimated bucket regions (kc_stats)
    bool have_result = false;
    bool batch_result = false;   // last result came from kc_count_sets
    uint64_t batch_low_bytes = 0;
    uint64_t root_total = 0, table_keys = 0;
    uint64_t root_counts[256] = {};

    // optional learned sizing hook (per-bucket repeat-key predictions)
    std::vector<double> pred_distinct, pred_table;  // learned sizing, per model bucket (4096)
    kc_sizing_fn sizing_cb = nullptr;  // learned sizing: called at each count's sizing point
    void* sizing_user = nullptr;
    bool side_in_ready = false;        // ev_side_in already recorded for this sizing

    // control-path mailbox: mapped pinned memory, [0, MBOX_UP) for uploads and
    // [MBOX_UP, MBOX_UP + MBOX_DOWN) for readbacks (put / get / sync_stream)
    static constexpr uint64_t MBOX_UP = 512ull << 10, MBOX_DOWN = 512ull << 10;
    uint8_t* mbox_h = nullptr;
    uint8_t* mbox_d = nullptr;
    uint64_t mbox_up_off = 0, mbox_down_off = 0;
    cudaEvent_t ev_mbox = nullptr;
    struct Readback {
        void* dst;
        uint64_t off, bytes;
    };
    std::vector<Readback> readbacks;

    // stage profiling: CUDA event pairs recorded on `stream` around each stage
    bool profiling = false;
    std::vector<cudaEvent_t> ev_pool;
    size_t ev_used = 0;
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> spans;
    uint64_t launches[KC_STAGE_COUNT] = {};
    double stage_ms[KC_STAGE_COUNT] = {};
};

namespace {

const char* const kStageNames[KC_STAGE_COUNT] = {"lines", "scan", "extract_hist", "extract_scatter", "count",
                                                  "rehash", "pack_low", "export", "sort", "init", "subroute"};

cudaEvent_t next_event(kc_context* c) {
    if (c->ev_used == c->ev_pool.size()) {
        cudaEvent_t e = nullptr;
        if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
        c->ev_pool.push_back(e);
    }
    return c->ev_pool[c->ev_used++];
}

// RAII span: records start/end events of a stage when profiling is on and
// counts the launches issued inside it.
struct Stage {
    kc_context* c;
    int id;
    cudaStream_t st;
    cudaEvent_t a = nullptr;
    Stage(kc_context* ctx, int s, uint64_t n_launch = 1, cudaStream_t on = nullptr)
        : c(ctx), id(s), st(on ? on : ctx->stream) {
        c->launches[s] += n_launch;
        if (c->profiling && (a = next_event(c))) cudaEventRecord(a, st);
    }
    ~Stage() {
        if (!a) return;
        cudaEvent_t b = next_event(c);
        if (!b) return;
        cudaEventRecord(b, st);
        c->spans.push_back({id, {a, b}});
    }
};

// CTAs of a grid-stride kernel that are resident at once on the device (at
// most `cap`): launching more leaves a second, partial wave.
template <class Kernel>
uint64_t resident_grid(const kc_context* c, Kernel k, int threads, uint64_t cap) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, threads, 0) != cudaSuccess || per_sm < 1) {
        cudaGetLastError();
        per_sm = 1;
    }
    return std::max<uint64_t>(1, std::min<uint64_t>(cap, (uint64_t)c->sm_count * (uint64_t)per_sm));
}

// `stream` waits for the table initialisation launched on `side`.
int join_init(kc_context* c) {
    if (!c->init_pending) return KC_OK;
    c->init_pending = false;
    CK(cudaStreamWaitEvent(c->stream, c->ev_init, 0));
    return KC_OK;
}

int setup_shape(kc_context* c) {
    const kc_config& g = c->cfg;
    if (g.k < 1 || g.k > 128) return fail(KC_ERR_INVALID, "k=%u out of range: 1..128", g.k);
    if (g.canonical != 1) return fail(KC_ERR_INVALID, "only canonical counting is supported (the reference has no other mode)");
    if (g.max_count < g.min_count) return fail(KC_ERR_INVALID, "max_count < min_count");
    if (g.n_buckets != 256 && g.n_buckets != 4096) return fail(KC_ERR_INVALID, "n_buckets must be 256 or 4096");
    if (g.bloom_bits <= 0.0 || g.table_load <= 0.05 || g.table_load > 0.95 || g.repeat_ratio <= 0.0)
        return fail(KC_ERR_INVALID, "bloom_bits, table_load (0.05..0.95) and repeat_ratio must be positive");
    if (g.batch_bytes < (1ull << 20)) return fail(KC_ERR_INVALID, "batch_bytes must be at least 1 MiB");
    if (g.device_batch_bytes && g.device_batch_bytes < (1ull << 20))
        return fail(KC_ERR_INVALID, "device_batch_bytes must be 0 or at least 1 MiB");
    if (g.priority != 0 && g.priority != 1) return fail(KC_ERR_INVALID, "priority must be 0 or 1");
    c->nw = g.k <= 32 ? 1 : (g.k <= 64 ? 2 : 4);
    c->n_buckets = g.n_buckets;
    c->bucket_bits = g.n_buckets == 256 ? 8 : 12;
    c->bucket_shift = 64 - c->bucket_bits;
    c->slot_bytes = c->nw == 1 ? sizeof(kc::Slot1) : (c->nw == 2 ? sizeof(kc::Slot2) : sizeof(kc::Slot4));
    c->record_bytes = kc_record_bytes(g.k);
    c->packed_bytes = kc_packed_bytes(g.k);
    return KC_OK;
}

// Control-path transfers on `stream`.  The copy engines carry the bulk
// FASTQ batches (h2d stream) and output pieces (d2h stream); a small
// cudaMemcpyAsync/cudaMemsetAsync on `stream` would queue behind them and
// hold up the batch it belongs to.  So: fills run as a kernel, uploads are
// staged in the mapped mailbox and copied in by a kernel, readbacks are
// copied out to the mailbox by a kernel and land in their host destination
// at the next sync_stream().  Sizes and addresses must be 4-byte multiples;
// anything else, or larger than the mailbox, takes cudaMemcpyAsync.
int fill_dev(kc_context* c, void* dst, uint64_t bytes, uint32_t word) {
    if (!bytes) return KC_OK;
    if (bytes % 4 || reinterpret_cast<uintptr_t>(dst) % 4) {
        CK(cudaMemsetAsync(dst, (int)(word & 0xFF), bytes, c->stream));
        return KC_OK;
    }
    const uint64_t n = bytes / 4;
    kc::fill_words<<<std::min<uint64_t>(ceil_div(n, 256), (uint64_t)c->sm_count * 16), 256, 0, c->stream>>>(
        static_cast<uint32_t*>(dst), n, word);
    CK(cudaGetLastError());
    return KC_OK;
}

int put(kc_context* c, void* dst, const void* src, uint64_t bytes) {
    if (!bytes) return KC_OK;
    if (bytes % 4 || reinterpret_cast<uintptr_t>(dst) % 4 || bytes > kc_context::MBOX_UP) {
        CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->stream));
        return KC_OK;
    }
    if (c->mbox_up_off + bytes > kc_context::MBOX_UP) {
        // wrap: every earlier upload kernel has to have read its bytes
        CK(cudaEventSynchronize(c->ev_mbox));
        c->mbox_up_off = 0;
    }
    std::memcpy(c->mbox_h + c->mbox_up_off, src, bytes);
    const uint64_t n = bytes / 4;
    kc::copy_words<<<std::min<uint64_t>(ceil_div(n, 256), 64), 256, 0, c->stream>>>(
        reinterpret_cast<const uint32_t*>(c->mbox_d + c->mbox_up_off), static_cast<uint32_t*>(dst), n);
    CK(cudaGetLastError());
    CK(cudaEventRecord(c->ev_mbox, c->stream));
    c->mbox_up_off += (bytes + 15) & ~15ull;
    return KC_OK;
}

int get(kc_context* c, void* dst, const void* src, uint64_t bytes) {
    if (!bytes) return KC_OK;
    if (bytes % 4 || reinterpret_cast<uintptr_t>(src) % 4 || c->mbox_down_off + bytes > kc_context::MBOX_DOWN) {
        CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->stream));
        return KC_OK;
    }
    const uint64_t off = kc_context::MBOX_UP + c->mbox_down_off;
    const uint64_t n = bytes / 4;
    kc::copy_words<<<std::min<uint64_t>(ceil_div(n, 256), 64), 256, 0, c->stream>>>(
        static_cast<const uint32_t*>(src), reinterpret_cast<uint32_t*>(c->mbox_d + off), n);
    CK(cudaGetLastError());
    c->readbacks.push_back({dst, off, bytes});
    c->mbox_down_off += (bytes + 15) & ~15ull;
    return KC_OK;
}

// Wait for `stream`, then deliver the pending readbacks.
int sync_stream(kc_context* c) {
    CK(cudaStreamSynchronize(c->stream));
    for (const auto& r : c->readbacks) std::memcpy(r.dst, c->mbox_h + r.off, r.bytes);
    c->readbacks.clear();
    c->mbox_down_off = 0;
    c->mbox_up_off = 0;
    return KC_OK;
}

#define CKR(x)                   \
    do {                         \
        const int r_ = (x);      \
        if (r_) return r_;       \
    } while (0)

// Exclusive scan of n values of type TI into TO out[], plus base; optional
// device total in scalars[slot].
template <class TI, class TO>
int device_scan(kc_context* c, const TI* in, uint64_t n, TO* out, uint64_t base, uint64_t* d_total) {
    const uint64_t nb = std::max<uint64_t>(1, ceil_div(n, kc::SCAN_TILE));
    CK(c->scan_sums.ensure(nb * sizeof(uint64_t)));
    Stage st(c, KC_STAGE_SCAN, n ? 3 : 1);
    uint64_t* sums = c->scan_sums.as<uint64_t>();
    if (n) kc::scan_reduce<TI><<<nb, kc::SCAN_BLOCK, 0, c->stream>>>(in, n, sums);
    else CKR(fill_dev(c, sums, sizeof(uint64_t), 0));
    kc::scan_sums<<<1, kc::SCAN_BLOCK, 0, c->stream>>>(sums, n ? nb : 1, base, d_total);
    if (n) kc::scan_apply<TI, TO><<<nb, kc::SCAN_BLOCK, 0, c->stream>>>(in, n, sums, out);
    CK(cudaGetLastError());
    return KC_OK;
}

// Allocate filter and tables from per-bucket k-mer totals of the first batch
// (batch_bytes of FASTQ; 0 when no extraction follows).
int size_structures(kc_context* c, const std::vector<uint64_t>& kb, double scale, uint64_t batch_bytes) {
    const kc_config& g = c->cfg;
    const uint32_t nb = c->n_buckets;
    c->h_meta.assign(nb, kc::BucketMeta{});
    uint64_t bw = 0, ts = 0;
    const bool learned = g.sizing == KC_SIZING_LEARNED && c->pred_table.size() == KC_MODEL_BUCKETS;
    const uint32_t per = KC_MODEL_BUCKETS / nb;  // model buckets per engine bucket (16 or 1)
    for (uint32_t b = 0; b < nb; ++b) {
        const double kest = (double)kb[b] * scale;
        uint64_t words, slots;
        if (learned) {
            // filter: 12 bits per predicted distinct key; table: predicted
            // table keys with 15% headroom at the target load
            double d = 0, t = 0;
            for (uint32_t q = 0; q < per; ++q) {
                d += c->pred_distinct[b * per + q];
                t += c->pred_table[b * per + q];
            }
            words = pow2_at_least(std::max<uint64_t>((uint64_t)(d * 12.0 / 64.0), 256));
            slots = pow2_at_least(std::max<uint64_t>((uint64_t)(t * 1.15 / g.table_load), 256));
        } else {
            words = pow2_at_least(std::max<uint64_t>((uint64_t)(kest * g.bloom_bits / 64.0), 256));
            slots = pow2_at_least(std::max<uint64_t>((uint64_t)(kest * g.repeat_ratio / g.table_load), 256));
        }
        if (c->nw == 1) {
            // 64-bit keys: the filter is the 32-bit pad field of the table
            // cells, at the index of the first table probe, so one read serves
            // both; cells = the larger of the table's slots and the filter's
            // 32-bit words.  After a table grows, the old cells stay the filter.
            slots = std::max<uint64_t>(slots, 2 * words);
            c->h_meta[b].bloom_off = ts;
            c->h_meta[b].bloom_mask = slots - 1;
        } else {
            c->h_meta[b].bloom_off = bw;
            c->h_meta[b].bloom_mask = words - 1;
            bw += words;
        }
        c->h_meta[b].tab_off = ts;
        c->h_meta[b].tab_mask = slots - 1;
        ts += slots;
    }
    c->bloom_words = c->nw == 1 ? ts / 2 : bw;  // in 64-bit words (cells hold 32 filter bits each)
    c->table_slots_used = ts;
    c->win_ready = false;
    CK(c->bloom.ensure(bw * sizeof(uint64_t)));
    CK(c->table.ensure(ts * c->slot_bytes + ts * c->slot_bytes / 4));  // room for a few in-place growths
    CK(c->meta.ensure(nb * sizeof(kc::BucketMeta)));
    CKR(put(c, c->meta.p, c->h_meta.data(), nb * sizeof(kc::BucketMeta)));
    {
        // Filter and table initialisation.  When it is small against the
        // first batch (under 4 bytes per FASTQ byte; the extraction moves
        // ~0.33 GB of FASTQ per ms, the initialisation 2-5 GB per ms) it runs
        // on the side stream, two CTAs per SM, after the work already queued
        // on `stream` (a previous count may still read the table), beside
        // the extraction, which is bound by instruction issue, not by HBM;
        // the count joins it.  Otherwise it runs first at full width: 48 GB
        // of 128-bit tables behind a 2 GiB batch slowed that batch's
        // extraction and still held up the count.
        const uint64_t init_bytes = bw * sizeof(uint64_t) + ts * c->slot_bytes;
        const bool beside = init_bytes < 4 * batch_bytes;
        cudaStream_t is = c->stream;
        if (beside) {
            // after the work queued before this batch's extraction (recorded
            // before it when sizing follows the extraction's launch)
            if (!c->side_in_ready) CK(cudaEventRecord(c->ev_side_in, c->stream));
            CK(cudaStreamWaitEvent(c->side, c->ev_side_in, 0));
            is = c->side;
        }
        c->side_in_ready = false;
        Stage st(c, KC_STAGE_INIT, bw ? 2 : 1, is);
        const int ig = c->sm_count * (beside ? 2 : 8);
        if (bw) kc::zero16<<<ig, 256, 0, is>>>(c->bloom.as<uint4>(), bw / 2);  // bw: a sum of powers of two >= 256
        if (c->nw == 1) kc::init_slots<1><<<ig, 256, 0, is>>>(c->table.p, ts);
        else if (c->nw == 2) kc::init_slots<2><<<ig, 256, 0, is>>>(c->table.p, ts);
        else kc::init_slots<4><<<ig, 256, 0, is>>>(c->table.p, ts);
        CK(cudaGetLastError());
        if (beside) {
            CK(cudaEventRecord(c->ev_init, c->side));
            c->init_pending = true;
        }
    }
    CK(c->overflow.ensure(nb * sizeof(uint32_t)));
    CKR(fill_dev(c, c->overflow.p, nb * sizeof(uint32_t), 0));
    c->h_overflow.assign(nb, 0);
    c->sized = true;
    return KC_OK;
}

template <int NW>
void launch_count(kc_context* c, uint64_t n_keys, int use_filter) {
    constexpr int TILE = kc::count_tile<NW>();
    join_init(c);
    // each CTA covers CNT_SEGS_PER_WARP segments per warp, in blockIdx order
    const uint64_t tiles = ceil_div(n_keys, (uint64_t)TILE * kc::CNT_SEGS_PER_WARP);
    if (!tiles) return;
    kc::CountArgs a{};
    a.routed = c->routed.p;
    a.n_keys = n_keys;
    a.meta = c->meta.as<kc::BucketMeta>();
    a.bloom = c->bloom.as<uint64_t>();
    a.table = c->table.p;
    a.seg_low = c->tile_low.as<uint32_t>();
    a.seg_fail = c->tile_fail.as<uint32_t>();
    a.bucket_overflow = c->overflow.as<uint32_t>();
    a.error = c->scalars.as<uint32_t>() + 13;
    a.bucket_shift = c->bucket_shift;
    a.n_buckets = c->n_buckets;
    a.use_filter = use_filter;
    a.filter_in_table = c->nw == 1;
    Stage st(c, use_filter ? KC_STAGE_COUNT_ROUTED : KC_STAGE_REHASH);
    kc::count_routed<NW><<<tiles, kc::CNT_THREADS, 0, c->stream>>>(a);
}

// Grow the tables of the given buckets x4 (again x4 for a bucket whose keys
// still met a full probe window): per round one arena growth for all of them,
// their new tables initialised and filled by two launches, one
// synchronisation; c->h_meta is updated (not uploaded).
template <int NW>
int grow_buckets(kc_context* c, const std::vector<uint32_t>& buckets) {
    std::vector<uint32_t> pending = buckets;
    std::vector<uint64_t> new_slots(buckets.size());
    std::vector<uint32_t> idx(buckets.size());
    for (size_t i = 0; i < buckets.size(); ++i) {
        new_slots[i] = (c->h_meta[buckets[i]].tab_mask + 1) * 4;
        idx[i] = (uint32_t)i;
    }
    std::vector<uint32_t> todo = idx;
    for (int round = 0; !todo.empty(); ++round) {
        if (round > 12) return fail(KC_ERR_OVERFLOW, "a table kept overflowing while it was grown");
        uint64_t total = 0, max_slots = 0;
        for (uint32_t i : todo) {
            total += new_slots[i];
            max_slots = std::max<uint64_t>(max_slots, new_slots[i]);
        }
        CK(c->table.grow_keep((c->table_slots_used + total) * c->slot_bytes, c->table_slots_used * c->slot_bytes,
                              c->stream));
        std::vector<kc::GrowJob> jobs(todo.size());
        for (size_t j = 0; j < todo.size(); ++j) {
            const kc::BucketMeta& m = c->h_meta[buckets[todo[j]]];
            jobs[j] = kc::GrowJob{m.tab_off, m.tab_mask + 1, c->table_slots_used, new_slots[todo[j]] - 1};
            c->table_slots_used += new_slots[todo[j]];
        }
        CK(c->grow_jobs.ensure(jobs.size() * sizeof(kc::GrowJob)));
        CK(c->grow_failed.ensure(jobs.size() * sizeof(uint32_t)));
        CK(cudaMemcpyAsync(c->grow_jobs.p, jobs.data(), jobs.size() * sizeof(kc::GrowJob), cudaMemcpyHostToDevice,
                           c->stream));
        CKR(fill_dev(c, c->grow_failed.p, jobs.size() * sizeof(uint32_t), 0));
        std::vector<uint32_t> failed(jobs.size());
        for (size_t j0 = 0; j0 < jobs.size(); j0 += 65535) {  // grid y limit
            const uint32_t nj = (uint32_t)std::min<size_t>(65535, jobs.size() - j0);
            const dim3 grid((uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(256, ceil_div(max_slots, 4096))), nj);
            Stage st(c, KC_STAGE_REHASH, 2);
            kc::grow_init<NW><<<grid, 256, 0, c->stream>>>(c->table.p, c->grow_jobs.as<kc::GrowJob>() + j0);
            kc::grow_move<NW><<<grid, 256, 0, c->stream>>>(c->table.p, c->grow_jobs.as<kc::GrowJob>() + j0,
                                                           c->grow_failed.as<uint32_t>() + j0);
            CK(cudaGetLastError());
        }
        CK(cudaMemcpyAsync(failed.data(), c->grow_failed.p, jobs.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                           c->stream));
        CKR(sync_stream(c));
        std::vector<uint32_t> again;
        for (size_t j = 0; j < todo.size(); ++j) {
            const uint32_t i = todo[j];
            if (failed[j]) {  // pathological clustering: grow again
                new_slots[i] *= 4;
                again.push_back(i);
                continue;
            }
            kc::BucketMeta& m = c->h_meta[buckets[i]];
            m.tab_off = jobs[j].new_off;
            m.tab_mask = new_slots[i] - 1;
            ++c->rehashes;
        }
        todo.swap(again);
    }
    return KC_OK;
}

// Grow the tables of overflowed buckets (x4) and re-insert the keys that
// met a full table, until none is left.
template <int NW>
int rehash_loop(kc_context* c, uint64_t n_keys) {
    const uint32_t nb = c->n_buckets;
    for (int round = 0;; ++round) {
        CKR(get(c, c->h_overflow.data(), c->overflow.p, nb * sizeof(uint32_t)));
        CKR(sync_stream(c));
        std::vector<uint32_t> grow;
        for (uint32_t b = 0; b < nb; ++b)
            if (c->h_overflow[b]) grow.push_back(b);
        if (grow.empty()) return KC_OK;
        if (round > 24) return fail(KC_ERR_OVERFLOW, "repeat tables kept overflowing after %d growth rounds", round);
        CKR(fill_dev(c, c->overflow.p, nb * sizeof(uint32_t), 0));
        CKR(grow_buckets<NW>(c, grow));
        CKR(put(c, c->meta.p, c->h_meta.data(), nb * sizeof(kc::BucketMeta)));
        c->win_ready = false;  // grown buckets leave the windowed count (their filter and table part)
        launch_count<NW>(c, n_keys, 0);
        CK(cudaGetLastError());
    }
}

// Windows of the current table layout, or false when some bucket's filter and
// table have parted (a table that grew after an overflow keeps its old cells
// as the filter): the windowed count needs the filter word in the first probe
// cell of the key's own table.
bool build_windows(kc_context* c) {
    const uint32_t nb = c->n_buckets;
    c->h_bucket_win.assign(nb, kc::BucketWin{});
    c->h_win_info.clear();
    for (uint32_t b = 0; b < nb; ++b) {
        const kc::BucketMeta& m = c->h_meta[b];
        if (m.bloom_off != m.tab_off || m.bloom_mask != m.tab_mask) return false;
        const uint64_t cells = m.tab_mask + 1;
        const uint32_t n = cells <= (uint64_t)kc::WIN_Z ? 1u : (uint32_t)(cells >> kc::WIN_ZSHIFT);
        c->h_bucket_win[b] = kc::BucketWin{(uint32_t)c->h_win_info.size(), n == 1 ? kc::WIN_SINGLE : kc::WIN_ZSHIFT};
        for (uint32_t q = 0; q < n; ++q) c->h_win_info.push_back(kc::WinInfo{b, q});
    }
    c->n_wins = c->h_win_info.size();
    // launch order: the first phase's windows (one-window buckets and even
    // windows), then the second's (odd windows)
    c->h_win_order.clear();
    for (int ph = 0; ph < 2; ++ph) {
        for (uint32_t r = 0; r < (uint32_t)c->n_wins; ++r) {
            const kc::WinInfo& wi = c->h_win_info[r];
            const bool single = c->h_bucket_win[wi.bucket].zshift >= kc::WIN_SINGLE;
            if ((single ? 0u : (wi.sub & 1u)) == (uint32_t)ph) c->h_win_order.push_back(r);
        }
        if (ph == 0) c->n_wins_phase0 = c->h_win_order.size();
    }
    return true;
}

// Count the keys [off, off + n) of `routed` (off a multiple of the count
// segment) with count_routed: the spill area of the windowed count.
template <int NW>
void launch_count_range(kc_context* c, uint64_t off, uint64_t n, int use_filter) {
    constexpr int TILE = kc::count_tile<NW>();
    constexpr int SEG = kc::count_seg<NW>();
    join_init(c);
    const uint64_t tiles = ceil_div(n, (uint64_t)TILE * kc::CNT_SEGS_PER_WARP);
    if (!tiles) return;
    kc::CountArgs a{};
    a.routed = c->routed.as<uint8_t>() + off * (uint64_t)(8 * NW);
    a.n_keys = n;
    a.meta = c->meta.as<kc::BucketMeta>();
    a.bloom = c->bloom.as<uint64_t>();
    a.table = c->table.p;
    a.seg_low = c->tile_low.as<uint32_t>() + off / SEG;
    a.seg_fail = c->tile_fail.as<uint32_t>() + off / SEG;
    a.bucket_overflow = c->overflow.as<uint32_t>();
    a.error = c->scalars.as<uint32_t>() + 13;
    a.bucket_shift = c->bucket_shift;
    a.n_buckets = c->n_buckets;
    a.use_filter = use_filter;
    a.filter_in_table = c->nw == 1;
    Stage st(c, KC_STAGE_COUNT_ROUTED);
    kc::count_routed<NW><<<tiles, kc::CNT_THREADS, 0, c->stream>>>(a);
}

// Windowed count of one batch of 64-bit keys in `routed` (kc_window.cuh):
// group the keys by window (ranges estimated from every 16th chunk, the
// overflow of a window to a spill area; exact ranges for small batches or
// when the spill area overflows), count every window in shared memory, even
// windows first, then the spilled keys with count_routed.  `routed` then
// holds the window-grouped keys with per-segment first occurrences and
// overflowed keys as count_routed leaves them, and n_keys becomes its length.
int window_count(kc_context* c, uint64_t& n_keys) {
    const uint64_t nw = c->n_wins;
    if (!c->win_ready) {
        CK(c->bucket_win.ensure(c->n_buckets * sizeof(kc::BucketWin)));
        CK(c->win_info.ensure(nw * sizeof(kc::WinInfo)));
        CK(c->win_order.ensure(nw * sizeof(uint32_t)));
        CK(cudaMemcpyAsync(c->win_order.p, c->h_win_order.data(), nw * sizeof(uint32_t), cudaMemcpyHostToDevice,
                           c->stream));
        CK(cudaMemcpyAsync(c->bucket_win.p, c->h_bucket_win.data(), c->n_buckets * sizeof(kc::BucketWin),
                           cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(c->win_info.p, c->h_win_info.data(), nw * sizeof(kc::WinInfo), cudaMemcpyHostToDevice,
                           c->stream));
        CK(c->win_count.ensure(nw * sizeof(uint32_t)));
        CK(c->win_padded.ensure(nw * sizeof(uint32_t)));  // capacities
        CK(c->win_start.ensure(nw * sizeof(uint64_t)));
        CK(c->win_cursor.ensure(nw * sizeof(uint64_t)));
        CK(c->win_end.ensure(nw * sizeof(uint64_t)));
        c->win_ready = true;
    }
    uint64_t* d_scal = c->scalars.as<uint64_t>();
    uint32_t* d_spill_full = c->scalars.as<uint32_t>() + 14;
    const auto* meta = c->meta.as<kc::BucketMeta>();
    const auto* bwin = c->bucket_win.as<kc::BucketWin>();
    const uint64_t cchunks = ceil_div(n_keys, kc::SUB_CHUNK);
    const uint64_t small_grid = std::min<uint64_t>(ceil_div(nw, 256), (uint64_t)c->sm_count * 8);
    // sampled ranges need enough sampled chunks per window to be worth it
    uint32_t stride = cchunks >= 64ull * 16 ? 16u : 1u;
    uint64_t total = 0, spill_start = 0, spill_used = 0;
    for (;;) {
        CKR(fill_dev(c, c->win_count.p, nw * sizeof(uint32_t), 0));
        {
            Stage st(c, KC_STAGE_SUBROUTE, 2);
            const uint64_t g = ceil_div(cchunks, stride);
            if (g)
                kc::subroute_count<<<g, kc::SUB_THREADS, 0, c->stream>>>(
                    c->routed.as<uint64_t>(), n_keys, meta, bwin, c->bucket_shift, stride, c->win_count.as<uint32_t>());
            kc::window_caps<<<small_grid, 256, 0, c->stream>>>(c->win_count.as<uint32_t>(), nw, stride,
                                                                c->win_padded.as<uint32_t>());
            CK(cudaGetLastError());
        }
        int rc;
        if ((rc = device_scan<uint32_t, uint64_t>(c, c->win_padded.as<uint32_t>(), nw, c->win_start.as<uint64_t>(), 0,
                                                  d_scal + 3)))
            return rc;
        CKR(get(c, &total, d_scal + 3, sizeof(uint64_t)));
        CKR(sync_stream(c));
        spill_start = total;
        const uint64_t spill_cap = stride > 1 ? std::max<uint64_t>(1ull << 16, (total / 16 + 63) & ~63ull) : 0;
        const uint64_t arr = total + spill_cap;
        CK(c->routed2.ensure(std::max<uint64_t>(arr, 1) * sizeof(uint64_t)));
        CK(c->tile_low.ensure(std::max<uint64_t>(arr / kc::WIN_SEG, 1) * sizeof(uint32_t)));
        CK(c->tile_fail.ensure(std::max<uint64_t>(arr / kc::WIN_SEG, 1) * sizeof(uint32_t)));
        CK(c->tile_low_prefix.ensure(std::max<uint64_t>(arr / kc::WIN_SEG, 1) * sizeof(uint64_t)));
        CKR(put(c, d_scal + 5, &spill_start, sizeof(uint64_t)));
        CKR(fill_dev(c, d_spill_full, sizeof(uint32_t), 0));
        {
            Stage st(c, KC_STAGE_SUBROUTE, n_keys ? 2 : 1);
            kc::window_bounds<<<small_grid, 256, 0, c->stream>>>(c->win_start.as<uint64_t>(), c->win_padded.as<uint32_t>(),
                                                                 nw, c->win_cursor.as<uint64_t>(), c->win_end.as<uint64_t>());
            kc::ScatterArgs sa{};
            sa.keys = c->routed.as<uint64_t>();
            sa.n = n_keys;
            sa.meta = meta;
            sa.bw = bwin;
            sa.bucket_shift = c->bucket_shift;
            sa.win_cursor = c->win_cursor.as<unsigned long long>();
            sa.win_end = c->win_end.as<uint64_t>();
            sa.spill_cursor = reinterpret_cast<unsigned long long*>(d_scal + 5);
            sa.spill_end = arr;
            sa.spill_full = d_spill_full;
            sa.out = c->routed2.as<uint64_t>();
            if (n_keys)
                kc::subroute_scatter<<<ceil_div(n_keys, kc::SCAT_CHUNK), kc::SCAT_THREADS, kc::scatter_smem_bytes(),
                                       c->stream>>>(sa);
            CK(cudaGetLastError());
        }
        uint32_t full = 0;
        uint64_t spill_end = 0;
        CKR(get(c, &spill_end, d_scal + 5, sizeof(uint64_t)));
        CKR(get(c, &full, d_spill_full, sizeof(uint32_t)));
        CKR(sync_stream(c));
        if (full && stride > 1) {  // the estimate missed by more than the spill area: exact ranges
            stride = 1;
            continue;
        }
        if (full) return fail(KC_ERR_DEVICE, "internal error: exact window ranges overflowed");
        spill_used = spill_end - spill_start;
        break;
    }
    std::swap(c->routed, c->routed2);
    n_keys = spill_start + spill_used;
    CKR(join_init(c));
    kc::WindowArgs a{};
    a.keys = c->routed.as<uint64_t>();
    a.win_start = c->win_start.as<uint64_t>();
    a.win_fill = c->win_cursor.as<unsigned long long>();
    a.win_cap = c->win_padded.as<uint32_t>();
    a.wins = c->win_info.as<kc::WinInfo>();
    a.order = c->win_order.as<uint32_t>();
    a.bw = bwin;
    a.meta = meta;
    a.table = c->table.as<kc::Slot1>();
    a.seg_low = c->tile_low.as<uint32_t>();
    a.seg_fail = c->tile_fail.as<uint32_t>();
    a.bucket_overflow = c->overflow.as<uint32_t>();
    {
        Stage st(c, KC_STAGE_COUNT_ROUTED, 2);
        for (uint32_t ph = 0; ph < 2; ++ph) {
            a.phase = ph;
            a.order_base = ph ? (uint32_t)c->n_wins_phase0 : 0u;
            const uint64_t grid = ph ? nw - c->n_wins_phase0 : c->n_wins_phase0;
            if (grid) kc::count_window<<<grid, kc::WIN_THREADS, kc::window_smem_bytes(), c->stream>>>(a);
        }
        CK(cudaGetLastError());
    }
    if (spill_used) launch_count_range<1>(c, spill_start, spill_used, 1);
    c->window_spill += spill_used;
    CK(cudaGetLastError());
    return KC_OK;
}

// mode HIST: totals of `bins` buckets (the top log2(bins) key bits) over
// every `stride`-th tile.  mode SCATTER: keys into the regions of `bins`
// routing buckets (estimated regions with an overflow area when `estimated`,
// else exact).
template <int NW>
int launch_extract(kc_context* c, const uint8_t* buf, uint64_t n, int has_halo, int mode, uint32_t bins,
                   uint32_t stride = 1, bool estimated = false, uint64_t overflow_start = 0,
                   uint64_t overflow_end = 0) {
    const uint64_t tiles = ceil_div(ceil_div(n, kc::EXT_TILE), std::max<uint32_t>(stride, 1));
    if (!tiles) return KC_OK;
    kc::ExtractArgs a{};
    a.buf = buf;
    a.n = n;
    a.has_halo = has_halo;
    a.tile_line = c->tile_line.as<uint64_t>();
    a.k = c->cfg.k;
    a.bucket_shift = 64 - (bins == 4096 ? 12 : 8);
    a.n_buckets = bins;
    a.bucket_count = c->bucket_count.as<unsigned long long>();
    a.bucket_cursor = c->bucket_cursor.as<unsigned long long>();
    a.routed = c->routed.p;
    a.error = c->scalars.as<uint32_t>() + 12;
    a.tile_stride = stride;
    if (estimated) {
        a.region_end = c->region_end.as<unsigned long long>();
        a.region_fill = c->region_fill.as<unsigned long long>();
        a.overflow_cursor = reinterpret_cast<unsigned long long*>(c->scalars.as<uint64_t>() + 2);
        a.overflow_start = overflow_start;
        a.overflow_end = overflow_end;
    }
    Stage st(c, mode == kc::HIST ? KC_STAGE_EXTRACT_HIST : KC_STAGE_EXTRACT_SCATTER);
    if (mode == kc::HIST)
        kc::extract_kernel<NW, kc::HIST>
            <<<tiles, kc::EXT_THREADS, kc::extract_smem_bytes<NW, kc::HIST>(bins), c->stream>>>(a);
    else
        kc::extract_kernel<NW, kc::SCATTER>
            <<<tiles, kc::EXT_THREADS, kc::extract_smem_bytes<NW, kc::SCATTER>(bins), c->stream>>>(a);
    CK(cudaGetLastError());
    return KC_OK;
}

template <int NW>
int count_and_pack(kc_context* c, uint64_t n_keys, uint32_t ext_err);

// Count one batch of FASTQ bytes already in device memory.  route_only:
// route it exactly (every tile's histogram, no estimated regions) into
// `routed`, bucket-contiguous in bucket order, and stop there (filter and
// tables untouched; kc_route_device).
template <int NW>
int process_batch(kc_context* c, const uint8_t* buf, uint64_t n, int has_halo, bool route_only = false) {
    if (reinterpret_cast<uintptr_t>(buf) % 16)
        return fail(KC_ERR_INVALID, "device FASTQ batch must be 16-byte aligned");
    const uint32_t nb = c->n_buckets;
    const uint64_t tiles = ceil_div(n, kc::EXT_TILE);
    c->last_batch_low = 0;  // a batch without k-mers packs nothing
    CK(c->tile_nl.ensure(std::max<uint64_t>(tiles, 1) * sizeof(uint32_t)));
    CK(c->tile_line.ensure(std::max<uint64_t>(tiles, 1) * sizeof(uint64_t)));
    CK(c->scalars.ensure(64));
    uint64_t* d_scal = c->scalars.as<uint64_t>();
    CKR(fill_dev(c, c->scalars.as<uint32_t>() + 12, 2 * sizeof(uint32_t), 0));  // extraction and count error words
    if (tiles) {
        Stage st(c, KC_STAGE_LINES);
        kc::lines_per_tile<<<tiles, kc::EXT_THREADS, 0, c->stream>>>(buf, n, c->tile_nl.as<uint32_t>());
    }
    CK(cudaGetLastError());
    int rc = device_scan<uint32_t, uint64_t>(c, c->tile_nl.as<uint32_t>(), tiles, c->tile_line.as<uint64_t>(),
                                             c->line_base, d_scal + 0);
    if (rc) return rc;

    CK(c->bucket_count.ensure(nb * sizeof(uint64_t)));
    CK(c->bucket_cursor.ensure(nb * sizeof(uint64_t)));
    CK(c->region_end.ensure(nb * sizeof(uint64_t)));
    CK(c->region_fill.ensure(nb * sizeof(uint64_t)));

    // Bucket regions.  A large batch takes them from a histogram of every
    // EST_STRIDE-th tile: region = estimate x 1.02 + 4 standard deviations +
    // 256 keys, and a CTA's keys past its region go to an overflow area after
    // the regions (counted like the rest; the unfilled region tails hold EMPTY
    // keys, which the count kernel skips).  If the overflow area itself fills,
    // the batch is routed again from an exact histogram of every tile.
    //
    // Keys are routed by their top 8 bits (rb = 256 routing buckets) whatever
    // the table partition: with 4096 table buckets, the 16 that share a
    // routing bucket are adjacent in the filter and table arenas, so a routed
    // region still touches one contiguous working set, and the scatter keeps
    // its 256-bucket shared-memory footprint.  The histogram counts all nb
    // table buckets (sizing is per table bucket).
    constexpr int CT = kc::count_tile<NW>();
    constexpr int SEG = kc::count_seg<NW>();
    const uint32_t rb = std::min<uint32_t>(nb, 256), per = nb / rb;
    bool est = tiles >= kc::EST_MIN_TILES && !route_only;
    std::vector<uint64_t> start(rb), end(rb), cursor(rb);
    uint64_t n_keys = 0, kb = 0;
    for (int attempt = 0;; ++attempt) {
        const uint32_t stride = est ? kc::EST_STRIDE : 1u;
        CKR(fill_dev(c, c->bucket_count.p, nb * sizeof(uint64_t), 0));
        if ((rc = launch_extract<NW>(c, buf, n, has_halo, kc::HIST, nb, stride))) return rc;
        c->h_bucket_count.resize(nb);
        uint64_t line_end = 0;
        CKR(get(c, c->h_bucket_count.data(), c->bucket_count.p, nb * sizeof(uint64_t)));
        CKR(get(c, &line_end, d_scal + 0, sizeof(uint64_t)));
        CKR(sync_stream(c));
        if (attempt == 0) c->line_base = line_end;

        std::vector<uint64_t> kest(nb);
        uint64_t total_cap = 0;
        const double f = est ? (double)tiles / (double)ceil_div(tiles, stride) : 1.0;
        for (uint32_t b = 0; b < nb; ++b) kest[b] = (uint64_t)((double)c->h_bucket_count[b] * f);
        if (route_only) c->route_counts.assign(rb, 0);
        for (uint32_t r = 0; r < rb; ++r) {
            uint64_t exact = 0;
            for (uint32_t q = 0; q < per; ++q) exact += c->h_bucket_count[r * per + q];
            if (route_only) c->route_counts[r] = exact;
            const double e = (double)exact * f;
            const uint64_t cap = est ? (uint64_t)(e * 1.02 + 4.0 * std::sqrt(e) + 256.0) : exact;
            start[r] = total_cap;
            total_cap += cap;
            end[r] = total_cap;
        }
        // at least 65536 keys: one CTA's run of a bucket (<= 8192 keys) always fits
        const uint64_t ovf_cap = est ? std::max<uint64_t>(1ull << 16, total_cap / 32) : 0;
        // filter and tables are sized from these totals after the extraction
        // is enqueued (it does not read them), so that a learned-sizing
        // callback's work and the structures' initialisation run beside it
        const bool size_here = !c->sized && !route_only;
        const double scale =
            (c->expected_total_bytes > n && n > 0) ? (double)c->expected_total_bytes / (double)n : 1.0;
        if (size_here && !total_cap && (rc = size_structures(c, kest, scale, n))) return rc;
        if (!total_cap) {  // no k-mers in this batch
            if (route_only) c->routed_keys = 0;
            return KC_OK;
        }

        const uint64_t cap_keys = total_cap + ovf_cap;
        const uint64_t ctiles = ceil_div(cap_keys, CT);
        CK(c->routed.ensure(ctiles * CT * (uint64_t)(8 * NW)));
        CK(c->tile_low.ensure(ctiles * (CT / SEG) * sizeof(uint32_t)));
        CK(c->tile_fail.ensure(ctiles * (CT / SEG) * sizeof(uint32_t)));
        CK(c->tile_low_prefix.ensure(ctiles * (CT / SEG) * sizeof(uint64_t)));
        CKR(put(c, c->bucket_cursor.p, start.data(), rb * sizeof(uint64_t)));
        if (est) {
            CKR(put(c, c->region_end.p, end.data(), rb * sizeof(uint64_t)));
            CKR(put(c, d_scal + 2, &total_cap, sizeof(uint64_t)));
            CKR(fill_dev(c, c->region_fill.p, rb * sizeof(uint64_t), 0xFFFFFFFFu));
        }
        if (size_here) {
            CK(cudaEventRecord(c->ev_side_in, c->stream));
            c->side_in_ready = true;
        }
        if ((rc = launch_extract<NW>(c, buf, n, has_halo, kc::SCATTER, rb, 1, est, total_cap, cap_keys))) return rc;
        if (size_here) {
            if (c->cfg.sizing == KC_SIZING_LEARNED && c->sizing_cb && c->sizing_cb(c->sizing_user, c) != 0)
                return fail(KC_ERR_INVALID, "the sizing callback failed");
            if ((rc = size_structures(c, kest, scale, n))) return rc;
        }
        if (!est) {
            n_keys = kb = total_cap;
            break;
        }
        uint64_t ovf_used = 0;
        uint32_t flags = 0;
        CKR(get(c, cursor.data(), c->bucket_cursor.p, rb * sizeof(uint64_t)));
        CKR(get(c, &ovf_used, d_scal + 2, sizeof(uint64_t)));
        CKR(get(c, &flags, c->scalars.as<uint32_t>() + 12, sizeof(uint32_t)));
        CKR(sync_stream(c));
        if (flags & 2u) {  // overflow area full: route this batch again, exactly
            CKR(fill_dev(c, c->scalars.as<uint32_t>() + 12, sizeof(uint32_t), 0));
            est = false;
            ++c->reroutes;
            continue;
        }
        c->overflow_keys += ovf_used - total_cap;
        kb = 0;
        for (uint32_t r = 0; r < rb; ++r) kb += cursor[r] - start[r];
        n_keys = ovf_used;  // regions, then the used part of the overflow area
        {
            Stage st(c, KC_STAGE_EXTRACT_SCATTER);
            kc::fill_region_gaps<NW><<<rb, 256, 0, c->stream>>>(
                c->routed.p, c->bucket_cursor.as<unsigned long long>(), c->region_fill.as<unsigned long long>(),
                c->region_end.as<unsigned long long>(), rb);
            CK(cudaGetLastError());
        }
        break;
    }
    c->K += kb;
    if (c->after_scatter) CK(cudaEventRecord(c->after_scatter, c->stream));
    uint32_t ext_err = 0;
    CKR(get(c, &ext_err, c->scalars.as<uint32_t>() + 12, sizeof(uint32_t)));
    if (route_only) {
        CKR(sync_stream(c));
        if (ext_err) return fail(KC_ERR_DEVICE, "internal error: routing bucket disagreed with its reservation");
        c->routed_keys = n_keys;
        return KC_OK;
    }
    return count_and_pack<NW>(c, n_keys, ext_err);
}

// Filter, tables and low.bin packing of the n_keys keys in `routed`
// (EMPTY keys are skipped); ext_err is the extraction's error word, read back
// with the count's.
template <int NW>
int count_and_pack(kc_context* c, uint64_t n_keys, uint32_t ext_err) {
    constexpr int SEG = kc::count_seg<NW>();
    uint64_t* d_scal = c->scalars.as<uint64_t>();
    int rc;
    bool windowed = false;
    if constexpr (NW == 1) {
        // 64-bit keys count in shared-memory windows while every bucket's
        // filter sits in its table's cells (no table has grown yet)
        // (windows pay a read and a write of every table cell per batch:
        // worth it from 2 keys per cell, e.g. a whole input in one pass,
        // not for the host path's batches against the whole input's tables)
        if (c->window_count && n_keys >= 2 * c->table_slots_used && (c->win_ready || build_windows(c))) {
            if ((rc = window_count(c, n_keys))) return rc;
            windowed = true;
        }
    }
    if (!windowed) launch_count<NW>(c, n_keys, 1);
    const uint64_t nsegs = ceil_div(n_keys, SEG);
    CK(cudaGetLastError());
    if ((rc = rehash_loop<NW>(c, n_keys))) return rc;

    // first occurrences -> packed low.bin bytes
    if ((rc = device_scan<uint32_t, uint64_t>(c, c->tile_low.as<uint32_t>(), nsegs,
                                              c->tile_low_prefix.as<uint64_t>(), 0, d_scal + 1)))
        return rc;
    uint64_t nlow = 0;
    uint32_t cnt_err = 0;
    CKR(get(c, &nlow, d_scal + 1, sizeof(uint64_t)));
    CKR(get(c, &cnt_err, c->scalars.as<uint32_t>() + 13, sizeof(uint32_t)));
    CKR(sync_stream(c));
    if (ext_err) return fail(KC_ERR_DEVICE, "internal error: routing bucket disagreed with its reservation");
    if (cnt_err) return fail(KC_ERR_DEVICE, "internal error: a 256-bit table slot was never published");
    uint8_t* low_dst;
    uint64_t low_base;
    if (c->stream_low) {
        // this batch's first occurrences go to a ring slot that the previous
        // user (two batches ago) has finished copying out
        DevBuf& ring = c->lowring[c->batches & 1];
        if (ring.cap < nlow * c->packed_bytes + 64) {
            CK(cudaStreamSynchronize(c->d2h));
            CK(ring.ensure(nlow * c->packed_bytes + 64));
        }
        CK(cudaStreamWaitEvent(c->stream, c->ev_lowfree[c->batches & 1], 0));
        low_dst = ring.as<uint8_t>();
        low_base = 0;
    } else {
        // first occurrences accumulate over the batches; size the buffer for
        // the whole input from the share seen so far (+10%), so that it is
        // reallocated (old and new both live during the copy) about once
        uint64_t need = (c->low_total + nlow) * c->packed_bytes + 64;
        if (need > c->low_packed.cap && c->expected_total_bytes > c->input_bytes && c->input_bytes > 0)
            need = std::max<uint64_t>(need, (uint64_t)((double)need * 1.1 * (double)c->expected_total_bytes /
                                                       (double)c->input_bytes));
        CK(c->low_packed.grow_keep(need, c->low_total * c->packed_bytes, c->stream));
        low_dst = c->low_packed.as<uint8_t>();
        low_base = c->low_total;
    }
    {
        Stage st(c, KC_STAGE_PACK_LOW);
        kc::pack_low<NW><<<resident_grid(c, kc::pack_low<NW>, 256, ceil_div(nsegs, 256)), 256, 0, c->stream>>>(
            c->routed.p, c->tile_low.as<uint32_t>(), c->tile_low_prefix.as<uint64_t>(), nsegs, c->cfg.k, low_dst,
            low_base);
    }
    CK(cudaGetLastError());
    c->low_total += nlow;
    c->last_batch_low = nlow;
    return KC_OK;
}

// Export every table slot whose count passes min..max: per-chunk counts
// (export_count), their scan in chunk order = each chunk's first output
// record, then one read of the table that places the records
// (export_write).  Chunks are listed group by group (root id, or set x root
// id), so each group's records are contiguous; totals[g] receives group g's
// record count and totals[n_groups] the occupied slots.
template <int NW>
int run_export(kc_context* c, const std::vector<kc::ExportChunk>& ch, uint64_t n_groups,
               std::vector<uint64_t>& totals) {
    const uint64_t nch = ch.size();
    c->n_chunks = nch;
    CKR(join_init(c));
    CK(c->chunks.ensure(std::max<uint64_t>(nch, 1) * sizeof(kc::ExportChunk)));
    CK(c->chunk_pass.ensure(std::max<uint64_t>(nch, 1) * sizeof(uint32_t)));
    CK(c->chunk_off.ensure(std::max<uint64_t>(nch, 1) * sizeof(uint64_t)));
    CK(c->root_count.ensure((n_groups + 1) * sizeof(uint64_t)));
    if (nch) CKR(put(c, c->chunks.p, ch.data(), nch * sizeof(kc::ExportChunk)));
    CKR(fill_dev(c, c->root_count.p, (n_groups + 1) * sizeof(uint64_t), 0));
    unsigned long long* rcd = c->root_count.as<unsigned long long>();
    const uint64_t grid = std::min<uint64_t>(std::max<uint64_t>(nch, 1), (uint64_t)c->sm_count * 8);
    // the counting pass leaves a bit per passing slot when every chunk is whole
    // 32-slot words (bucket tables are powers of two of at least 64 slots at
    // offsets that are multiples of 64), and the writing pass reads only those
    uint32_t* bits = nullptr;
    bool whole_words = true;
    for (const kc::ExportChunk& e : ch) whole_words = whole_words && e.slot_begin % 32 == 0 && e.n_slots % 32 == 0;
    if (whole_words && nch) {
        CK(c->pass_bits.ensure(ceil_div(c->table_slots_used, 32) * sizeof(uint32_t)));
        bits = c->pass_bits.as<uint32_t>();
    }
    if (nch) {
        Stage st(c, KC_STAGE_EXPORT);
        const uint64_t cgrid = resident_grid(c, kc::export_count<NW>, kc::EXP_THREADS, nch);
        kc::export_count<NW><<<cgrid, kc::EXP_THREADS, 0, c->stream>>>(
            c->table.p, c->chunks.as<kc::ExportChunk>(), nch, c->cfg.min_count, c->cfg.max_count,
            c->chunk_pass.as<uint32_t>(), rcd, rcd + n_groups, bits);
        CK(cudaGetLastError());
    }
    int rc;
    if ((rc = device_scan<uint32_t, uint64_t>(c, c->chunk_pass.as<uint32_t>(), nch, c->chunk_off.as<uint64_t>(), 0,
                                              nullptr)))
        return rc;
    totals.assign(n_groups + 1, 0);
    CKR(get(c, totals.data(), rcd, (n_groups + 1) * sizeof(uint64_t)));
    CKR(sync_stream(c));
    uint64_t R = 0;
    for (uint64_t g = 0; g < n_groups; ++g) R += totals[g];
    CK(c->roots.ensure(std::max<uint64_t>(R, 1) * c->record_bytes));
    if (nch && R) {
        Stage st(c, KC_STAGE_EXPORT);
        if (bits)
            kc::export_write_bits<NW><<<resident_grid(c, kc::export_write_bits<NW>, kc::EXP_THREADS, nch),
                                        kc::EXP_THREADS, 0, c->stream>>>(
                c->table.p, bits, c->chunks.as<kc::ExportChunk>(), nch, c->chunk_off.as<uint64_t>(),
                c->roots.as<uint8_t>());
        else
            kc::export_write<NW><<<grid, kc::EXP_THREADS, 0, c->stream>>>(
                c->table.p, c->chunks.as<kc::ExportChunk>(), nch, c->cfg.min_count, c->cfg.max_count,
                c->chunk_off.as<uint64_t>(), c->roots.as<uint8_t>());
        CK(cudaGetLastError());
    }
    return KC_OK;
}

template <int NW>
int export_tables(kc_context* c) {
    const uint32_t nb = c->n_buckets;
    std::vector<kc::ExportChunk> ch;
    const uint32_t CH = 16384;
    for (uint32_t b = 0; b < nb; ++b) {
        const uint64_t slots = c->h_meta[b].tab_mask + 1;
        for (uint64_t s = 0; s < slots; s += CH) {
            kc::ExportChunk e;
            e.slot_begin = c->h_meta[b].tab_off + s;
            e.n_slots = (uint32_t)std::min<uint64_t>(CH, slots - s);
            e.root = b >> (c->bucket_bits - 8);
            ch.push_back(e);
        }
    }
    std::vector<uint64_t> h;
    int rc;
    if ((rc = run_export<NW>(c, ch, 256, h))) return rc;
    uint64_t tot = 0;
    for (int r = 0; r < 256; ++r) {
        c->root_counts[r] = h[r];
        tot += h[r];
    }
    c->root_total = tot;
    c->table_keys = h[256];
    // Record order inside a root file is unspecified in the reference (DFS and
    // hash-bucket order, src/NewKmerTree.h:773-859); here it is table order,
    // and sorting is applied by the caller of export_tables when
    // cfg.sort_output is set.
    return KC_OK;
}

int begin_run(kc_context* c, uint64_t total_bytes) {
    CK(cudaSetDevice(c->device));
    c->line_base = 0;
    c->low_total = 0;
    c->K = 0;
    c->readbacks.clear();  // a failed earlier call may have left some behind
    c->mbox_up_off = c->mbox_down_off = 0;
    c->rehashes = 0;
    c->overflow_keys = 0;
    c->reroutes = 0;
    c->window_spill = 0;
    c->batches = 0;
    c->input_bytes = 0;
    c->sized = false;
    c->have_result = false;
    c->batch_result = false;
    c->expected_total_bytes = total_bytes;
    c->ev_used = 0;
    c->spans.clear();
    std::memset(c->launches, 0, sizeof c->launches);
    std::memset(c->stage_ms, 0, sizeof c->stage_ms);
    return KC_OK;
}

// After the final synchronize: fold event spans into per-stage totals.
void collect_stage_times(kc_context* c) {
    for (auto& sp : c->spans) {
        float ms = 0;
        if (cudaEventElapsedTime(&ms, sp.second.first, sp.second.second) == cudaSuccess) c->stage_ms[sp.first] += ms;
    }
    c->spans.clear();
    c->ev_used = 0;
}

int finish_run(kc_context* c) {
    int rc;
    if (!c->sized) {
        // empty input: allocate minimal structures so the export is uniform
        std::vector<uint64_t> zero(c->n_buckets, 0);
        if ((rc = size_structures(c, zero, 1.0, 0))) return rc;
    }
    rc = c->nw == 1 ? export_tables<1>(c) : (c->nw == 2 ? export_tables<2>(c) : export_tables<4>(c));
    if (rc) return rc;
    if (c->cfg.sort_output && c->root_total > 1) {
        uint64_t bt, bh, bo, bs;
        kc_sort_scratch_bytes(c->root_total, c->record_bytes, &bt, &bh, &bo, &bs);
        CK(c->sort_tmp.ensure(bt));
        CK(c->sort_hist.ensure(bh));
        CK(c->sort_offs.ensure(bo));
        CK(c->sort_sums.ensure(bs));
        const KcSortScratch w{c->sort_tmp.p, c->sort_hist.p, c->sort_offs.p, c->sort_sums.p};
        Stage st(c, KC_STAGE_SORT, 4 * ((2 * c->cfg.k + 7) / 8));
        rc = kc_sort_roots(c->roots.p, c->root_total, c->record_bytes, c->cfg.k, w, c->stream);
        if (rc) return fail(rc, "root record sort failed: %s", kc_sort_error());
    }
    CKR(sync_stream(c));
    c->have_result = true;
    return KC_OK;
}

void fill_stats(kc_context* c, kc_stats* s, double dev_ms, double wall_ms) {
    if (!s) return;
    std::memset(s, 0, sizeof *s);
    s->input_bytes = c->input_bytes;
    s->total_kmers = c->K;
    s->low_records = c->low_total;
    s->root_records = c->root_total;
    s->table_keys = c->table_keys;
    s->rehashes = c->rehashes;
    s->batches = c->batches;
    std::memcpy(s->root_counts, c->root_counts, sizeof s->root_counts);
    s->device_ms = dev_ms;
    s->wall_ms = wall_ms;
    uint64_t live = 0;
    for (const auto& m : c->h_meta) {
        live += m.tab_mask + 1;
        s->max_bucket_table_slots = std::max<uint64_t>(s->max_bucket_table_slots, m.tab_mask + 1);
        s->max_bucket_filter_words =
            std::max<uint64_t>(s->max_bucket_filter_words, c->nw == 1 ? (m.bloom_mask + 1) / 2 : m.bloom_mask + 1);
    }
    s->table_slots = live;
    s->filter_words = c->bloom_words;
    s->overflow_keys = c->overflow_keys;
    s->reroutes = c->reroutes;
}

// Output delivery thread: waits for each device->host piece in FIFO order and
// hands it to the sink, so that the thread issuing the counting work never
// waits for a copy it does not need.  A piece with slot -1 is an empty root
// file (sink called with no bytes).  Pieces still queued at stop are drained.
void deliver_loop(kc_context* c) {
    cudaSetDevice(c->device);
    std::unique_lock<std::mutex> lk(c->pin_mu);
    for (;;) {
        c->pin_cv.wait(lk, [&] { return c->deliver_stop || !c->pending.empty(); });
        if (c->pending.empty()) return;
        const kc_context::Piece p = c->pending.front();
        const bool skip = c->sink_rc || c->deliver_err;
        lk.unlock();
        bool copy_ok = true;
        int r = 0;
        if (p.slot >= 0) copy_ok = cudaEventSynchronize(c->ev_pin[p.slot]) == cudaSuccess;
        if (copy_ok && !skip) r = c->sink(c->sink_user, p.kind, p.root, p.slot >= 0 ? c->pin[p.slot] : nullptr, p.bytes);
        lk.lock();
        if (!copy_ok) c->deliver_err = true;
        if (r && !c->sink_rc) c->sink_rc = r;
        c->pending.pop_front();
        if (p.slot >= 0) c->slot_busy[p.slot] = false;
        c->pin_cv.notify_all();
    }
}

int sink_status(kc_context* c) {
    std::lock_guard<std::mutex> lk(c->pin_mu);
    if (c->deliver_err) return fail(KC_ERR_DEVICE, "device->host copy of an output piece failed");
    if (c->sink_rc) return fail(KC_ERR_IO, "output sink returned %d", c->sink_rc);
    return KC_OK;
}

// Wait until every queued piece was delivered.
int drain_pieces(kc_context* c) {
    {
        std::unique_lock<std::mutex> lk(c->pin_mu);
        c->pin_cv.wait(lk, [&] { return c->pending.empty(); });
    }
    return sink_status(c);
}

// Copy `bytes` at device `src` (ready once `ready` fires on `stream`) out
// through the pinned slots, PIN_BYTES at a time.
int stream_piece(kc_context* c, int kind, uint32_t root, const uint8_t* src, uint64_t bytes, cudaEvent_t ready) {
    if (bytes == 0) {
        if (kind == KC_SINK_ROOT) {
            std::lock_guard<std::mutex> lk(c->pin_mu);
            c->pending.push_back({kind, root, 0, -1});
            c->pin_cv.notify_all();
        }
        return sink_status(c);
    }
    CK(cudaStreamWaitEvent(c->d2h, ready, 0));
    for (uint64_t off = 0; off < bytes; off += kc_context::PIN_BYTES) {
        const uint64_t m = std::min<uint64_t>(kc_context::PIN_BYTES, bytes - off);
        int slot = -1;
        {
            std::unique_lock<std::mutex> lk(c->pin_mu);
            c->pin_cv.wait(lk, [&] {
                for (int q = 0; q < kc_context::PIN_SLOTS; ++q)
                    if (!c->slot_busy[q]) {
                        slot = q;
                        return true;
                    }
                return c->sink_rc != 0 || c->deliver_err;
            });
            if (slot < 0) break;  // the sink failed: stop producing
            c->slot_busy[slot] = true;
        }
        CK(cudaMemcpyAsync(c->pin[slot], src + off, m, cudaMemcpyDeviceToHost, c->d2h));
        CK(cudaEventRecord(c->ev_pin[slot], c->d2h));
        std::lock_guard<std::mutex> lk(c->pin_mu);
        c->pending.push_back({kind, root, m, slot});
        c->pin_cv.notify_all();
    }
    return sink_status(c);
}

int stream_out_low(kc_context* c) {
    const int ring = (int)((c->batches) & 1);  // ring slot used by the batch just packed
    CK(cudaEventRecord(c->ev_pack, c->stream));
    int rc = stream_piece(c, KC_SINK_LOW, 0, c->lowring[ring].as<uint8_t>(), c->last_batch_low * c->packed_bytes,
                          c->ev_pack);
    if (rc) return rc;
    // the ring slot is free for reuse once these copies are done
    CK(cudaEventRecord(c->ev_lowfree[ring], c->d2h));
    return KC_OK;
}

int stream_out_roots(kc_context* c) {
    CK(cudaEventRecord(c->ev_pack, c->stream));
    uint64_t off = 0;
    for (uint32_t r = 0; r < 256; ++r) {
        const uint64_t bytes = c->root_counts[r] * c->record_bytes;
        int rc = stream_piece(c, KC_SINK_ROOT, r, c->roots.as<uint8_t>() + off, bytes, c->ev_pack);
        if (rc) return rc;
        off += bytes;
    }
    return KC_OK;
}

int run_batch(kc_context* c, const uint8_t* buf, uint64_t n, int has_halo) {
    c->batches++;
    c->input_bytes += n;
    if (c->nw == 1) return process_batch<1>(c, buf, n, has_halo);
    if (c->nw == 2) return process_batch<2>(c, buf, n, has_halo);
    return process_batch<4>(c, buf, n, has_halo);
}

// Count n_keys canonical keys already extracted and routed elsewhere (the
// owner side of a sharded count): size from the per-routing-bucket totals,
// copy the keys into `routed`, then filter, tables and packing as for a
// batch of FASTQ.
template <int NW>
int count_keys(kc_context* c, const void* d_keys, uint64_t n_keys, const uint64_t* counts) {
    constexpr int CT = kc::count_tile<NW>();
    constexpr int SEG = kc::count_seg<NW>();
    const uint32_t nb = c->n_buckets;
    const uint32_t per = nb / 256;  // table buckets per routing bucket (1 or 16)
    std::vector<uint64_t> kest(nb);
    for (uint32_t b = 0; b < nb; ++b) {
        const uint64_t r = counts[b / per];
        kest[b] = r / per + ((b % per) < (r % per) ? 1 : 0);
    }
    int rc;
    if ((rc = size_structures(c, kest, 1.0, 0))) return rc;
    const uint64_t ctiles = ceil_div(n_keys, CT);
    CK(c->routed.ensure(ctiles * CT * (uint64_t)(8 * NW)));
    CK(c->tile_low.ensure(ctiles * (CT / SEG) * sizeof(uint32_t)));
    CK(c->tile_fail.ensure(ctiles * (CT / SEG) * sizeof(uint32_t)));
    CK(c->tile_low_prefix.ensure(ctiles * (CT / SEG) * sizeof(uint64_t)));
    CK(c->scalars.ensure(64));
    CKR(fill_dev(c, c->scalars.as<uint32_t>() + 12, 2 * sizeof(uint32_t), 0));
    CK(cudaMemcpyAsync(c->routed.p, d_keys, n_keys * (uint64_t)(8 * NW), cudaMemcpyDefault, c->stream));
    c->K += n_keys;
    c->batches++;
    return count_and_pack<NW>(c, n_keys, 0);
}

}  // namespace

// ------------------------------------------------------------------ C ABI

extern "C" {

void kc_config_default(kc_config* g) {
    if (!g) return;
    std::memset(g, 0, sizeof *g);
    g->k = 31;
    g->canonical = 1;
    g->min_count = 1;
    g->max_count = 0xFFFFFFFFu;
    g->n_buckets = 256;
    g->sizing = KC_SIZING_SAMPLED;
    g->device = 0;
    g->sort_output = 0;
    g->chunk_bytes = 256ull << 20;
    g->batch_bytes = 1ull << 30;
    g->bloom_bits = 5.0;  // the reference sizes its filters at 4.81 bits per estimated k-mer (src/main.cpp:88-108)
    g->table_load = 0.7;
    g->repeat_ratio = 0.125;
    g->device_batch_bytes = 8ull << 30;
}

const char* kc_last_error(void) { return g_err.c_str(); }

uint64_t kc_packed_bytes(uint32_t k) { return (uint64_t)(k / 32) * 8 + (2 * (k % 32) + 7) / 8; }

uint64_t kc_record_bytes(uint32_t k) { return k <= 32 ? 16 : (k <= 64 ? 24 : 40); }

int kc_create(const kc_config* cfg, kc_context** out) {
    if (!cfg || !out) return fail(KC_ERR_INVALID, "null argument");
    *out = nullptr;
    kc_context* c = new kc_context();
    c->cfg = *cfg;
    int rc = setup_shape(c);
    if (rc) {
        delete c;
        return rc;
    }
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        delete c;
        return fail(KC_ERR_DEVICE, "no CUDA device available (%s)", cudaGetErrorString(e));
    }
    if (cfg->device < 0 || cfg->device >= ndev) {
        delete c;
        return fail(KC_ERR_INVALID, "device %d out of range (%d devices)", cfg->device, ndev);
    }
    c->device = cfg->device;
    cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, cfg->device);
    int prio_low = 0, prio_high = 0;
    if ((e = cudaSetDevice(c->device)) != cudaSuccess ||
        (e = cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high)) != cudaSuccess ||
        (e = cudaStreamCreateWithPriority(&c->stream, cudaStreamNonBlocking, cfg->priority ? prio_high : 0)) !=
            cudaSuccess ||
        (e = cudaEventCreate(&c->ev0)) != cudaSuccess || (e = cudaEventCreate(&c->ev1)) != cudaSuccess) {
        delete c;
        return fail(KC_ERR_DEVICE, "stream/event creation failed: %s", cudaGetErrorString(e));
    }
    if ((e = cudaStreamCreateWithFlags(&c->h2d, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&c->d2h, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaStreamCreateWithPriority(&c->side, cudaStreamNonBlocking, prio_high)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&c->ev_side_in, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&c->ev_init, cudaEventDisableTiming)) != cudaSuccess) {
        kc_destroy(c);
        return fail(KC_ERR_DEVICE, "stream creation failed: %s", cudaGetErrorString(e));
    }
    for (int i = 0; i < 2; ++i) {
        cudaEventCreateWithFlags(&c->ev_h2d[i], cudaEventDisableTiming);
        cudaEventCreateWithFlags(&c->ev_free[i], cudaEventDisableTiming);
        cudaEventCreateWithFlags(&c->ev_lowfree[i], cudaEventDisableTiming);
    }
    for (int i = 0; i < kc_context::PIN_SLOTS; ++i) cudaEventCreateWithFlags(&c->ev_pin[i], cudaEventDisableTiming);
    cudaEventCreateWithFlags(&c->ev_pack, cudaEventDisableTiming);
    cudaEventCreateWithFlags(&c->ev_mbox, cudaEventDisableTiming);
    if ((e = cudaHostAlloc(reinterpret_cast<void**>(&c->mbox_h), kc_context::MBOX_UP + kc_context::MBOX_DOWN,
                           cudaHostAllocMapped | cudaHostAllocPortable)) != cudaSuccess ||
        (e = cudaHostGetDevicePointer(reinterpret_cast<void**>(&c->mbox_d), c->mbox_h, 0)) != cudaSuccess) {
        kc_destroy(c);
        return fail(KC_ERR_DEVICE, "mapped control mailbox allocation failed: %s", cudaGetErrorString(e));
    }
    // 4096-bucket extraction and the scatter staging area exceed 48 KiB.
    cudaFuncSetAttribute(kc::extract_kernel<1, kc::HIST>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)kc::extract_smem_bytes<1, kc::HIST>(4096));
    cudaFuncSetAttribute(kc::extract_kernel<1, kc::SCATTER>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)kc::extract_smem_bytes<1, kc::SCATTER>(4096));
    cudaFuncSetAttribute(kc::extract_kernel<2, kc::HIST>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)kc::extract_smem_bytes<2, kc::HIST>(4096));
    cudaFuncSetAttribute(kc::extract_kernel<2, kc::SCATTER>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)kc::extract_smem_bytes<2, kc::SCATTER>(4096));
    cudaFuncSetAttribute(kc::extract_kernel<4, kc::HIST>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)kc::extract_smem_bytes<4, kc::HIST>(4096));
    cudaFuncSetAttribute(kc::extract_kernel<4, kc::SCATTER>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)kc::extract_smem_bytes<4, kc::SCATTER>(4096));
    cudaFuncSetAttribute(kc::count_window, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kc::window_smem_bytes());
    cudaFuncSetAttribute(kc::loads_table_pass<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kc::loads_table_smem());
    cudaFuncSetAttribute(kc::loads_table_pass<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kc::loads_table_smem());
    cudaFuncSetAttribute(kc::loads_table_pass<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kc::loads_table_smem());
    cudaFuncSetAttribute(kc::subroute_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)kc::scatter_smem_bytes());
    if ((e = cudaGetLastError()) != cudaSuccess) {
        delete c;
        return fail(KC_ERR_DEVICE, "kernel attribute setup failed: %s", cudaGetErrorString(e));
    }
    if (const char* w = std::getenv("KC_WINDOW_COUNT")) c->window_count = std::strcmp(w, "0") != 0;
    *out = c;
    return KC_OK;
}

void kc_destroy(kc_context* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->side) cudaStreamSynchronize(c->side);
    DevBuf* bufs[] = {&c->stage,  &c->tile_nl,   &c->tile_line, &c->bucket_count, &c->bucket_cursor, &c->region_end, &c->region_fill, &c->routed,
                      &c->tile_low, &c->tile_fail, &c->tile_low_prefix, &c->scan_sums, &c->scalars, &c->overflow,
                      &c->meta,   &c->bloom,     &c->table,     &c->low_packed,   &c->roots,         &c->chunks,
                      &c->root_count, &c->chunk_pass, &c->chunk_off, &c->sort_tmp, &c->sort_hist, &c->sort_offs, &c->sort_sums,
                      &c->set_tiles, &c->tile_prefix, &c->set_info, &c->hist_tiles, &c->pass_bits, &c->loads, &c->routed2,
                      &c->grow_jobs, &c->grow_failed,
                      &c->bucket_win, &c->win_info, &c->win_order, &c->win_count, &c->win_padded, &c->win_start, &c->win_cursor,
                      &c->win_end};
    for (DevBuf* b : bufs) b->release();
    for (cudaEvent_t e : c->ev_pool) cudaEventDestroy(e);
    if (c->h2d) cudaStreamSynchronize(c->h2d);
    if (c->d2h) cudaStreamSynchronize(c->d2h);
    for (int i = 0; i < 2; ++i) {
        for (cudaEvent_t e : {c->ev_h2d[i], c->ev_free[i], c->ev_lowfree[i]})
            if (e) cudaEventDestroy(e);
        c->lowring[i].release();
    }
    for (int i = 0; i < kc_context::PIN_SLOTS; ++i) {
        if (c->ev_pin[i]) cudaEventDestroy(c->ev_pin[i]);
        if (c->pin[i]) cudaFreeHost(c->pin[i]);
    }
    for (int i = 0; i < kc_context::RING_SLOTS; ++i) {
        if (c->ev_ring[i]) cudaEventDestroy(c->ev_ring[i]);
        if (c->ring[i]) cudaFreeHost(c->ring[i]);
    }
    for (cudaGraphExec_t& x : c->sets_exec)
        if (x) cudaGraphExecDestroy(x);
    if (c->ev_pack) cudaEventDestroy(c->ev_pack);
    if (c->ev_mbox) cudaEventDestroy(c->ev_mbox);
    if (c->mbox_h) cudaFreeHost(c->mbox_h);
    c->stage2.release();
    if (c->h2d) cudaStreamDestroy(c->h2d);
    if (c->d2h) cudaStreamDestroy(c->d2h);
    if (c->side) cudaStreamDestroy(c->side);
    if (c->ev_side_in) cudaEventDestroy(c->ev_side_in);
    if (c->ev_init) cudaEventDestroy(c->ev_init);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

void* kc_stream(kc_context* c) { return c ? (void*)c->stream : nullptr; }

int kc_set_profiling(kc_context* c, int enable) {
    if (!c) return fail(KC_ERR_INVALID, "null context");
    c->profiling = enable != 0;
    return KC_OK;
}

int kc_stage_times(kc_context* c, double* ms, uint64_t* launches, int cap) {
    if (!c) return fail(KC_ERR_INVALID, "null context");
    for (int i = 0; i < cap && i < KC_STAGE_COUNT; ++i) {
        if (ms) ms[i] = c->stage_ms[i];
        if (launches) launches[i] = c->launches[i];
    }
    return KC_STAGE_COUNT;
}

const char* kc_stage_name(int stage) {
    return stage >= 0 && stage < KC_STAGE_COUNT ? kStageNames[stage] : "";
}

int kc_count_device(kc_context* c, const uint8_t* d_fastq, uint64_t n, kc_stats* stats) {
    if (!c || (!d_fastq && n)) return fail(KC_ERR_INVALID, "null argument");
    const auto t0 = std::chrono::steady_clock::now();
    int rc = begin_run(c, n);
    if (rc) return rc;
    CK(cudaEventRecord(c->ev0, c->stream));
    const uint64_t want = c->cfg.device_batch_bytes ? c->cfg.device_batch_bytes : c->cfg.batch_bytes;
    const uint64_t B = std::max<uint64_t>(kc::EXT_TILE, want & ~(uint64_t)(kc::EXT_TILE - 1));
    for (uint64_t off = 0; off < n || (n == 0 && off == 0); off += B) {
        if (n == 0) break;
        const uint64_t len = std::min<uint64_t>(B, n - off);
        if ((rc = run_batch(c, d_fastq + off, len, off > 0))) return rc;
    }
    if ((rc = finish_run(c))) return rc;
    CK(cudaEventRecord(c->ev1, c->stream));
    CK(cudaEventSynchronize(c->ev1));
    collect_stage_times(c);
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    const double wall = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    fill_stats(c, stats, ms, wall);
    return KC_OK;
}

// Batch lengths of a host input: batch_bytes B each, except that a long
// input (at least 4 B, B >= 64 MiB) ramps up over its first batches (B/8,
// B/4, B/2) and down over its last ones, so that the first output leaves
// early and the last batch is counted soon after its bytes arrived.
std::vector<uint64_t> plan_batches(uint64_t n, uint64_t B) {
    std::vector<uint64_t> v;
    if (!n) return v;
    const uint64_t T = kc::EXT_TILE;
    auto al = [&](uint64_t x) { return std::max<uint64_t>(T, x & ~(T - 1)); };
    if (n < 4 * B || B < (64ull << 20)) {
        for (uint64_t off = 0; off < n; off += B) v.push_back(std::min<uint64_t>(B, n - off));
        return v;
    }
    const uint64_t ramp[3] = {al(B / 8), al(B / 4), al(B / 2)};
    const uint64_t ends = 2 * (ramp[0] + ramp[1] + ramp[2]);
    const uint64_t mid = n - ends;  // > 2 B
    const uint64_t k = ceil_div(mid, B);
    const uint64_t each = al(mid / k);
    v.assign(ramp, ramp + 3);
    for (uint64_t i = 0; i + 1 < k; ++i) v.push_back(each);
    v.push_back(mid - (k - 1) * each);
    for (int i = 2; i >= 0; --i) v.push_back(ramp[i]);
    return v;
}

// pread of [off, off + n) into dst by up to 8 threads (page-cache copies run
// at memory speed per thread, so a few threads read several times faster).
static bool read_parallel(int fd, uint8_t* dst, uint64_t off, uint64_t n) {
    const uint64_t parts = std::max<uint64_t>(1, std::min<uint64_t>(8, n >> 23));  // >= 8 MiB each
    const uint64_t each = (n + parts - 1) / parts;
    std::vector<std::thread> th;
    std::vector<char> ok(parts, 0);
    auto work = [&](uint64_t p) {
        const uint64_t a = p * each, b = std::min<uint64_t>(n, a + each);
        uint64_t got = a;
        while (got < b) {
            const ssize_t r = ::pread(fd, dst + got, b - got, (off_t)(off + got));
            if (r < 0 && errno == EINTR) continue;
            if (r <= 0) return;
            got += (uint64_t)r;
        }
        ok[p] = 1;
    };
    for (uint64_t p = 1; p < parts; ++p) th.emplace_back(work, p);
    work(0);
    for (auto& t : th) t.join();
    for (char v : ok)
        if (!v) return false;
    return true;
}

// Host input, double-buffered: batch i+1 is copied host->device on its own
// stream (chunk_bytes pieces) while batch i is counted.  Staging buffers are
// [HALO | batch | pad]; the HALO bytes before a batch are copied from the
// host too, so windows that straddle a batch split are seen once, as the
// reference reader's k-1 overlap does (src/FastqReader.h:338-365).
int host_pipeline(kc_context* c, const uint8_t* fastq, uint64_t n) {
    const uint64_t B = std::max<uint64_t>(kc::EXT_TILE, c->cfg.batch_bytes & ~(uint64_t)(kc::EXT_TILE - 1));
    const std::vector<uint64_t> plan = plan_batches(n, B);
    const uint64_t nbatch = plan.size();
    std::vector<uint64_t> offs(nbatch);
    uint64_t cap = 1;
    for (uint64_t i = 0, o = 0; i < nbatch; o += plan[i], ++i) {
        offs[i] = o;
        cap = std::max<uint64_t>(cap, plan[i]);
    }
    CK(c->stage.ensure(kc::HALO + cap + kc::EXT_TILE));
    if (nbatch > 1) CK(c->stage2.ensure(kc::HALO + cap + kc::EXT_TILE));
    uint8_t* slots[2] = {c->stage.as<uint8_t>(), c->stage2.as<uint8_t>()};
    const uint64_t chunk = std::max<uint64_t>(c->cfg.chunk_bytes, 1 << 20);
    const bool from_file = c->src_fd >= 0;
    auto enqueue_copy = [&](uint64_t i) -> int {
        const int slot = (int)(i & 1);
        const uint64_t off = offs[i], len = plan[i];
        uint8_t* dst = slots[slot];
        if (i >= 2) CK(cudaStreamWaitEvent(c->h2d, c->ev_free[slot], 0));
        if (from_file) {
            // [HALO before the batch | batch] from the file, through the ring
            const uint64_t start = off >= (uint64_t)kc::HALO ? off - kc::HALO : off;
            uint8_t* d = off >= (uint64_t)kc::HALO ? dst : dst + kc::HALO;
            const uint64_t total = off + len - start;
            for (uint64_t q = 0; q < total; q += kc_context::RING_BYTES) {
                const uint64_t m = std::min<uint64_t>(kc_context::RING_BYTES, total - q);
                const int s = (int)(c->ring_next++ % kc_context::RING_SLOTS);
                CK(cudaEventSynchronize(c->ev_ring[s]));  // its previous copy has left
                if (!read_parallel(c->src_fd, c->ring[s], start + q, m))
                    return fail(KC_ERR_IO, "Failed to read fastq data at byte %llu", (unsigned long long)(start + q));
                CK(cudaMemcpyAsync(d + q, c->ring[s], m, cudaMemcpyHostToDevice, c->h2d));
                CK(cudaEventRecord(c->ev_ring[s], c->h2d));
            }
        } else {
            if (off >= (uint64_t)kc::HALO)
                CK(cudaMemcpyAsync(dst, fastq + off - kc::HALO, kc::HALO, cudaMemcpyHostToDevice, c->h2d));
            for (uint64_t q = 0; q < len; q += chunk)
                CK(cudaMemcpyAsync(dst + kc::HALO + q, fastq + off + q, std::min<uint64_t>(chunk, len - q),
                                   cudaMemcpyHostToDevice, c->h2d));
        }
        CK(cudaEventRecord(c->ev_h2d[slot], c->h2d));
        return KC_OK;
    };
    int rc;
    if (nbatch && (rc = enqueue_copy(0))) return rc;
    for (uint64_t i = 0; i < nbatch; ++i) {
        // host memory: the next batch's copy is queued before this batch's
        // work; from a file, its read follows this batch's launches, so that
        // the device counts while the host reads
        if (!from_file && i + 1 < nbatch && (rc = enqueue_copy(i + 1))) return rc;
        const int slot = (int)(i & 1);
        CK(cudaStreamWaitEvent(c->stream, c->ev_h2d[slot], 0));
        c->after_scatter = c->ev_free[slot];
        rc = run_batch(c, slots[slot] + kc::HALO, plan[i], offs[i] > 0);
        c->after_scatter = nullptr;
        if (rc) return rc;
        if (c->stream_low && (rc = stream_out_low(c))) return rc;
        if (from_file && i + 1 < nbatch && (rc = enqueue_copy(i + 1))) return rc;
    }
    return KC_OK;
}

int kc_route_device(kc_context* c, const uint8_t* d_fastq, uint64_t n, uint64_t* counts) {
    if (!c || (!d_fastq && n) || !counts) return fail(KC_ERR_INVALID, "null argument");
    int rc = begin_run(c, n);
    if (rc) return rc;
    c->have_route = false;
    c->routed_keys = 0;
    c->route_counts.assign(256, 0);
    if (n) {
        c->batches = 1;
        c->input_bytes = n;
        rc = c->nw == 1 ? process_batch<1>(c, d_fastq, n, 0, true)
                        : (c->nw == 2 ? process_batch<2>(c, d_fastq, n, 0, true) : process_batch<4>(c, d_fastq, n, 0, true));
        if (rc) return rc;
    }
    CKR(sync_stream(c));
    collect_stage_times(c);
    for (int r = 0; r < 256; ++r) counts[r] = r < (int)c->route_counts.size() ? c->route_counts[r] : 0;
    c->have_route = true;
    return KC_OK;
}

int kc_routed_keys(kc_context* c, const void** d_keys, uint64_t* n_keys) {
    if (!c || !d_keys || !n_keys) return fail(KC_ERR_INVALID, "null argument");
    if (!c->have_route) return fail(KC_ERR_STATE, "no routed keys: call kc_route_device first");
    CK(cudaStreamSynchronize(c->stream));
    *d_keys = c->routed.p;
    *n_keys = c->routed_keys;
    return KC_OK;
}

int kc_copy_routed(kc_context* c, void* dst, uint64_t cap) {
    if (!c) return fail(KC_ERR_INVALID, "null context");
    if (!c->have_route) return fail(KC_ERR_STATE, "no routed keys: call kc_route_device first");
    const uint64_t bytes = c->routed_keys * 8ull * c->nw;
    if (!bytes) return KC_OK;
    if (!dst || cap < bytes) return fail(KC_ERR_INVALID, "destination holds %llu bytes, %llu needed",
                                         (unsigned long long)cap, (unsigned long long)bytes);
    CK(cudaMemcpyAsync(dst, c->routed.p, bytes, cudaMemcpyDefault, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return KC_OK;
}

int kc_count_keys_device(kc_context* c, const void* d_keys, uint64_t n_keys, const uint64_t* counts,
                         kc_stats* stats) {
    if (!c || (!d_keys && n_keys) || !counts) return fail(KC_ERR_INVALID, "null argument");
    uint64_t total = 0;
    for (int r = 0; r < 256; ++r) total += counts[r];
    if (total != n_keys) return fail(KC_ERR_INVALID, "bucket counts sum to %llu, not n_keys = %llu",
                                     (unsigned long long)total, (unsigned long long)n_keys);
    const auto t0 = std::chrono::steady_clock::now();
    int rc = begin_run(c, 0);
    if (rc) return rc;
    c->have_route = false;  // `routed` is overwritten
    CK(cudaEventRecord(c->ev0, c->stream));
    if (n_keys) {
        rc = c->nw == 1 ? count_keys<1>(c, d_keys, n_keys, counts)
                        : (c->nw == 2 ? count_keys<2>(c, d_keys, n_keys, counts) : count_keys<4>(c, d_keys, n_keys, counts));
        if (rc) return rc;
    }
    if ((rc = finish_run(c))) return rc;
    CK(cudaEventRecord(c->ev1, c->stream));
    CK(cudaEventSynchronize(c->ev1));
    collect_stage_times(c);
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    const double wall = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    fill_stats(c, stats, ms, wall);
    return KC_OK;
}

int kc_count_host(kc_context* c, const uint8_t* fastq, uint64_t n, kc_stats* stats) {
    if (!c || (!fastq && n)) return fail(KC_ERR_INVALID, "null argument");
    const auto t0 = std::chrono::steady_clock::now();
    int rc = begin_run(c, n);
    if (rc) return rc;
    c->stream_low = false;
    CK(cudaEventRecord(c->ev0, c->stream));
    if ((rc = host_pipeline(c, fastq, n))) return rc;
    if ((rc = finish_run(c))) return rc;
    CK(cudaEventRecord(c->ev1, c->stream));
    CK(cudaEventSynchronize(c->ev1));
    collect_stage_times(c);
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    const double wall = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    fill_stats(c, stats, ms, wall);
    return KC_OK;
}

}  // extern "C"

namespace {

// The streamed count of n input bytes from host memory (fastq) or from a file
// descriptor (fd >= 0, read in pieces through the pinned ring).
int count_stream_impl(kc_context* c, const uint8_t* fastq, int fd, uint64_t n, kc_sink_fn sink, void* user,
                      kc_stats* stats) {
    const auto t0 = std::chrono::steady_clock::now();
    int rc = begin_run(c, n);
    if (rc) return rc;
    // a streamed result is never kept on the device: drop the previous
    // result's packed first occurrences (they can be tens of GB)
    c->low_packed.release();
    for (int i = 0; i < kc_context::PIN_SLOTS; ++i) {
        if (!c->pin[i]) {
            if (cudaHostAlloc(reinterpret_cast<void**>(&c->pin[i]), kc_context::PIN_BYTES, cudaHostAllocDefault) !=
                cudaSuccess) {
                cudaGetLastError();
                c->pin[i] = nullptr;
                return fail(KC_ERR_NOMEM, "pinned staging allocation failed");
            }
        }
    }
    for (int i = 0; i < 2; ++i) CK(cudaEventRecord(c->ev_lowfree[i], c->d2h));
    c->stream_low = true;
    c->sink = sink;
    c->sink_user = user;
    {
        std::lock_guard<std::mutex> lk(c->pin_mu);
        c->sink_rc = 0;
        c->deliver_err = false;
        c->deliver_stop = false;
        c->pending.clear();
        for (bool& b : c->slot_busy) b = false;
    }
    try {
        c->deliverer = std::thread(deliver_loop, c);
    } catch (...) {
        c->stream_low = false;
        return fail(KC_ERR_NOMEM, "could not start the output delivery thread");
    }
    // stops the delivery thread on every exit path, after it delivered (or,
    // once the sink failed, skipped) every queued piece
    struct StopDelivery {
        kc_context* c;
        ~StopDelivery() {
            {
                std::lock_guard<std::mutex> lk(c->pin_mu);
                c->deliver_stop = true;
            }
            c->pin_cv.notify_all();
            if (c->deliverer.joinable()) c->deliverer.join();
            c->stream_low = false;
        }
    } stop{c};
    if (fd >= 0) {
        for (int i = 0; i < kc_context::RING_SLOTS; ++i) {
            if (!c->ring[i] && cudaHostAlloc(reinterpret_cast<void**>(&c->ring[i]), kc_context::RING_BYTES,
                                             cudaHostAllocDefault) != cudaSuccess) {
                cudaGetLastError();
                c->ring[i] = nullptr;
                return fail(KC_ERR_NOMEM, "pinned read ring allocation failed");
            }
            if (!c->ev_ring[i]) CK(cudaEventCreateWithFlags(&c->ev_ring[i], cudaEventDisableTiming));
        }
    }
    struct SourceGuard {
        kc_context* c;
        ~SourceGuard() { c->src_fd = -1; }
    } src{c};
    c->src_fd = fd;
    CK(cudaEventRecord(c->ev0, c->stream));
    rc = host_pipeline(c, fastq, n);
    if (!rc) rc = finish_run(c);
    if (!rc) rc = stream_out_roots(c);
    const int drc = drain_pieces(c);
    if (rc) return rc;
    if (drc) return drc;
    CK(cudaEventRecord(c->ev1, c->stream));
    CK(cudaEventSynchronize(c->ev1));
    collect_stage_times(c);
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    const double wall = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    fill_stats(c, stats, ms, wall);
    return KC_OK;
}

}  // namespace

extern "C" {

int kc_count_host_stream(kc_context* c, const uint8_t* fastq, uint64_t n, kc_sink_fn sink, void* user,
                         kc_stats* stats) {
    if (!c || (!fastq && n) || !sink) return fail(KC_ERR_INVALID, "null argument");
    return count_stream_impl(c, fastq, -1, n, sink, user, stats);
}

}  // extern "C"

// The streamed count of a plain FASTQ file's n bytes read from fd (kc_count_fastq).
int kc_internal_count_fd_stream(kc_context* c, int fd, uint64_t n, kc_sink_fn sink, void* user, kc_stats* stats) {
    if (!c || fd < 0 || !sink) return fail(KC_ERR_INVALID, "null argument");
    return count_stream_impl(c, nullptr, fd, n, sink, user, stats);
}

namespace {

// Merged-count histogram kernels: low.bin keys looked up (and marked) in
// their tables, then every unmarked key of each live bucket table (regions
// left behind by a rehash are stale copies and are not walked).
template <int NW>
void histogram_kernels(kc_context* c, uint32_t min_freq, uint32_t max_freq, unsigned long long* d, uint64_t bins) {
    const int grid = c->sm_count * 8;
    kc::hist_clear_marks<NW><<<grid, 256, 0, c->stream>>>(c->table.p, c->table_slots_used);
    kc::hist_low_pass<NW><<<grid, 256, 0, c->stream>>>(c->low_packed.as<uint8_t>(), c->low_total, c->cfg.k,
                                                       c->meta.as<kc::BucketMeta>(), c->bucket_shift, c->table.p,
                                                       min_freq, max_freq, d);
    // the export's chunk list covers exactly the live bucket tables
    if (c->n_chunks)
        kc::hist_table_pass<NW><<<std::min<uint64_t>(c->n_chunks, (uint64_t)grid), 256, 0, c->stream>>>(
            c->table.p, c->chunks.as<kc::ExportChunk>(), c->n_chunks, min_freq, max_freq, d, d + bins);
}

// Per model bucket loads: dd[0..4096) distinct, [4096..8192) table keys,
// [8192..12288) k-mer occurrences.
template <int NW>
void loads_kernels(kc_context* c, unsigned long long* dd) {
    const int grid = c->sm_count * 8;
    kc::hist_clear_marks<NW><<<grid, 256, 0, c->stream>>>(c->table.p, c->table_slots_used);
    // per-CTA shared-memory totals: a few CTAs per SM, each flushing 4096 bins once
    const uint64_t lgrid = std::max<uint64_t>(1, std::min<uint64_t>(ceil_div(c->low_total, 4096),
                                                                      (uint64_t)c->sm_count * 2));
    kc::loads_low_pass<NW><<<lgrid, 512, kc::loads_low_smem(), c->stream>>>(
        c->low_packed.as<uint8_t>(), c->low_total, c->cfg.k, c->meta.as<kc::BucketMeta>(), c->bucket_shift,
        c->table.p, dd, dd + 2 * KC_MODEL_BUCKETS);
    if (c->n_chunks)
        kc::loads_table_pass<NW><<<std::min<uint64_t>(c->n_chunks, (uint64_t)c->sm_count * 2), 512,
                                   kc::loads_table_smem(), c->stream>>>(
            c->table.p, c->chunks.as<kc::ExportChunk>(), c->n_chunks, dd, dd + KC_MODEL_BUCKETS,
            dd + 2 * KC_MODEL_BUCKETS);
}

}  // namespace

extern "C" {

// Merged count histogram and distinct keys of the last device-held result.
int kc_histogram(kc_context* c, uint32_t min_freq, uint32_t max_freq, uint64_t* hist, uint64_t* distinct) {
    if (!c) return fail(KC_ERR_INVALID, "null context");
    if (!c->have_result) return fail(KC_ERR_STATE, "no result: run a count first");
    if (c->batch_result) return fail(KC_ERR_STATE, "a multi-set result has one histogram per set; not supported");
    if (c->stream_low) return fail(KC_ERR_STATE, "streamed results are not kept on the device");
    if (max_freq < min_freq || min_freq == 0) return fail(KC_ERR_INVALID, "need 1 <= min_freq <= max_freq");
    const uint64_t bins = (uint64_t)max_freq - min_freq + 1;
    if (bins > (1ull << 26)) return fail(KC_ERR_INVALID, "histogram range too large");
    DevBuf gh;
    CK(gh.ensure((bins + 1) * sizeof(unsigned long long)));
    unsigned long long* d = gh.as<unsigned long long>();
    CK(cudaMemsetAsync(d, 0, (bins + 1) * sizeof(unsigned long long), c->stream));
    if (c->nw == 1) histogram_kernels<1>(c, min_freq, max_freq, d, bins);
    else if (c->nw == 2) histogram_kernels<2>(c, min_freq, max_freq, d, bins);
    else histogram_kernels<4>(c, min_freq, max_freq, d, bins);
    CK(cudaGetLastError());
    std::vector<unsigned long long> h(bins + 1);
    CK(cudaMemcpyAsync(h.data(), d, (bins + 1) * sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    gh.release();
    if (hist)
        for (uint64_t i = 0; i < bins; ++i) hist[i] = h[i];
    if (distinct) *distinct = c->low_total + h[bins];
    return KC_OK;
}

int kc_result_sizes(kc_context* c, uint64_t* low_bytes, uint64_t* n_root, uint64_t* root_counts) {
    if (!c) return fail(KC_ERR_INVALID, "null context");
    if (!c->have_result) return fail(KC_ERR_STATE, "no result: run a count first");
    if (low_bytes) *low_bytes = c->batch_result ? c->batch_low_bytes : c->low_total * c->packed_bytes;
    if (n_root) *n_root = c->root_total;
    if (root_counts) std::memcpy(root_counts, c->root_counts, sizeof c->root_counts);
    return KC_OK;
}

int kc_copy_low(kc_context* c, uint8_t* dst, uint64_t cap) {
    if (!c) return fail(KC_ERR_INVALID, "null context");
    if (!c->have_result) return fail(KC_ERR_STATE, "no result: run a count first");
    const uint64_t bytes = c->batch_result ? c->batch_low_bytes : c->low_total * c->packed_bytes;
    if (cap < bytes) return fail(KC_ERR_INVALID, "destination too small: %llu < %llu", (unsigned long long)cap,
                                 (unsigned long long)bytes);
    if (bytes) {
        CK(cudaMemcpyAsync(dst, c->low_packed.p, bytes, cudaMemcpyDefault, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
    return KC_OK;
}

int kc_copy_roots(kc_context* c, uint8_t* dst, uint64_t cap) {
    if (!c) return fail(KC_ERR_INVALID, "null context");
    if (!c->have_result) return fail(KC_ERR_STATE, "no result: run a count first");
    const uint64_t bytes = c->root_total * c->record_bytes;
    if (cap < bytes) return fail(KC_ERR_INVALID, "destination too small: %llu < %llu", (unsigned long long)cap,
                                 (unsigned long long)bytes);
    if (bytes) {
        CK(cudaMemcpyAsync(dst, c->roots.p, bytes, cudaMemcpyDefault, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
    return KC_OK;
}

int kc_device_results(kc_context* c, const void** d_low, uint64_t* low_bytes, const void** d_roots, uint64_t* n_roots) {
    if (!c) return fail(KC_ERR_INVALID, "null context");
    if (!c->have_result) return fail(KC_ERR_STATE, "no result: run a count first");
    if (d_low) *d_low = c->low_packed.p;
    if (low_bytes) *low_bytes = c->batch_result ? c->batch_low_bytes : c->low_total * c->packed_bytes;
    if (d_roots) *d_roots = c->roots.p;
    if (n_roots) *n_roots = c->root_total;
    return KC_OK;
}

void* kc_host_alloc(uint64_t bytes) {
    void* p = nullptr;
    if (cudaHostAlloc(&p, bytes ? bytes : 1, cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        fail(KC_ERR_NOMEM, "cudaHostAlloc(%llu) failed", (unsigned long long)bytes);
        return nullptr;
    }
    return p;
}

void kc_host_free(void* p) {
    if (p) cudaFreeHost(p);
}

}  // extern "C"

extern "C" int kc_set_predicted_loads(kc_context* c, const double* distinct, const double* table_keys) {
    if (!c) return fail(KC_ERR_INVALID, "null context");
    if (!distinct || !table_keys) {
        c->pred_distinct.clear();
        c->pred_table.clear();
        return KC_OK;
    }
    for (int i = 0; i < KC_MODEL_BUCKETS; ++i)
        if (!(distinct[i] >= 0.0) || !(table_keys[i] >= 0.0) || !std::isfinite(distinct[i]) ||
            !std::isfinite(table_keys[i]))
            return fail(KC_ERR_INVALID, "predicted loads must be finite and non-negative");
    c->pred_distinct.assign(distinct, distinct + KC_MODEL_BUCKETS);
    c->pred_table.assign(table_keys, table_keys + KC_MODEL_BUCKETS);
    return KC_OK;
}

extern "C" int kc_bucket_loads(kc_context* c, uint64_t* distinct, uint64_t* table_keys, uint64_t* kmers) {
    if (!c) return fail(KC_ERR_INVALID, "null context");
    if (!c->have_result) return fail(KC_ERR_STATE, "no result: run a count first");
    if (c->batch_result) return fail(KC_ERR_STATE, "not available for a multi-set result");
    if (c->stream_low) return fail(KC_ERR_STATE, "streamed results are not kept on the device");
    CK(c->loads.ensure(3 * KC_MODEL_BUCKETS * sizeof(unsigned long long)));
    unsigned long long* dd = c->loads.as<unsigned long long>();
    CK(cudaMemsetAsync(dd, 0, 3 * KC_MODEL_BUCKETS * sizeof(unsigned long long), c->stream));
    if (c->nw == 1) loads_kernels<1>(c, dd);
    else if (c->nw == 2) loads_kernels<2>(c, dd);
    else loads_kernels<4>(c, dd);
    CK(cudaGetLastError());
    std::vector<unsigned long long> h(3 * KC_MODEL_BUCKETS);
    CK(cudaMemcpyAsync(h.data(), dd, h.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (int i = 0; i < KC_MODEL_BUCKETS; ++i) {
        if (distinct) distinct[i] = h[i];
        if (table_keys) table_keys[i] = h[KC_MODEL_BUCKETS + i];
        if (kmers) kmers[i] = h[2 * KC_MODEL_BUCKETS + i];
    }
    return KC_OK;
}

int kc_internal_set_error(int code, const char* msg) { return fail(code, "%s", msg); }

namespace {
template <int NW>
int prefix_counts_impl(kc_context* c, const uint8_t* host, uint64_t n, uint64_t* counts) {
    const uint64_t tiles = ceil_div(n, kc::EXT_TILE);
    CK(c->stage.ensure(kc::HALO + n + kc::EXT_TILE));
    uint8_t* buf = c->stage.as<uint8_t>() + kc::HALO;
    CK(cudaMemcpyAsync(buf, host, n, cudaMemcpyHostToDevice, c->stream));
    CK(c->tile_nl.ensure(std::max<uint64_t>(tiles, 1) * sizeof(uint32_t)));
    CK(c->tile_line.ensure(std::max<uint64_t>(tiles, 1) * sizeof(uint64_t)));
    CK(c->scalars.ensure(64));
    CK(c->bucket_count.ensure(256 * sizeof(uint64_t)));
    CKR(fill_dev(c, c->scalars.as<uint32_t>() + 12, sizeof(uint32_t), 0));
    CKR(fill_dev(c, c->bucket_count.p, 256 * sizeof(uint64_t), 0));
    if (tiles) {
        kc::lines_per_tile<<<tiles, kc::EXT_THREADS, 0, c->stream>>>(buf, n, c->tile_nl.as<uint32_t>());
        CK(cudaGetLastError());
        int rc = device_scan<uint32_t, uint64_t>(c, c->tile_nl.as<uint32_t>(), tiles, c->tile_line.as<uint64_t>(), 0,
                                                 c->scalars.as<uint64_t>());
        if (rc) return rc;
        if ((rc = launch_extract<NW>(c, buf, n, 0, kc::HIST, 256, 1))) return rc;
    }
    CKR(get(c, counts, c->bucket_count.p, 256 * sizeof(uint64_t)));
    return sync_stream(c);
}
}  // namespace

// Canonical k-mers per root prefix (key word 0 >> 56) of FASTQ bytes in host
// memory, counted exactly on the context's device (every tile's histogram).
int kc_internal_prefix_counts(kc_context* c, const uint8_t* host, uint64_t n, uint64_t* counts) {
    if (!c || (!host && n) || !counts) return fail(KC_ERR_INVALID, "null argument");
    CK(cudaSetDevice(c->device));
    c->readbacks.clear();
    c->mbox_up_off = c->mbox_down_off = 0;
    return c->nw == 1 ? prefix_counts_impl<1>(c, host, n, counts)
                      : (c->nw == 2 ? prefix_counts_impl<2>(c, host, n, counts) : prefix_counts_impl<4>(c, host, n, counts));
}

uint64_t kc_internal_record_bytes(const kc_context* c) { return c ? c->record_bytes : 0; }
uint32_t kc_internal_k(const kc_context* c) { return c ? c->cfg.k : 0; }

// ------------------------------------------------------------------ batches
//
// Many independent read sets in one device buffer, counted in one pass: every
// pipeline stage is ONE launch over all sets.  Set s owns buckets
// [256 s, 256 s + 256) and a routed region aligned to a count segment (the gap
// holds EMPTY keys, which the count kernel skips), so segments, filter and
// tables never mix sets.  Host synchronisation happens only at the sizing
// points (after the histogram, after counting, after the low scan, after the
// export count) instead of per set; the scatter -> gap fill -> count sequence
// runs as one captured CUDA graph.

namespace {

// Per-set first-occurrence totals from the per-segment exclusive scan.  A set
// whose routed region is empty starts at segment index nsegs, one past the end
// of the scan, so that index reads the grand total instead.
__global__ void set_low_counts(const uint64_t* seg_prefix, const uint64_t* set_seg_start, uint32_t n_sets,
                               uint64_t nsegs, const uint64_t* total, uint64_t* out) {
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n_sets; s += gridDim.x * blockDim.x) {
        const uint64_t sa = set_seg_start[s];
        const uint64_t sb = (s + 1 < n_sets) ? set_seg_start[s + 1] : nsegs;
        const uint64_t a = sa < nsegs ? seg_prefix[sa] : *total;
        const uint64_t b = sb < nsegs ? seg_prefix[sb] : *total;
        out[s] = b - a;
    }
}

template <int NW>
int count_sets_impl(kc_context* c, const uint8_t* buf, const kc_set_desc* sets, uint32_t n_sets, kc_set_result* res) {
    constexpr int SEG = kc::count_seg<NW>();
    constexpr int CT = kc::count_tile<NW>();
    constexpr uint32_t NB = 256;
    const kc_config& g = c->cfg;
    const uint64_t nbk = (uint64_t)n_sets * NB;
    using KeyT = typename kc::KeyOf<NW>::T;

    // tiles
    std::vector<kc::SetTile> tiles;
    for (uint32_t s = 0; s < n_sets; ++s) {
        const uint32_t first = (uint32_t)tiles.size();
        for (uint64_t off = 0; off < sets[s].bytes; off += kc::EXT_TILE)
            tiles.push_back(kc::SetTile{sets[s].offset + off, sets[s].offset + sets[s].bytes, s, sets[s].k, first, 0});
    }
    const uint64_t nt = tiles.size();
    CK(c->set_tiles.ensure(std::max<uint64_t>(nt, 1) * sizeof(kc::SetTile)));
    CK(c->tile_nl.ensure(std::max<uint64_t>(nt, 1) * sizeof(uint32_t)));
    CK(c->tile_line.ensure(std::max<uint64_t>(nt, 1) * sizeof(uint64_t)));
    CK(c->tile_prefix.ensure(std::max<uint64_t>(nt, 1) * sizeof(uint64_t)));
    CK(c->scalars.ensure(64));
    uint64_t* d_scal = c->scalars.as<uint64_t>();
    CK(cudaMemsetAsync(c->scalars.as<uint32_t>() + 12, 0, sizeof(uint32_t), c->stream));
    if (nt) CK(cudaMemcpyAsync(c->set_tiles.p, tiles.data(), nt * sizeof(kc::SetTile), cudaMemcpyHostToDevice, c->stream));
    const kc::SetTile* d_tiles = c->set_tiles.as<kc::SetTile>();
    int rc;
    if (nt) {
        Stage st(c, KC_STAGE_LINES, 2);
        kc::lines_per_set_tile<<<nt, kc::EXT_THREADS, 0, c->stream>>>(buf, d_tiles, c->tile_nl.as<uint32_t>());
    }
    if ((rc = device_scan<uint32_t, uint64_t>(c, c->tile_nl.as<uint32_t>(), nt, c->tile_prefix.as<uint64_t>(), 0,
                                              d_scal + 0)))
        return rc;
    if (nt) kc::rebase_set_lines<<<std::min<uint64_t>(ceil_div(nt, 256), 1184), 256, 0, c->stream>>>(
        c->tile_prefix.as<uint64_t>(), d_tiles, nt, c->tile_line.as<uint64_t>());

    kc::ExtractArgs a{};
    a.tiles = d_tiles;
    a.buf = buf;
    a.tile_line = c->tile_line.as<uint64_t>();
    a.bucket_shift = 56;
    a.n_buckets = NB;
    CK(c->bucket_count.ensure(nbk * sizeof(uint64_t)));
    CK(c->bucket_cursor.ensure(nbk * sizeof(uint64_t)));
    a.bucket_count = c->bucket_count.as<unsigned long long>();
    a.bucket_cursor = c->bucket_cursor.as<unsigned long long>();
    a.error = c->scalars.as<uint32_t>() + 12;
    // Routing regions per (set, bucket).  A set of at least EST_MIN_TILES
    // tiles is histogrammed on every EST_STRIDE-th of its tiles: its regions
    // are estimates (x 1.02 + 4 standard deviations + 256 keys) followed by
    // an overflow area of its own (at least 65536 keys, so one CTA's run of a
    // bucket always fits), which a CTA's run that does not fit its region
    // takes whole.  A smaller set is histogrammed on every tile and gets exact
    // regions.  A pass whose overflow area filled is routed again, exactly.
    bool exact_only = false;
route_again:
    std::vector<uint8_t> sampled(n_sets, 0);
    std::vector<double> factor(n_sets, 1.0);
    std::vector<uint32_t> hist_list;
    bool any_sampled = false;
    {
        uint64_t t0 = 0;
        for (uint32_t s = 0; s < n_sets; ++s) {
            const uint64_t tn = ceil_div(sets[s].bytes, (uint64_t)kc::EXT_TILE);
            sampled[s] = !exact_only && tn >= kc::EST_MIN_TILES;
            uint64_t listed = 0;
            for (uint64_t q = 0; q < tn; ++q)
                if (!sampled[s] || q % kc::EST_STRIDE == 0) {
                    hist_list.push_back((uint32_t)(t0 + q));
                    ++listed;
                }
            if (sampled[s]) {
                factor[s] = (double)tn / (double)listed;
                any_sampled = true;
            }
            t0 += tn;
        }
    }
    CK(cudaMemsetAsync(c->bucket_count.p, 0, nbk * sizeof(uint64_t), c->stream));
    if (nt) {
        if (any_sampled) {
            CK(c->hist_tiles.ensure(hist_list.size() * sizeof(uint32_t)));
            CK(cudaMemcpyAsync(c->hist_tiles.p, hist_list.data(), hist_list.size() * sizeof(uint32_t),
                               cudaMemcpyHostToDevice, c->stream));
            a.tile_list = c->hist_tiles.as<uint32_t>();
        }
        Stage st(c, KC_STAGE_EXTRACT_HIST);
        kc::extract_kernel<NW, kc::HIST><<<any_sampled ? hist_list.size() : nt, kc::EXT_THREADS,
                                           kc::extract_smem_bytes<NW, kc::HIST>(NB), c->stream>>>(a);
        a.tile_list = nullptr;
    }
    CK(cudaGetLastError());
    std::vector<uint64_t> cnt(nbk);
    CK(cudaMemcpyAsync(cnt.data(), c->bucket_count.p, nbk * sizeof(uint64_t), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));

    // layout: each set's routed region starts on a segment boundary
    std::vector<uint64_t> start(nbk), rend(nbk), set_key0(n_sets), set_key1(n_sets), set_next(n_sets), set_seg(n_sets);
    std::vector<uint64_t> ovf_start(n_sets), ovf_end(n_sets);
    uint64_t pos = 0;
    c->h_meta.assign(nbk, kc::BucketMeta{});
    uint64_t bw = 0, ts = 0, K = 0;
    // learned sizing (kc_set_predicted_set_rates) when predictions for these
    // n_sets sets were handed over: predicted rates x the bucket's exact
    // k-mer total, 12 filter bits per distinct key, table keys with 15%
    // headroom at the target load; else (and for a negative rate) the sampled
    // rule on the exact per-bucket k-mer totals
    const bool learned = g.sizing == KC_SIZING_LEARNED && c->set_pred_table.size() == nbk;
    for (uint32_t s = 0; s < n_sets; ++s) {
        pos = ceil_div(pos, SEG) * SEG;
        set_key0[s] = pos;
        set_seg[s] = pos / SEG;
        uint64_t set_cap = 0;
        for (uint32_t b = 0; b < NB; ++b) {
            // k-mers of the bucket (estimated for a sampled set) and its region
            const double e = (double)cnt[(uint64_t)s * NB + b] * factor[s];
            const uint64_t kb = sampled[s] ? (uint64_t)e : cnt[(uint64_t)s * NB + b];
            const uint64_t cap = sampled[s] ? (uint64_t)(e * 1.02 + 4.0 * std::sqrt(e) + 256.0) : kb;
            start[(uint64_t)s * NB + b] = pos;
            pos += cap;
            rend[(uint64_t)s * NB + b] = pos;
            set_cap += cap;
            K += kb;
            uint64_t words, slots;
            const uint64_t q = (uint64_t)s * NB + b;
            if (learned && c->set_pred_distinct[q] >= 0.0 && c->set_pred_table[q] >= 0.0) {
                const double d = std::min(c->set_pred_distinct[q], 1.0) * (double)kb;
                const double t = std::min(c->set_pred_table[q], 1.0) * (double)kb;
                words = pow2_at_least(std::max<uint64_t>((uint64_t)(d * 12.0 / 64.0), 64));
                slots = pow2_at_least(std::max<uint64_t>((uint64_t)(t * 1.15 / g.table_load), 64));
            } else {
                words = pow2_at_least(std::max<uint64_t>((uint64_t)(kb * g.bloom_bits / 64.0), 64));
                slots = pow2_at_least(std::max<uint64_t>((uint64_t)(kb * g.repeat_ratio / g.table_load), 64));
            }
            c->h_meta[(uint64_t)s * NB + b] = kc::BucketMeta{bw, words - 1, ts, slots - 1};
            bw += words;
            ts += slots;
        }
        ovf_start[s] = pos;
        if (sampled[s]) pos += std::max<uint64_t>(1ull << 16, set_cap / 32);
        ovf_end[s] = pos;
        set_key1[s] = pos;
    }
    const uint64_t n_keys = ceil_div(pos, SEG) * SEG;
    for (uint32_t s = 0; s < n_sets; ++s) set_next[s] = (s + 1 < n_sets) ? set_key0[s + 1] : n_keys;
    c->K = K;
    c->bloom_words = bw;
    c->table_slots_used = ts;
    CK(c->bloom.ensure(bw * sizeof(uint64_t)));
    CK(c->table.ensure(ts * c->slot_bytes + ts * c->slot_bytes / 4));  // room for a few in-place growths
    CK(c->meta.ensure(nbk * sizeof(kc::BucketMeta)));
    CK(c->overflow.ensure(nbk * sizeof(uint32_t)));
    const uint64_t nsegs = n_keys / SEG;
    CK(c->routed.ensure(std::max<uint64_t>(ceil_div(n_keys, CT) * CT, 1) * sizeof(KeyT)));
    CK(c->tile_low.ensure(std::max<uint64_t>(nsegs, 1) * sizeof(uint32_t)));
    CK(c->tile_fail.ensure(std::max<uint64_t>(nsegs, 1) * sizeof(uint32_t)));
    CK(c->tile_low_prefix.ensure(std::max<uint64_t>(nsegs, 1) * sizeof(uint64_t)));
    CK(c->set_info.ensure((size_t)n_sets * 9 * sizeof(uint64_t) + 64));
    uint64_t* d_seg = c->set_info.as<uint64_t>();              // set_seg_start[n_sets]
    uint64_t* d_end = d_seg + n_sets;                          // set_key1
    uint64_t* d_next = d_end + n_sets;                         // next set's first key
    uint64_t* d_low = d_next + n_sets;                         // low count per set
    uint64_t* d_lowbase = d_low + n_sets;                      // low byte base per set
    uint64_t* d_ovs = d_lowbase + n_sets;                      // overflow area per set: start,
    uint64_t* d_ove = d_ovs + n_sets;                          //   end,
    uint64_t* d_ovc = d_ove + n_sets;                          //   cursor (end of the set's keys after the scatter)
    uint32_t* d_k = reinterpret_cast<uint32_t*>(d_ovc + n_sets);
    std::vector<uint32_t> ks(n_sets);
    for (uint32_t s = 0; s < n_sets; ++s) ks[s] = sets[s].k;
    CK(cudaMemcpyAsync(d_seg, set_seg.data(), n_sets * sizeof(uint64_t), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(d_end, set_key1.data(), n_sets * sizeof(uint64_t), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(d_next, set_next.data(), n_sets * sizeof(uint64_t), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(d_k, ks.data(), n_sets * sizeof(uint32_t), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->meta.p, c->h_meta.data(), nbk * sizeof(kc::BucketMeta), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->bucket_cursor.p, start.data(), nbk * sizeof(uint64_t), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(d_ovs, ovf_start.data(), n_sets * sizeof(uint64_t), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(d_ove, ovf_end.data(), n_sets * sizeof(uint64_t), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(d_ovc, ovf_start.data(), n_sets * sizeof(uint64_t), cudaMemcpyHostToDevice, c->stream));
    if (any_sampled) {
        CK(c->region_end.ensure(nbk * sizeof(uint64_t)));
        CK(c->region_fill.ensure(nbk * sizeof(uint64_t)));
        CK(cudaMemcpyAsync(c->region_end.p, rend.data(), nbk * sizeof(uint64_t), cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemsetAsync(c->region_fill.p, 0xFF, nbk * sizeof(uint64_t), c->stream));
        a.region_end = c->region_end.as<unsigned long long>();
        a.region_fill = c->region_fill.as<unsigned long long>();
        a.set_ovf_start = d_ovs;
        a.set_ovf_end = d_ove;
        a.set_ovf_cursor = reinterpret_cast<unsigned long long*>(d_ovc);
    } else {
        a.region_end = nullptr;
        a.region_fill = nullptr;
        a.set_ovf_start = a.set_ovf_end = nullptr;
        a.set_ovf_cursor = nullptr;
    }
    {
        Stage st(c, KC_STAGE_INIT, 1);
        CK(cudaMemsetAsync(c->bloom.p, 0, bw * sizeof(uint64_t), c->stream));
        kc::init_slots<NW><<<c->sm_count * 8, 256, 0, c->stream>>>(c->table.p, ts);
        CK(cudaMemsetAsync(c->overflow.p, 0, nbk * sizeof(uint32_t), c->stream));
    }
    CK(cudaGetLastError());

    kc::CountArgs ca{};
    ca.routed = c->routed.p;
    ca.n_keys = n_keys;
    ca.meta = c->meta.as<kc::BucketMeta>();
    ca.bloom = c->bloom.as<uint64_t>();
    ca.table = c->table.p;
    ca.seg_low = c->tile_low.as<uint32_t>();
    ca.seg_fail = c->tile_fail.as<uint32_t>();
    ca.bucket_overflow = c->overflow.as<uint32_t>();
    ca.bucket_shift = 56;
    ca.n_buckets = (uint32_t)std::min<uint64_t>(nbk, 0xFFFFFFFFu);
    ca.set_seg_start = d_seg;
    ca.n_sets = n_sets;
    ca.set_buckets = NB;
    ca.use_filter = 1;
    const uint64_t cgrid = ceil_div(n_keys, (uint64_t)CT * kc::CNT_SEGS_PER_WARP);

    // scatter -> gap fill(s) -> count as one graph.  The context keeps the
    // instantiated graph of each shape: a later call captures its own
    // launches (the same kernels, new arguments and grids) and updates the
    // instantiated graph of its shape in place (cudaGraphExecUpdate),
    // instantiating only when the update is refused; the replay is one launch
    // of the whole sequence.
    {
        Stage st(c, KC_STAGE_COUNT_ROUTED, 3);
        a.routed = c->routed.p;
        cudaGraph_t graph = nullptr;
        CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        if (nt)
            kc::extract_kernel<NW, kc::SCATTER>
                <<<nt, kc::EXT_THREADS, kc::extract_smem_bytes<NW, kc::SCATTER>(NB), c->stream>>>(a);
        if (any_sampled)  // EMPTY keys into the unfilled tails of the estimated regions
            kc::fill_region_gaps<NW><<<nbk, 256, 0, c->stream>>>(
                c->routed.p, c->bucket_cursor.as<unsigned long long>(), c->region_fill.as<unsigned long long>(),
                c->region_end.as<unsigned long long>(), (uint32_t)nbk);
        // and after each set's keys (its overflow area's unused part, the alignment gap)
        kc::fill_set_gaps<NW><<<n_sets, 256, 0, c->stream>>>(c->routed.p, d_ovc, d_next, n_sets);
        if (cgrid) kc::count_routed<NW><<<cgrid, kc::CNT_THREADS, 0, c->stream>>>(ca);
        const cudaError_t ce = cudaStreamEndCapture(c->stream, &graph);
        if (ce != cudaSuccess) return fail(KC_ERR_DEVICE, "graph capture failed: %s", cudaGetErrorString(ce));
        cudaError_t e = cudaSuccess;
        bool updated = false;
        const int nodes = (nt ? 1 : 0) + (any_sampled ? 1 : 0) + 1 + (cgrid ? 1 : 0);
        const int key = NW * 16 + nodes + (any_sampled ? 8 : 0);
        int slot = -1;
        for (int i = 0; i < kc_context::SETS_EXECS; ++i)
            if (c->sets_exec[i] && c->sets_exec_key[i] == key) slot = i;
        if (slot >= 0) {
            cudaGraphExecUpdateResultInfo info{};
            updated = cudaGraphExecUpdate(c->sets_exec[slot], graph, &info) == cudaSuccess;
            if (!updated) cudaGetLastError();
        } else {
            slot = c->sets_exec_next;
            c->sets_exec_next = (c->sets_exec_next + 1) % kc_context::SETS_EXECS;
        }
        cudaGraphExec_t& ex = c->sets_exec[slot];
        if (!updated) {
            if (ex) cudaGraphExecDestroy(ex);
            ex = nullptr;
            e = cudaGraphInstantiate(&ex, graph, 0);
            c->sets_exec_key[slot] = key;
            ++c->sets_instantiations;
        }
        if (e == cudaSuccess) e = cudaGraphLaunch(ex, c->stream);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
            if (ex) cudaGraphExecDestroy(ex);
            ex = nullptr;
            return fail(KC_ERR_DEVICE, "graph launch failed: %s", cudaGetErrorString(e));
        }
    }

    // exact k-mers per (set, bucket): a region's cursor advanced by every run
    // of its bucket, those sent to the overflow area included
    std::vector<uint64_t> exact(nbk);
    {
        uint32_t flags = 0;
        CK(cudaMemcpyAsync(exact.data(), c->bucket_cursor.p, nbk * sizeof(uint64_t), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaMemcpyAsync(&flags, c->scalars.as<uint32_t>() + 12, sizeof flags, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        if (flags & 2u) {  // an overflow area was full: route this pass again, exactly
            CK(cudaMemsetAsync(c->scalars.as<uint32_t>() + 12, 0, sizeof(uint32_t), c->stream));
            exact_only = true;
            ++c->reroutes;
            goto route_again;
        }
        K = 0;
        for (uint64_t q = 0; q < nbk; ++q) {
            exact[q] -= start[q];
            K += exact[q];
        }
        c->K = K;
    }

    // overflowed tables: grow x4, move, retry only the failed keys
    for (int round = 0;; ++round) {
        std::vector<uint32_t> ov(nbk);
        CK(cudaMemcpyAsync(ov.data(), c->overflow.p, nbk * sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        bool any = false;
        for (uint64_t b = 0; b < nbk; ++b) any |= ov[b] != 0;
        if (!any) break;
        if (round > 24) return fail(KC_ERR_OVERFLOW, "repeat tables kept overflowing");
        CK(cudaMemsetAsync(c->overflow.p, 0, nbk * sizeof(uint32_t), c->stream));
        std::vector<uint32_t> grow;
        for (uint64_t b = 0; b < nbk; ++b)
            if (ov[b]) grow.push_back((uint32_t)b);
        if ((rc = grow_buckets<NW>(c, grow))) return rc;
        CK(cudaMemcpyAsync(c->meta.p, c->h_meta.data(), nbk * sizeof(kc::BucketMeta), cudaMemcpyHostToDevice, c->stream));
        ca.table = c->table.p;
        ca.use_filter = 0;
        Stage st(c, KC_STAGE_REHASH);
        if (cgrid) kc::count_routed<NW><<<cgrid, kc::CNT_THREADS, 0, c->stream>>>(ca);
        CK(cudaGetLastError());
    }

    // first occurrences: per-set counts, byte bases, packing
    if ((rc = device_scan<uint32_t, uint64_t>(c, c->tile_low.as<uint32_t>(), nsegs, c->tile_low_prefix.as<uint64_t>(), 0,
                                              d_scal + 1)))
        return rc;
    set_low_counts<<<std::max<uint64_t>(1, ceil_div(n_sets, 256)), 256, 0, c->stream>>>(
        c->tile_low_prefix.as<uint64_t>(), d_seg, n_sets, nsegs, d_scal + 1, d_low);
    CK(cudaGetLastError());
    std::vector<uint64_t> lows(n_sets);
    CK(cudaMemcpyAsync(lows.data(), d_low, n_sets * sizeof(uint64_t), cudaMemcpyDeviceToHost, c->stream));
    uint32_t ext_err = 0;
    CK(cudaMemcpyAsync(&ext_err, c->scalars.as<uint32_t>() + 12, sizeof ext_err, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (ext_err) return fail(KC_ERR_DEVICE, "internal error: routing bucket disagreed with its reservation");
    std::vector<uint64_t> lowbase(n_sets);
    uint64_t lb = 0, total_low = 0;
    for (uint32_t s = 0; s < n_sets; ++s) {  // each set's low.bin bytes start 16-byte aligned
        total_low += lows[s];
        lb = (lb + 15) & ~15ull;
        lowbase[s] = lb;
        lb += lows[s] * kc_packed_bytes(sets[s].k);
    }
    CK(cudaMemcpyAsync(d_lowbase, lowbase.data(), n_sets * sizeof(uint64_t), cudaMemcpyHostToDevice, c->stream));
    CK(c->low_packed.ensure(lb + 64));
    if (nsegs) {
        Stage st(c, KC_STAGE_PACK_LOW);
        kc::pack_low_sets<NW><<<std::min<uint64_t>(ceil_div(nsegs, 8 * 32), (uint64_t)c->sm_count * 16), 256, 0,
                                c->stream>>>(
            c->routed.p, c->tile_low.as<uint32_t>(), c->tile_low_prefix.as<uint64_t>(), nsegs, d_seg, d_k, d_lowbase,
            n_sets, c->low_packed.as<uint8_t>());
    }
    CK(cudaGetLastError());

    // root records grouped by (set, root id)
    std::vector<kc::ExportChunk> ch;
    const uint32_t CH = 16384;
    for (uint64_t b = 0; b < nbk; ++b) {
        const uint64_t slots = c->h_meta[b].tab_mask + 1;
        for (uint64_t q = 0; q < slots; q += CH)
            ch.push_back(kc::ExportChunk{c->h_meta[b].tab_off + q, (uint32_t)std::min<uint64_t>(CH, slots - q), (uint32_t)b});
    }
    std::vector<uint64_t> rc_h;
    if ((rc = run_export<NW>(c, ch, nbk, rc_h))) return rc;
    std::vector<uint64_t> rstart(nbk);
    uint64_t R = 0;
    for (uint64_t b = 0; b < nbk; ++b) {
        rstart[b] = R;
        R += rc_h[b];
    }
    CK(cudaStreamSynchronize(c->stream));

    // per-set results; per-set table keys from the live table regions
    for (uint32_t s = 0; s < n_sets; ++s) {
        kc_set_result& r = res[s];
        std::memset(&r, 0, sizeof r);
        uint64_t km = 0;
        for (uint32_t b = 0; b < NB; ++b) {
            km += exact[(uint64_t)s * NB + b];
            r.root_counts[b] = rc_h[(uint64_t)s * NB + b];
            r.root_records += r.root_counts[b];
        }
        r.total_kmers = km;
        r.low_records = lows[s];
        r.low_offset = lowbase[s];
        r.low_bytes = lows[s] * kc_packed_bytes(sets[s].k);
        r.root_offset = rstart[(uint64_t)s * NB];
    }
    c->low_total = total_low;
    c->batch_low_bytes = lb;
    c->root_total = R;
    c->table_keys = rc_h[nbk];
    std::memset(c->root_counts, 0, sizeof c->root_counts);
    for (uint64_t b = 0; b < nbk; ++b) c->root_counts[b % NB] += rc_h[b];
    c->batch_result = true;
    c->have_result = true;
    return KC_OK;
}

}  // namespace

extern "C" int kc_count_sets(kc_context* c, const uint8_t* d_fastq, const kc_set_desc* sets, uint32_t n_sets,
                             kc_set_result* results, kc_stats* stats) {
    if (!c || !sets || !results || n_sets == 0 || (!d_fastq)) return fail(KC_ERR_INVALID, "null argument");
    if (c->n_buckets != 256) return fail(KC_ERR_INVALID, "read-set batches use 256 buckets per set");
    for (uint32_t s = 0; s < n_sets; ++s) {
        const uint32_t k = sets[s].k;
        const uint32_t nw = k <= 32 ? 1 : (k <= 64 ? 2 : 4);
        if (k < 1 || k > 128 || nw != c->nw)
            return fail(KC_ERR_INVALID, "set %u: k=%u must be in the key width of the context's k (%u)", s, k, c->cfg.k);
        if (sets[s].offset % 16) return fail(KC_ERR_INVALID, "set %u: offset must be 16-byte aligned", s);
    }
    const auto t0 = std::chrono::steady_clock::now();
    int rc = begin_run(c, 0);
    if (rc) return rc;
    c->stream_low = false;
    CK(cudaEventRecord(c->ev0, c->stream));
    uint64_t bytes = 0;
    for (uint32_t s = 0; s < n_sets; ++s) bytes += sets[s].bytes;
    c->input_bytes = bytes;
    c->batches = 1;
    rc = c->nw == 1 ? count_sets_impl<1>(c, d_fastq, sets, n_sets, results)
                    : (c->nw == 2 ? count_sets_impl<2>(c, d_fastq, sets, n_sets, results)
                                  : count_sets_impl<4>(c, d_fastq, sets, n_sets, results));
    if (rc) return rc;
    CK(cudaEventRecord(c->ev1, c->stream));
    CK(cudaEventSynchronize(c->ev1));
    collect_stage_times(c);
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    const double wall = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    fill_stats(c, stats, ms, wall);
    if (stats) stats->low_records = c->low_total;
    return KC_OK;
}

namespace {

// Per set, k-mers per model bucket (the top 12 bits of the canonical key) of
// bytes [offset, offset + bytes) of each set: the extraction's histogram pass
// over per-set tiles.
template <int NW>
int set_prefix_kmers_impl(kc_context* c, const uint8_t* buf, const kc_set_desc* sets, uint32_t n_sets, uint64_t* counts) {
    constexpr uint32_t NB = KC_MODEL_BUCKETS;
    std::vector<kc::SetTile> tiles;
    for (uint32_t s = 0; s < n_sets; ++s) {
        const uint32_t first = (uint32_t)tiles.size();
        for (uint64_t off = 0; off < sets[s].bytes; off += kc::EXT_TILE)
            tiles.push_back(kc::SetTile{sets[s].offset + off, sets[s].offset + sets[s].bytes, s, sets[s].k, first, 0});
    }
    const uint64_t nt = tiles.size(), nbk = (uint64_t)n_sets * NB;
    CK(c->set_tiles.ensure(std::max<uint64_t>(nt, 1) * sizeof(kc::SetTile)));
    CK(c->tile_nl.ensure(std::max<uint64_t>(nt, 1) * sizeof(uint32_t)));
    CK(c->tile_line.ensure(std::max<uint64_t>(nt, 1) * sizeof(uint64_t)));
    CK(c->tile_prefix.ensure(std::max<uint64_t>(nt, 1) * sizeof(uint64_t)));
    CK(c->scalars.ensure(64));
    CK(c->bucket_count.ensure(nbk * sizeof(uint64_t)));
    CK(cudaMemsetAsync(c->bucket_count.p, 0, nbk * sizeof(uint64_t), c->stream));
    CK(cudaMemsetAsync(c->scalars.as<uint32_t>() + 12, 0, sizeof(uint32_t), c->stream));
    if (nt) {
        CK(cudaMemcpyAsync(c->set_tiles.p, tiles.data(), nt * sizeof(kc::SetTile), cudaMemcpyHostToDevice, c->stream));
        const kc::SetTile* d_tiles = c->set_tiles.as<kc::SetTile>();
        kc::lines_per_set_tile<<<nt, kc::EXT_THREADS, 0, c->stream>>>(buf, d_tiles, c->tile_nl.as<uint32_t>());
        int rc;
        if ((rc = device_scan<uint32_t, uint64_t>(c, c->tile_nl.as<uint32_t>(), nt, c->tile_prefix.as<uint64_t>(), 0,
                                                  c->scalars.as<uint64_t>())))
            return rc;
        kc::rebase_set_lines<<<std::min<uint64_t>(ceil_div(nt, 256), 1184), 256, 0, c->stream>>>(
            c->tile_prefix.as<uint64_t>(), d_tiles, nt, c->tile_line.as<uint64_t>());
        kc::ExtractArgs a{};
        a.tiles = d_tiles;
        a.buf = buf;
        a.tile_line = c->tile_line.as<uint64_t>();
        a.bucket_shift = 64 - 12;
        a.n_buckets = NB;
        a.bucket_count = c->bucket_count.as<unsigned long long>();
        a.error = c->scalars.as<uint32_t>() + 12;
        kc::extract_kernel<NW, kc::HIST><<<nt, kc::EXT_THREADS, kc::extract_smem_bytes<NW, kc::HIST>(NB), c->stream>>>(a);
        CK(cudaGetLastError());
    }
    CK(cudaMemcpyAsync(counts, c->bucket_count.p, nbk * sizeof(uint64_t), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return KC_OK;
}

}  // namespace

extern "C" int kc_set_prefix_kmers(kc_context* c, const uint8_t* d_fastq, const kc_set_desc* sets, uint32_t n_sets,
                                   uint64_t* counts) {
    if (!c || !sets || !counts || n_sets == 0 || !d_fastq) return fail(KC_ERR_INVALID, "null argument");
    for (uint32_t s = 0; s < n_sets; ++s) {
        const uint32_t k = sets[s].k;
        const uint32_t nw = k <= 32 ? 1 : (k <= 64 ? 2 : 4);
        if (k < 1 || k > 128 || nw != c->nw)
            return fail(KC_ERR_INVALID, "set %u: k=%u must be in the key width of the context's k (%u)", s, k, c->cfg.k);
        if (sets[s].offset % 16) return fail(KC_ERR_INVALID, "set %u: offset must be 16-byte aligned", s);
    }
    CK(cudaSetDevice(c->device));
    return c->nw == 1 ? set_prefix_kmers_impl<1>(c, d_fastq, sets, n_sets, counts)
                      : (c->nw == 2 ? set_prefix_kmers_impl<2>(c, d_fastq, sets, n_sets, counts)
                                    : set_prefix_kmers_impl<4>(c, d_fastq, sets, n_sets, counts));
}

extern "C" uint64_t kc_sets_graph_instantiations(const kc_context* c) { return c ? c->sets_instantiations : 0; }

extern "C" int kc_set_sizing_callback(kc_context* c, kc_sizing_fn fn, void* user) {
    if (!c) return fail(KC_ERR_INVALID, "null context");
    c->sizing_cb = fn;
    c->sizing_user = fn ? user : nullptr;
    return KC_OK;
}

extern "C" int kc_set_predicted_set_rates(kc_context* c, uint32_t n_sets, const double* distinct,
                                          const double* table_keys) {
    if (!c) return fail(KC_ERR_INVALID, "null context");
    if (!distinct || !table_keys || n_sets == 0) {
        c->set_pred_distinct.clear();
        c->set_pred_table.clear();
        return KC_OK;
    }
    const uint64_t n = (uint64_t)n_sets * 256;
    c->set_pred_distinct.assign(distinct, distinct + n);
    c->set_pred_table.assign(table_keys, table_keys + n);
    return KC_OK;
}
