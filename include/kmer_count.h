/* kmer_count.h -- C ABI of the B200 exact canonical k-mer counter
 * (libkmertree_b200.so).
 *
 * Drop-in for the counting path of ScorchShana/KmerTreeCounter (tree_v4):
 * FASTQ bytes -> exact (canonical k-mer, count) records written in the
 * reference's own file formats, so tool/ExportReader.h,
 * tool/FinalDrainReader.h, tool/histogram_tool.cpp and tool/PostProcess.h
 * read the output unchanged:
 *
 *   <out_dir>/low.bin        headerless packed keys, one per first occurrence
 *                            (src/ExportWriter.h:339-342, :522-550)
 *   <out_dir>/root_{id}.bin  headerless ExportRecord<N> = {u64 key[N]; u32
 *                            count; u32 pad=0}, id = key word 0 >> 56, one
 *                            file per id 0..255, created even when empty
 *                            (src/definition.h:159-163,
 *                            src/FinalDrainWriter.h:31-90)
 *
 * Exact count of a key = its root record count + [key in low.bin], the
 * merged view tool/histogram_tool.cpp "precise" computes.
 *
 * All plain C types.  The library owns its device and pinned memory; caller
 * strings and buffers are borrowed for the duration of a call.  Every call is
 * synchronous at the API level and runs on one CUDA stream per context.  The
 * library never calls exit(); errors are negative return codes with a
 * message from kc_last_error() (thread-local).
 */
#ifndef KMER_COUNT_H
#define KMER_COUNT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define KC_OK 0
#define KC_ERR_INVALID (-1)  /* bad argument (reference: usage error, exit 1) */
#define KC_ERR_IO (-2)       /* open/read/write failure (reference: exit(-1)) */
#define KC_ERR_OVERFLOW (-3) /* count table could not be grown to fit */
#define KC_ERR_DEVICE (-4)   /* CUDA error, extension missing, no device */
#define KC_ERR_NOMEM (-5)    /* device or pinned allocation failed */
#define KC_ERR_STATE (-6)    /* call order: no result available yet */

/* ---- sizing modes -------------------------------------------------------- */
#define KC_SIZING_SAMPLED 0 /* per-bucket loads from the routing histogram and a
                               fixed repeat ratio; rehash on overflow */
#define KC_SIZING_LEARNED 1 /* per-bucket loads from a sizing model; the sampled
                               rule is the fallback on overflow */

/* Counting configuration.  Replaces the positional arguments of
 * `Tree <fastq> <k> <n_thread> <mem_gb> [map_capacity] [min] [max]`
 * (src/main.cpp:314-374); n_thread, mem_gb and map_capacity have no meaning on
 * the device and are accepted and ignored by the CLI. */
typedef struct kc_config {
    uint32_t k;            /* 1..128; key words N = 1 for k<=32, 2 for k<=64, 4 for k<=128.
                            * k = 96 differs from the reference on purpose: the
                            * reference leaves bases older than the window in key
                            * word 3 of F-oriented keys (its forward register is
                            * masked only in the last word, src/GetKmer.h:58-82),
                            * so one k-mer can get several root records; here word
                            * 3 is 0 and every k-mer has one key. */
    uint32_t canonical;    /* must be 1: the reference always counts canonical */
    uint32_t min_count;    /* root-record filter, inclusive (src/NewKmerTree.h:1159-1168) */
    uint32_t max_count;
    uint32_t n_buckets;    /* internal partitions: 256 or 4096 */
    uint32_t sizing;       /* KC_SIZING_* */
    int32_t device;        /* CUDA device ordinal */
    uint32_t sort_output;  /* 1: root records sorted by key inside each root file */
    uint64_t chunk_bytes;  /* host->device streaming chunk (default 256 MiB) */
    uint64_t batch_bytes;  /* FASTQ bytes counted per device pass (default 1 GiB) */
    double bloom_bits;     /* first-occurrence filter bits per k-mer occurrence */
    double table_load;     /* target load factor of the repeat tables */
    double repeat_ratio;   /* sampled sizing: distinct repeat keys per k-mer */
    uint64_t device_batch_bytes; /* FASTQ bytes per pass when the input is already in
                                  * device memory (kc_count_device; default 8 GiB, 0 =
                                  * batch_bytes).  Larger passes reuse each bucket's
                                  * filter and table lines more often in L2; the cost is
                                  * the routed-key buffer, about 3 bytes per FASTQ byte
                                  * for k <= 32 and 6 for k <= 64. */
    int32_t priority;      /* 1: the context's main stream at the device's highest
                            * priority, so its kernels are scheduled ahead of work
                            * already queued on other streams (a sizing prediction
                            * made beside another context's count); 0 = default */
} kc_config;

/* Counters of one run.  total_kmers and root_records match the reference's
 * "Total read k-mer count" and "High frequency unique k-mer" lines
 * (src/main.cpp:266, :309). */
typedef struct kc_stats {
    uint64_t input_bytes;
    uint64_t total_kmers;     /* K: valid windows */
    uint64_t low_records;     /* L: keys written to low.bin */
    uint64_t root_records;    /* R: records written to root files (after filter) */
    uint64_t table_keys;      /* distinct keys held by the repeat tables */
    uint64_t rehashes;        /* table growth steps taken after an overflow */
    uint64_t batches;         /* device passes */
    uint64_t root_counts[256];/* records per root file */
    double device_ms;         /* time spent in kernels and copies on the stream */
    double wall_ms;
    uint64_t table_slots;     /* repeat-table slots in use at the end (after any growth) */
    uint64_t filter_words;    /* 64-bit words of the first-occurrence filter */
    uint64_t overflow_keys;   /* keys routed past their estimated bucket region */
    uint64_t reroutes;        /* batches routed again from an exact histogram */
    uint64_t max_bucket_filter_words;  /* largest per-bucket filter (the reference's "Max Bloom
                                        * Filter capacity", src/main.cpp:88-108, in 64-bit words) */
    uint64_t max_bucket_table_slots;   /* largest per-bucket repeat table */
} kc_stats;

typedef struct kc_context kc_context;

/* Defaults: k=31, canonical=1, min=1, max=UINT32_MAX, 256 buckets, sampled
 * sizing, device 0, unsorted roots, 256 MiB chunks, 1 GiB host batches,
 * 8 GiB device batches, 5 filter bits per k-mer, table load 0.7, repeat
 * ratio 0.125. */
void kc_config_default(kc_config* cfg);

/* Thread-local message for the last failing call on this thread. */
const char* kc_last_error(void);

/* Bytes of one packed low.bin record for k (src/ExportWriter.h:339-342). */
uint64_t kc_packed_bytes(uint32_t k);

/* sizeof(ExportRecord<N>) for k: 16, 24 (src/definition.h:159-163). */
uint64_t kc_record_bytes(uint32_t k);

/* ---- one-shot file API --------------------------------------------------- */

/* Count the FASTQ (plain or gzip, detected by magic bytes as
 * src/FastqReader.h:93-104 does) at fastq_path and write low.bin and
 * root_0..255.bin into out_dir (created if missing).
 * Replaces process_main<N> (src/main.cpp:111-312). */
int kc_count_fastq(const kc_config* cfg, const char* fastq_path, const char* out_dir, kc_stats* stats);

/* ---- context API ------------------------------------------------------- */

int kc_create(const kc_config* cfg, kc_context** out);
void kc_destroy(kc_context* ctx);

/* Count a FASTQ byte stream held in host memory (pinned or pageable); the
 * bytes are streamed to the device in chunk_bytes pieces.  Results stay on
 * the device until copied out or written. */
int kc_count_host(kc_context* ctx, const uint8_t* fastq, uint64_t n, kc_stats* stats);

/* Streaming form of kc_count_host for large inputs: results are handed to
 * `sink` as they reach host memory, so device->host copies overlap the
 * counting of later batches.  The sink runs on a delivery thread the library
 * starts for the call and joins before returning (one call at a time, in
 * the order below); it must not call back into this context.
 *   kind KC_SINK_LOW   packed low.bin bytes, in file order (first
 *                      occurrences of a batch are final when emitted)
 *   kind KC_SINK_ROOT  ExportRecord<N> bytes of root file `root`, roots in
 *                      order 0..255; an empty root is one call with bytes 0
 * `data` is page-locked library memory valid only during the call.  A
 * non-zero return from the sink stops the count with KC_ERR_IO. */
#define KC_SINK_LOW 0
#define KC_SINK_ROOT 1
typedef int (*kc_sink_fn)(void* user, int kind, uint32_t root, const uint8_t* data, uint64_t bytes);
int kc_count_host_stream(kc_context* ctx, const uint8_t* fastq, uint64_t n, kc_sink_fn sink, void* user,
                         kc_stats* stats);

/* Same, with the FASTQ already in device memory (a device pointer). */
int kc_count_device(kc_context* ctx, const uint8_t* d_fastq, uint64_t n, kc_stats* stats);

/* ---- one input over several GPUs (bucket owners) ------------------------
 * The reference partitions its Bloom filters and trees by root prefix
 * (key word 0 >> 56; src/FastqClassifier.h:211-240, src/main.cpp:38-86).
 * Sharded, every GPU extracts and routes its slice of the FASTQ records, the
 * slices' keys are exchanged so that each GPU receives the keys of a
 * contiguous range of root prefixes (one all-to-all), and each GPU counts
 * them: its root files are the root files of its prefixes, and the low.bin
 * bytes of all GPUs concatenated are the input's low.bin.
 *
 * kc_route_device: extract and route whole 4-line records (the slice must
 * start at a record) in device memory; the keys stay in the context, in
 * root-prefix order, counts[256] receiving the keys per prefix (so prefix p's
 * keys are at index sum(counts[0..p)) ).  The slice is routed in one pass
 * (device_batch_bytes does not split it): its keys take 8N bytes per k-mer,
 * about 2.5N times the slice's FASTQ bytes for 150 bp reads.
 * kc_copy_routed: copy those keys (8N bytes each) to dst (device or host),
 * dst_bytes >= 8N x sum(counts).
 * kc_count_keys_device: count n_keys canonical keys in device memory (8N
 * bytes each, as routed, any order) as one input; counts[256] are the keys
 * per root prefix (they size the filter and tables, and must sum to
 * n_keys).  Results as after kc_count_device. */
int kc_route_device(kc_context* ctx, const uint8_t* d_fastq, uint64_t n, uint64_t* counts);
int kc_copy_routed(kc_context* ctx, void* dst, uint64_t dst_bytes);
/* kc_routed_keys: the routed keys where they are (device pointer into the
 * context, 8N bytes per key, sum(counts) keys), e.g. as the send buffer of
 * the exchange, without a copy.  Valid until the next call on the context;
 * the caller must let its reads finish before that call (a later count on
 * the context overwrites them). */
int kc_routed_keys(kc_context* ctx, const void** d_keys, uint64_t* n_keys);
int kc_count_keys_device(kc_context* ctx, const void* d_keys, uint64_t n_keys, const uint64_t* counts,
                         kc_stats* stats);

/* ---- many read sets in one pass ----------------------------------------
 * Benchmark pattern "batched uneven samples": independent read sets of uneven
 * size and read length counted together -- every pipeline stage is one launch
 * over all sets, with host synchronisation only at the sizing points.  Set s
 * is bytes [offset, offset + bytes) of one device buffer (offset 16-byte
 * aligned) counted with its own k (all sets in the key width of the
 * context's k: all <= 32 or all 33..64) into its own filter, tables, low.bin
 * range and 256 root files.  No counterpart in the reference, which counts one
 * file per process. */
typedef struct kc_set_desc {
    uint64_t offset;
    uint64_t bytes;
    uint32_t k;
    uint32_t reserved;
} kc_set_desc;

typedef struct kc_set_result {
    uint64_t total_kmers;
    uint64_t low_records;
    uint64_t low_offset;      /* byte offset of this set's low.bin in kc_copy_low's buffer */
    uint64_t low_bytes;
    uint64_t root_records;
    uint64_t root_offset;     /* record offset of this set's root files in kc_copy_roots's buffer */
    uint64_t root_counts[256];/* records per root file, files in order 0..255 */
} kc_set_result;

int kc_count_sets(kc_context* ctx, const uint8_t* d_fastq, const kc_set_desc* sets, uint32_t n_sets,
                  kc_set_result* results, kc_stats* stats);
/* Graph instantiations kc_count_sets has made on this context (a diagnostic:
 * later calls with a shape seen before update and replay its graph). */
uint64_t kc_sets_graph_instantiations(const kc_context* ctx);

/* Sizes of the last result: packed low.bin bytes, number of root records,
 * and per-root record counts (256 entries, may be NULL). */
int kc_result_sizes(kc_context* ctx, uint64_t* low_bytes, uint64_t* n_root_records, uint64_t* root_counts);

/* Copy the packed low.bin bytes into dst (cap bytes; host or device memory). */
int kc_copy_low(kc_context* ctx, uint8_t* dst, uint64_t cap);

/* Copy all root records (ExportRecord<N>, grouped by root id 0..255 in
 * order) into dst (cap bytes; host or device memory). */
int kc_copy_roots(kc_context* ctx, uint8_t* dst, uint64_t cap);

/* Merged count histogram of the last device-held result (kc_count_host or
 * kc_count_device): hist[i] = number of distinct keys whose exact count
 * (root count + [key in low.bin]) equals min_freq + i, for i in
 * 0..max_freq-min_freq; *distinct = number of distinct keys.  The device form
 * of tool/histogram_tool.cpp "precise" (tool/HighFrequencyInsertThreadPool.h:
 * 150-177, tool/LowFrequencyQueryThreadPool.h:375-432). */
int kc_histogram(kc_context* ctx, uint32_t min_freq, uint32_t max_freq, uint64_t* hist, uint64_t* distinct);

/* Write low.bin and root_0..255.bin of the last result into out_dir. */
int kc_write_outputs(kc_context* ctx, const char* out_dir);

/* Device pointers to the last result (valid until the next count or
 * kc_destroy): packed low bytes and the grouped root-record array. */
int kc_device_results(kc_context* ctx, const void** d_low, uint64_t* low_bytes, const void** d_roots,
                      uint64_t* n_roots);

/* Page-locked host memory for callers that stream input (cudaHostAlloc). */
void* kc_host_alloc(uint64_t bytes);
void kc_host_free(void* p);

/* CUDA stream of the context (as void*), for callers that time it. */
void* kc_stream(kc_context* ctx);

/* ---- post-processing (tool/PostProcess.h) -------------------------------
 * The reference's PostProcess::merge_all (tool/PostProcess.h:63-139) turns a
 * count's low.bin and root files into
 *   final_root.bin  all root records, root files 0..255 in order, unchanged
 *   final_low.bin   the low.bin keys that are no root file's key, sorted
 *                   (lexicographic over the key words) and unique, each as
 *                   its N raw little-endian 64-bit words (kmer<N>)
 *   freq_hist.txt   "count\tnum_kmers" then "c\tn" lines in ascending c:
 *                   each root record counts at its count + 1, each
 *                   final_low.bin key at 1; not written when both are empty.
 * The reference reads low.bin as raw kmer<N> records, which matches its
 * packed layout only when that is 8N bytes (k = 29..32, 61..64, 93..96,
 * 125..128); here low.bin is unpacked with k, so every k is handled. */
typedef struct kc_post_stats {
    uint64_t root_records;  /* records in final_root.bin */
    uint64_t low_in;        /* keys read from low.bin */
    uint64_t low_in_roots;  /* of those, keys that are also root keys (left out) */
    uint64_t final_low;     /* keys in final_low.bin */
    uint64_t hist_lines;    /* count lines in freq_hist.txt (0: not written) */
} kc_post_stats;

/* From the last single-input result held on the device (after kc_count_host,
 * kc_count_device or kc_count_keys_device); files go to out_dir (created if
 * missing).  The sorting and filtering run on the context's device. */
int kc_post_process(kc_context* ctx, const char* out_dir, kc_post_stats* stats);

/* From low.bin and root_0..255.bin in temp_dir (as Tree writes them; missing
 * root files count as empty), counted with cfg->k, on cfg->device. */
int kc_post_process_dir(const kc_config* cfg, const char* temp_dir, const char* out_dir, kc_post_stats* stats);

/* ---- Stage-0 figures of the reference -----------------------------------
 * Before counting, the reference samples at most 256 MB of the FASTQ (three
 * thirds of that from the start, middle and end of a plain file; the head of
 * a gzip file; src/FastqPreReader.h:110-330), counts the sample's canonical
 * k-mers per root prefix (key word 0 >> 56), raises counts below 1000 to
 * 1000, assigns prefixes to its classifier threads by the longest-processing-
 * time rule (src/main.cpp:38-86) and sizes one Bloom filter per prefix
 * (src/main.cpp:88-108).  This build sizes from exact per-bucket totals or a
 * learned model; these entry points compute the reference's figures for
 * side-by-side diagnostics (bin/Tree prints them as the reference does). */
typedef struct kc_stage0 {
    uint64_t estimated_file_size;        /* raw FASTQ bytes assumed: file size, 4x for gzip */
    uint64_t sample_bytes;               /* FASTQ bytes the sampler parsed */
    uint64_t sampled_kmers;              /* canonical k-mers in the sample (before raising) */
    uint64_t average_prefix_count;       /* "Average prefix count" */
    uint64_t max_bloom_filter_capacity;  /* "Max Bloom Filter capacity", 64-bit words */
    uint32_t classifier_num;             /* classifier threads for n_thread (src/main.cpp:114-117) */
    uint32_t reserved;
    uint64_t prefix_count[256];          /* sampled k-mers per root prefix, raised to >= 1000 */
    uint64_t bloom_filter_capacity[256]; /* filter words per root prefix */
    uint32_t prefix_owner[256];          /* classifier of each root prefix */
    uint32_t load_order[256];            /* classifiers in the order the reference prints their loads */
    uint64_t classifier_load[256];       /* total prefix count per classifier */
} kc_stage0;

/* The rules alone, from per-prefix sampled counts (256 entries), the raw
 * FASTQ size and the thread count (6 or more, as the reference requires).
 * Needs no device. */
int kc_stage0_rule(const uint64_t* prefix_counts, uint64_t estimated_file_size, uint32_t n_thread, kc_stage0* out);

/* Sample the FASTQ at fastq_path as the reference does, count the sample's
 * k-mers (cfg->k) per root prefix on cfg->device, and apply the rules. */
int kc_stage0_file(const kc_config* cfg, const char* fastq_path, uint32_t n_thread, kc_stage0* out);

/* ---- diagnostics ----------------------------------------------------------
 * The reference prints per-stage timers and, with TEST_MODE, cycle counters
 * (src/main.cpp:270-309, src/definition.h:4).  Here: with profiling on, every
 * stage of a count is bracketed by CUDA events on the context's stream. */
#define KC_STAGE_LINES 0
#define KC_STAGE_SCAN 1
#define KC_STAGE_EXTRACT_HIST 2
#define KC_STAGE_EXTRACT_SCATTER 3
#define KC_STAGE_COUNT_ROUTED 4
#define KC_STAGE_REHASH 5
#define KC_STAGE_PACK_LOW 6
#define KC_STAGE_EXPORT 7
#define KC_STAGE_SORT 8
#define KC_STAGE_INIT 9
#define KC_STAGE_SUBROUTE 10 /* 64-bit keys: grouping a batch's keys by table window */
#define KC_STAGE_COUNT 11

int kc_set_profiling(kc_context* ctx, int enable);

/* Device milliseconds and kernel launches per stage of the last count
 * (arrays of `cap` entries; either may be NULL).  Returns KC_STAGE_COUNT. */
int kc_stage_times(kc_context* ctx, double* ms, uint64_t* launches, int cap);

const char* kc_stage_name(int stage);

/* ---- allocation-free entry point ------------------------------------------
 * No counterpart in the reference.  For callers that must not allocate device
 * memory on this path: a framework whose caching allocator owns the device
 * budget and forbids raw cudaMalloc, or a latency-sensitive thread that cannot
 * afford cudaMalloc/cudaFree (cudaFree synchronises the device).
 *
 * Counts a FASTQ already in device memory (16-byte aligned, at most
 * KC_NOALLOC_MAX_FASTQ_BYTES, 256 buckets, k 1..64, canonical only) on
 * `stream` (a cudaStream_t, NULL = default stream) and writes the packed
 * low.bin bytes to d_low and the root records, grouped by root id, to d_roots
 * (16-byte aligned device buffers with the given byte capacities); stats receives the
 * counters.  All scratch comes from one static device array of
 * KC_NOALLOC_SCRATCH_BYTES per GPU, held until exit.  With CUDA's lazy module
 * loading (the default since CUDA 12.2) that array is reserved when the first
 * call on a device looks up its address, not when the library is loaded: make
 * that first call before the caller's allocator claims the device budget (or
 * run with CUDA_MODULE_LOADING=EAGER), and before any stream capture.  Calls
 * share the array: overlapping calls on the GPU race and must be serialised
 * by the caller.  Larger inputs, other k or bucket counts, unaligned buffers
 * and output buffers too small for the result are rejected with
 * KC_ERR_INVALID; a table that outgrows the array ends the call with
 * KC_ERR_OVERFLOW. */
#define KC_NOALLOC_SCRATCH_BYTES (64ull << 20)
#define KC_NOALLOC_MAX_FASTQ_BYTES (1ull << 20)

int kc_count_device_noalloc(const kc_config* cfg, const uint8_t* d_fastq, uint64_t n, uint8_t* d_low,
                            uint64_t low_cap, uint8_t* d_roots, uint64_t roots_cap, void* stream, kc_stats* stats);

#ifdef __cplusplus
}
#endif

#endif /* KMER_COUNT_H */
