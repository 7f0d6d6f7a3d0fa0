// Stage-0 figures of the reference: its sample of the FASTQ, the per-prefix
// k-mer counts of that sample, and the sizing rules it derives from them.
//
// The reference reads at most 256 MB before counting (FastqPreReader::pre_read,
// src/FastqPreReader.h:110-330): for a plain file, three reads of a third of
// that each -- from the start, from the middle and from the end of the file,
// the last two moved forward to the next "\n@" (find_next_record_start) -- and
// for a gzip file the first 256 MB-or-file-size of decompressed bytes.  Its
// line state machine is reset to the header state when the read that ends a
// segment arrives, i.e. before the head and the middle read are parsed, not
// before the tail read, which continues the state where the middle read left
// it; a sequence line cut by a reset continues with the next sequence line
// (no line break is inserted).  The sequence lines it collects are counted
// per root prefix (key word 0 >> 56) of their canonical k-mers
// (FastqPrefixCounter::count_prefixes), and
//   * every count below 1000 is raised to 1000; "Average prefix count" is the
//     mean (src/main.cpp:174-186);
//   * prefixes go to classifier threads by the longest-processing-time rule
//     (src/main.cpp:38-86), classifier_num from n_thread as
//     src/main.cpp:114-117;
//   * each prefix's Bloom filter gets max(bit_ceil(file/3 x share x 4.81 / 64),
//     2^15) words (src/main.cpp:88-108).
// Here the sampled lines are counted on the device by the extraction kernel,
// after being laid out as a FASTQ of their own (one record per collected
// line), and the rules are applied on the host with the same arithmetic.
//
// This build does not size anything from these figures (it uses exact
// per-bucket totals, or a learned model); they are reported for comparison.

#include <algorithm>
#include <bit>
#include <cerrno>
#include <cstdio>
#include <cstring>
#include <queue>
#include <string>
#include <vector>

#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>
#include <zlib.h>

#include "../../include/kmer_count.h"
#include "kc_internal.h"

namespace {

constexpr uint64_t kSampleLimit = 256ull * 1024 * 1024;
constexpr uint64_t kChunk = 2ull * 1024 * 1024;     // FASTQ_FILE_CHUNK_SIZE
constexpr uint64_t kMinCapacity = 1ull << 15;       // smallest filter, in 64-bit words
constexpr uint32_t kMinPrefixCount = 1000;

int s0_fail(int code, const std::string& m) { return kc_internal_set_error(code, m.c_str()); }

// Line state of the reference's reader: 0 header, 1 sequence, 2 plus, 3 quality.
struct SeqCollector {
    int state = 0;
    std::string lines;  // collected sequence bytes, '\n' between lines
    void reset() { state = 0; }
    void feed(const uint8_t* p, uint64_t n) {
        uint64_t pos = 0;
        while (pos < n) {
            const void* nl = std::memchr(p + pos, '\n', n - pos);
            const uint64_t end = nl ? (uint64_t)(static_cast<const uint8_t*>(nl) - p) : n;
            if (state == 1) lines.append(reinterpret_cast<const char*>(p + pos), end - pos);
            if (!nl) return;
            if (state == 1) lines.push_back('\n');
            state = (state + 1) & 3;
            pos = end + 1;
        }
    }
};

bool pread_all(int fd, uint8_t* dst, uint64_t n, uint64_t off, uint64_t* got) {
    *got = 0;
    while (*got < n) {
        const ssize_t r = ::pread(fd, dst + *got, n - *got, (off_t)(off + *got));
        if (r < 0 && errno == EINTR) continue;
        if (r < 0) return false;
        if (r == 0) break;
        *got += (uint64_t)r;
    }
    return true;
}

// find_next_record_start: the first "\n@" within 64 KiB after `start` (the
// position of the '@'), else `start`.
uint64_t next_record_start(int fd, uint64_t start) {
    std::vector<uint8_t> buf(65536);
    uint64_t n = 0;
    if (!pread_all(fd, buf.data(), buf.size(), start, &n) || n <= 1) return start;
    for (uint64_t i = 1; i < n; ++i)
        if (buf[i - 1] == '\n' && buf[i] == '@') return start + i;
    return start;
}

int sample_plain(int fd, uint64_t size, SeqCollector& col, uint64_t* sampled) {
    const uint64_t need = std::min(size, kSampleLimit);
    uint64_t part = need / 3;
    if (part == 0) part = 1;
    const uint64_t chunk = std::max(part, kChunk);
    const uint64_t offsets[3] = {0, size / 2 >= part / 2 ? size / 2 - part / 2 : 0, size >= part ? size - part : 0};
    std::vector<uint8_t> buf(chunk);
    uint64_t pos = 0, have = 0, seg_read = 0;
    int seg = 0;
    *sampled = 0;
    for (;;) {
        uint64_t n = 0;
        if (!pread_all(fd, buf.data(), chunk, pos, &n)) return s0_fail(KC_ERR_IO, "read failed while sampling");
        if (n == 0) break;
        pos += n;
        seg_read += n;
        have += n;
        if (seg_read >= part && seg < 2) {  // the read that ends a segment resets the state
            col.reset();
            ++seg;
            seg_read = 0;
            pos = next_record_start(fd, offsets[seg]);
        }
        col.feed(buf.data(), n);
        *sampled += n;
        if (have >= need) break;
    }
    return KC_OK;
}

int sample_gzip(const char* path, uint64_t compressed, SeqCollector& col, uint64_t* sampled) {
    gzFile gz = gzopen(path, "rb");
    if (!gz) return s0_fail(KC_ERR_IO, std::string("Failed to open gzip file: ") + path);
    const uint64_t need = std::min(compressed, kSampleLimit);
    std::vector<uint8_t> buf(kChunk);
    uint64_t have = 0;
    *sampled = 0;
    for (;;) {
        const int r = gzread(gz, buf.data(), (unsigned)buf.size());
        if (r < 0) {
            gzclose(gz);
            return s0_fail(KC_ERR_IO, "gzip error while sampling");
        }
        if (r == 0 || have >= need) break;  // the read that finds enough is not parsed
        col.feed(buf.data(), (uint64_t)r);
        have += (uint64_t)r;
        *sampled += (uint64_t)r;
    }
    gzclose(gz);
    return KC_OK;
}

}  // namespace

extern "C" {

int kc_stage0_rule(const uint64_t* prefix_counts, uint64_t estimated_file_size, uint32_t n_thread, kc_stage0* out) {
    if (!prefix_counts || !out) return s0_fail(KC_ERR_INVALID, "null argument");
    if (n_thread < 6) return s0_fail(KC_ERR_INVALID, "n_thread must be >= 6");
    std::memset(out, 0, sizeof *out);
    // thread split of process_main: parsers n/8 (at least 1), two fixed
    // threads, the rest halved between classifiers and tree workers
    const uint32_t parser = n_thread / 8 > 0 ? n_thread / 8 : 1u;
    const uint32_t budget = n_thread - 2 - parser;
    const uint32_t classifiers = std::max<uint32_t>(1u, (uint32_t)(budget / 2.0));
    if (classifiers > 256) return s0_fail(KC_ERR_INVALID, "n_thread too large for the Stage-0 report (256 classifiers at most)");
    out->classifier_num = classifiers;
    out->estimated_file_size = estimated_file_size;

    // counts as the reference stores them (32-bit), small ones raised
    uint32_t c32[256];
    uint64_t total = 0;
    for (int p = 0; p < 256; ++p) {
        c32[p] = (uint32_t)prefix_counts[p];
        out->sampled_kmers += prefix_counts[p];
        if (c32[p] < kMinPrefixCount) c32[p] = kMinPrefixCount;
        out->prefix_count[p] = c32[p];
        total += c32[p];
    }
    out->average_prefix_count = total / 256;

    // longest processing time first: prefixes by count, largest first, each
    // to the least-loaded classifier (ties resolved as the standard library's
    // sort and heap resolve them for the same input order)
    struct Pref {
        uint64_t prefix;
        uint32_t count;
    };
    Pref order[256];
    for (int p = 0; p < 256; ++p) order[p] = Pref{(uint64_t)p, c32[p]};
    std::sort(order, order + 256, [](const Pref& a, const Pref& b) { return a.count > b.count; });
    struct Load {
        uint32_t index;
        uint32_t count;
        bool operator<(const Load& o) const { return count > o.count; }
    };
    std::priority_queue<Load, std::vector<Load>> heap;
    for (uint32_t i = 0; i < classifiers; ++i) heap.push(Load{i, 0});
    for (int i = 0; i < 256; ++i) {
        Load w = heap.top();
        heap.pop();
        out->prefix_owner[order[i].prefix] = w.index;
        w.count += order[i].count;
        heap.push(w);
    }
    for (uint32_t i = 0; !heap.empty(); ++i) {
        out->load_order[i] = heap.top().index;
        out->classifier_load[heap.top().index] = heap.top().count;
        heap.pop();
    }

    // filter capacity per prefix, in 64-bit words
    const uint64_t est_kmers = estimated_file_size / 3;
    for (int p = 0; p < 256; ++p) {
        const double share = (double)c32[p] / (double)total;
        const uint64_t est = (uint64_t)((double)est_kmers * share * 4.81 / 64);
        out->bloom_filter_capacity[p] = std::max<uint64_t>(std::bit_ceil(est), kMinCapacity);
        out->max_bloom_filter_capacity = std::max(out->max_bloom_filter_capacity, out->bloom_filter_capacity[p]);
    }
    return KC_OK;
}

int kc_stage0_file(const kc_config* cfg, const char* fastq_path, uint32_t n_thread, kc_stage0* out) {
    if (!cfg || !fastq_path || !out) return s0_fail(KC_ERR_INVALID, "null argument");
    const int fd = ::open(fastq_path, O_RDONLY);
    if (fd < 0) return s0_fail(KC_ERR_IO, std::string("Failed to open file ") + fastq_path + ": " + std::strerror(errno));
    struct stat st;
    if (fstat(fd, &st) != 0) {
        ::close(fd);
        return s0_fail(KC_ERR_IO, std::string("Failed to get file size of ") + fastq_path);
    }
    const uint64_t size = (uint64_t)st.st_size;
    uint8_t magic[2] = {0, 0};
    uint64_t got = 0;
    pread_all(fd, magic, 2, 0, &got);
    const bool gz = got == 2 && magic[0] == 0x1F && magic[1] == 0x8B;
    SeqCollector col;
    uint64_t sampled = 0;
    int rc = gz ? sample_gzip(fastq_path, size, col, &sampled) : sample_plain(fd, size, col, &sampled);
    ::close(fd);
    if (rc) return rc;
    // the collected lines as a FASTQ of their own: "@\n<line>\n+\n\n" each
    std::string fq;
    fq.reserve(col.lines.size() + col.lines.size() / 8 + 16);
    uint64_t start = 0;
    while (start < col.lines.size()) {
        const size_t nl = col.lines.find('\n', start);
        const uint64_t end = nl == std::string::npos ? col.lines.size() : nl;
        fq += "@\n";
        fq.append(col.lines, start, end - start);
        fq += "\n+\n\n";
        start = end + 1;
    }
    uint64_t counts[256] = {};
    kc_context* ctx = nullptr;
    if ((rc = kc_create(cfg, &ctx))) return rc;
    rc = kc_internal_prefix_counts(ctx, reinterpret_cast<const uint8_t*>(fq.data()), fq.size(), counts);
    kc_destroy(ctx);
    if (rc) return rc;
    rc = kc_stage0_rule(counts, gz ? size * 4 : size, n_thread, out);
    if (!rc) out->sample_bytes = sampled;
    return rc;
}

}  // extern "C"
