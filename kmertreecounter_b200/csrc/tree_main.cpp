// `Tree` -- command-line drop-in for the reference binary (src/main.cpp:314-596).
//
//   Tree <fastq_file> <k_len> <n_thread> <memory_limit_gb> [map_capacity] [min_count] [max_count]
//
// Same positional arguments, validation and exit codes as the reference:
//   * wrong argument count or unparsable numbers -> usage on stderr, exit 1
//   * n_thread < 6                                -> message, exit 255 (exit(-1))
//   * map_capacity <= 1 or >= 16 Mi, max < min   -> usage, exit 1
//   * k_len > 128                                 -> message, exit 1
// Outputs go to ./tmp/ relative to the working directory (src/definition.h:169),
// created when missing (the reference requires it to exist).  n_thread,
// memory_limit_gb and map_capacity describe the CPU pipeline and are accepted
// and ignored.  Stdout carries the two counters the reference prints:
// "Total read k-mer count: X" (src/main.cpp:266) and
// "High frequency unique k-mer : R" (src/main.cpp:309).
//
// Before counting it prints the reference's Stage-0 lines ("Thread split",
// "Average prefix count", "Classifier i total prefix count", "Max Bloom
// Filter capacity"), computed from the reference's own sample and rules.
// Extra environment knobs (not in the reference): KC_DEVICE, KC_BUCKETS,
// KC_SORT (0/1), KC_OUT_DIR, KC_STAGE0 (0: skip the Stage-0 report).

#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <limits>
#include <string>
#include <thread>

#include "../../include/kmer_count.h"

namespace {

void usage(const char* argv0) {
    std::cerr << "Usage: " << argv0
              << " <fastq_file> <k_len> <n_thread> <memory_limit_gb> [map_capacity] [min_count] [max_count]"
              << std::endl;
}

}  // namespace

int main(int argc, char* argv[]) {
    if (argc < 5 || argc > 8) {
        usage(argv[0]);
        return 1;
    }
    unsigned long k_len = 0, n_thread = 0, map_capacity = 1024;
    unsigned long long memory_limit = 0;
    unsigned long min_count = 1, max_count = std::numeric_limits<uint32_t>::max();
    std::string filename;
    try {
        filename = argv[1];
        k_len = std::stoul(argv[2]);
        n_thread = std::stoul(argv[3]);
        memory_limit = std::stoull(argv[4]);
        if (argc >= 6) map_capacity = std::stoul(argv[5]);
        if (argc >= 7) min_count = std::stoul(argv[6]);
        if (argc >= 8) max_count = std::stoul(argv[7]);
        if (n_thread < 6) {
            std::cerr << "n_thread must be >= 6" << std::endl;
            std::exit(-1);
        }
    } catch (const std::exception&) {
        usage(argv[0]);
        return 1;
    }
    (void)memory_limit;
    if (map_capacity <= 1 || map_capacity >= 16ull * 1024 * 1024 || max_count < min_count) {
        usage(argv[0]);
        return 1;
    }
    if (k_len == 0 || k_len > 128) {
        std::cerr << "k_len must be <= 128" << std::endl;
        return 1;
    }
    std::cout << "Input parameters:" << std::endl;
    std::cout << "  Fastq file: " << filename << std::endl;
    std::cout << "  k-mer length: " << k_len << std::endl;
    std::cout << "  Min count: " << min_count << std::endl;
    std::cout << "  Max count: " << max_count << std::endl;

    kc_config cfg;
    kc_config_default(&cfg);
    cfg.k = (uint32_t)k_len;
    cfg.min_count = (uint32_t)min_count;
    cfg.max_count = (uint32_t)max_count;
    if (const char* d = std::getenv("KC_DEVICE")) cfg.device = std::atoi(d);
    if (const char* b = std::getenv("KC_BUCKETS")) cfg.n_buckets = (uint32_t)std::atoi(b);
    if (const char* s = std::getenv("KC_SORT")) cfg.sort_output = (uint32_t)std::atoi(s);
    const char* out_dir = std::getenv("KC_OUT_DIR");

    // Stage 0 as the reference reports it (src/main.cpp:111-186): thread
    // split, then the sampled prefix counts' average, the classifier loads and
    // the largest filter.  Informational: the count below sizes its
    // structures from exact per-bucket totals, so the report is computed on a
    // second thread while the count runs and printed before the count's
    // lines.  KC_STAGE0=0 skips it.
    const char* s0 = std::getenv("KC_STAGE0");
    const bool stage0 = !s0 || std::string(s0) != "0";
    kc_stage0 s{};
    int src = KC_OK;
    std::string s0_err;
    std::thread s0_thread;
    if (stage0)
        s0_thread = std::thread([&] {
            src = kc_stage0_file(&cfg, filename.c_str(), (uint32_t)n_thread, &s);
            if (src != KC_OK) s0_err = kc_last_error();
        });

    kc_stats st;
    const int rc = kc_count_fastq(&cfg, filename.c_str(), out_dir ? out_dir : "./tmp/", &st);
    const std::string count_err = rc != KC_OK ? kc_last_error() : "";
    if (stage0) {
        s0_thread.join();
        const unsigned long parsers = n_thread / 8 > 0 ? n_thread / 8 : 1;
        const unsigned long budget = n_thread - 2 - parsers;
        const unsigned long classifiers = budget / 2 ? budget / 2 : 1;
        std::cout << "Thread split:" << std::endl;
        std::cout << "  parser threads: " << parsers << std::endl;
        std::cout << "  classifier threads: " << classifiers << std::endl;
        std::cout << "  task threads: " << budget - classifiers << std::endl;
        if (src != KC_OK) {
            std::cerr << s0_err << std::endl;
            return src == KC_ERR_INVALID ? 1 : 255;
        }
        std::cout << "Average prefix count: " << s.average_prefix_count << std::endl;
        for (uint32_t i = 0; i < s.classifier_num; ++i)
            std::cout << "Classifier " << s.load_order[i] << " total prefix count: "
                      << s.classifier_load[s.load_order[i]] << std::endl;
        std::cout << "Max Bloom Filter capacity: " << s.max_bloom_filter_capacity << std::endl;
    }
    if (rc != KC_OK) {
        std::cerr << count_err << std::endl;
        return rc == KC_ERR_INVALID ? 1 : 255;
    }
    std::cout << "Largest filter of this count (64-bit words): " << st.max_bucket_filter_words << std::endl;
    std::cout << "Largest repeat table of this count (slots): " << st.max_bucket_table_slots << std::endl;
    std::cout << "Total read k-mer count: " << st.total_kmers << std::endl;
    std::cout << "Low frequency k-mer (low.bin records): " << st.low_records << std::endl;
    std::cout << "Device elapsed ms: " << st.device_ms << std::endl;
    std::cout << "Total elapsed us: " << (uint64_t)(st.wall_ms * 1000.0) << std::endl;
    std::cout << "High frequency unique k-mer : " << st.root_records << std::endl;
    return 0;
}
