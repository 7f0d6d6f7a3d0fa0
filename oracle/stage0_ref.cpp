// Test infrastructure only: runs the REFERENCE's own Stage-0 sizing rules on
// given per-prefix counts, so the library's restatement can be checked
// against them.  Linked with the reference's src/main.cpp (its `main` renamed
// by the build recipe, oracle/Makefile), whose lpt() (src/main.cpp:38-86) and
// calculate_bloom_filter_capacity() (src/main.cpp:88-108) are called here.
//
// stdin:  estimated_file_size n_thread count_0 .. count_255   (whitespace separated)
// stdout: the reference's own lines ("Classifier i total prefix count: c",
//         "Max Bloom Filter capacity: M"), preceded by "Average prefix count: A"
//         and the classifier count, followed by "owner p o" and
//         "capacity p c" for every prefix p.
//
// The raise of small counts to 1000, the average and the thread split are
// the few lines of process_main (src/main.cpp:114-117, :174-186) that sit
// around those two calls; they are restated here.
#include <atomic>
#include <cstdint>
#include <iostream>
#include <vector>

#include "definition.h"

void lpt(std::vector<std::atomic<uint32_t>>& prefix_counts, uint32_t classifier_num);
void calculate_bloom_filter_capacity(std::vector<std::atomic<uint32_t>>& prefix_counts, uint64_t estimated_file_size);

int main() {
    uint64_t est = 0, n_thread = 0;
    std::cin >> est >> n_thread;
    std::vector<std::atomic<uint32_t>> counts(256);
    for (auto& c : counts) {
        uint64_t v = 0;
        std::cin >> v;
        c.store((uint32_t)v);
    }
    if (!std::cin) return 2;
    const uint32_t parser = n_thread / 8 > 0 ? (uint32_t)(n_thread / 8) : 1u;
    const uint32_t budget = (uint32_t)n_thread - 2 - parser;
    const uint32_t classifiers = (budget / 2.0 == 0) ? 1u : (uint32_t)(budget / 2.0);
    uint64_t avg = 0;
    for (auto& c : counts) {
        if (c.load() < 1000) c.store(1000);
        avg += c.load();
    }
    std::cout << "Average prefix count: " << avg / 256 << "\n";
    std::cout << "classifiers " << classifiers << "\n";
    lpt(counts, classifiers);
    calculate_bloom_filter_capacity(counts, est);
    for (int p = 0; p < 256; ++p) std::cout << "owner " << p << " " << (unsigned)prefix_owners[p] << "\n";
    for (int p = 0; p < 256; ++p) std::cout << "capacity " << p << " " << bloom_filter_capacity[p] << "\n";
    return 0;
}
