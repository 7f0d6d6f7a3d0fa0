// `PostProcess` -- the reference's post-processing step (tool/PostProcess.h,
// driven by tool/PostProcessMain.cpp) on the device:
//
//   PostProcess <temp_dir> <output_dir> [k_len]
//
// Reads <temp_dir>/low.bin and root_{0..255}.bin and writes
// <output_dir>/final_root.bin, final_low.bin and freq_hist.txt as
// PostProcess::merge_all does (tool/PostProcess.h:63-139).  The reference's
// main hard-codes kmer<2> (k 33..64); here k_len (default 63) gives the key
// width and unpacks low.bin.  Exit 1 on a usage error, 255 on failure (the
// reference's std::exit(-1)).  KC_DEVICE picks the GPU.
#include <cstdlib>
#include <iostream>
#include <string>

#include "../../include/kmer_count.h"

int main(int argc, char* argv[]) {
    if (argc < 3 || argc > 4) {
        std::cerr << "Usage: " << argv[0] << " [temp_dir] [output_dir] [k_len]" << std::endl;
        return 1;
    }
    kc_config cfg;
    kc_config_default(&cfg);
    cfg.k = 63;
    try {
        if (argc == 4) cfg.k = (uint32_t)std::stoul(argv[3]);
    } catch (const std::exception&) {
        std::cerr << "Usage: " << argv[0] << " [temp_dir] [output_dir] [k_len]" << std::endl;
        return 1;
    }
    if (const char* d = std::getenv("KC_DEVICE")) cfg.device = std::atoi(d);
    kc_post_stats st;
    const int rc = kc_post_process_dir(&cfg, argv[1], argv[2], &st);
    if (rc != KC_OK) {
        std::cerr << "[PostProcess] " << kc_last_error() << std::endl;
        return rc == KC_ERR_INVALID ? 1 : 255;
    }
    std::cout << "Root records: " << st.root_records << std::endl;
    std::cout << "low.bin keys: " << st.low_in << " (" << st.low_in_roots << " also in root files)" << std::endl;
    std::cout << "final_low.bin keys: " << st.final_low << std::endl;
    return 0;
}
