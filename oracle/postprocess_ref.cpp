// Test infrastructure only: runs the REFERENCE's own post-processing,
// PostProcess<N>::merge_all (tool/PostProcess.h:63-139, header-only), on a
// directory of low.bin + root_{id}.bin, so that the build's device version
// can be compared with it byte for byte.  (The reference's own
// tool/PostProcessMain.cpp calls methods that do not exist and does not
// compile.)
//
//   postprocess <temp_dir/> <output_dir/> <N: 1|2|4>
#include <cstdlib>
#include <string>

#include "PostProcess.h"

int main(int argc, char** argv) {
    if (argc != 4) return 1;
    temp_dir = argv[1];
    output_dir = argv[2];
    const int n = std::atoi(argv[3]);
    if (n == 1) {
        PostProcess<1> p(4);
        p.merge_all();
    } else if (n == 2) {
        PostProcess<2> p(4);
        p.merge_all();
    } else if (n == 4) {
        PostProcess<4> p(4);
        p.merge_all();
    } else {
        return 1;
    }
    return 0;
}
