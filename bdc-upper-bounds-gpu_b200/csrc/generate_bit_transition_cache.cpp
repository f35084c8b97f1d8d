// generate_bit_transition_cache.cpp -- drop-in for the reference generator
// (backend/generate_bit_transition_cache.cpp:46-77): `./generate_bit_transition_cache N`
// writes ./transition_counts/cache_{n'}_{k'} for every 0 <= k' < n' <= N in
// the same binary format (uint32, index (x << k') | y).  The counts are
// computed on the GPU (bdc_generate_cache); a file that cannot be opened
// exits with status 2 like the reference's try_to_open_file (backend/utils.cc:46-53).
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "bdc_b200.h"

int main(int argc, char const* argv[]) {
    if (argc != 2) {
        fprintf(stderr, "Usage %s n k\n", argv[0]);
        return 1;
    }
    const int N = atoi(argv[1]);
    if (N < 0 || N > 17) {
        fprintf(stderr, "n must be in 0..17\n");
        return 1;
    }
    std::vector<uint32_t> buf;
    for (int n = 0; n <= N; ++n) {
        for (int k = 0; k < n; ++k) {
            buf.resize((size_t)1 << (n + k));
            if (bdc_generate_cache(n, k, 0, buf.data()) != BDC_OK) {
                fprintf(stderr, "Error: %s\n", bdc_last_error());
                return 2;
            }
            const std::string path = "./transition_counts/cache_" + std::to_string(n) + "_" + std::to_string(k);
            if (bdc_write_cache_file(path.c_str(), n, k, buf.data()) != BDC_OK) {
                fprintf(stderr, "Error: failed to open file %s.\n", path.c_str());
                return 2;
            }
        }
    }
    return 0;
}
