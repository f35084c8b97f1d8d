// main_BAA.cpp -- drop-in for the reference CLI (backend/main_BAA.cu:134-170):
//
//   ./main_BAA n k [read_from_file] [a] [save_iterations]
//
// Same positional arguments and defaults (read_from_file 0, a 0.005,
// save_iterations 100), same relative paths (./transition_counts/cache_n_k,
// distributions/dist_n_k.txt), same stopping rule (iterate while mx >= a,
// main_BAA.cu:73) and the same result line.  The BA iterations run on the
// device through the C ABI (include/bdc_b200.h).
//
// Differences, on purpose: a missing or wrong-sized distribution file is an
// error (exit 2) instead of continuing with an empty vector; the dist file is
// replaced atomically; BDC_TABLES=device builds the half tables on the GPU
// instead of reading transition_counts/; BDC_ENGINE=count|factored|count-fp32c
// picks the engine (default: fastest available; count-fp32c also prints the
// last bound's error against FP64); BDC_SOLVE=<gap bits> runs the certified
// solver (bdc_solve) instead of the plain loop and prints the bracket.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "bdc_b200.h"

static int die(const char* what) {
    fprintf(stderr, "Error: %s: %s\n", what, bdc_last_error());
    return 2;
}

static int compute_C_n_k(int n, int k, double a, bool read_from_file, long save_iterations) {
    const std::string file = "distributions/dist_" + std::to_string(n) + "_" + std::to_string(k) + ".txt";
    bdc_options o;
    bdc_default_options(&o);
    const char* tables = getenv("BDC_TABLES");
    o.cache_dir = (tables && strcmp(tables, "device") == 0) ? nullptr : "./transition_counts";
    const char* eng = getenv("BDC_ENGINE");
    if (eng && strcmp(eng, "count") == 0) o.engine = BDC_ENGINE_COUNT;
    if (eng && strcmp(eng, "factored") == 0) o.engine = BDC_ENGINE_FACTORED;
    const bool c32 = eng && strcmp(eng, "count-fp32c") == 0;
    if (c32) o.engine = BDC_ENGINE_COUNT_FP32C;
    o.verbose = 1;

    bdc_handle_t h = nullptr;
    if (bdc_create(n, k, &o, &h) != BDC_OK) return die("load_cache");
    int64_t R = 0;
    bdc_info(h, nullptr, nullptr, &R, nullptr);

    if (read_from_file) {
        printf("Loading distribution from file: %s\n", file.c_str());
        int64_t cnt = 0;
        if (bdc_read_dist_file(file.c_str(), nullptr, 0, &cnt) != BDC_OK) return die("read_distribution_file");
        if (cnt != R) {
            fprintf(stderr, "Error: %s holds %lld values, BDC_{%d,%d} has %lld representatives\n", file.c_str(),
                    (long long)cnt, n, k, (long long)R);
            return 2;
        }
        std::vector<double> p(R);
        if (bdc_read_dist_file(file.c_str(), p.data(), R, &cnt) != BDC_OK) return die("read_distribution_file");
        if (bdc_set_p(h, p.data(), R) != BDC_OK) return die("set distribution");
    } else {
        printf("Initializing uniform distribution\n");
        if (bdc_set_p_uniform(h) != BDC_OK) return die("set distribution");
    }
    // BDC_SOLVE=<gap in bits>: the certified solver instead of the plain loop
    const char* solve = getenv("BDC_SOLVE");
    if (solve && *solve) {
        const double gap = atof(solve);
        printf("Starting the certified solver (bracket below %g bits)...\n", gap);
        fflush(stdout);
        auto t0 = std::chrono::high_resolution_clock::now();
        bdc_stats st;
        if (bdc_solve(h, gap, 1000000, &st) != BDC_OK) return die("bdc_solve");
        auto t1 = std::chrono::high_resolution_clock::now();
        std::vector<double> p(R);
        if (bdc_get_p(h, p.data(), R) != BDC_OK) return die("read distribution");
        if (bdc_write_dist_file(file.c_str(), p.data(), R) != BDC_OK) return die("save distribution");
        printf("Final distribution saved to %s\n", file.c_str());
        bdc_destroy(h);
        printf("Certified C_{%d,%d} in [%.15f, %.15f] bits (%lld BA evaluations, %.3f s)\n", n, k, st.best_rate,
               st.best_upper_bound, (long long)st.iters, std::chrono::duration<double>(t1 - t0).count());
        return st.converged ? 0 : 3;
    }
    printf("Starting BAA iterations...\n");
    fflush(stdout);

    double mx = a;
    long i = 1;
    std::vector<double> p(R);
    while (mx >= a) {
        auto t0 = std::chrono::high_resolution_clock::now();
        bdc_stats st;
        if (bdc_iterate(h, 1, a, &st) != BDC_OK) return die("baa_iteration");
        mx = st.mx;
        if (save_iterations > 0 && i % save_iterations == 0) {
            auto s0 = std::chrono::high_resolution_clock::now();
            if (bdc_get_p(h, p.data(), R) != BDC_OK) return die("read distribution");
            if (bdc_write_dist_file(file.c_str(), p.data(), R) != BDC_OK) return die("save distribution");
            auto s1 = std::chrono::high_resolution_clock::now();
            printf("Distribution saved in %.3f seconds\n", std::chrono::duration<double>(s1 - s0).count());
        }
        auto t1 = std::chrono::high_resolution_clock::now();
        printf("Iteration %ld: mx = %.6f, time = %.3f s\n", i, mx, std::chrono::duration<double>(t1 - t0).count());
        fflush(stdout);
        ++i;
    }
    double ub_err = 0, rate_err = 0;
    if (c32 && bdc_bound_error(h, &ub_err, &rate_err) != BDC_OK) return die("bound error");
    if (bdc_get_p(h, p.data(), R) != BDC_OK) return die("read distribution");
    if (bdc_write_dist_file(file.c_str(), p.data(), R) != BDC_OK) return die("save distribution");
    printf("Final distribution saved to %s\n", file.c_str());
    double rate = 0;
    if (bdc_rate(h, &rate) != BDC_OK) return die("compute_rate");
    rate /= std::log(2.0);
    bdc_destroy(h);
    printf("Computed C_{%d,%d} = %.6f bits (max deviation %.6f)\n", n, k, rate, mx);
    if (c32)
        printf("Compensated FP32: last bound %.3e bits and rate %.3e bits from their FP64 values\n", ub_err,
               rate_err);
    return 0;
}

int main(int argc, char* argv[]) {
    if (argc < 3) {
        fprintf(stderr, "Usage: %s <n> <k> [reed_from_file] [a] [save_iterations]\n", argv[0]);
        fprintf(stderr, "Exemple: %s 21 20\n", argv[0]);
        fprintf(stderr, "Exemple: %s 21 20 1 0.01 200\n", argv[0]);
        return 1;
    }
    const int n = (int)std::stoul(argv[1]);
    const int k = (int)std::stoul(argv[2]);
    bool read_from_file = false;
    double a = 0.005;
    long save_iterations = 100;
    if (argc > 3) read_from_file = std::stoi(argv[3]) != 0;
    if (argc > 4) a = std::stod(argv[4]);
    if (argc > 5) save_iterations = (long)std::stoul(argv[5]);
    return compute_C_n_k(n, k, a, read_from_file, save_iterations);
}
