// ref_harness.cu -- drives the reference's own BA path (backend/BAA.cu, compiled
// unchanged from the reference sources) through its host API and dumps every
// intermediate vector in full double precision.
//
// TEST INFRASTRUCTURE ONLY: this program produces golden vectors for the
// parity tests; the product never links or runs it.  It must be started in a
// directory that holds transition_counts/cache_n_k files, because the
// reference loads them by relative path (backend/cache_io.h:7-14).
//
// usage: ref_harness n k iters init outdir
//   init   "uniform" (main_BAA.cu:64) or a path to raw little-endian doubles,
//          one per canonical representative in ascending order
//   outdir receives raw double files:
//     p_0.bin                 starting vector
//     lnq_<t>.bin             compute_all_log_D on p_t   (BAA.cu:642-724)
//     logw_<t>.bin            compute_all_log_W          (BAA.cu:727-814)
//     p_<t+1>.bin             baa_iteration              (BAA.cu:590-639)
//     kl_final.bin            compute_KL_kernel on the final p (BAA.cu:533-571)
//     lnq_final.bin           compute_all_log_D on the final p
//   and meta.txt with one line per iteration "iter mx" (BAA.cu:916-946) plus
//   "rate_nats <v>" from compute_rate (BAA.cu:836-913), and timing lines
//   "time_iter_s <t>" measured around baa_iteration + compute_max_deviation
//   (the body of the reference loop, main_BAA.cu:80-99) with cudaEvents.
#include "BAA.cuh"

#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

static void dump(const std::string& path, const std::vector<double>& v) {
    FILE* f = fopen(path.c_str(), "wb");
    if (!f) { fprintf(stderr, "cannot write %s\n", path.c_str()); exit(3); }
    fwrite(v.data(), sizeof(double), v.size(), f);
    fclose(f);
}

static std::vector<double> load(const std::string& path, size_t n) {
    std::vector<double> v(n);
    FILE* f = fopen(path.c_str(), "rb");
    if (!f) { fprintf(stderr, "cannot read %s\n", path.c_str()); exit(3); }
    size_t got = fread(v.data(), sizeof(double), n, f);
    fclose(f);
    if (got != n) { fprintf(stderr, "short read %s: %zu of %zu\n", path.c_str(), got, n); exit(3); }
    return v;
}

int main(int argc, char** argv) {
    if (argc < 6) {
        fprintf(stderr, "usage: %s n k iters init outdir\n", argv[0]);
        return 1;
    }
    size_t n = std::stoul(argv[1]);
    size_t k = std::stoul(argv[2]);
    int iters = std::stoi(argv[3]);
    std::string init = argv[4];
    std::string out = argv[5];

    std::vector<uint32_t> reps;
    for (uint32_t x = 0; x < (1u << n); ++x)
        if (rep(x, (int)n) == x) reps.push_back(x);

    std::vector<double> Q(reps.size());
    if (init == "uniform") {
        std::fill(Q.begin(), Q.end(), 1.0 / (double)(1u << n));
    } else {
        Q = load(init, reps.size());
    }
    dump(out + "/p_0.bin", Q);

    load_cache(n, k);

    FILE* meta = fopen((out + "/meta.txt").c_str(), "w");
    fprintf(meta, "n %zu\nk %zu\nreps %zu\n", n, k, reps.size());
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    for (int t = 0; t < iters; ++t) {
        std::vector<double> lnq = compute_all_log_D(Q, reps, n, k);
        std::vector<double> lw = compute_all_log_W(Q, lnq, reps, n, k);
        dump(out + "/lnq_" + std::to_string(t) + ".bin", lnq);
        dump(out + "/logw_" + std::to_string(t) + ".bin", lw);
        std::vector<double> Qb = Q;
        cudaEventRecord(e0);
        Q = baa_iteration(Q, reps, n, k);
        double mx = compute_max_deviation(Q, Qb);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        dump(out + "/p_" + std::to_string(t + 1) + ".bin", Q);
        fprintf(meta, "iter %d mx %.17g\n", t, mx);
        fprintf(meta, "time_iter_s %d %.9g\n", t, ms * 1e-3);
    }

    std::vector<double> lnq = compute_all_log_D(Q, reps, n, k);
    dump(out + "/lnq_final.bin", lnq);

    // KL(x) per representative, via the reference kernel
    uint32_t* d_reps = nullptr;
    double* d_lnq = nullptr;
    double* d_kl = nullptr;
    CUDA_CHECK(cudaMalloc(&d_reps, reps.size() * sizeof(uint32_t)));
    CUDA_CHECK(cudaMalloc(&d_lnq, lnq.size() * sizeof(double)));
    CUDA_CHECK(cudaMalloc(&d_kl, reps.size() * sizeof(double)));
    CUDA_CHECK(cudaMemcpy(d_reps, reps.data(), reps.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemcpy(d_lnq, lnq.data(), lnq.size() * sizeof(double), cudaMemcpyHostToDevice));
    compute_KL_kernel<<<reps.size(), 1024>>>(d_reps, d_lnq, d_kl, (uint8_t)n, (uint8_t)k);
    CUDA_CHECK(cudaGetLastError());
    CUDA_CHECK(cudaDeviceSynchronize());
    std::vector<double> kl(reps.size());
    CUDA_CHECK(cudaMemcpy(kl.data(), d_kl, reps.size() * sizeof(double), cudaMemcpyDeviceToHost));
    dump(out + "/kl_final.bin", kl);
    cudaFree(d_reps);
    cudaFree(d_lnq);
    cudaFree(d_kl);

    double rate = compute_rate(lnq, Q, reps, (uint8_t)n, (uint8_t)k);
    fprintf(meta, "rate_nats %.17g\n", rate);
    fclose(meta);
    return 0;
}
