// bdc_kernels.cuh -- launch entry points shared between the engine's .cu files.
#pragma once

#include "bdc_common.cuh"

namespace bdc {

struct CountLaunch {
    Split s;
    HalfTables A;             // cache_{n1, j} bundles, rows indexed by x_hi, stored rotated
                              // (launch_rotate_bundle with count_tile_tb(k))
    HalfTables B;             // cache_{n2, m} bundles, rows indexed by x_lo
    const uint32_t* reps;     // canonical representatives, ascending
    int64_t R;
    int grid;                 // CTAs of the q / D passes
    cudaStream_t stream;
    int c32 = 0;              // q and D sums in compensated FP32 (counts must be < 2^24)
};

// ---- count path (bdc_count.cu)
int count_cta_threads(int k);
int count_ctas_per_sm(int k);  // CTAs per SM in the grid of the q / D passes
int count_tile_tb(int k);      // top bits of y per thread tile (the rotation of the A bundle)
// the A bundle with each segment j >= tb rotated so that a tile's entries are adjacent
cudaError_t launch_rotate_bundle(const HalfTables& A, int tb, uint16_t* dst, cudaStream_t stream);
cudaError_t launch_count_pairs(const Split& s, const HalfTables& A, const HalfTables& B,
                               const uint32_t* xs, const uint32_t* ys, int64_t npairs,
                               uint32_t* out, cudaStream_t stream);
cudaError_t launch_qpass(const CountLaunch& L, const double* p0, const double* p1, double* part,
                         const DevState* st, int use_state);
cudaError_t launch_qfold(const double* part, int nparts, int k, double inv_c, double* lnq,
                         double* q_out, const DevState* st, int use_state, cudaStream_t stream);
cudaError_t launch_dpass(const CountLaunch& L, const double* lnq, const double* h, double inv_c,
                         double log_c, double* out, const DevState* st, int use_state);
cudaError_t launch_hpass(const CountLaunch& L, double inv_c, double log_c, double* out, uint32_t* nnz);

// ---- tables (bdc_tables.cu)
cudaError_t launch_gen_cache(int n, int k, uint32_t* out, cudaStream_t stream);
cudaError_t launch_build_bundle(int h, int mmax, int stride, const uint32_t* const* caches_dev,
                                uint16_t* rows, int* overflow, cudaStream_t stream);
cudaError_t launch_gen_bundle(int h, int mmax, int stride, uint16_t* rows, cudaStream_t stream);
cudaError_t build_reps(int n, uint32_t* reps_out, int64_t* count_out, void* scratch,
                       size_t scratch_bytes, cudaStream_t stream);
size_t build_reps_scratch_bytes(int n);

// ---- BA update (bdc_update.cu)
struct UpdateLaunch {
    int n;
    const uint32_t* reps;
    int64_t R;
    double* p0;        // the two iterate buffers; DevState::cur selects the current one
    double* p1;
    const double* d;   // D(x) per representative (nats)
    double* logw;      // scratch [R]
    double* part;      // block partials [3 * nblocks]
    int nblocks;
    double a;          // stopping threshold on mx (bits)
    DevState* st;
    cudaStream_t stream;
};
cudaError_t launch_update(const UpdateLaunch& U);
// stages 1 (logW, max logW = shift, max D, rate), 2 (e = exp(logW - shift),
// ln Z) and 3 (p' = e / exp(DevState::log_z), mx, buffer flip): first..last
cudaError_t launch_update_stages(const UpdateLaunch& U, int first, int last);
cudaError_t launch_logw(int n, const uint32_t* reps, int64_t R, const double* p, const double* d,
                        double* logw, cudaStream_t stream);
cudaError_t launch_mi_grad(int n, const uint32_t* reps, int64_t R, const double* d, double* grad,
                           cudaStream_t stream);
cudaError_t launch_rate(int n, const uint32_t* reps, int64_t R, const double* p, const double* d,
                        double* part, int nblocks, double* out, cudaStream_t stream);
cudaError_t launch_vec_max(const double* v, int64_t R, double* part, int nblocks, double* out,
                           cudaStream_t stream);
cudaError_t launch_max_dev(const double* p, const double* pb, int64_t R, double* part, int nblocks,
                           double* out, cudaStream_t stream);

}  // namespace bdc
