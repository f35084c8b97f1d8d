// bdc_engine.cuh -- the handle behind bdc_handle_t and the engine interface.
#pragma once

#include <string>

#include "bdc_common.cuh"
#include "bdc_kernels.cuh"

struct FactoredState;  // bdc_factored.cu

struct bdc_handle {
    // problem
    int n = 0, k = 0;
    bdc::Split s{};
    double C = 0, inv_c = 0, log_c = 0;
    int64_t R = 0;
    // placement / options
    int device = 0;
    int shard_rank = 0, shard_world = 1;  // factored engine over several GPUs: this handle's share of the rows
    int engine = BDC_ENGINE_COUNT;
    int c32 = 0;  // count engine with compensated-FP32 sums (BDC_ENGINE_COUNT_FP32C)
    int verbose = 0;
    int num_sms = 148;
    std::string cache_dir;
    cudaStream_t stream = nullptr;      // where work is queued
    cudaStream_t own_stream = nullptr;  // created by the handle
    size_t bytes = 0;  // device bytes held
    // tables (the representatives, the bundles and h below are shared by
    // every handle of the same n, k and table source on the device:
    // bdc_engine.cu, TableSet)
    void* tables = nullptr;
    uint32_t* d_reps = nullptr;
    uint16_t* d_bundle_hi = nullptr;
    uint16_t* d_bundle_lo = nullptr;  // equal to d_bundle_hi when n is even
    bdc::HalfTables A{}, B{};
    uint16_t* d_bundle_rot = nullptr;  // the A bundle rotated for the count passes' vector loads
    bdc::HalfTables Ar{};
    // per-representative vectors
    double* d_p[2] = {nullptr, nullptr};
    double* d_h = nullptr;     // sum_y W ln W
    double* d_d = nullptr;     // D(x)
    double* d_logw = nullptr;  // scratch
    // output side
    double* d_lnq = nullptr;   // [2^{k-1}]
    double* d_q = nullptr;     // [2^{k-1}]
    double* d_qpart = nullptr; // [grid][2^k]
    // FP64 re-evaluation of a compensated-FP32 handle's bound
    double* d_lnq64 = nullptr; // [2^{k-1}]
    double* d_d64 = nullptr;   // [R]
    // reductions / state
    double* d_red = nullptr;
    double* d_scalar = nullptr;
    double* d_shard = nullptr;   // [2^k] summed q partials of a sharded iteration (on first use)
    bdc::DevState* d_st = nullptr;
    bdc::DevState* h_st = nullptr;  // pinned mirror
    int grid_count = 0;
    int nb_upd = 0;
    bool p_set = false;
    int64_t nonzero_pairs = 0;  // sum over reps of distinct length-k subsequences
    // factored engine
    FactoredState* fac = nullptr;
    // scratch blocks of the certified solver, reused across its calls (bdc_solve.cu)
    void* solve_pool = nullptr;
};

namespace bdc {

bdc_status fail(bdc_status st, const char* fmt, ...) __attribute__((format(printf, 2, 3)));

int select_engine(int requested, int n, int k);
bdc_status engine_init(bdc_handle* H);
void engine_free(bdc_handle* H);
bdc_status engine_after_set_p(bdc_handle* H, int strict_zero = 0);
bdc_status engine_current_p(bdc_handle* H, const double** p);
bdc_status engine_iterate(bdc_handle* H, int64_t max_iters, double a, bdc_stats* stats);
bdc_status engine_log_q(bdc_handle* H);       // ln q of the current p into H->d_lnq
bdc_status engine_divergence(bdc_handle* H);  // D from H->d_lnq into H->d_d
// compensated-FP32 handles: the last bound and rate re-evaluated in FP64 at
// the same iterate; the absolute differences in bits (0 for FP64 engines)
bdc_status engine_bound_error(bdc_handle* H, double* ub_err_bits, double* rate_err_bits);

CountLaunch count_launch(const bdc_handle* H);
UpdateLaunch update_launch(const bdc_handle* H, double a);
bdc_status engine_profile(bdc_handle* H, int iters, bdc_profile_t* out);
cudaError_t engine_enqueue_iteration(bdc_handle* H, double a);  // one iteration, gated by done
int count_group_size(int k);

// factored engine (bdc_factored.cu)
// factored engine sharded by rows (bdc_factored.cu): this handle's window,
// and one iteration in three parts around the two exchanges
void factored_shard_range(const bdc_handle* H, int* row0, int* rows, int64_t* i0, int64_t* i1);
bdc_status factored_shard_q(bdc_handle* H, double* acc);
bdc_status factored_shard_d(bdc_handle* H, const double* acc, double* part5);
bdc_status factored_shard_finish(bdc_handle* H, const double* part5, double a);

// the certified solver (bdc_solve.cu) with its first phase chosen: 0 Anderson
// (bdc_solve), 1 the momentum loop (bdc_accelerate), 2 none (the handle's
// iterate is already near the optimum: support phases only)
constexpr double kSupportSwitchBits = 1e-4;  // bracket at which the support phases take over
bdc_status solve_impl(bdc_handle* H, double gap_bits, int64_t max_evals, bdc_stats* stats, int phase1);

// frees the certified solver's scratch blocks (bdc_solve.cu)
void solve_pool_release(bdc_handle* H);

bool factored_supports(int n, int k);
bdc_status factored_init(bdc_handle* H);
void factored_free(bdc_handle* H);
// d_p[0] -> dense state; strict_zero: a zero entry stays zero (ln p = -inf)
// instead of the reference's ln 0 = 0
bdc_status factored_load_p(bdc_handle* H, int strict_zero = 0);
bdc_status factored_store_p(bdc_handle* H, double* p_out);  // dense state -> p per rep
bdc_status factored_iterate(bdc_handle* H, int64_t max_iters, double a, bdc_stats* stats);
bdc_status factored_profile(bdc_handle* H, int iters, bdc_profile_t* out);
bdc_status factored_accelerate(bdc_handle* H, int64_t max_evals, double gap_bits, bdc_stats* stats);
// the accelerated loop's pieces, for callers that queue its steps themselves
// (batches): the step length, the start (snapshots of the current iterate,
// the device stop at gap_bits) and `steps` steps queued on H->stream
double factored_acc_eta();
bdc_status factored_acc_start(bdc_handle* H, double gap_bits);
bdc_status factored_acc_buffers(bdc_handle* H);  // the loop's snapshot vectors (before any capture)
cudaError_t factored_enqueue_acc_steps(bdc_handle* H, int steps, double eta);
cudaError_t factored_enqueue_iteration(bdc_handle* H, double a);
// finishes an iteration that stopped on an exp-shift overflow (on H->stream);
// any other device error is returned as BDC_ERR_NUMERIC
bdc_status factored_recover(bdc_handle* H, double a);
bdc_status factored_map(bdc_handle* H, const double* p_in, double* p_out, double* D_out);
// Device buffers for dgemm_nt: one product descriptor and a tile map (every
// tile on descriptor 0) of up to `tiles` 64x64 tiles, allocated once by the
// caller and reused by every call on one stream.
struct DgemmScratch {
    void* desc = nullptr;
    int* map = nullptr;
    int tiles = 0;
};
cudaError_t dgemm_scratch_alloc(DgemmScratch& sc, int max_tiles, cudaStream_t s);
void dgemm_scratch_free(DgemmScratch& sc);
// C (M x N) = alpha A B^T (+ C) on the FP64 tensor-core path, queued on s
// without allocating or synchronising
cudaError_t dgemm_nt(const DgemmScratch& sc, const double* A, int lda, const double* B, int ldb, double* C, int ldc,
                     int M, int N, int K, double alpha, int accumulate, cudaStream_t s);

}  // namespace bdc
