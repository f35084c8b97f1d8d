// bdc_capi.cu -- the C ABI of include/bdc_b200.h: handle life cycle, device
// buffers, the iteration driver and the reference-shaped single calls.
//
// Reference host layer replaced here (Pintz45/BDC-Upper-Bounds-GPU):
//   backend/BAA.cu:27-188   load_gpu_cache / compute_normalizers /
//                           load_log_counts / load_cache (device globals, one
//                           (n,k) per process, never freed)
//   backend/BAA.cu:590-946  baa_iteration, compute_all_log_D,
//                           compute_all_log_W, compute_rate,
//                           compute_max_deviation (host vectors in and out,
//                           cudaMalloc/cudaFree and H2D/D2H on every call)
//   backend/main_BAA.cu:39-131  the BA loop
// Here a handle owns all device state for one (n,k); the iterate never leaves
// the device inside bdc_iterate; errors are status codes.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "bdc_common.cuh"
#include "bdc_engine.cuh"
#include "bdc_kernels.cuh"

using namespace bdc;

namespace bdc {

bdc_status fail(bdc_status st, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    set_last_error("%s", buf);
    return st;
}

}  // namespace bdc

extern "C" {

void bdc_default_options(bdc_options* o) {
    if (!o) return;
    o->engine = BDC_ENGINE_AUTO;
    o->device = 0;
    o->cache_dir = nullptr;
    o->verbose = 0;
}

const char* bdc_version(void) { return "bdc-b200 0.1.0 (sm_100a)"; }

static bdc_status create_handle(int n, int k, const bdc_options* opts, int rank, int world, bdc_handle_t* out);

// a handle that holds only a window of the rows (bdc_create_sharded) runs
// the sharded iteration only
static bdc_status refuse_sharded(bdc_handle_t H, const char* what) {
    if (H && H->shard_world > 1)
        return fail(BDC_ERR_STATE, "%s: this handle holds a shard of the rows; use the bdc_fshard_* calls", what);
    return BDC_OK;
}

bdc_status bdc_create(int n, int k, const bdc_options* opts, bdc_handle_t* out) {
    return create_handle(n, k, opts, 0, 1, out);
}

bdc_status bdc_create_sharded(int n, int k, const bdc_options* opts, int rank, int world, bdc_handle_t* out) {
    if (world < 1 || rank < 0 || rank >= world)
        return fail(BDC_ERR_ARG, "bdc_create_sharded: rank %d of %d", rank, world);
    bdc_options o;
    bdc_default_options(&o);
    if (opts) o = *opts;
    if (o.engine != BDC_ENGINE_AUTO && o.engine != BDC_ENGINE_FACTORED)
        return fail(BDC_ERR_UNSUPPORTED, "bdc_create_sharded: rows are sharded on the factored engine only");
    o.engine = BDC_ENGINE_FACTORED;
    return create_handle(n, k, &o, rank, world, out);
}

static bdc_status create_handle(int n, int k, const bdc_options* opts, int rank, int world, bdc_handle_t* out) {
    if (!out) return fail(BDC_ERR_ARG, "bdc_create: out is NULL");
    *out = nullptr;
    bdc_options o;
    bdc_default_options(&o);
    if (opts) o = *opts;
    if (n < 1 || n > 30 || k < 1 || k > n)
        return fail(BDC_ERR_ARG, "bdc_create: need 1 <= k <= n <= 30 (got n=%d k=%d)", n, k);
    if (k > 14)
        return fail(BDC_ERR_UNSUPPORTED, "bdc_create: output length k=%d above 14 is not built", k);
    const Split s = make_split(n, k);
    if (s.n1 > kMaxHalf) return fail(BDC_ERR_UNSUPPORTED, "half length %d above %d", s.n1, kMaxHalf);
    if (cudaSetDevice(o.device) != cudaSuccess)
        return fail(BDC_ERR_CUDA, "cudaSetDevice(%d) failed", o.device);

    bdc_handle* H = new bdc_handle();
    H->n = n;
    H->k = k;
    H->s = s;
    H->device = o.device;
    H->shard_rank = rank;
    H->shard_world = world;
    H->verbose = o.verbose;
    H->cache_dir = o.cache_dir ? std::string(o.cache_dir) : std::string();
    H->C = (double)binom(n, k);
    H->inv_c = 1.0 / H->C;  // d_normalizers (backend/BAA.cu:108)
    H->log_c = std::log(H->C);
    H->engine = select_engine(o.engine, n, k);
    if (H->engine < 0) {
        delete H;
        return fail(BDC_ERR_UNSUPPORTED, "requested engine does not support n=%d k=%d", n, k);
    }
    if (H->engine == BDC_ENGINE_COUNT_FP32C) {
        H->engine = BDC_ENGINE_COUNT;
        H->c32 = 1;
    }
    bdc_status rc = engine_init(H);
    if (rc != BDC_OK) {
        engine_free(H);
        delete H;
        return rc;
    }
    *out = H;
    return BDC_OK;
}

bdc_status bdc_destroy(bdc_handle_t H) {
    if (!H) return BDC_OK;
    BDC_CUDA_TRY(cudaSetDevice(H->device));
    engine_free(H);
    delete H;
    return BDC_OK;
}

bdc_status bdc_info(bdc_handle_t H, int* n, int* k, int64_t* num_reps, int* engine) {
    if (!H) return fail(BDC_ERR_ARG, "bdc_info: NULL handle");
    if (n) *n = H->n;
    if (k) *k = H->k;
    if (num_reps) *num_reps = H->R;
    if (engine) *engine = H->c32 ? BDC_ENGINE_COUNT_FP32C : H->engine;
    return BDC_OK;
}

bdc_status bdc_get_reps(bdc_handle_t H, uint32_t* reps, int64_t R) {
    if (!H || !reps) return fail(BDC_ERR_ARG, "bdc_get_reps: NULL argument");
    if (R != H->R) return fail(BDC_ERR_ARG, "bdc_get_reps: %lld slots for %lld representatives", (long long)R, (long long)H->R);
    BDC_CUDA_TRY(cudaSetDevice(H->device));
    BDC_CUDA_TRY(cudaMemcpyAsync(reps, H->d_reps, sizeof(uint32_t) * R, cudaMemcpyDeviceToHost, H->stream));
    BDC_CUDA_TRY(cudaStreamSynchronize(H->stream));
    return BDC_OK;
}

bdc_status bdc_set_p(bdc_handle_t H, const double* p, int64_t R) {
    if (!H || !p) return fail(BDC_ERR_ARG, "bdc_set_p: NULL argument");
    if (R != H->R)
        return fail(BDC_ERR_ARG, "bdc_set_p: distribution has %lld entries, (n=%d) has %lld representatives",
                    (long long)R, H->n, (long long)H->R);
    BDC_CUDA_TRY(cudaSetDevice(H->device));
    BDC_CUDA_TRY(cudaMemcpyAsync(H->d_p[0], p, sizeof(double) * R, cudaMemcpyHostToDevice, H->stream));
    return engine_after_set_p(H);
}

bdc_status bdc_set_p_device(bdc_handle_t H, const double* p, int64_t R) {
    if (!H || !p) return fail(BDC_ERR_ARG, "bdc_set_p_device: NULL argument");
    if (R != H->R) return fail(BDC_ERR_ARG, "bdc_set_p_device: size mismatch");
    BDC_CUDA_TRY(cudaSetDevice(H->device));
    BDC_CUDA_TRY(cudaMemcpyAsync(H->d_p[0], p, sizeof(double) * R, cudaMemcpyDeviceToDevice, H->stream));
    return engine_after_set_p(H);
}

bdc_status bdc_set_p_uniform(bdc_handle_t H) {
    if (!H) return fail(BDC_ERR_ARG, "bdc_set_p_uniform: NULL handle");
    BDC_CUDA_TRY(cudaSetDevice(H->device));
    std::vector<double> u(H->R, 1.0 / (double)(1ull << H->n));  // backend/main_BAA.cu:64
    BDC_CUDA_TRY(cudaMemcpyAsync(H->d_p[0], u.data(), sizeof(double) * H->R, cudaMemcpyHostToDevice, H->stream));
    BDC_CUDA_TRY(cudaStreamSynchronize(H->stream));
    return engine_after_set_p(H);
}

bdc_status bdc_get_p(bdc_handle_t H, double* p, int64_t R) {
    if (!H || !p) return fail(BDC_ERR_ARG, "bdc_get_p: NULL argument");
    if (bdc_status rs = refuse_sharded(H, "bdc_get_p")) return rs;
    if (R != H->R) return fail(BDC_ERR_ARG, "bdc_get_p: size mismatch");
    if (!H->p_set) return fail(BDC_ERR_STATE, "bdc_get_p: no distribution set");
    BDC_CUDA_TRY(cudaSetDevice(H->device));
    const double* src = nullptr;
    bdc_status rc = engine_current_p(H, &src);
    if (rc != BDC_OK) return rc;
    BDC_CUDA_TRY(cudaMemcpyAsync(p, src, sizeof(double) * R, cudaMemcpyDeviceToHost, H->stream));
    BDC_CUDA_TRY(cudaStreamSynchronize(H->stream));
    return BDC_OK;
}

bdc_status bdc_get_p_device(bdc_handle_t H, double* p, int64_t R) {
    if (!H || !p) return fail(BDC_ERR_ARG, "bdc_get_p_device: NULL argument");
    if (bdc_status rs = refuse_sharded(H, "bdc_get_p_device")) return rs;
    if (R != H->R) return fail(BDC_ERR_ARG, "bdc_get_p_device: size mismatch");
    if (!H->p_set) return fail(BDC_ERR_STATE, "bdc_get_p_device: no distribution set");
    BDC_CUDA_TRY(cudaSetDevice(H->device));
    const double* src = nullptr;
    bdc_status rc = engine_current_p(H, &src);
    if (rc != BDC_OK) return rc;
    BDC_CUDA_TRY(cudaMemcpyAsync(p, src, sizeof(double) * R, cudaMemcpyDeviceToDevice, H->stream));
    BDC_CUDA_TRY(cudaStreamSynchronize(H->stream));
    return BDC_OK;
}

bdc_status bdc_iterate(bdc_handle_t H, int64_t max_iters, double a, bdc_stats* stats) {
    if (!H) return fail(BDC_ERR_ARG, "bdc_iterate: NULL handle");
    if (bdc_status rs = refuse_sharded(H, "bdc_iterate")) return rs;
    if (!H->p_set) return fail(BDC_ERR_STATE, "bdc_iterate: no distribution set");
    if (max_iters < 0) return fail(BDC_ERR_ARG, "bdc_iterate: max_iters < 0");
    BDC_CUDA_TRY(cudaSetDevice(H->device));
    return engine_iterate(H, max_iters, a, stats);
}

bdc_status bdc_bound_error(bdc_handle_t H, double* ub_err, double* rate_err) {
    if (!H || !ub_err || !rate_err) return fail(BDC_ERR_ARG, "bdc_bound_error: NULL argument");
    if (bdc_status rs = refuse_sharded(H, "bdc_bound_error")) return rs;
    if (!H->p_set) return fail(BDC_ERR_STATE, "bdc_bound_error: no distribution set");
    BDC_CUDA_TRY(cudaSetDevice(H->device));
    return engine_bound_error(H, ub_err, rate_err);
}

bdc_status bdc_accelerate(bdc_handle_t H, int64_t max_evals, double gap_bits, bdc_stats* stats) {
    if (!H) return fail(BDC_ERR_ARG, "bdc_accelerate: NULL handle");
    if (bdc_status rs = refuse_sharded(H, "bdc_accelerate")) return rs;
    if (!H->p_set) return fail(BDC_ERR_STATE, "bdc_accelerate: no distribution set");
    if (H->engine != BDC_ENGINE_FACTORED)
        return fail(BDC_ERR_UNSUPPORTED, "bdc_accelerate: needs the factored engine (k < n)");
    if (max_evals < 0) return fail(BDC_ERR_ARG, "bdc_accelerate: max_evals < 0");
    BDC_CUDA_TRY(cudaSetDevice(H->device));
    // a target below the support switch: the momentum phase, then the
    // support phases (restricted BA, Newton on the support, the full-space
    // check) finish, as in the certified solver (counts exact in FP32: n <= 26)
    if (gap_bits > 0.0 && gap_bits < kSupportSwitchBits && H->n <= 26 && max_evals > 0)
        return solve_impl(H, gap_bits, max_evals, stats, 1);
    return factored_accelerate(H, max_evals, gap_bits, stats);
}

// The factored engine evaluates I(p;W) and D(x) with one BA map (the G
// product's epilogue yields both); the map advances the dense iterate, which
// is then reloaded from p so that the handle still holds p.
static bdc_status factored_eval(bdc_handle_t H, bool with_d) {
    const double* cur = nullptr;
    bdc_status rc = engine_current_p(H, &cur);  // p in d_p[0]
    if (rc != BDC_OK) return rc;
    rc = factored_map(H, H->d_p[0], H->d_p[1], with_d ? H->d_d : nullptr);
    if (rc != BDC_OK) return rc;
    const double rate = H->h_st->rate;
    rc = engine_after_set_p(H);
    H->h_st->rate = rate;
    return rc;
}

bdc_status bdc_mi_forward(bdc_handle_t H, const double* p, int64_t R, double* I_nats) {
    if (!H || !I_nats) return fail(BDC_ERR_ARG, "bdc_mi_forward: NULL argument");
    if (bdc_status rs = refuse_sharded(H, "bdc_mi_forward")) return rs;
    if (p) {
        bdc_status rc = bdc_set_p(H, p, R);
        if (rc != BDC_OK) return rc;
    }
    if (H->engine == BDC_ENGINE_FACTORED) {
        if (!H->p_set) return fail(BDC_ERR_STATE, "bdc_mi_forward: no distribution set");
        BDC_CUDA_TRY(cudaSetDevice(H->device));
        bdc_status rc = factored_eval(H, false);
        if (rc != BDC_OK) return rc;
        *I_nats = H->h_st->rate;
        return BDC_OK;
    }
    return bdc_rate(H, I_nats);
}

bdc_status bdc_mi_backward(bdc_handle_t H, double* grad, int64_t R) {
    if (!H || !grad) return fail(BDC_ERR_ARG, "bdc_mi_backward: NULL argument");
    if (bdc_status rs = refuse_sharded(H, "bdc_mi_backward")) return rs;
    if (R != H->R) return fail(BDC_ERR_ARG, "bdc_mi_backward: %lld slots for %lld representatives", (long long)R, (long long)H->R);
    if (!H->p_set) return fail(BDC_ERR_STATE, "bdc_mi_backward: no distribution set");
    BDC_CUDA_TRY(cudaSetDevice(H->device));
    bdc_status rc = BDC_OK;
    if (H->engine == BDC_ENGINE_FACTORED) {
        rc = factored_eval(H, true);
    } else {
        rc = engine_log_q(H);
        if (rc == BDC_OK) rc = engine_divergence(H);
    }
    if (rc != BDC_OK) return rc;
    BDC_CUDA_TRY(launch_mi_grad(H->n, H->d_reps, H->R, H->d_d, H->d_logw, H->stream));
    BDC_CUDA_TRY(cudaMemcpyAsync(grad, H->d_logw, sizeof(double) * R, cudaMemcpyDeviceToHost, H->stream));
    BDC_CUDA_TRY(cudaStreamSynchronize(H->stream));
    return BDC_OK;
}

bdc_status bdc_mi_backward_device(bdc_handle_t H, double* grad_dev, int64_t R) {
    if (!H || !grad_dev) return fail(BDC_ERR_ARG, "bdc_mi_backward_device: NULL argument");
    if (bdc_status rs = refuse_sharded(H, "bdc_mi_backward_device")) return rs;
    if (R != H->R)
        return fail(BDC_ERR_ARG, "bdc_mi_backward_device: %lld slots for %lld representatives", (long long)R,
                    (long long)H->R);
    if (!H->p_set) return fail(BDC_ERR_STATE, "bdc_mi_backward_device: no distribution set");
    BDC_CUDA_TRY(cudaSetDevice(H->device));
    bdc_status rc = BDC_OK;
    if (H->engine == BDC_ENGINE_FACTORED) {
        rc = factored_eval(H, true);
    } else {
        rc = engine_log_q(H);
        if (rc == BDC_OK) rc = engine_divergence(H);
    }
    if (rc != BDC_OK) return rc;
    BDC_CUDA_TRY(launch_mi_grad(H->n, H->d_reps, H->R, H->d_d, grad_dev, H->stream));
    BDC_CUDA_TRY(cudaStreamSynchronize(H->stream));
    return BDC_OK;
}

bdc_status bdc_baa_iteration(bdc_handle_t H, const double* p_in, double* p_out, int64_t R) {
    if (!H || !p_in || !p_out) return fail(BDC_ERR_ARG, "bdc_baa_iteration: NULL argument");
    if (bdc_status rs = refuse_sharded(H, "bdc_baa_iteration")) return rs;
    bdc_status rc = bdc_set_p(H, p_in, R);
    if (rc != BDC_OK) return rc;
    rc = engine_iterate(H, 1, -INFINITY, nullptr);
    if (rc != BDC_OK) return rc;
    return bdc_get_p(H, p_out, R);
}

bdc_status bdc_log_q(bdc_handle_t H, double* lnq, int64_t nq) {
    if (!H || !lnq) return fail(BDC_ERR_ARG, "bdc_log_q: NULL argument");
    if (bdc_status rs = refuse_sharded(H, "bdc_log_q")) return rs;
    const int64_t want = (H->k >= 1) ? (1ll << (H->k - 1)) : 1;
    if (nq != want) return fail(BDC_ERR_ARG, "bdc_log_q: %lld slots, expected 2^(k-1) = %lld", (long long)nq, (long long)want);
    if (!H->p_set) return fail(BDC_ERR_STATE, "bdc_log_q: no distribution set");
    BDC_CUDA_TRY(cudaSetDevice(H->device));
    bdc_status rc = engine_log_q(H);
    if (rc != BDC_OK) return rc;
    BDC_CUDA_TRY(cudaMemcpyAsync(lnq, H->d_lnq, sizeof(double) * nq, cudaMemcpyDeviceToHost, H->stream));
    BDC_CUDA_TRY(cudaStreamSynchronize(H->stream));
    return BDC_OK;
}

static bdc_status divergence_common(bdc_handle_t H, const double* lnq, int64_t R, bool with_lnp, double* out) {
    if (R != H->R) return fail(BDC_ERR_ARG, "size mismatch: %lld for %lld representatives", (long long)R, (long long)H->R);
    if (!H->p_set) return fail(BDC_ERR_STATE, "no distribution set");
    BDC_CUDA_TRY(cudaSetDevice(H->device));
    bdc_status rc;
    if (lnq) {
        const int64_t nq = (H->k >= 1) ? (1ll << (H->k - 1)) : 1;
        BDC_CUDA_TRY(cudaMemcpyAsync(H->d_lnq, lnq, sizeof(double) * nq, cudaMemcpyHostToDevice, H->stream));
    } else {
        rc = engine_log_q(H);
        if (rc != BDC_OK) return rc;
    }
    rc = engine_divergence(H);  // D per rep into H->d_d from H->d_lnq
    if (rc != BDC_OK) return rc;
    const double* src = H->d_d;
    if (with_lnp) {
        const double* p = nullptr;
        rc = engine_current_p(H, &p);
        if (rc != BDC_OK) return rc;
        BDC_CUDA_TRY(launch_logw(H->n, H->d_reps, H->R, p, H->d_d, H->d_logw, H->stream));
        src = H->d_logw;
    }
    BDC_CUDA_TRY(cudaMemcpyAsync(out, src, sizeof(double) * R, cudaMemcpyDeviceToHost, H->stream));
    BDC_CUDA_TRY(cudaStreamSynchronize(H->stream));
    return BDC_OK;
}

bdc_status bdc_log_w(bdc_handle_t H, const double* lnq, double* logw, int64_t R) {
    if (!H || !logw) return fail(BDC_ERR_ARG, "bdc_log_w: NULL argument");
    if (bdc_status rs = refuse_sharded(H, "bdc_log_w")) return rs;
    return divergence_common(H, lnq, R, true, logw);
}

bdc_status bdc_divergence(bdc_handle_t H, const double* lnq, double* d, int64_t R) {
    if (!H || !d) return fail(BDC_ERR_ARG, "bdc_divergence: NULL argument");
    if (bdc_status rs = refuse_sharded(H, "bdc_divergence")) return rs;
    return divergence_common(H, lnq, R, false, d);
}

bdc_status bdc_rate(bdc_handle_t H, double* rate_nats) {
    if (!H || !rate_nats) return fail(BDC_ERR_ARG, "bdc_rate: NULL argument");
    if (bdc_status rs = refuse_sharded(H, "bdc_rate")) return rs;
    if (!H->p_set) return fail(BDC_ERR_STATE, "bdc_rate: no distribution set");
    BDC_CUDA_TRY(cudaSetDevice(H->device));
    bdc_status rc = engine_log_q(H);
    if (rc != BDC_OK) return rc;
    rc = engine_divergence(H);
    if (rc != BDC_OK) return rc;
    const double* p = nullptr;
    rc = engine_current_p(H, &p);
    if (rc != BDC_OK) return rc;
    BDC_CUDA_TRY(launch_rate(H->n, H->d_reps, H->R, p, H->d_d, H->d_red, H->nb_upd, H->d_scalar, H->stream));
    BDC_CUDA_TRY(cudaMemcpyAsync(rate_nats, H->d_scalar, sizeof(double), cudaMemcpyDeviceToHost, H->stream));
    BDC_CUDA_TRY(cudaStreamSynchronize(H->stream));
    return BDC_OK;
}

bdc_status bdc_max_deviation(bdc_handle_t H, const double* p, const double* pb, int64_t R, double* mx) {
    if (!H || !p || !pb || !mx) return fail(BDC_ERR_ARG, "bdc_max_deviation: NULL argument");
    if (R != H->R) return fail(BDC_ERR_ARG, "bdc_max_deviation: size mismatch");
    BDC_CUDA_TRY(cudaSetDevice(H->device));
    // d_logw and d_d are scratch here
    BDC_CUDA_TRY(cudaMemcpyAsync(H->d_logw, p, sizeof(double) * R, cudaMemcpyHostToDevice, H->stream));
    BDC_CUDA_TRY(cudaMemcpyAsync(H->d_d, pb, sizeof(double) * R, cudaMemcpyHostToDevice, H->stream));
    BDC_CUDA_TRY(launch_max_dev(H->d_logw, H->d_d, R, H->d_red, H->nb_upd, H->d_scalar, H->stream));
    BDC_CUDA_TRY(cudaMemcpyAsync(mx, H->d_scalar, sizeof(double), cudaMemcpyDeviceToHost, H->stream));
    BDC_CUDA_TRY(cudaStreamSynchronize(H->stream));
    return BDC_OK;
}

bdc_status bdc_counts(bdc_handle_t H, const uint32_t* xs, const uint32_t* ys, int64_t npairs, uint32_t* out) {
    if (!H || (npairs > 0 && (!xs || !ys || !out)) || npairs < 0)
        return fail(BDC_ERR_ARG, "bdc_counts: bad arguments");
    if (npairs == 0) return BDC_OK;
    BDC_CUDA_TRY(cudaSetDevice(H->device));
    const uint32_t xmask = low_mask(H->n), ymask = low_mask(H->k);
    for (int64_t i = 0; i < npairs; ++i)
        if ((xs[i] & ~xmask) || (ys[i] & ~ymask))
            return fail(BDC_ERR_ARG, "bdc_counts: pair %lld (x=%u, y=%u) out of range for n=%d k=%d",
                        (long long)i, xs[i], ys[i], H->n, H->k);
    uint32_t *dx = nullptr, *dy = nullptr, *dout = nullptr;
    const size_t bytes = sizeof(uint32_t) * npairs;
    bdc_status rc = BDC_OK;
    if (cudaMalloc(&dx, bytes) != cudaSuccess || cudaMalloc(&dy, bytes) != cudaSuccess ||
        cudaMalloc(&dout, bytes) != cudaSuccess) {
        rc = fail(BDC_ERR_CUDA, "bdc_counts: cudaMalloc failed");
    } else if (cudaMemcpyAsync(dx, xs, bytes, cudaMemcpyHostToDevice, H->stream) != cudaSuccess ||
               cudaMemcpyAsync(dy, ys, bytes, cudaMemcpyHostToDevice, H->stream) != cudaSuccess ||
               launch_count_pairs(H->s, H->A, H->B, dx, dy, npairs, dout, H->stream) != cudaSuccess ||
               cudaMemcpyAsync(out, dout, bytes, cudaMemcpyDeviceToHost, H->stream) != cudaSuccess ||
               cudaStreamSynchronize(H->stream) != cudaSuccess) {
        rc = fail(BDC_ERR_CUDA, "bdc_counts: %s", cudaGetErrorString(cudaGetLastError()));
    }
    cudaFree(dx);
    cudaFree(dy);
    cudaFree(dout);
    return rc;
}

bdc_status bdc_work(bdc_handle_t H, int64_t* nonzero_pairs, int* split_terms) {
    if (!H) return fail(BDC_ERR_ARG, "bdc_work: NULL handle");
    if (nonzero_pairs) *nonzero_pairs = H->nonzero_pairs;
    if (split_terms) *split_terms = H->s.jhi - H->s.jlo + 1;
    return BDC_OK;
}

bdc_status bdc_profile(bdc_handle_t H, int iters, bdc_profile_t* out) {
    if (!H || !out || iters < 1) return fail(BDC_ERR_ARG, "bdc_profile: bad arguments");
    if (bdc_status rs = refuse_sharded(H, "bdc_profile")) return rs;
    if (!H->p_set) return fail(BDC_ERR_STATE, "bdc_profile: no distribution set");
    BDC_CUDA_TRY(cudaSetDevice(H->device));
    return engine_profile(H, iters, out);
}

bdc_status bdc_set_stream(bdc_handle_t H, void* stream) {
    if (!H) return fail(BDC_ERR_ARG, "bdc_set_stream: NULL handle");
    BDC_CUDA_TRY(cudaSetDevice(H->device));
    BDC_CUDA_TRY(cudaStreamSynchronize(H->stream));
    H->stream = stream ? (cudaStream_t)stream : H->own_stream;
    return BDC_OK;
}

bdc_status bdc_generate_cache(int n, int k, int device, uint32_t* out) {
    if (!out || n < 0 || k < 0 || n > kMaxN || k > kMaxN || n + k > 34)
        return fail(BDC_ERR_ARG, "bdc_generate_cache: need 0 <= n, k and n + k <= 34");
    if (cudaSetDevice(device) != cudaSuccess) return fail(BDC_ERR_CUDA, "cudaSetDevice(%d) failed", device);
    const size_t bytes = sizeof(uint32_t) << (n + k);
    uint32_t* d = nullptr;
    if (cudaMalloc(&d, bytes) != cudaSuccess) return fail(BDC_ERR_NOMEM, "bdc_generate_cache: cudaMalloc(%zu) failed", bytes);
    bdc_status rc = BDC_OK;
    if (launch_gen_cache(n, k, d, 0) != cudaSuccess ||
        cudaMemcpy(out, d, bytes, cudaMemcpyDeviceToHost) != cudaSuccess)
        rc = fail(BDC_ERR_CUDA, "bdc_generate_cache: %s", cudaGetErrorString(cudaGetLastError()));
    cudaFree(d);
    return rc;
}

}  // extern "C"
