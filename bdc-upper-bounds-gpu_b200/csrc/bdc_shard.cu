// bdc_shard.cu -- one rank's share of a BA iteration on the count engine, for
// BA sharded by input strings over several GPUs (no counterpart in the
// reference, which runs one (n,k) on one GPU: backend/main_BAA.cu:39-131).
//
// Rank r owns the representatives [r0, r1) and only ever touches p there.
// One iteration is four calls with three exchanges between them:
//
//   bdc_shard_q            partial sums acc_r[y] = sum_{x in shard} |O(x)| p(x) N(x,y)
//   -- all-reduce (sum) of acc over ranks: 2^k doubles --
//   bdc_shard_set_q        ln q from the summed acc (orbit fold, as one CTA partial)
//   bdc_shard_update_begin D pass and logW = ln p + D on the shard; local shift
//                          s_r = max logW, Z_r = sum |O| exp(logW - s_r), max D,
//                          sum |O| p D, input-zero flag
//   -- all-reduce of S = max s_r, then Z = sum Z_r exp(s_r - S), max D, rate --
//   bdc_shard_update_end   p' = exp(logW - s_r) / exp(ln Z + S - s_r) on the
//                          shard, local mx = max log2 p'/p
//   -- all-reduce (max) of mx: the stopping statistic --
//
// The q and D passes and the update are the single-GPU kernels on a
// sub-range of the representatives.  Every call makes the handle's device
// current on the calling thread (as every other handle call does).  After a
// sharded iteration the handle's own statistics (its last bound, rate and mx)
// describe its shard, not the whole problem; its best-bound trackers are left
// as the handle's own iterations set them.
#include "bdc_engine.cuh"

namespace bdc {

// out[y] = sum over the nparts rows of part (fixed order)
__global__ void k_sum_rows(const double* __restrict__ part, int nparts, int ny, double* __restrict__ out) {
    for (int y = blockIdx.x * blockDim.x + threadIdx.x; y < ny; y += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int c = 0; c < nparts; ++c) s += part[(int64_t)c * ny + y];
        out[y] = s;
    }
}

static bdc_status shard_check(bdc_handle* H, int64_t r0, int64_t r1, const char* what) {
    if (!H) return fail(BDC_ERR_ARG, "%s: NULL handle", what);
    if (H->engine != BDC_ENGINE_COUNT) return fail(BDC_ERR_UNSUPPORTED, "%s: needs the count engine", what);
    if (!H->p_set) return fail(BDC_ERR_STATE, "%s: no distribution set", what);
    if (r0 < 0 || r1 <= r0 || r1 > H->R)
        return fail(BDC_ERR_ARG, "%s: representative range [%lld, %lld) outside [0, %lld)", what, (long long)r0,
                    (long long)r1, (long long)H->R);
    BDC_CUDA_TRY(cudaSetDevice(H->device));
    if (!H->d_shard) {
        BDC_CUDA_TRY(cudaMalloc(&H->d_shard, sizeof(double) << H->k));
        H->bytes += sizeof(double) << H->k;
    }
    return BDC_OK;
}

static CountLaunch shard_launch(bdc_handle* H, int64_t r0, int64_t r1) {
    CountLaunch L = count_launch(H);
    L.reps = H->d_reps + r0;
    L.R = r1 - r0;
    return L;
}

static UpdateLaunch shard_update(bdc_handle* H, int64_t r0, int64_t r1) {
    UpdateLaunch U = update_launch(H, -INFINITY);
    U.reps = H->d_reps + r0;
    U.R = r1 - r0;
    U.p0 = H->d_p[0] + r0;
    U.p1 = H->d_p[1] + r0;
    U.d = H->d_d + r0;
    U.logw = H->d_logw + r0;
    return U;
}

static bdc_status pull_state(bdc_handle* H) {
    BDC_CUDA_TRY(cudaMemcpyAsync(H->h_st, H->d_st, sizeof(DevState), cudaMemcpyDeviceToHost, H->stream));
    BDC_CUDA_TRY(cudaStreamSynchronize(H->stream));
    return BDC_OK;
}

}  // namespace bdc

using namespace bdc;

extern "C" {

bdc_status bdc_shard_q(bdc_handle_t H, int64_t r0, int64_t r1, double* acc, int64_t ny) {
    bdc_status rc = shard_check(H, r0, r1, "bdc_shard_q");
    if (rc != BDC_OK) return rc;
    if (!acc || ny != ((int64_t)1 << H->k)) return fail(BDC_ERR_ARG, "bdc_shard_q: acc must hold 2^k values");
    const double* p = H->d_p[H->h_st->cur & 1] + r0;
    BDC_CUDA_TRY(launch_qpass(shard_launch(H, r0, r1), p, p, H->d_qpart, H->d_st, 0));
    const int ny_i = (int)ny;
    k_sum_rows<<<(ny_i + 255) / 256, 256, 0, H->stream>>>(H->d_qpart, H->grid_count, ny_i, H->d_shard);
    BDC_CUDA_TRY(cudaGetLastError());
    BDC_CUDA_TRY(cudaMemcpyAsync(acc, H->d_shard, sizeof(double) * ny, cudaMemcpyDeviceToHost, H->stream));
    BDC_CUDA_TRY(cudaStreamSynchronize(H->stream));
    return BDC_OK;
}

bdc_status bdc_shard_set_q(bdc_handle_t H, const double* acc, int64_t ny) {
    if (!H || !acc) return fail(BDC_ERR_ARG, "bdc_shard_set_q: NULL argument");
    bdc_status rc = shard_check(H, 0, H->R, "bdc_shard_set_q");
    if (rc != BDC_OK) return rc;
    if (ny != ((int64_t)1 << H->k)) return fail(BDC_ERR_ARG, "bdc_shard_set_q: acc must hold 2^k values");
    BDC_CUDA_TRY(cudaMemcpyAsync(H->d_shard, acc, sizeof(double) * ny, cudaMemcpyHostToDevice, H->stream));
    BDC_CUDA_TRY(launch_qfold(H->d_shard, 1, H->k, H->inv_c, H->d_lnq, H->d_q, H->d_st, 0, H->stream));
    BDC_CUDA_TRY(cudaStreamSynchronize(H->stream));
    return BDC_OK;
}

bdc_status bdc_shard_update_begin(bdc_handle_t H, int64_t r0, int64_t r1, double* stats) {
    bdc_status rc = shard_check(H, r0, r1, "bdc_shard_update_begin");
    if (rc != BDC_OK) return rc;
    if (!stats) return fail(BDC_ERR_ARG, "bdc_shard_update_begin: NULL stats");
    // the update's first stage folds its (shard-local) max D and rate into the
    // handle's best-bound trackers; they are put back afterwards, so that they
    // keep describing only the handle's own single-GPU iterations
    rc = pull_state(H);
    if (rc != BDC_OK) return rc;
    const double keep[2] = {H->h_st->best_ub, H->h_st->best_rate};
    BDC_CUDA_TRY(cudaMemsetAsync(&H->d_st->done, 0, sizeof(int), H->stream));
    BDC_CUDA_TRY(launch_dpass(shard_launch(H, r0, r1), H->d_lnq, H->d_h + r0, H->inv_c, H->log_c, H->d_d + r0,
                              H->d_st, 0));
    BDC_CUDA_TRY(launch_update_stages(shard_update(H, r0, r1), 1, 2));
    rc = pull_state(H);
    if (rc != BDC_OK) return rc;
    stats[0] = H->h_st->shift;       // max logW on the shard
    stats[1] = exp(H->h_st->log_z);  // sum |O| exp(logW - shift) on the shard
    stats[2] = H->h_st->max_d;       // max D on the shard (nats)
    stats[3] = H->h_st->rate;        // sum |O| p D on the shard (nats)
    stats[4] = H->h_st->zero_p ? 1.0 : 0.0;
    BDC_CUDA_TRY(cudaMemcpyAsync(&H->d_st->best_ub, &keep[0], sizeof(double), cudaMemcpyHostToDevice, H->stream));
    BDC_CUDA_TRY(cudaMemcpyAsync(&H->d_st->best_rate, &keep[1], sizeof(double), cudaMemcpyHostToDevice, H->stream));
    return pull_state(H);
}

bdc_status bdc_shard_update_end(bdc_handle_t H, int64_t r0, int64_t r1, double log_z, double* mx) {
    bdc_status rc = shard_check(H, r0, r1, "bdc_shard_update_end");
    if (rc != BDC_OK) return rc;
    if (!mx) return fail(BDC_ERR_ARG, "bdc_shard_update_end: NULL mx");
    BDC_CUDA_TRY(cudaMemcpyAsync(&H->d_st->log_z, &log_z, sizeof(double), cudaMemcpyHostToDevice, H->stream));
    BDC_CUDA_TRY(launch_update_stages(shard_update(H, r0, r1), 3, 3));
    rc = pull_state(H);
    if (rc != BDC_OK) return rc;
    *mx = H->h_st->mx;
    return BDC_OK;
}

// ---------------------------------------------- factored engine, rows sharded
static bdc_status fshard_check(bdc_handle* H, const char* what) {
    if (!H) return fail(BDC_ERR_ARG, "%s: NULL handle", what);
    if (H->engine != BDC_ENGINE_FACTORED || !H->fac)
        return fail(BDC_ERR_UNSUPPORTED, "%s: needs a handle from bdc_create_sharded", what);
    if (!H->p_set) return fail(BDC_ERR_STATE, "%s: no distribution set", what);
    BDC_CUDA_TRY(cudaSetDevice(H->device));
    return BDC_OK;
}

bdc_status bdc_fshard_range(bdc_handle_t H, int* row0, int* rows, int64_t* rep_begin, int64_t* rep_end) {
    if (!H || !H->fac || !row0 || !rows || !rep_begin || !rep_end)
        return fail(BDC_ERR_ARG, "bdc_fshard_range: NULL argument or not a factored handle");
    factored_shard_range(H, row0, rows, rep_begin, rep_end);
    return BDC_OK;
}

bdc_status bdc_fshard_q(bdc_handle_t H, double* acc, int64_t ny) {
    bdc_status rc = fshard_check(H, "bdc_fshard_q");
    if (rc != BDC_OK) return rc;
    if (!acc || ny != ((int64_t)1 << H->k)) return fail(BDC_ERR_ARG, "bdc_fshard_q: acc must hold 2^k values");
    return factored_shard_q(H, acc);
}

bdc_status bdc_fshard_d(bdc_handle_t H, const double* acc, int64_t ny, double* part5) {
    bdc_status rc = fshard_check(H, "bdc_fshard_d");
    if (rc != BDC_OK) return rc;
    if (!acc || !part5 || ny != ((int64_t)1 << H->k))
        return fail(BDC_ERR_ARG, "bdc_fshard_d: acc must hold 2^k values, part5 five");
    return factored_shard_d(H, acc, part5);
}

bdc_status bdc_fshard_finish(bdc_handle_t H, const double* part5, double a, bdc_stats* stats) {
    bdc_status rc = fshard_check(H, "bdc_fshard_finish");
    if (rc != BDC_OK) return rc;
    if (!part5) return fail(BDC_ERR_ARG, "bdc_fshard_finish: NULL part5");
    rc = factored_shard_finish(H, part5, a);
    if (rc != BDC_OK) return rc;
    if (stats) {
        const double ln2 = 0.69314718055994530942;
        const DevState* s = H->h_st;
        stats->iters = 1;
        stats->total_iters = s->iter;
        stats->mx = s->mx;
        stats->upper_bound = s->max_d / ln2;
        stats->rate = s->rate / ln2;
        stats->lse = s->lse / ln2;
        stats->best_upper_bound = s->best_ub / ln2;
        stats->best_rate = s->best_rate / ln2;
        stats->converged = s->done;
    }
    return BDC_OK;
}

bdc_status bdc_fshard_get_p(bdc_handle_t H, double* p, int64_t count) {
    bdc_status rc = fshard_check(H, "bdc_fshard_get_p");
    if (rc != BDC_OK) return rc;
    int row0 = 0, rows = 0;
    int64_t i0 = 0, i1 = 0;
    factored_shard_range(H, &row0, &rows, &i0, &i1);
    if (!p || count != i1 - i0) return fail(BDC_ERR_ARG, "bdc_fshard_get_p: %lld slots for %lld representatives",
                                            (long long)count, (long long)(i1 - i0));
    // the dense state of the held rows -> p of their representatives
    BDC_CUDA_TRY(cudaMemsetAsync(H->d_d, 0, sizeof(double) * H->R, H->stream));
    rc = factored_store_p(H, H->d_d);
    if (rc != BDC_OK) return rc;
    BDC_CUDA_TRY(cudaMemcpyAsync(p, H->d_d + i0, sizeof(double) * count, cudaMemcpyDeviceToHost, H->stream));
    BDC_CUDA_TRY(cudaStreamSynchronize(H->stream));
    return BDC_OK;
}

}  // extern "C"
