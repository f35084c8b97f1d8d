// bdc_engine.cu -- handle set-up shared by both engines and the count engine's
// iteration driver.
//
// Set-up replaces load_cache (backend/BAA.cu:183-188) and the canonical list
// (backend/main_BAA.cu:46-50): representatives are compacted on the device,
// the two half-table bundles are built (from cache files or by the device
// generator), and the entropy term h(x) = sum_y W ln W is computed once.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "bdc_engine.cuh"

namespace bdc {

template <typename T>
static cudaError_t dalloc(bdc_handle* H, T** p, size_t count) {
    H->bytes += count * sizeof(T);
    return cudaMalloc((void**)p, count * sizeof(T) + 16);
}

static int mmax_for_high(const Split& s) {
    // stored sub-lengths j of the high half: jlo <= j <= jhi and j < n1
    const int hi = s.jhi < s.n1 - 1 ? s.jhi : s.n1 - 1;
    return (hi >= s.jlo) ? hi : -1;
}

static int mmax_for_low(const Split& s) {
    // stored sub-lengths m = k - j of the low half, m < n2
    const int mlo = s.k - s.jhi, mhi0 = s.k - s.jlo;
    const int hi = mhi0 < s.n2 - 1 ? mhi0 : s.n2 - 1;
    return (hi >= mlo) ? hi : -1;
}

static int bundle_stride(int mmax) {
    const int st = (mmax >= 0) ? (1 << (mmax + 1)) : 8;
    return st < 8 ? 8 : st;
}

// one bundle for half length hlen, from cache files or by the device generator
static bdc_status make_bundle(bdc_handle* H, int hlen, int mmax, uint16_t** rows_out, int* stride_out) {
    const int stride = bundle_stride(mmax);
    const size_t entries = ((size_t)stride) << hlen;
    uint16_t* rows = nullptr;
    BDC_CUDA_TRY(dalloc(H, &rows, entries));
    *rows_out = rows;
    *stride_out = stride;
    if (mmax < 0) {
        BDC_CUDA_TRY(cudaMemsetAsync(rows, 0, entries * sizeof(uint16_t), H->stream));
        return BDC_OK;
    }
    if (H->cache_dir.empty()) {
        BDC_CUDA_TRY(launch_gen_bundle(hlen, mmax, stride, rows, H->stream));
        return BDC_OK;
    }
    // cache_{hlen, m} for m <= mmax: the reference loads every n' <= ceil(n/2),
    // k' < n' (backend/BAA.cu:48-57) but only these two half lengths are read.
    std::vector<uint32_t*> dev(mmax + 1, nullptr);
    std::vector<uint32_t> host;
    int* d_over = nullptr;
    bdc_status rc = BDC_OK;
    if (cudaMalloc(&d_over, sizeof(int)) != cudaSuccess || cudaMemset(d_over, 0, sizeof(int)) != cudaSuccess)
        return fail(BDC_ERR_CUDA, "cudaMalloc of the overflow flag failed");
    for (int m = 0; m <= mmax && rc == BDC_OK; ++m) {
        const size_t cnt = (size_t)1 << (hlen + m);
        host.resize(cnt);
        const std::string path = H->cache_dir + "/cache_" + std::to_string(hlen) + "_" + std::to_string(m);
        rc = bdc_read_cache_file(path.c_str(), hlen, m, host.data());
        if (rc != BDC_OK) break;
        if (cudaMalloc(&dev[m], cnt * sizeof(uint32_t)) != cudaSuccess ||
            cudaMemcpy(dev[m], host.data(), cnt * sizeof(uint32_t), cudaMemcpyHostToDevice) != cudaSuccess)
            rc = fail(BDC_ERR_CUDA, "uploading %s failed", path.c_str());
    }
    if (rc == BDC_OK) {
        if (launch_build_bundle(hlen, mmax, stride, dev.data(), rows, d_over, H->stream) != cudaSuccess ||
            cudaStreamSynchronize(H->stream) != cudaSuccess)
            rc = fail(BDC_ERR_CUDA, "building the half-table bundle failed");
        int over = 0;
        if (rc == BDC_OK && cudaMemcpy(&over, d_over, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
            rc = fail(BDC_ERR_CUDA, "reading the overflow flag failed");
        if (rc == BDC_OK && over)
            rc = fail(BDC_ERR_IO, "a cache_%d_m file holds a count above 65535 (not a subsequence count)", hlen);
    }
    for (auto p : dev)
        if (p) cudaFree(p);
    cudaFree(d_over);
    return rc;
}

int select_engine(int requested, int n, int k) {
    switch (requested) {
        case BDC_ENGINE_COUNT: return BDC_ENGINE_COUNT;
        // FP32 holds the counts exactly only below 2^24: max N(x,y) <= C(n,k)
        // and C(26,13) = 10,400,600 < 2^24 < C(27,13)
        case BDC_ENGINE_COUNT_FP32C: return n <= 26 ? BDC_ENGINE_COUNT_FP32C : -1;
        case BDC_ENGINE_FACTORED: return factored_supports(n, k) ? BDC_ENGINE_FACTORED : -1;
        case BDC_ENGINE_AUTO: return factored_supports(n, k) ? BDC_ENGINE_FACTORED : BDC_ENGINE_COUNT;
        default: return -1;
    }
}

CountLaunch count_launch(const bdc_handle* H) {
    CountLaunch L;
    L.s = H->s;
    L.A = H->Ar;
    L.B = H->B;
    L.reps = H->d_reps;
    L.R = H->R;
    L.grid = H->grid_count;
    L.stream = H->stream;
    L.c32 = H->c32;
    return L;
}

// number of representatives of {id, r, c, rc} on n-bit strings (Burnside)
static int64_t num_reps_of(int n) {
    const int64_t all = 1ll << n;
    const int64_t fixed_r = 1ll << ((n + 1) / 2);
    const int64_t fixed_rc = (n % 2 == 0) ? (1ll << (n / 2)) : 0;
    return (all + fixed_r + fixed_rc) / 4;
}

// The p-independent data of a handle -- the representatives, the half-table
// bundles, the rotated A bundle and h(x) per representative -- is read-only
// after set-up and the same for every handle of one n, k and table source on
// one device (the seeds of a batch, the ranks of a sharded problem on one
// device), so those handles share one set, freed with its last handle.
struct TableSet {
    int device = 0, n = 0, k = 0;
    std::string source;  // the cache directory, empty for the device generator
    int refs = 0;
    uint32_t* reps = nullptr;
    uint16_t *hi = nullptr, *lo = nullptr, *rot = nullptr;
    double* h = nullptr;
    HalfTables A{}, B{}, Ar{};
    int64_t nonzero_pairs = 0;
};
static std::mutex g_tables_mu;
static std::vector<TableSet*> g_tables;

static TableSet* find_tables(const bdc_handle* H) {
    for (TableSet* t : g_tables)
        if (t->device == H->device && t->n == H->n && t->k == H->k && t->source == H->cache_dir) return t;
    return nullptr;
}

static void release_tables(bdc_handle* H) {
    std::lock_guard<std::mutex> lock(g_tables_mu);
    TableSet* t = (TableSet*)H->tables;
    H->tables = nullptr;
    if (!t) {
        // set-up failed before its tables were published: they are the handle's own
        cudaFree(H->d_reps);
        if (H->d_bundle_lo && H->d_bundle_lo != H->d_bundle_hi) cudaFree(H->d_bundle_lo);
        cudaFree(H->d_bundle_hi);
        cudaFree(H->d_bundle_rot);
        cudaFree(H->d_h);
    } else if (--t->refs == 0) {
        cudaFree(t->reps);
        if (t->lo && t->lo != t->hi) cudaFree(t->lo);
        cudaFree(t->hi);
        cudaFree(t->rot);
        cudaFree(t->h);
        g_tables.erase(std::find(g_tables.begin(), g_tables.end(), t));
        delete t;
    }
    H->d_reps = nullptr;
    H->d_bundle_hi = H->d_bundle_lo = H->d_bundle_rot = nullptr;
    H->d_h = nullptr;
}

// the representatives, the half-table bundles and the rotated A bundle of a
// new table set
static bdc_status build_tables(bdc_handle* H, int mA, int mB) {
    const Split& s = H->s;
    const int64_t R = H->R;
    // representatives
    BDC_CUDA_TRY(dalloc(H, &H->d_reps, (size_t)R));
    {
        const size_t sb = build_reps_scratch_bytes(H->n);
        void* scratch = nullptr;
        int64_t* d_cnt = nullptr;
        BDC_CUDA_TRY(cudaMalloc(&scratch, sb));
        BDC_CUDA_TRY(cudaMalloc(&d_cnt, sizeof(int64_t)));
        cudaError_t e = build_reps(H->n, H->d_reps, d_cnt, scratch, sb, H->stream);
        int64_t got = -1;
        if (e == cudaSuccess) e = cudaMemcpyAsync(&got, d_cnt, sizeof(int64_t), cudaMemcpyDeviceToHost, H->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(H->stream);
        cudaFree(scratch);
        cudaFree(d_cnt);
        BDC_CUDA_TRY(e);
        if (got != R) return fail(BDC_ERR_CUDA, "representative count %lld, expected %lld", (long long)got, (long long)R);
    }

    // half tables
    int strideA = 0, strideB = 0;
    bdc_status rc;
    if (s.n1 == s.n2) {
        const int mm = mA > mB ? mA : mB;
        rc = make_bundle(H, s.n1, mm, &H->d_bundle_hi, &strideA);
        if (rc != BDC_OK) return rc;
        H->d_bundle_lo = H->d_bundle_hi;
        strideB = strideA;
        H->A = HalfTables{H->d_bundle_hi, s.n1, mm, strideA};
        H->B = HalfTables{H->d_bundle_lo, s.n2, mm, strideB};
    } else {
        rc = make_bundle(H, s.n1, mA, &H->d_bundle_hi, &strideA);
        if (rc != BDC_OK) return rc;
        rc = make_bundle(H, s.n2, mB, &H->d_bundle_lo, &strideB);
        if (rc != BDC_OK) return rc;
        H->A = HalfTables{H->d_bundle_hi, s.n1, mA, strideA};
        H->B = HalfTables{H->d_bundle_lo, s.n2, mB, strideB};
    }

    // the A bundle rotated for the count passes (their tiles read 2^TB
    // entries of one row at once)
    {
        const size_t cnt = ((size_t)H->A.stride) << H->A.h;
        BDC_CUDA_TRY(cudaMalloc(&H->d_bundle_rot, cnt * sizeof(uint16_t)));
        H->bytes += cnt * sizeof(uint16_t);
        BDC_CUDA_TRY(launch_rotate_bundle(H->A, count_tile_tb(H->k), H->d_bundle_rot, H->stream));
        H->Ar = H->A;
        H->Ar.rows = H->d_bundle_rot;
    }
    return BDC_OK;
}

bdc_status engine_init(bdc_handle* H) {
    BDC_CUDA_TRY(cudaStreamCreateWithFlags(&H->own_stream, cudaStreamNonBlocking));
    H->stream = H->own_stream;
    BDC_CUDA_TRY(cudaDeviceGetAttribute(&H->num_sms, cudaDevAttrMultiProcessorCount, H->device));
    const Split& s = H->s;
    const int64_t R = num_reps_of(H->n);
    H->R = R;

    // the table set is looked up and, when new, built and published under
    // the registry's lock
    std::unique_lock<std::mutex> tables_lock(g_tables_mu);
    TableSet* shared = find_tables(H);

    // memory estimate (the reference checks 95% of free memory with an
    // assert, backend/BAA.cu:31-44, which vanishes under NDEBUG)
    const int mA = mmax_for_high(s), mB = mmax_for_low(s);
    size_t need = 0;
    if (!shared) {
        need += ((size_t)bundle_stride(mA) << s.n1) * 2 * 2;  // and its rotated copy
        if (s.n2 != s.n1) need += ((size_t)bundle_stride(mB) << s.n2) * 2;
        need += (size_t)R * (4 + 8);
    }
    need += (size_t)R * 8 * 4;
    size_t free_b = 0, total_b = 0;
    BDC_CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
    if (need > (size_t)(0.95 * (double)free_b))
        return fail(BDC_ERR_NOMEM, "need about %zu MB of device memory, %zu MB free", need >> 20, free_b >> 20);

    if (shared) {
        ++shared->refs;
        H->tables = shared;
        H->d_reps = shared->reps;
        H->d_bundle_hi = shared->hi;
        H->d_bundle_lo = shared->lo;
        H->d_bundle_rot = shared->rot;
        H->d_h = shared->h;
        H->A = shared->A;
        H->B = shared->B;
        H->Ar = shared->Ar;
        H->nonzero_pairs = shared->nonzero_pairs;
        tables_lock.unlock();
    }

    if (!shared) {
        bdc_status rc = build_tables(H, mA, mB);
        if (rc != BDC_OK) return rc;
    }

    // per-representative vectors and reductions
    for (int b = 0; b < 2; ++b) BDC_CUDA_TRY(dalloc(H, &H->d_p[b], (size_t)R));
    if (!shared) BDC_CUDA_TRY(dalloc(H, &H->d_h, (size_t)R));
    BDC_CUDA_TRY(dalloc(H, &H->d_d, (size_t)R));
    BDC_CUDA_TRY(dalloc(H, &H->d_logw, (size_t)R));
    const size_t nq = (size_t)1 << (H->k >= 1 ? H->k - 1 : 0);
    BDC_CUDA_TRY(dalloc(H, &H->d_lnq, nq));
    BDC_CUDA_TRY(dalloc(H, &H->d_q, nq));
    if (H->c32) {
        BDC_CUDA_TRY(dalloc(H, &H->d_lnq64, nq));
        BDC_CUDA_TRY(dalloc(H, &H->d_d64, (size_t)R));
    }
    const int group = count_group_size(H->k);
    const int cta = count_cta_threads(H->k);
    const int gpc = cta / group > 0 ? cta / group : 1;
    int64_t grid = (R + gpc - 1) / gpc;
    const int64_t gmax = (int64_t)H->num_sms * count_ctas_per_sm(H->k);
    if (grid > gmax) grid = gmax;
    if (grid < 1) grid = 1;
    H->grid_count = (int)grid;
    BDC_CUDA_TRY(dalloc(H, &H->d_qpart, (size_t)grid << H->k));
    int64_t nb = (R + 1023) / 1024;
    if (nb > (int64_t)H->num_sms * 4) nb = (int64_t)H->num_sms * 4;
    if (nb < 1) nb = 1;
    H->nb_upd = (int)nb;
    BDC_CUDA_TRY(dalloc(H, &H->d_red, (size_t)nb * 6));
    BDC_CUDA_TRY(dalloc(H, &H->d_scalar, 8));
    BDC_CUDA_TRY(cudaMalloc(&H->d_st, sizeof(DevState)));
    BDC_CUDA_TRY(cudaMemsetAsync(H->d_st, 0, sizeof(DevState), H->stream));
    BDC_CUDA_TRY(cudaMallocHost(&H->h_st, sizeof(DevState)));
    memset(H->h_st, 0, sizeof(DevState));

    // h(x) = (1/C) sum_y N ln N - ln C, once per table set; the same pass
    // counts the distinct subsequences of every representative
    if (!shared) {
        uint32_t* d_nnz = nullptr;
        BDC_CUDA_TRY(cudaMalloc(&d_nnz, sizeof(uint32_t) * R + 16));
        cudaError_t e = launch_hpass(count_launch(H), H->inv_c, H->log_c, H->d_h, d_nnz);
        std::vector<uint32_t> nnz((size_t)R);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(nnz.data(), d_nnz, sizeof(uint32_t) * R, cudaMemcpyDeviceToHost, H->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(H->stream);
        cudaFree(d_nnz);
        BDC_CUDA_TRY(e);
        int64_t tot = 0;
        for (uint32_t v : nnz) tot += v;
        H->nonzero_pairs = tot;
        // publish the set (every kernel that wrote it has completed)
        TableSet* t = new TableSet();
        t->device = H->device;
        t->n = H->n;
        t->k = H->k;
        t->source = H->cache_dir;
        t->refs = 1;
        t->reps = H->d_reps;
        t->hi = H->d_bundle_hi;
        t->lo = H->d_bundle_lo;
        t->rot = H->d_bundle_rot;
        t->h = H->d_h;
        t->A = H->A;
        t->B = H->B;
        t->Ar = H->Ar;
        t->nonzero_pairs = tot;
        g_tables.push_back(t);
        H->tables = t;
        tables_lock.unlock();
    }

    if (H->engine == BDC_ENGINE_FACTORED) {
        bdc_status rc = factored_init(H);
        if (rc != BDC_OK) return rc;
    }
    if (H->verbose)
        printf("bdc: n=%d k=%d reps=%lld engine=%s tables=%s device bytes=%.1f MB\n", H->n, H->k,
               (long long)R, H->engine == BDC_ENGINE_FACTORED ? "factored" : (H->c32 ? "count-fp32c" : "count"),
               H->cache_dir.empty() ? "generated" : H->cache_dir.c_str(), H->bytes / 1048576.0);
    return BDC_OK;
}

void engine_free(bdc_handle* H) {
    if (H->stream) cudaStreamSynchronize(H->stream);
    solve_pool_release(H);
    if (H->fac) factored_free(H);
    if (H->stream) cudaStreamSynchronize(H->stream);
    release_tables(H);
    for (int b = 0; b < 2; ++b) cudaFree(H->d_p[b]);
    cudaFree(H->d_d);
    cudaFree(H->d_logw);
    cudaFree(H->d_lnq);
    cudaFree(H->d_q);
    cudaFree(H->d_qpart);
    cudaFree(H->d_lnq64);
    cudaFree(H->d_d64);
    cudaFree(H->d_shard);
    cudaFree(H->d_red);
    cudaFree(H->d_scalar);
    cudaFree(H->d_st);
    if (H->h_st) cudaFreeHost(H->h_st);
    if (H->own_stream) cudaStreamDestroy(H->own_stream);
    H->own_stream = nullptr;
    H->stream = nullptr;
}

static bdc_status reset_state(bdc_handle* H) {
    memset(H->h_st, 0, sizeof(DevState));
    H->h_st->best_ub = DBL_MAX;
    H->h_st->best_rate = -DBL_MAX;
    BDC_CUDA_TRY(cudaMemcpyAsync(H->d_st, H->h_st, sizeof(DevState), cudaMemcpyHostToDevice, H->stream));
    BDC_CUDA_TRY(cudaStreamSynchronize(H->stream));
    return BDC_OK;
}

bdc_status engine_after_set_p(bdc_handle* H, int strict_zero) {
    bdc_status rc = reset_state(H);
    if (rc != BDC_OK) return rc;
    H->p_set = true;
    if (H->engine == BDC_ENGINE_FACTORED) {
        rc = factored_load_p(H, strict_zero);
        if (rc != BDC_OK) return rc;
    }
    BDC_CUDA_TRY(cudaStreamSynchronize(H->stream));
    return BDC_OK;
}

bdc_status engine_current_p(bdc_handle* H, const double** p) {
    if (H->engine == BDC_ENGINE_FACTORED) {
        bdc_status rc = factored_store_p(H, H->d_p[0]);
        if (rc != BDC_OK) return rc;
        *p = H->d_p[0];
        return BDC_OK;
    }
    *p = H->d_p[H->h_st->cur & 1];
    return BDC_OK;
}

bdc_status engine_log_q(bdc_handle* H) {
    const double* p = nullptr;
    bdc_status rc = engine_current_p(H, &p);
    if (rc != BDC_OK) return rc;
    const CountLaunch L = count_launch(H);
    BDC_CUDA_TRY(launch_qpass(L, p, p, H->d_qpart, H->d_st, 0));
    BDC_CUDA_TRY(launch_qfold(H->d_qpart, H->grid_count, H->k, H->inv_c, H->d_lnq, H->d_q, H->d_st, 0, H->stream));
    return BDC_OK;
}

bdc_status engine_divergence(bdc_handle* H) {
    const CountLaunch L = count_launch(H);
    BDC_CUDA_TRY(launch_dpass(L, H->d_lnq, H->d_h, H->inv_c, H->log_c, H->d_d, H->d_st, 0));
    return BDC_OK;
}

UpdateLaunch update_launch(const bdc_handle* H, double a) {
    UpdateLaunch U;
    U.n = H->n;
    U.reps = H->d_reps;
    U.R = H->R;
    U.p0 = H->d_p[0];
    U.p1 = H->d_p[1];
    U.d = H->d_d;
    U.logw = H->d_logw;
    U.part = H->d_red;
    U.nblocks = H->nb_upd;
    U.a = a;
    U.st = H->d_st;
    U.stream = H->stream;
    return U;
}

// one count-engine iteration, gated by DevState::done
static cudaError_t enqueue_count_iteration(bdc_handle* H, double a) {
    const CountLaunch L = count_launch(H);
    cudaError_t e = launch_qpass(L, H->d_p[0], H->d_p[1], H->d_qpart, H->d_st, 1);
    if (e == cudaSuccess)
        e = launch_qfold(H->d_qpart, H->grid_count, H->k, H->inv_c, H->d_lnq, H->d_q, H->d_st, 1, H->stream);
    if (e == cudaSuccess) e = launch_dpass(L, H->d_lnq, H->d_h, H->inv_c, H->log_c, H->d_d, H->d_st, 1);
    if (e == cudaSuccess) e = launch_update(update_launch(H, a));
    return e;
}

bdc_status engine_profile(bdc_handle* H, int iters, bdc_profile_t* out) {
    if (H->engine == BDC_ENGINE_FACTORED) return factored_profile(H, iters, out);
    BDC_CUDA_TRY(cudaMemsetAsync(&H->d_st->done, 0, sizeof(int), H->stream));
    cudaEvent_t ev[5];
    for (auto& e : ev) BDC_CUDA_TRY(cudaEventCreate(&e));
    double acc[4] = {0, 0, 0, 0}, tot = 0;
    const CountLaunch L = count_launch(H);
    bdc_status rc = BDC_OK;
    for (int it = 0; it < iters && rc == BDC_OK; ++it) {
        cudaError_t e = cudaEventRecord(ev[0], H->stream);
        if (e == cudaSuccess) e = launch_qpass(L, H->d_p[0], H->d_p[1], H->d_qpart, H->d_st, 1);
        if (e == cudaSuccess) e = cudaEventRecord(ev[1], H->stream);
        if (e == cudaSuccess)
            e = launch_qfold(H->d_qpart, H->grid_count, H->k, H->inv_c, H->d_lnq, H->d_q, H->d_st, 1, H->stream);
        if (e == cudaSuccess) e = cudaEventRecord(ev[2], H->stream);
        if (e == cudaSuccess) e = launch_dpass(L, H->d_lnq, H->d_h, H->inv_c, H->log_c, H->d_d, H->d_st, 1);
        if (e == cudaSuccess) e = cudaEventRecord(ev[3], H->stream);
        if (e == cudaSuccess) {
            UpdateLaunch U = update_launch(H, -INFINITY);
            e = launch_update(U);
        }
        if (e == cudaSuccess) e = cudaEventRecord(ev[4], H->stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(ev[4]);
        if (e != cudaSuccess) {
            rc = fail(BDC_ERR_CUDA, "bdc_profile: %s", cudaGetErrorString(e));
            break;
        }
        float ms;
        for (int j = 0; j < 4; ++j) {
            cudaEventElapsedTime(&ms, ev[j], ev[j + 1]);
            acc[j] += ms;
        }
        cudaEventElapsedTime(&ms, ev[0], ev[4]);
        tot += ms;
    }
    for (auto& e : ev) cudaEventDestroy(e);
    if (rc != BDC_OK) return rc;
    BDC_CUDA_TRY(cudaMemcpyAsync(H->h_st, H->d_st, sizeof(DevState), cudaMemcpyDeviceToHost, H->stream));
    BDC_CUDA_TRY(cudaStreamSynchronize(H->stream));
    out->ms_q = acc[0] / iters;
    out->ms_fold = acc[1] / iters;
    out->ms_d = acc[2] / iters;
    out->ms_update = acc[3] / iters;
    out->ms_iter = tot / iters;
    out->ms_main = out->ms_d;
    out->work_main = (double)H->nonzero_pairs * (double)(H->s.jhi - H->s.jlo + 1);
    out->launches = 6;
    out->iters = iters;
    out->main_kind = 0;
    out->bytes_main = 0.0;
    return BDC_OK;
}

bdc_status engine_bound_error(bdc_handle* H, double* ub_err_bits, double* rate_err_bits) {
    *ub_err_bits = 0.0;
    *rate_err_bits = 0.0;
    if (!H->c32) return BDC_OK;
    BDC_CUDA_TRY(cudaMemcpyAsync(H->h_st, H->d_st, sizeof(DevState), cudaMemcpyDeviceToHost, H->stream));
    BDC_CUDA_TRY(cudaStreamSynchronize(H->stream));
    if (H->h_st->iter == 0) return fail(BDC_ERR_STATE, "bdc_bound_error: no iteration since the distribution was set");
    // the update wrote p' into the other buffer and flipped cur, so the
    // iterate the last D pass used is still in d_p[cur ^ 1]
    const double* pt = H->d_p[(H->h_st->cur ^ 1) & 1];
    CountLaunch L = count_launch(H);
    L.c32 = 0;
    BDC_CUDA_TRY(launch_qpass(L, pt, pt, H->d_qpart, H->d_st, 0));
    BDC_CUDA_TRY(launch_qfold(H->d_qpart, H->grid_count, H->k, H->inv_c, H->d_lnq64, nullptr, H->d_st, 0, H->stream));
    BDC_CUDA_TRY(launch_dpass(L, H->d_lnq64, H->d_h, H->inv_c, H->log_c, H->d_d64, H->d_st, 0));
    BDC_CUDA_TRY(launch_vec_max(H->d_d64, H->R, H->d_red, H->nb_upd, H->d_scalar + 6, H->stream));
    BDC_CUDA_TRY(launch_rate(H->n, H->d_reps, H->R, pt, H->d_d64, H->d_red + H->nb_upd, H->nb_upd, H->d_scalar + 7,
                             H->stream));
    double v[2];
    BDC_CUDA_TRY(cudaMemcpyAsync(v, H->d_scalar + 6, sizeof(v), cudaMemcpyDeviceToHost, H->stream));
    BDC_CUDA_TRY(cudaStreamSynchronize(H->stream));
    const double ln2 = 0.69314718055994530942;
    *ub_err_bits = fabs(H->h_st->max_d - v[0]) / ln2;
    *rate_err_bits = fabs(H->h_st->rate - v[1]) / ln2;
    return BDC_OK;
}

cudaError_t engine_enqueue_iteration(bdc_handle* H, double a) {
    if (H->engine == BDC_ENGINE_FACTORED) return factored_enqueue_iteration(H, a);
    return enqueue_count_iteration(H, a);
}

bdc_status engine_iterate(bdc_handle* H, int64_t max_iters, double a, bdc_stats* stats) {
    if (H->engine == BDC_ENGINE_FACTORED) return factored_iterate(H, max_iters, a, stats);
    BDC_CUDA_TRY(cudaMemsetAsync(&H->d_st->done, 0, sizeof(int), H->stream));
    const long long it0 = H->h_st->iter;
    int64_t remaining = max_iters;
    int64_t chunk = 1;
    while (remaining > 0) {
        const int64_t c = chunk < remaining ? chunk : remaining;
        for (int64_t i = 0; i < c; ++i) BDC_CUDA_TRY(enqueue_count_iteration(H, a));
        BDC_CUDA_TRY(cudaMemcpyAsync(H->h_st, H->d_st, sizeof(DevState), cudaMemcpyDeviceToHost, H->stream));
        BDC_CUDA_TRY(cudaStreamSynchronize(H->stream));
        remaining -= c;
        if (H->h_st->done) break;
        if (chunk < 64) chunk *= 2;
    }
    if (stats) {
        const double ln2 = 0.69314718055994530942;
        stats->iters = H->h_st->iter - it0;
        stats->total_iters = H->h_st->iter;
        stats->mx = H->h_st->mx;
        stats->upper_bound = H->h_st->max_d / ln2;
        stats->rate = H->h_st->rate / ln2;
        stats->lse = H->h_st->lse / ln2;
        stats->best_upper_bound = H->h_st->best_ub / ln2;
        stats->best_rate = H->h_st->best_rate / ln2;
        stats->converged = H->h_st->done;
    }
    return BDC_OK;
}

}  // namespace bdc
