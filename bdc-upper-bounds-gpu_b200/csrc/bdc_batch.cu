// bdc_batch.cu -- many BA instances (different (n,k) and starting
// distributions) iterated together from one captured CUDA graph.
//
// No counterpart in the reference, which runs one (n,k) per process
// (backend/BAA.cu:3-7 keeps its tables in device globals).  Here each
// instance is an ordinary handle (its own tables, tuned tile shapes and
// iterate); the batch captures kBatchIters iterations of every instance, each
// on its own branch forked from one origin stream, into a single graph and
// replays it.  An instance whose stopping test has fired turns its later
// kernels into no-ops through its device done flag, so the others go on.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "bdc_engine.cuh"

struct bdc_batch {
    std::vector<bdc_handle*> hs;
    int device = 0;
    cudaStream_t origin = nullptr;  // the batch's own stream: captures run here
    cudaStream_t launch = nullptr;  // where iterations are queued (origin unless set)
    std::vector<cudaStream_t> lanes;
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> joins;
    cudaGraphExec_t exec = nullptr;
    double a = 0.0;
    cudaGraphExec_t acc_exec = nullptr;  // accelerated steps of every instance (bdc_batch_accelerate)
    double acc_eta = 0.0;
};

namespace bdc {

constexpr int kBatchIters = 8;

static void batch_free(bdc_batch* B) {
    if (B->exec) cudaGraphExecDestroy(B->exec);
    if (B->acc_exec) cudaGraphExecDestroy(B->acc_exec);
    for (auto s : B->lanes) cudaStreamDestroy(s);
    for (auto e : B->joins) cudaEventDestroy(e);
    if (B->fork) cudaEventDestroy(B->fork);
    if (B->origin) cudaStreamDestroy(B->origin);
    delete B;
}

// kBatchIters iterations of every instance, one branch per instance
static bdc_status batch_capture(bdc_batch* B, double a) {
    if (B->exec && B->a == a) return BDC_OK;
    if (B->exec) {
        cudaGraphExecDestroy(B->exec);
        B->exec = nullptr;
    }
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(B->origin, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) e = cudaEventRecord(B->fork, B->origin);
    for (size_t i = 0; i < B->hs.size() && e == cudaSuccess; ++i) {
        bdc_handle* H = B->hs[i];
        e = cudaStreamWaitEvent(B->lanes[i], B->fork, 0);
        cudaStream_t keep = H->stream;
        H->stream = B->lanes[i];
        for (int it = 0; it < kBatchIters && e == cudaSuccess; ++it) e = engine_enqueue_iteration(H, a);
        H->stream = keep;
        if (e == cudaSuccess) e = cudaEventRecord(B->joins[i], B->lanes[i]);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(B->origin, B->joins[i], 0);
    }
    cudaError_t e2 = cudaStreamEndCapture(B->origin, &g);
    if (e == cudaSuccess) e = e2;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&B->exec, g, 0);
    if (g) cudaGraphDestroy(g);
    BDC_CUDA_TRY(e);
    B->a = a;
    return BDC_OK;
}

// kAccBatchSteps accelerated steps of every instance, one branch per instance
constexpr int kAccBatchSteps = 8;

static bdc_status batch_capture_acc(bdc_batch* B, double eta) {
    if (B->acc_exec && B->acc_eta == eta) return BDC_OK;
    // every instance's snapshot vectors exist before its steps are captured
    for (auto* H : B->hs) {
        bdc_status rc = factored_acc_buffers(H);
        if (rc != BDC_OK) return rc;
    }
    if (B->acc_exec) {
        cudaGraphExecDestroy(B->acc_exec);
        B->acc_exec = nullptr;
    }
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(B->origin, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) e = cudaEventRecord(B->fork, B->origin);
    for (size_t i = 0; i < B->hs.size() && e == cudaSuccess; ++i) {
        bdc_handle* H = B->hs[i];
        e = cudaStreamWaitEvent(B->lanes[i], B->fork, 0);
        cudaStream_t keep = H->stream;
        H->stream = B->lanes[i];
        if (e == cudaSuccess) e = factored_enqueue_acc_steps(H, kAccBatchSteps, eta);
        H->stream = keep;
        if (e == cudaSuccess) e = cudaEventRecord(B->joins[i], B->lanes[i]);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(B->origin, B->joins[i], 0);
    }
    cudaError_t e2 = cudaStreamEndCapture(B->origin, &g);
    if (e == cudaSuccess) e = e2;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&B->acc_exec, g, 0);
    if (g) cudaGraphDestroy(g);
    BDC_CUDA_TRY(e);
    B->acc_eta = eta;
    return BDC_OK;
}

}  // namespace bdc

using namespace bdc;

extern "C" {

bdc_status bdc_batch_create(bdc_handle_t* handles, int count, bdc_batch_t* out) {
    if (!handles || count < 1 || !out) return fail(BDC_ERR_ARG, "bdc_batch_create: need count >= 1 handles");
    *out = nullptr;
    bdc_batch* B = new bdc_batch();
    B->device = handles[0] ? handles[0]->device : 0;
    for (int i = 0; i < count; ++i) {
        if (!handles[i]) {
            batch_free(B);
            return fail(BDC_ERR_ARG, "bdc_batch_create: handle %d is NULL", i);
        }
        if (handles[i]->shard_world > 1) {
            batch_free(B);
            return fail(BDC_ERR_STATE, "bdc_batch_create: handle %d holds a shard of the rows", i);
        }
        if (handles[i]->device != B->device) {
            batch_free(B);
            return fail(BDC_ERR_ARG, "bdc_batch_create: handles on different devices");
        }
        for (int j = 0; j < i; ++j)
            if (handles[j] == handles[i]) {
                batch_free(B);
                return fail(BDC_ERR_ARG, "bdc_batch_create: handle %d appears twice", i);
            }
        B->hs.push_back(handles[i]);
    }
    cudaError_t e = cudaSetDevice(B->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&B->origin, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&B->fork, cudaEventDisableTiming);
    B->lanes.resize(count, nullptr);
    B->joins.resize(count, nullptr);
    for (int i = 0; i < count && e == cudaSuccess; ++i) {
        e = cudaStreamCreateWithFlags(&B->lanes[i], cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&B->joins[i], cudaEventDisableTiming);
    }
    if (e != cudaSuccess) {
        batch_free(B);
        return fail(BDC_ERR_CUDA, "bdc_batch_create: %s", cudaGetErrorString(e));
    }
    B->launch = B->origin;
    *out = B;
    return BDC_OK;
}

bdc_status bdc_batch_set_stream(bdc_batch_t B, void* stream) {
    if (!B) return fail(BDC_ERR_ARG, "bdc_batch_set_stream: NULL batch");
    B->launch = stream ? (cudaStream_t)stream : B->origin;
    return BDC_OK;
}

bdc_status bdc_batch_destroy(bdc_batch_t B) {
    if (!B) return BDC_OK;
    BDC_CUDA_TRY(cudaSetDevice(B->device));
    cudaStreamSynchronize(B->launch);
    cudaStreamSynchronize(B->origin);
    batch_free(B);
    return BDC_OK;
}

bdc_status bdc_batch_iterate(bdc_batch_t B, int64_t max_iters, double a, bdc_stats* stats) {
    if (!B || max_iters < 0) return fail(BDC_ERR_ARG, "bdc_batch_iterate: bad arguments");
    BDC_CUDA_TRY(cudaSetDevice(B->device));
    const size_t N = B->hs.size();
    for (auto* H : B->hs)
        if (!H->p_set) return fail(BDC_ERR_STATE, "bdc_batch_iterate: an instance has no distribution set");
    for (auto* H : B->hs) {
        BDC_CUDA_TRY(cudaStreamSynchronize(H->stream));
        BDC_CUDA_TRY(cudaMemsetAsync(&H->d_st->done, 0, sizeof(int), B->launch));
        BDC_CUDA_TRY(cudaMemcpyAsync(H->h_st, H->d_st, sizeof(DevState), cudaMemcpyDeviceToHost, B->launch));
    }
    BDC_CUDA_TRY(cudaStreamSynchronize(B->launch));
    // Each instance runs to its own target: one interrupted by a re-scale
    // lags the others, and one that reached its target is parked (done = 1,
    // which the kernels read as "skip") so that the shared graph cannot
    // take it past max_iters.
    std::vector<long long> it0(N), target(N);
    std::vector<char> parked(N, 0);
    for (size_t i = 0; i < N; ++i) {
        it0[i] = B->hs[i]->h_st->iter;
        target[i] = it0[i] + max_iters;
    }
    static const int kOne = 1, kZero = 0;
    int64_t chunk = 1;
    for (int guard = 0; guard < 1000000; ++guard) {
        int64_t minrem = INT64_MAX;
        bool any = false;
        for (size_t i = 0; i < N; ++i) {
            bdc_handle* H = B->hs[i];
            if (H->h_st->done) continue;
            const int64_t rem = target[i] - H->h_st->iter;
            if (rem <= 0) {
                BDC_CUDA_TRY(cudaMemcpyAsync(&H->d_st->done, &kOne, sizeof(int), cudaMemcpyHostToDevice, B->launch));
                H->h_st->done = 1;
                parked[i] = 1;
                continue;
            }
            any = true;
            minrem = std::min(minrem, rem);
        }
        if (!any) break;
        const int64_t c = std::min<int64_t>(chunk, minrem);
        const int64_t ng = c / kBatchIters;
        if (ng > 0) {
            bdc_status rc = batch_capture(B, a);
            if (rc != BDC_OK) return rc;
            for (int64_t g = 0; g < ng; ++g) BDC_CUDA_TRY(cudaGraphLaunch(B->exec, B->launch));
        }
        for (int64_t r = ng * kBatchIters; r < c; ++r)
            for (auto* H : B->hs) {
                if (H->h_st->done) continue;
                cudaStream_t keep = H->stream;
                H->stream = B->launch;
                cudaError_t e = engine_enqueue_iteration(H, a);
                H->stream = keep;
                BDC_CUDA_TRY(e);
            }
        for (auto* H : B->hs)
            BDC_CUDA_TRY(cudaMemcpyAsync(H->h_st, H->d_st, sizeof(DevState), cudaMemcpyDeviceToHost, B->launch));
        BDC_CUDA_TRY(cudaStreamSynchronize(B->launch));
        for (auto* H : B->hs) {
            if (!H->h_st->error) continue;
            if (H->engine != BDC_ENGINE_FACTORED)
                return fail(BDC_ERR_NUMERIC, "bdc_batch_iterate: device error %d", H->h_st->error);
            cudaStream_t keep = H->stream;
            H->stream = B->launch;
            bdc_status rc = factored_recover(H, a);  // finishes the interrupted iteration
            H->stream = keep;
            if (rc != BDC_OK) return rc;
            BDC_CUDA_TRY(cudaMemcpyAsync(H->h_st, H->d_st, sizeof(DevState), cudaMemcpyDeviceToHost, B->launch));
            BDC_CUDA_TRY(cudaStreamSynchronize(B->launch));
        }
        if (chunk < 256) chunk *= 2;
    }
    // un-park: the handles are left as a single iterate would leave them
    for (size_t i = 0; i < N; ++i)
        if (parked[i]) {
            BDC_CUDA_TRY(cudaMemcpyAsync(&B->hs[i]->d_st->done, &kZero, sizeof(int), cudaMemcpyHostToDevice, B->launch));
            B->hs[i]->h_st->done = 0;
        }
    BDC_CUDA_TRY(cudaStreamSynchronize(B->launch));
    if (stats) {
        const double ln2 = 0.69314718055994530942;
        for (size_t i = 0; i < N; ++i) {
            const DevState* s = B->hs[i]->h_st;
            bdc_stats& o = stats[i];
            o.iters = s->iter - it0[i];
            o.total_iters = s->iter;
            o.mx = s->mx;
            o.upper_bound = s->max_d / ln2;
            o.rate = s->rate / ln2;
            o.lse = s->lse / ln2;
            o.best_upper_bound = s->best_ub / ln2;
            o.best_rate = s->best_rate / ln2;
            o.converged = s->done;
        }
    }
    return BDC_OK;
}

bdc_status bdc_batch_accelerate(bdc_batch_t B, int64_t max_evals, double gap_bits, bdc_stats* stats,
                                double* seconds) {
    if (!B || max_evals < 0) return fail(BDC_ERR_ARG, "bdc_batch_accelerate: bad arguments");
    BDC_CUDA_TRY(cudaSetDevice(B->device));
    const size_t N = B->hs.size();
    const double ln2 = 0.69314718055994530942;
    for (auto* H : B->hs) {
        if (!H->p_set) return fail(BDC_ERR_STATE, "bdc_batch_accelerate: an instance has no distribution set");
        if (H->engine != BDC_ENGINE_FACTORED)
            return fail(BDC_ERR_UNSUPPORTED, "bdc_batch_accelerate: every instance needs the factored engine");
    }
    const double eta = factored_acc_eta();
    // a target below the support switch: the batched momentum phase runs to
    // the switch, then each instance's support phases finish (n <= 26)
    bool support = gap_bits > 0.0 && gap_bits < kSupportSwitchBits;
    for (auto* H : B->hs) support = support && H->n <= 26;
    const double phase_gap = support ? kSupportSwitchBits : gap_bits;
    std::vector<long long> it0(N);
    std::vector<double> sec(N, -1.0);
    std::vector<char> fin(N, 0);
    bdc_status rc = batch_capture_acc(B, eta);
    if (rc != BDC_OK) return rc;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    BDC_CUDA_TRY(cudaEventCreate(&e0));
    BDC_CUDA_TRY(cudaEventCreate(&e1));
    // start: the plain first step where the iterate still carries the
    // caller's exact zeros, then each instance's snapshots and device stop
    for (auto* H : B->hs) BDC_CUDA_TRY(cudaStreamSynchronize(H->stream));
    BDC_CUDA_TRY(cudaEventRecord(e0, B->launch));
    for (size_t i = 0; i < N; ++i) {
        bdc_handle* H = B->hs[i];
        cudaStream_t keep = H->stream;
        H->stream = B->launch;
        rc = BDC_OK;
        cudaError_t ce = cudaMemsetAsync(&H->d_st->done, 0, sizeof(int), B->launch);
        if (ce == cudaSuccess) ce = cudaMemcpyAsync(H->h_st, H->d_st, sizeof(DevState), cudaMemcpyDeviceToHost, B->launch);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(B->launch);
        if (ce != cudaSuccess) rc = fail(BDC_ERR_CUDA, "bdc_batch_accelerate: %s", cudaGetErrorString(ce));
        it0[i] = H->h_st->iter;
        if (rc == BDC_OK && H->h_st->iter == 0 && max_evals > 0) rc = factored_iterate(H, 1, -INFINITY, nullptr);
        if (rc == BDC_OK) rc = factored_acc_start(H, phase_gap);
        H->stream = keep;
        if (rc != BDC_OK) return rc;
    }
    static const int kOne = 1;
    for (int guard = 0; guard < 10000000; ++guard) {
        // park the instances that are finished or out of evaluations
        bool any = false;
        for (size_t i = 0; i < N; ++i) {
            bdc_handle* H = B->hs[i];
            if (fin[i]) continue;
            if (H->h_st->done || H->h_st->iter - it0[i] >= max_evals) {
                fin[i] = 1;
                if (!H->h_st->done) {
                    BDC_CUDA_TRY(cudaMemcpyAsync(&H->d_st->done, &kOne, sizeof(int), cudaMemcpyHostToDevice, B->launch));
                    H->h_st->done = 1;
                }
                continue;
            }
            any = true;
        }
        if (!any) break;
        BDC_CUDA_TRY(cudaGraphLaunch(B->acc_exec, B->launch));
        BDC_CUDA_TRY(cudaEventRecord(e1, B->launch));
        for (auto* H : B->hs)
            BDC_CUDA_TRY(cudaMemcpyAsync(H->h_st, H->d_st, sizeof(DevState), cudaMemcpyDeviceToHost, B->launch));
        BDC_CUDA_TRY(cudaStreamSynchronize(B->launch));
        float ms = 0.f;
        BDC_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
        for (size_t i = 0; i < N; ++i) {
            bdc_handle* H = B->hs[i];
            if (H->h_st->error) {
                // an exp shift out of range finishes by re-scaling; any other
                // device error is returned
                cudaStream_t keep = H->stream;
                H->stream = B->launch;
                bdc_status r2 = factored_recover(H, -INFINITY);
                H->stream = keep;
                if (r2 != BDC_OK) return r2;
                BDC_CUDA_TRY(cudaMemcpyAsync(H->h_st, H->d_st, sizeof(DevState), cudaMemcpyDeviceToHost, B->launch));
                BDC_CUDA_TRY(cudaStreamSynchronize(B->launch));
            }
            if (!fin[i] && sec[i] < 0 && (H->h_st->best_ub - H->h_st->best_rate) / ln2 < phase_gap) sec[i] = ms * 1e-3;
        }
    }
    for (auto* H : B->hs) BDC_CUDA_TRY(cudaMemsetAsync(&H->d_st->done, 0, sizeof(int), B->launch));
    BDC_CUDA_TRY(cudaStreamSynchronize(B->launch));
    // the support phases, instance by instance on the launch stream; an
    // instance's time is its momentum phase in the batch plus its own
    // support phases
    std::vector<bdc_stats> sup(N);
    std::vector<char> used_sup(N, 0);
    std::vector<long long> mom(N);
    for (size_t i = 0; i < N; ++i) mom[i] = B->hs[i]->h_st->iter - it0[i];  // momentum-phase evaluations
    if (support) {
        for (size_t i = 0; i < N; ++i) {
            bdc_handle* H = B->hs[i];
            if (sec[i] < 0) continue;  // the momentum phase did not reach the switch
            cudaStream_t keep = H->stream;
            H->stream = B->launch;
            BDC_CUDA_TRY(cudaEventRecord(e0, B->launch));
            bdc_status r2 = solve_impl(H, gap_bits, max_evals, &sup[i], 2);
            BDC_CUDA_TRY(cudaEventRecord(e1, B->launch));
            H->stream = keep;
            if (r2 != BDC_OK) return r2;
            BDC_CUDA_TRY(cudaEventSynchronize(e1));
            float ms = 0.f;
            BDC_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
            used_sup[i] = 1;
            sec[i] = sup[i].converged ? sec[i] + ms * 1e-3 : -1.0;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    for (size_t i = 0; i < N; ++i) {
        const DevState* s = B->hs[i]->h_st;
        if (used_sup[i]) {
            if (stats) {
                stats[i] = sup[i];
                stats[i].iters += mom[i];  // the batched momentum evaluations too
            }
            if (seconds) seconds[i] = sec[i];
            continue;
        }
        if (stats) {
            bdc_stats& o = stats[i];
            o.iters = s->iter - it0[i];
            o.total_iters = s->iter;
            o.mx = s->mx;
            o.upper_bound = s->max_d / ln2;
            o.rate = s->rate / ln2;
            o.lse = s->lse / ln2;
            o.best_upper_bound = s->best_ub / ln2;
            o.best_rate = s->best_rate / ln2;
            o.converged = (s->best_ub - s->best_rate) / ln2 < gap_bits;
        }
        if (seconds) seconds[i] = sec[i];
    }
    return BDC_OK;
}

}  // extern "C"
