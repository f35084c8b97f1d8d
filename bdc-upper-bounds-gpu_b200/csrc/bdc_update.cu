// bdc_update.cu -- the normalised BA update, the stopping statistic and the
// reported scalars, as three streaming kernels over the representatives.
//
// Reference (Pintz45/BDC-Upper-Bounds-GPU):
//   backend/BAA.cu:590-639   baa_iteration: max logW, exp(logW - max),
//                            sum |O| exp(..), divide (four Thrust passes and a
//                            host round trip of every vector)
//   backend/BAA.cu:916-946   compute_max_deviation: max log2 p' - log2 p
//   backend/BAA.cu:820-913   compute_rate: sum |O| p KL
//   backend/main_BAA.cu:73   the loop runs while (mx >= a)
//
// Here everything stays resident: each kernel streams the R-vectors once,
// reduces per block, and the last block to finish folds the block partials
// in a fixed order (deterministic) into DevState.  DevState::done makes every
// later kernel a no-op once mx < a, so a chunk of iterations can be queued or
// captured in a graph without a host round trip per iteration.
#include <atomic>
#include <cfloat>

#include "bdc_common.cuh"
#include "bdc_engine.cuh"
#include "bdc_kernels.cuh"

namespace bdc {

constexpr int kUpdThreads = 256;

__device__ __forceinline__ double log_keep0(double v) { return v != 0.0 ? log(v) : 0.0; }

template <typename Op>
__device__ __forceinline__ double block_reduce(double v, Op op, double ident) {
    __shared__ double sh[kUpdThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v = op(v, __shfl_xor_sync(0xFFFFFFFFu, v, off));
    __syncthreads();
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    double r = ident;
    if (threadIdx.x < 32) {
        r = (lane < kUpdThreads / 32) ? sh[lane] : ident;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) r = op(r, __shfl_xor_sync(0xFFFFFFFFu, r, off));
    }
    return r;  // valid in thread 0
}

struct OpMax {
    __device__ double operator()(double a, double b) const {
        // NaN propagates: a NaN deviation stops the loop as in the reference
        // (while (mx >= a) is false for NaN)
        if (a != a) return a;
        if (b != b) return b;
        return a > b ? a : b;
    }
};
struct OpSum {
    __device__ double operator()(double a, double b) const { return a + b; }
};

// true in exactly one block: the last one to arrive
__device__ __forceinline__ bool last_block(unsigned int* ticket) {
    __shared__ bool is_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned int t = atomicAdd(ticket, 1u);
        is_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    return is_last;
}

// fold nb partials (strided by `stride` doubles) with op in a fixed order
template <typename Op>
__device__ __forceinline__ double fold_partials(const double* part, int nb, Op op, double ident) {
    double v = ident;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) v = op(v, ((volatile const double*)part)[b]);
    return block_reduce(v, op, ident);
}

// stage 1: logW = ln p + D; block max logW, max D, sum |O| p D, any zero p
__global__ void __launch_bounds__(kUpdThreads)
k_upd_logw(int n, const uint32_t* __restrict__ reps, int64_t R, const double* __restrict__ p0,
           const double* __restrict__ p1, const double* __restrict__ d, double* __restrict__ logw,
           double* __restrict__ part, DevState* st) {
    if (st->done) return;
    const double* __restrict__ p = st->cur ? p1 : p0;
    double mlw = -DBL_MAX, md = -DBL_MAX, rate = 0.0, zero = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < R;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double pi = p[i];
        const double di = d[i];
        const double lw = log_keep0(pi) + di;
        logw[i] = lw;
        mlw = OpMax()(mlw, lw);
        md = OpMax()(md, di);
        rate = fma((double)orbit_size(reps[i], n) * pi, di, rate);
        if (pi == 0.0) zero = 1.0;
    }
    const int nb = gridDim.x;
    double r0 = block_reduce(mlw, OpMax(), -DBL_MAX);
    double r1 = block_reduce(md, OpMax(), -DBL_MAX);
    double r2 = block_reduce(rate, OpSum(), 0.0);
    double r3 = block_reduce(zero, OpMax(), 0.0);
    if (threadIdx.x == 0) {
        part[blockIdx.x] = r0;
        part[nb + blockIdx.x] = r1;
        part[2 * nb + blockIdx.x] = r2;
        part[3 * nb + blockIdx.x] = r3;
    }
    if (!last_block(&st->ticket[0])) return;
    r0 = fold_partials(part, nb, OpMax(), -DBL_MAX);
    r1 = fold_partials(part + nb, nb, OpMax(), -DBL_MAX);
    r2 = fold_partials(part + 2 * nb, nb, OpSum(), 0.0);
    r3 = fold_partials(part + 3 * nb, nb, OpMax(), 0.0);
    if (threadIdx.x == 0) {
        st->max_logw = r0;
        st->max_d = r1;
        st->rate = r2;
        st->best_ub = fmin(st->best_ub, r1);
        st->best_rate = fmax(st->best_rate, r2);
        st->zero_p = (r3 != 0.0);
        st->shift = r0;
        st->ticket[0] = 0;
    }
}

// stage 2: e = exp(logW - max) into the other buffer; Z = sum |O| e
__global__ void __launch_bounds__(kUpdThreads)
k_upd_exp(int n, const uint32_t* __restrict__ reps, int64_t R, double* __restrict__ p0,
          double* __restrict__ p1, const double* __restrict__ logw, double* __restrict__ part,
          DevState* st) {
    if (st->done) return;
    double* __restrict__ pn = st->cur ? p0 : p1;
    const double shift = st->shift;
    double z = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < R;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double e = exp(logw[i] - shift);
        pn[i] = e;
        z = fma((double)orbit_size(reps[i], n), e, z);
    }
    const int nb = gridDim.x;
    double r = block_reduce(z, OpSum(), 0.0);
    if (threadIdx.x == 0) part[4 * nb + blockIdx.x] = r;
    if (!last_block(&st->ticket[1])) return;
    r = fold_partials(part + 4 * nb, nb, OpSum(), 0.0);
    if (threadIdx.x == 0) {
        st->log_z = log(r);
        st->lse = st->shift + log(r);
        st->ticket[1] = 0;
    }
}

// stage 3: p' = e / Z; mx = max log2 p' - log2 p; flip buffers; stop test
__global__ void __launch_bounds__(kUpdThreads)
k_upd_norm(int64_t R, double* __restrict__ p0, double* __restrict__ p1, double* __restrict__ part,
           double a, DevState* st) {
    if (st->done) return;
    double* __restrict__ pn = st->cur ? p0 : p1;
    const double* __restrict__ pc = st->cur ? p1 : p0;
    const double z = exp(st->log_z);
    double mx = -DBL_MAX;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < R;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double v = pn[i] / z;
        pn[i] = v;
        mx = OpMax()(mx, log2(v) - log2(pc[i]));
    }
    const int nb = gridDim.x;
    double r = block_reduce(mx, OpMax(), -DBL_MAX);
    if (threadIdx.x == 0) part[5 * nb + blockIdx.x] = r;
    if (!last_block(&st->ticket[2])) return;
    r = fold_partials(part + 5 * nb, nb, OpMax(), -DBL_MAX);
    if (threadIdx.x == 0) {
        st->mx = r;
        st->cur ^= 1;
        st->iter += 1;
        st->done = !(r >= a);
        st->ticket[2] = 0;
    }
}

cudaError_t launch_update_stages(const UpdateLaunch& U, int first, int last) {
    if (first <= 1 && last >= 1)
        k_upd_logw<<<U.nblocks, kUpdThreads, 0, U.stream>>>(U.n, U.reps, U.R, U.p0, U.p1, U.d, U.logw,
                                                            U.part, U.st);
    if (first <= 2 && last >= 2)
        k_upd_exp<<<U.nblocks, kUpdThreads, 0, U.stream>>>(U.n, U.reps, U.R, U.p0, U.p1, U.logw, U.part,
                                                           U.st);
    if (first <= 3 && last >= 3) k_upd_norm<<<U.nblocks, kUpdThreads, 0, U.stream>>>(U.R, U.p0, U.p1, U.part, U.a, U.st);
    return cudaGetLastError();
}

cudaError_t launch_update(const UpdateLaunch& U) { return launch_update_stages(U, 1, 3); }

// ---------------------------------------------------------------- helpers
__global__ void k_logw(int n, const uint32_t* __restrict__ reps, int64_t R,
                       const double* __restrict__ p, const double* __restrict__ d,
                       double* __restrict__ logw) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < R;
         i += (int64_t)gridDim.x * blockDim.x)
        logw[i] = log_keep0(p[i]) + d[i];
}

cudaError_t launch_logw(int n, const uint32_t* reps, int64_t R, const double* p, const double* d,
                        double* logw, cudaStream_t stream) {
    int64_t b = (R + 255) / 256;
    if (b > 148 * 8) b = 148 * 8;
    if (b < 1) b = 1;
    k_logw<<<(int)b, 256, 0, stream>>>(n, reps, R, p, d, logw);
    return cudaGetLastError();
}

// single-kernel sum |O| p D (two kernels: block partials, then one block)
__global__ void __launch_bounds__(kUpdThreads)
k_rate_part(int n, const uint32_t* __restrict__ reps, int64_t R, const double* __restrict__ p,
            const double* __restrict__ d, double* __restrict__ part) {
    double s = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < R;
         i += (int64_t)gridDim.x * blockDim.x)
        s = fma((double)orbit_size(reps[i], n) * p[i], d[i], s);
    s = block_reduce(s, OpSum(), 0.0);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

__global__ void __launch_bounds__(kUpdThreads)
k_fold_sum(const double* __restrict__ part, int nb, double* out) {
    const double s = fold_partials(part, nb, OpSum(), 0.0);
    if (threadIdx.x == 0) *out = s;
}

__global__ void __launch_bounds__(kUpdThreads)
k_fold_max(const double* __restrict__ part, int nb, double* out) {
    const double s = fold_partials(part, nb, OpMax(), -DBL_MAX);
    if (threadIdx.x == 0) *out = s;
}

// adjoint of I(p;W) = sum_x p(x) D(x) over the representative parametrisation:
// dI/dp_rep = |O(rep)| (D(rep) - 1) -- the q-dependence of D cancels because
// sum_y W(y|x) = 1 (backend/BAA.cu:413-425 computes the same D)
__global__ void k_mi_grad(int n, const uint32_t* __restrict__ reps, int64_t R, const double* __restrict__ d,
                          double* __restrict__ grad) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < R; i += (int64_t)gridDim.x * blockDim.x)
        grad[i] = (double)orbit_size(reps[i], n) * (d[i] - 1.0);
}

cudaError_t launch_mi_grad(int n, const uint32_t* reps, int64_t R, const double* d, double* grad,
                           cudaStream_t stream) {
    int64_t b = (R + 255) / 256;
    if (b > 148 * 8) b = 148 * 8;
    if (b < 1) b = 1;
    k_mi_grad<<<(int)b, 256, 0, stream>>>(n, reps, R, d, grad);
    return cudaGetLastError();
}

cudaError_t launch_rate(int n, const uint32_t* reps, int64_t R, const double* p, const double* d,
                        double* part, int nblocks, double* out, cudaStream_t stream) {
    k_rate_part<<<nblocks, kUpdThreads, 0, stream>>>(n, reps, R, p, d, part);
    k_fold_sum<<<1, kUpdThreads, 0, stream>>>(part, nblocks, out);
    return cudaGetLastError();
}

__global__ void __launch_bounds__(kUpdThreads)
k_maxdev_part(const double* __restrict__ p, const double* __restrict__ pb, int64_t R,
              double* __restrict__ part) {
    double m = -DBL_MAX;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < R;
         i += (int64_t)gridDim.x * blockDim.x)
        m = OpMax()(m, log2(p[i]) - log2(pb[i]));
    m = block_reduce(m, OpMax(), -DBL_MAX);
    if (threadIdx.x == 0) part[blockIdx.x] = m;
}

__global__ void __launch_bounds__(kUpdThreads)
k_vmax_part(const double* __restrict__ v, int64_t R, double* __restrict__ part) {
    double m = -DBL_MAX;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < R;
         i += (int64_t)gridDim.x * blockDim.x)
        m = OpMax()(m, v[i]);
    m = block_reduce(m, OpMax(), -DBL_MAX);
    if (threadIdx.x == 0) part[blockIdx.x] = m;
}

cudaError_t launch_vec_max(const double* v, int64_t R, double* part, int nblocks, double* out,
                           cudaStream_t stream) {
    k_vmax_part<<<nblocks, kUpdThreads, 0, stream>>>(v, R, part);
    k_fold_max<<<1, kUpdThreads, 0, stream>>>(part, nblocks, out);
    return cudaGetLastError();
}

cudaError_t launch_max_dev(const double* p, const double* pb, int64_t R, double* part, int nblocks,
                           double* out, cudaStream_t stream) {
    k_maxdev_part<<<nblocks, kUpdThreads, 0, stream>>>(p, pb, R, part);
    k_fold_max<<<1, kUpdThreads, 0, stream>>>(part, nblocks, out);
    return cudaGetLastError();
}

}  // namespace bdc

// ===================================================================
// Allocation-free max deviation.
//
// For callers that cannot allocate device memory: code that owns every byte
// of its GPU memory through its own pool or arena (so a cudaMalloc behind its
// back would break its accounting or fail outright), code running where the
// allocator must not be called, and plugins that are handed buffers by a
// host application.  They pass their own device buffers for the inputs and
// for the one-double result; the block partials of the reduction live in a
// fixed array in the library's device memory instead of a buffer the library
// allocates.
//
// Limits and sharing:
//   * num_reps <= kNoAllocMaxReps (2^27 = 134,217,728 representatives, i.e.
//     every n <= 28); larger inputs return BDC_ERR_ARG.
//   * The array (kNoAllocSlots doubles, 128 KB) exists once per device that
//     loads the library and stays resident until the process exits.
//   * Every call on a device uses the same array.  Each call writes every
//     slot it later reads, so nothing has to start at zero and a call never
//     sees a previous call's values; but two calls whose kernels overlap on
//     the GPU (e.g. issued on different streams without ordering) race on
//     the array and may return wrong results.  Order such calls.
//   * The first call on each device looks up the array's device address
//     (cudaGetSymbolAddress, with that device current) and caches it; make
//     that first call before any stream capture is in progress on the
//     calling thread.
namespace bdc {

constexpr int kNoAllocSlots = 16384;
constexpr int kNoAllocTile = 8192;  // representatives reduced per block
constexpr int64_t kNoAllocMaxReps = (int64_t)kNoAllocSlots * kNoAllocTile;

static __device__ __align__(256) double g_noalloc_partials[kNoAllocSlots];

// block b reduces representatives [b * kNoAllocTile, (b + 1) * kNoAllocTile)
__global__ void __launch_bounds__(kUpdThreads)
k_maxdev_tile(const double* __restrict__ p, const double* __restrict__ pb, int64_t R, double* __restrict__ part) {
    const int64_t i0 = (int64_t)blockIdx.x * kNoAllocTile;
    const int64_t i1 = (i0 + kNoAllocTile < R) ? i0 + kNoAllocTile : R;
    double m = -DBL_MAX;
    for (int64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) m = OpMax()(m, log2(p[i]) - log2(pb[i]));
    m = block_reduce(m, OpMax(), -DBL_MAX);
    if (threadIdx.x == 0) part[blockIdx.x] = m;
}

// the array's device address per device, looked up on the first call there;
// null until then.  Two threads that make their first call on one device at
// the same time both look it up and store the same address.
static std::atomic<double*> g_noalloc_addr[64];

}  // namespace bdc

extern "C" bdc_status bdc_max_deviation_noalloc(const double* p_dev, const double* p_before_dev,
                                                int64_t num_reps, double* mx_dev, void* cuda_stream) {
    using namespace bdc;
    if (!p_dev || !p_before_dev || !mx_dev || num_reps < 1)
        return fail(BDC_ERR_ARG, "bdc_max_deviation_noalloc: NULL pointer or num_reps < 1");
    if (num_reps > kNoAllocMaxReps)
        return fail(BDC_ERR_ARG,
                    "bdc_max_deviation_noalloc: num_reps %lld exceeds the fixed scratch limit of %lld "
                    "(%d slots of %d); use bdc_max_deviation",
                    (long long)num_reps, (long long)kNoAllocMaxReps, kNoAllocSlots, kNoAllocTile);
    int dev = 0;
    BDC_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(BDC_ERR_ARG, "bdc_max_deviation_noalloc: device %d out of range", dev);
    double* part = g_noalloc_addr[dev].load(std::memory_order_acquire);
    if (!part) {
        void* addr = nullptr;
        BDC_CUDA_TRY(cudaGetSymbolAddress(&addr, g_noalloc_partials));
        part = (double*)addr;
        g_noalloc_addr[dev].store(part, std::memory_order_release);
    }
    cudaStream_t s = (cudaStream_t)cuda_stream;
    const int blocks = (int)((num_reps + kNoAllocTile - 1) / kNoAllocTile);
    k_maxdev_tile<<<blocks, kUpdThreads, 0, s>>>(p_dev, p_before_dev, num_reps, part);
    k_fold_max<<<1, kUpdThreads, 0, s>>>(part, blocks, mx_dev);
    BDC_CUDA_TRY(cudaGetLastError());
    return BDC_OK;
}
