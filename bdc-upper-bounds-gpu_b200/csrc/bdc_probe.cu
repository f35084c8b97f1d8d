// bdc_probe.cu -- measured throughput denominators for the roofline fractions
// of kernels that are bound by an arithmetic pipe other than the tensor cores
// (int32 multiply-add for the count path, FP64 FMA for the factored engine).
#include <cmath>

#include "bdc_engine.cuh"

namespace bdc {

// 8 independent multiply-add chains per thread, unrolled; the result is
// written only if it hits an impossible value so nothing is eliminated.
template <typename T>
__global__ void __launch_bounds__(256) k_peak(T* out, int iters, T seed) {
    T a[8];
    const T b = seed * (T)3 + (T)1;
    const T c = seed + (T)7;
#pragma unroll
    for (int j = 0; j < 8; ++j) a[j] = seed + (T)(threadIdx.x + j);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
#pragma unroll
            for (int j = 0; j < 8; ++j) a[j] = a[j] * b + c;
        }
    }
    T s = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) s += a[j];
    if (s == (T)-12345) out[0] = s;
}

// FP64 tensor-core path (mma.sync m8n8k4, 256 multiply-adds per warp
// instruction): 8 independent accumulator pairs per warp
__global__ void __launch_bounds__(256) k_peak_dmma(double* out, int iters, double seed) {
    double a = seed + threadIdx.x * 1e-3, b = seed * 0.5;
    double c[8][2];
#pragma unroll
    for (int j = 0; j < 8; ++j) c[j][0] = c[j][1] = seed * j;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
#pragma unroll
            for (int j = 0; j < 8; ++j)
                asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                             : "+d"(c[j][0]), "+d"(c[j][1])
                             : "d"(a), "d"(b));
        }
    }
    double s = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) s += c[j][0] + c[j][1];
    if (s == -12345.0) out[0] = s;
}

static bdc_status run_probe_dmma(int device, double ms_target, double* ops) {
    int sms = 148;
    BDC_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    double* out = nullptr;
    BDC_CUDA_TRY(cudaMalloc(&out, sizeof(double)));
    cudaEvent_t e0, e1;
    BDC_CUDA_TRY(cudaEventCreate(&e0));
    BDC_CUDA_TRY(cudaEventCreate(&e1));
    const int blocks = sms * 8, threads = 256;
    int iters = 16;
    float ms = 0.f;
    for (int rep = 0; rep < 12; ++rep) {
        BDC_CUDA_TRY(cudaEventRecord(e0));
        k_peak_dmma<<<blocks, threads>>>(out, iters, 0.999);
        BDC_CUDA_TRY(cudaEventRecord(e1));
        BDC_CUDA_TRY(cudaEventSynchronize(e1));
        BDC_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
        if (ms > ms_target * 0.5 && rep >= 2) break;
        if (ms < ms_target * 0.5) iters = (int)std::min<double>(1 << 22, iters * std::max(2.0, ms_target / (ms + 1e-3)));
    }
    float best = 1e30f;
    for (int rep = 0; rep < 3; ++rep) {
        BDC_CUDA_TRY(cudaEventRecord(e0));
        k_peak_dmma<<<blocks, threads>>>(out, iters, 0.999);
        BDC_CUDA_TRY(cudaEventRecord(e1));
        BDC_CUDA_TRY(cudaEventSynchronize(e1));
        BDC_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
        best = std::min(best, ms);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    // per warp instruction: 8 x 8 x 4 = 256 multiply-adds
    const double total = (double)blocks * (threads / 32) * (double)iters * 16.0 * 8.0 * 256.0;
    *ops = total / (best * 1e-3);
    return BDC_OK;
}

template <typename T>
static bdc_status run_probe(int device, double ms_target, T seed, double* ops) {
    int sms = 148;
    BDC_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    T* out = nullptr;
    BDC_CUDA_TRY(cudaMalloc(&out, sizeof(T)));
    cudaEvent_t e0, e1;
    BDC_CUDA_TRY(cudaEventCreate(&e0));
    BDC_CUDA_TRY(cudaEventCreate(&e1));
    const int blocks = sms * 8, threads = 256;
    int iters = 64;
    float ms = 0.f;
    // warm up, then grow the iteration count until the kernel runs ~ms_target
    for (int rep = 0; rep < 12; ++rep) {
        BDC_CUDA_TRY(cudaEventRecord(e0));
        k_peak<T><<<blocks, threads>>>(out, iters, seed);
        BDC_CUDA_TRY(cudaEventRecord(e1));
        BDC_CUDA_TRY(cudaEventSynchronize(e1));
        BDC_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
        if (ms > ms_target * 0.5 && rep >= 2) break;
        if (ms < ms_target * 0.5) iters = (int)std::min<double>(1 << 24, iters * std::max(2.0, ms_target / (ms + 1e-3)));
    }
    float best = 1e30f;
    for (int rep = 0; rep < 3; ++rep) {
        BDC_CUDA_TRY(cudaEventRecord(e0));
        k_peak<T><<<blocks, threads>>>(out, iters, seed);
        BDC_CUDA_TRY(cudaEventRecord(e1));
        BDC_CUDA_TRY(cudaEventSynchronize(e1));
        BDC_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
        best = std::min(best, ms);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    const double total = (double)blocks * threads * (double)iters * 16.0 * 8.0;
    *ops = total / (best * 1e-3);
    return BDC_OK;
}

}  // namespace bdc

extern "C" bdc_status bdc_peak_probe(int device, int kind, double ms, double* ops_per_s) {
    using namespace bdc;
    if (!ops_per_s || ms <= 0) return fail(BDC_ERR_ARG, "bdc_peak_probe: bad arguments");
    if (cudaSetDevice(device) != cudaSuccess) return fail(BDC_ERR_CUDA, "cudaSetDevice(%d) failed", device);
    switch (kind) {
        case 0: return run_probe<int>(device, ms, 3, ops_per_s);
        case 1: return run_probe<double>(device, ms, 0.999, ops_per_s);
        case 2: return run_probe<float>(device, ms, 0.999f, ops_per_s);
        case 3: return run_probe_dmma(device, ms, ops_per_s);
        default: return fail(BDC_ERR_ARG, "bdc_peak_probe: kind %d", kind);
    }
}
