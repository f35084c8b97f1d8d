// bdc_tables.cu -- half tables and the canonical representative list, built on
// the device.
//
// Reference counterparts (Pintz45/BDC-Upper-Bounds-GPU):
//   generate_bit_transition_cache.cpp:23-77  the cache_{n,k} generator (CPU DP
//       per (x, y) pair, written as uint32 at index (x << k) | y)
//   backend/BAA.cu:27-93                     load_gpu_cache: every cache_{n',k'}
//       with n' <= ceil(n/2) flattened into one array + a pointer table
//   backend/main_BAA.cu:46-50                canonical list: host loop over 2^n
//
// Here the generator is a kernel (one thread per pair, the same prefix DP),
// the engine keeps only the two half lengths it needs as uint16 "bundles"
// (see HalfTables), and the representative list is a device stream
// compaction over all 2^n strings that keeps ascending order.
#include "bdc_common.cuh"
#include "bdc_kernels.cuh"

namespace bdc {

// number of occurrences of y (k bits) as a subsequence of x (n bits); the
// prefix DP of generate_bit_transition_cache.cpp:23-44, rolled over i.
__device__ __forceinline__ uint32_t dp_count(uint32_t x, int n, uint32_t y, int k) {
    uint32_t dp[kMaxN + 1];
    dp[0] = 1;
    for (int j = 1; j <= k; ++j) dp[j] = 0;
    for (int i = 1; i <= n; ++i) {
        const uint32_t xi = (x >> (n - i)) & 1u;
        const int jt = i < k ? i : k;
        for (int j = jt; j >= 1; --j) {
            const uint32_t yj = (y >> (k - j)) & 1u;
            if (xi == yj) dp[j] += dp[j - 1];
        }
    }
    return dp[k];
}

__global__ void k_gen_cache(int n, int k, uint32_t* __restrict__ out) {
    const uint64_t total = 1ull << (n + k);
    for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < total;
         e += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t x = (uint32_t)(e >> k), y = (uint32_t)(e & low_mask(k));
        out[e] = (k > n) ? 0u : dp_count(x, n, y, k);
    }
}

cudaError_t launch_gen_cache(int n, int k, uint32_t* out, cudaStream_t stream) {
    const uint64_t total = 1ull << (n + k);
    uint64_t blocks = (total + 255) / 256;
    if (blocks > 148ull * 64) blocks = 148ull * 64;
    k_gen_cache<<<(unsigned)blocks, 256, 0, stream>>>(n, k, out);
    return cudaGetLastError();
}

// bundle row v: entry e in [1, 2^{mmax+1}) is cache_{h,m}[v][w] with
// m = floor(log2 e), w = e - 2^m; entry 0 is unused (0).
__global__ void k_gen_bundle(int h, int mmax, int stride, uint16_t* __restrict__ rows) {
    const uint64_t total = (uint64_t)stride << h;
    const int used = 1 << (mmax + 1);
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t v = (uint32_t)(i / stride);
        const int e = (int)(i % stride);
        uint16_t val = 0;
        if (e >= 1 && e < used) {
            const int m = 31 - __clz(e);
            const uint32_t w = (uint32_t)(e - (1 << m));
            val = (uint16_t)dp_count(v, h, w, m);
        }
        rows[i] = val;
    }
}

cudaError_t launch_gen_bundle(int h, int mmax, int stride, uint16_t* rows, cudaStream_t stream) {
    const uint64_t total = (uint64_t)stride << h;
    uint64_t blocks = (total + 255) / 256;
    if (blocks > 148ull * 64) blocks = 148ull * 64;
    k_gen_bundle<<<(unsigned)blocks, 256, 0, stream>>>(h, mmax, stride, rows);
    return cudaGetLastError();
}

// bundle from uploaded cache files: caches_dev[m] points to cache_{h,m}
// (2^{h+m} uint32, index (v << m) | w).  Values above 65535 set *overflow.
struct CachePtrs { const uint32_t* p[kMaxHalf + 1]; };

__global__ void k_build_bundle(int h, int mmax, int stride, CachePtrs caches,
                               uint16_t* __restrict__ rows, int* overflow) {
    const uint64_t total = (uint64_t)stride << h;
    const int used = 1 << (mmax + 1);
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t v = (uint32_t)(i / stride);
        const int e = (int)(i % stride);
        uint32_t val = 0;
        if (e >= 1 && e < used) {
            const int m = 31 - __clz(e);
            const uint32_t w = (uint32_t)(e - (1 << m));
            val = caches.p[m][((uint64_t)v << m) | w];
        }
        if (val > 0xFFFFu) { atomicExch(overflow, 1); val = 0xFFFFu; }
        rows[i] = (uint16_t)val;
    }
}

cudaError_t launch_build_bundle(int h, int mmax, int stride, const uint32_t* const* caches_dev,
                                uint16_t* rows, int* overflow, cudaStream_t stream) {
    if (mmax > kMaxHalf) return cudaErrorInvalidValue;
    CachePtrs cp{};
    for (int m = 0; m <= mmax; ++m) cp.p[m] = caches_dev[m];
    const uint64_t total = (uint64_t)stride << h;
    uint64_t blocks = (total + 255) / 256;
    if (blocks > 148ull * 64) blocks = 148ull * 64;
    k_build_bundle<<<(unsigned)blocks, 256, 0, stream>>>(h, mmax, stride, cp, rows, overflow);
    return cudaGetLastError();
}

// ------------------------------------------------- representative list
// Block b covers strings [b * 4096, (b + 1) * 4096): 256 threads x 16 strings.
constexpr int kRepThreads = 256;
constexpr int kRepPerThread = 16;
constexpr int kRepPerBlock = kRepThreads * kRepPerThread;

__device__ __forceinline__ int block_exclusive_scan(int v, int* total) {
    __shared__ int warp_sums[kRepThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int inc = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const int o = __shfl_up_sync(0xFFFFFFFFu, inc, off);
        if (lane >= off) inc += o;
    }
    if (lane == 31) warp_sums[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        int s = (lane < kRepThreads / 32) ? warp_sums[lane] : 0;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const int o = __shfl_up_sync(0xFFFFFFFFu, s, off);
            if (lane >= off) s += o;
        }
        if (lane < kRepThreads / 32) warp_sums[lane] = s;  // inclusive
    }
    __syncthreads();
    const int before = (warp > 0) ? warp_sums[warp - 1] : 0;
    *total = warp_sums[kRepThreads / 32 - 1];
    __syncthreads();
    return before + inc - v;
}

__global__ void k_rep_count(int n, int* __restrict__ counts) {
    const uint64_t total = 1ull << n;
    const uint64_t base = (uint64_t)blockIdx.x * kRepPerBlock + (uint64_t)threadIdx.x * kRepPerThread;
    int c = 0;
    for (int e = 0; e < kRepPerThread; ++e) {
        const uint64_t x = base + e;
        if (x < total && is_rep((uint32_t)x, n)) ++c;
    }
    int tot;
    block_exclusive_scan(c, &tot);
    if (threadIdx.x == 0) counts[blockIdx.x] = tot;
}

// exclusive scan of counts[0..nb) in place (one block), total to *count_out
__global__ void k_rep_scan(int* __restrict__ counts, int nb, int64_t* count_out) {
    __shared__ long long carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < nb; base += kRepThreads) {
        const int i = base + threadIdx.x;
        const int v = (i < nb) ? counts[i] : 0;
        int tot;
        const int ex = block_exclusive_scan(v, &tot);
        if (i < nb) counts[i] = (int)(carry + ex);
        __syncthreads();
        if (threadIdx.x == 0) carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) *count_out = carry;
}

__global__ void k_rep_write(int n, const int* __restrict__ offsets, uint32_t* __restrict__ reps) {
    const uint64_t total = 1ull << n;
    const uint64_t base = (uint64_t)blockIdx.x * kRepPerBlock + (uint64_t)threadIdx.x * kRepPerThread;
    int c = 0;
    for (int e = 0; e < kRepPerThread; ++e) {
        const uint64_t x = base + e;
        if (x < total && is_rep((uint32_t)x, n)) ++c;
    }
    int tot;
    int pos = offsets[blockIdx.x] + block_exclusive_scan(c, &tot);
    for (int e = 0; e < kRepPerThread; ++e) {
        const uint64_t x = base + e;
        if (x < total && is_rep((uint32_t)x, n)) reps[pos++] = (uint32_t)x;
    }
}

size_t build_reps_scratch_bytes(int n) {
    const uint64_t nb = ((1ull << n) + kRepPerBlock - 1) / kRepPerBlock;
    return nb * sizeof(int) + 16;
}

// reps_out must hold the representative count (<= 2^n / 4 + 2^{n/2+1});
// count_out is a device int64.
cudaError_t build_reps(int n, uint32_t* reps_out, int64_t* count_out, void* scratch,
                       size_t scratch_bytes, cudaStream_t stream) {
    const uint64_t nb = ((1ull << n) + kRepPerBlock - 1) / kRepPerBlock;
    if (scratch_bytes < nb * sizeof(int)) return cudaErrorInvalidValue;
    int* counts = (int*)scratch;
    k_rep_count<<<(unsigned)nb, kRepThreads, 0, stream>>>(n, counts);
    k_rep_scan<<<1, kRepThreads, 0, stream>>>(counts, (int)nb, count_out);
    k_rep_write<<<(unsigned)nb, kRepThreads, 0, stream>>>(n, counts, reps_out);
    return cudaGetLastError();
}

}  // namespace bdc
