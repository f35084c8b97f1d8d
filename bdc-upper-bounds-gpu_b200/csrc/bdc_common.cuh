// bdc_common.cuh -- shared definitions of the B200 Blahut-Arimoto engine for the
// binary deletion channel BDC_{n,k}.
//
// Conventions (kept identical to the reference, Pintz45/BDC-Upper-Bounds-GPU):
//   * a string of length L is an integer, MSB first: character i is bit L-1-i
//     (backend/generate_bit_transition_cache.cpp:15, backend/BAA.cu:271);
//   * the symmetry group is {id, reverse, complement, reverse-complement};
//     rep(x) is the minimum of the orbit and the orbit has 2 or 4 members
//     (backend/BAA.cu:216-241);
//   * p is stored per canonical representative, as the probability of EACH
//     string of the orbit, in ascending representative order
//     (backend/main_BAA.cu:46-50);
//   * q is stored over 2^{k-1} slots indexed by the representative's value
//     (backend/BAA.cu:649-652); slots that are not representatives hold ln 0
//     = 0, the reference's convention (backend/BAA.cu:573-580).
#pragma once

#include <cstdint>
#include <cstdio>
#include <cuda_runtime.h>

#include "../../include/bdc_b200.h"

namespace bdc {

constexpr int kMaxN = 32;      // strings are uint32
constexpr int kMaxHalf = 17;   // half tables are stored as uint16: C(17,8) = 24310 < 65536

// ---------------------------------------------------------------- symmetry
__host__ __device__ __forceinline__ uint32_t low_mask(int len) {
    return len >= 32 ? 0xFFFFFFFFu : ((1u << len) - 1u);
}

__host__ __device__ __forceinline__ uint32_t reverse_bits(uint32_t x, int len) {
#ifdef __CUDA_ARCH__
    return len == 0 ? 0u : (__brev(x) >> (32 - len));
#else
    uint32_t r = 0;
    for (int i = 0; i < len; ++i) r |= ((x >> i) & 1u) << (len - 1 - i);
    return r;
#endif
}

__host__ __device__ __forceinline__ uint32_t complement_bits(uint32_t x, int len) {
    return x ^ low_mask(len);
}

// canonical representative: min over the orbit (backend/BAA.cu:216-227)
__host__ __device__ __forceinline__ uint32_t orbit_rep(uint32_t x, int len) {
    uint32_t r = reverse_bits(x, len);
    uint32_t c = complement_bits(x, len);
    uint32_t rc = reverse_bits(c, len);
    uint32_t m1 = r < x ? r : x;
    uint32_t m2 = rc < c ? rc : c;
    return m2 < m1 ? m2 : m1;
}

// orbit size: 2 when reverse or reverse-complement fixes x, else 4
// (backend/BAA.cu:230-241)
__host__ __device__ __forceinline__ int orbit_size(uint32_t x, int len) {
    uint32_t r = reverse_bits(x, len);
    uint32_t rc = reverse_bits(complement_bits(x, len), len);
    return (x == r || x == rc) ? 2 : 4;
}

__host__ __device__ __forceinline__ bool is_rep(uint32_t x, int len) {
    return orbit_rep(x, len) == x;
}

__host__ __device__ inline uint32_t binom(uint32_t n, uint32_t k) {
    if (k > n) return 0;
    if (k > n - k) k = n - k;
    uint64_t r = 1;
    for (uint32_t i = 1; i <= k; ++i) r = r * (n - i + 1) / i;
    return (uint32_t)r;
}

// ------------------------------------------------------------ half tables
// Half-table "bundles": for a half length h the device holds one row per
// half-string v (2^h rows); the row holds cache_{h,m}[v][.] for m = 0 .. mmax
// at row(v)[2^m + w] (entry 0 is unused), so every segment with m >= 3 starts
// on a 16-byte boundary.  The row stride is 2^{mmax+1} entries.
// Entries are uint16 (exact: every count in a half table of length <= 17
// is < 65536).  m == h (the whole half) is an equality test, never stored.
#ifdef __CUDACC__
// The sum (MAX = false) or maximum (MAX = true) of n block partials v[i *
// stride] by one whole warp, in a fixed order: lane l combines i = l, l + 32,
// ... (eight loads in flight at a time), then a shuffle tree; every lane
// returns the result.  Replaces one thread walking the partials, whose loads
// would wait on one another.
template <bool MAX>
__device__ __forceinline__ double warp_parts(const double* __restrict__ v, int n, int stride) {
    const int lane = threadIdx.x & 31;
    double a = MAX ? -1.7976931348623157e308 : 0.0;
    int i = lane;
    for (; i + 7 * 32 < n; i += 8 * 32) {
        double t[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) t[u] = v[(size_t)(i + 32 * u) * stride];
#pragma unroll
        for (int u = 0; u < 8; ++u) a = MAX ? fmax(a, t[u]) : a + t[u];
    }
    for (; i < n; i += 32) a = MAX ? fmax(a, v[(size_t)i * stride]) : a + v[(size_t)i * stride];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double b = __shfl_xor_sync(0xFFFFFFFFu, a, o);
        a = MAX ? fmax(a, b) : a + b;
    }
    return a;
}
#endif

struct HalfTables {
    const uint16_t* rows = nullptr;  // [2^h][stride]
    int h = 0;                       // half length
    int mmax = -1;                   // largest stored sub-length
    int stride = 0;                  // entries per row
};

__host__ __device__ __forceinline__ int bundle_offset(int m) { return 1 << m; }

// the split of x = x_hi || x_lo and of y at split point j (backend/BAA.cu:340-395)
struct Split {
    int n, k, n1, n2;   // n1 = ceil(n/2) high bits, n2 = n - n1 low bits
    int jlo, jhi;       // valid split points: max(0, k - n2) .. min(k, n1)
};

__host__ __device__ inline Split make_split(int n, int k) {
    Split s;
    s.n = n; s.k = k;
    s.n1 = (n + 1) / 2;
    s.n2 = n - s.n1;
    s.jlo = k - s.n2 > 0 ? k - s.n2 : 0;
    s.jhi = k < s.n1 ? k : s.n1;
    return s;
}

// Exact N(x,y): the number of occurrences of y as a subsequence of x, by the
// split identity N = sum_j cache_{n1,j}[x_hi][y_hi] * cache_{n2,k-j}[x_lo][y_lo]
// (backend/BAA.cu:340-395).  A half whose sub-length equals its length is an
// equality test; sub-length 0 is the empty word (count 1).
__device__ __forceinline__ uint32_t split_count(const Split& s, const HalfTables& A,
                                                const HalfTables& B, uint32_t x, uint32_t y) {
    uint32_t xh = x >> s.n2, xl = x & low_mask(s.n2);
    const uint16_t* ar = A.rows + (size_t)xh * A.stride;
    const uint16_t* br = B.rows + (size_t)xl * B.stride;
    uint32_t tot = 0;
    for (int j = s.jlo; j <= s.jhi; ++j) {
        int m = s.k - j;
        uint32_t yh = (m >= 32) ? 0u : (y >> m), yl = y & low_mask(m);
        uint32_t c1 = (j == s.n1) ? (uint32_t)(xh == yh) : (uint32_t)__ldg(ar + bundle_offset(j) + yh);
        uint32_t c2 = (m == s.n2) ? (uint32_t)(xl == yl) : (uint32_t)__ldg(br + bundle_offset(m) + yl);
        tot += c1 * c2;
    }
    return tot;
}

// ------------------------------------------------------------- device state
// Scalars written by the device and read back once per chunk of iterations.
struct DevState {
    double max_logw;     // max_x logW of the last update
    double max_d;        // max_x D(x) of the last D pass (nats): the BA upper bound
    double log_z;        // ln Z of the last update, Z = sum |O| exp(logW - shift)
    double shift;        // the shift used for exp
    double mx;           // max_x log2 p' - log2 p of the last iteration
    double rate;         // sum |O| p D of the iterate the D pass used (nats)
    double lnp_max;      // max_x ln p of the current iterate
    double lse;          // ln sum |O| p e^D of the last D pass (nats)
    double best_ub;      // min over evaluated iterates of max_x D(x) (nats): still a bound
    double best_rate;    // max over evaluated iterates of I(p;W) (nats): a lower bound
    double ng_prev_rate; // accelerated loop: I(p;W) at the last accepted extrapolated point
    double ng_gap;       // accelerated loop: stop when best_ub - best_rate < this (nats)
    double ng_max;       // accelerated loop: max of the extrapolated log iterate
    long long ng_t;      // accelerated loop: steps since the last restart (momentum t / (t + 3))
    long long iter;      // iterations done since the last reset
    int cur;             // which of the two p buffers holds the current iterate
    int done;            // set when mx < a: later iterations do nothing
    int zero_p;          // the current iterate has a zero entry
    int error;           // device-detected error code (0 = none)
    int ng_mode;         // accelerated loop: 0 fresh start, 1 step accepted, 2 restart
    unsigned int ticket[4];  // last-block counters of the grid reductions
};

}  // namespace bdc

#define BDC_CUDA_TRY(expr)                                                         \
    do {                                                                           \
        cudaError_t _e = (expr);                                                   \
        if (_e != cudaSuccess) {                                                   \
            bdc::set_last_error("%s:%d: %s: %s", __FILE__, __LINE__, #expr,        \
                                cudaGetErrorString(_e));                           \
            return BDC_ERR_CUDA;                                                   \
        }                                                                          \
    } while (0)

namespace bdc {
void set_last_error(const char* fmt, ...);
}
