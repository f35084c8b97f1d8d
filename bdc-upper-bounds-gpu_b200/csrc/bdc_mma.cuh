// bdc_mma.cuh -- FP64 matrix products on the FP64 tensor-core path of sm_100
// (mma.sync.aligned.m8n8k4 .f64: 256 multiply-adds per warp instruction, the
// same peak as FP64 FMA on the CUDA cores but with 1/8 of the issue slots and
// operands read once per fragment).
//
// C(m, n) = sum_k A(m, k) B(k, n) over a "grouped" list of products
// (GemmDesc, bdc_gemm.cuh): CTA i runs tile i of the product whose
// tile_begin <= i.  A split of the contraction is expressed by several
// descriptors with offset operands and separate outputs.
//
// Tile: BM x BN x 16, 256 threads = WM x WN warps, warp tile (8 MT) x (8 NT).
// Global -> registers -> shared memory (k-major, rows padded by 4 doubles so
// that both the transposing stores and the fragment loads are 2 wavefronts per
// warp access), double buffered; the next k-slice is fetched into registers
// while the tensor cores work on the current one.
//
// Fragment layout of m8n8k4 .f64 (g = lane / 4, t = lane % 4):
//   A: a = A[g][t]   B: b = B[t][g]   C/D: c[i] = C[g][2t + i], i = 0, 1
#pragma once

#include "bdc_gemm.cuh"

namespace bdc {

__device__ __forceinline__ void mma_f64(double& c0, double& c1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}

__device__ __forceinline__ double opnd_load(const Operand& o, int64_t r, int64_t c) {
    if (o.kind == OP_EYE) return r == c ? 1.0 : 0.0;
    const int64_t idx = o.trans ? c * o.ld + r : r * o.ld + c;
    if (o.kind == OP_U16) return (double)__ldg((const uint16_t*)o.ptr + idx);
    return __ldg((const double*)o.ptr + idx);
}

template <int BM, int BN, int WM, int WN>
struct MmaCfg {
    static constexpr int BK = 16;
    static constexpr int MT = BM / (8 * WM);
    static constexpr int NT = BN / (8 * WN);
    static constexpr int PA = BM + 4;  // padded row of the k-major A tile
    static constexpr int PB = BN + 4;
    static constexpr int A_PER = BK * BM / 256;
    static constexpr int B_PER = BK * BN / 256;
    static_assert(WM * WN == 8, "256 threads");
    static_assert(MT >= 1 && NT >= 1, "warp tile");
    static_assert((BK * BM) % 256 == 0 && (BK * BN) % 256 == 0, "loader");
};

// Loads one k-slice of A (BM x 16) and B (16 x BN) into registers.  Threads
// walk the operand's contiguous direction so that global reads coalesce.
template <int BM, int BN, int WM, int WN>
struct MmaLoader {
    using C = MmaCfg<BM, BN, WM, WN>;
    double ra[C::A_PER], rb[C::B_PER];

    __device__ __forceinline__ void load(const Operand& A, const Operand& B, int M, int N, int K, int m0, int n0,
                                         int k0, bool a_rows, bool b_cols) {
        const int tid = threadIdx.x;
#pragma unroll
        for (int i = 0; i < C::A_PER; ++i) {
            const int e = tid + i * 256;
            const int kk = a_rows ? e / BM : e % C::BK;
            const int mm = a_rows ? e % BM : e / C::BK;
            const int m = m0 + mm, k = k0 + kk;
            ra[i] = (m < M && k < K) ? opnd_load(A, m, k) : 0.0;
        }
#pragma unroll
        for (int i = 0; i < C::B_PER; ++i) {
            const int e = tid + i * 256;
            const int kk = b_cols ? e / BN : e % C::BK;
            const int nn = b_cols ? e % BN : e / C::BK;
            const int n = n0 + nn, k = k0 + kk;
            rb[i] = (n < N && k < K) ? opnd_load(B, k, n) : 0.0;
        }
    }

    __device__ __forceinline__ void store(double* As, double* Bs, bool a_rows, bool b_cols) {
        const int tid = threadIdx.x;
#pragma unroll
        for (int i = 0; i < C::A_PER; ++i) {
            const int e = tid + i * 256;
            const int kk = a_rows ? e / BM : e % C::BK;
            const int mm = a_rows ? e % BM : e / C::BK;
            As[kk * C::PA + mm] = ra[i];
        }
#pragma unroll
        for (int i = 0; i < C::B_PER; ++i) {
            const int e = tid + i * 256;
            const int kk = b_cols ? e / BN : e % C::BK;
            const int nn = b_cols ? e % BN : e / C::BK;
            Bs[kk * C::PB + nn] = rb[i];
        }
    }
};

// The main loop: acc[MT][NT][2] += A_tile * B_tile over the whole contraction.
template <int BM, int BN, int WM, int WN>
__device__ __forceinline__ void mma_mainloop(const GemmDesc& d, int m0, int n0, double* smem,
                                             double (&acc)[MmaCfg<BM, BN, WM, WN>::MT][MmaCfg<BM, BN, WM, WN>::NT][2]) {
    using C = MmaCfg<BM, BN, WM, WN>;
    const Operand A = d.A, B = d.B;
    const int M = d.M, N = d.N, K = d.K;
    const bool a_rows = A.trans != 0;   // A(m,k) contiguous along m
    const bool b_cols = B.trans == 0;   // B(k,n) contiguous along n
    double* As[2] = {smem, smem + C::BK * C::PA};
    double* Bs[2] = {smem + 2 * C::BK * C::PA, smem + 2 * C::BK * C::PA + C::BK * C::PB};
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    const int wm0 = (warp / WN) * (8 * C::MT), wn0 = (warp % WN) * (8 * C::NT);
#pragma unroll
    for (int i = 0; i < C::MT; ++i)
#pragma unroll
        for (int j = 0; j < C::NT; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

    MmaLoader<BM, BN, WM, WN> ld;
    const int nk = (K + C::BK - 1) / C::BK;
    ld.load(A, B, M, N, K, m0, n0, 0, a_rows, b_cols);
    ld.store(As[0], Bs[0], a_rows, b_cols);
    __syncthreads();
    for (int s = 0; s < nk; ++s) {
        const int cur = s & 1;
        if (s + 1 < nk) ld.load(A, B, M, N, K, m0, n0, (s + 1) * C::BK, a_rows, b_cols);
        const double* as = As[cur];
        const double* bs = Bs[cur];
#pragma unroll
        for (int kq = 0; kq < C::BK / 4; ++kq) {
            double a[C::MT], b[C::NT];
#pragma unroll
            for (int i = 0; i < C::MT; ++i) a[i] = as[(kq * 4 + t) * C::PA + wm0 + i * 8 + g];
#pragma unroll
            for (int j = 0; j < C::NT; ++j) b[j] = bs[(kq * 4 + t) * C::PB + wn0 + j * 8 + g];
#pragma unroll
            for (int i = 0; i < C::MT; ++i)
#pragma unroll
                for (int j = 0; j < C::NT; ++j) mma_f64(acc[i][j][0], acc[i][j][1], a[i], b[j]);
        }
        if (s + 1 < nk) ld.store(As[cur ^ 1], Bs[cur ^ 1], a_rows, b_cols);
        __syncthreads();
    }
}

template <int BM, int BN, int WM, int WN>
constexpr int mma_smem_bytes() {
    return (int)sizeof(double) * 2 * MmaCfg<BM, BN, WM, WN>::BK * (MmaCfg<BM, BN, WM, WN>::PA + MmaCfg<BM, BN, WM, WN>::PB);
}

}  // namespace bdc

namespace bdc {

// ---------------------------------------------------------------------------
// Multi-stage variant for FP64 operands: tiles move global -> shared memory by
// cp.async (16-byte pieces, zero-filled past the operand's edge), STAGES deep,
// so that several k-slices are in flight without staging registers.  Each
// operand keeps its global orientation in shared memory:
//   AK: A k-major [BK][BM+4] (A contiguous along m) or m-major [BM][BK+4]
//   BKM: B k-major [BK][BN+4] (B contiguous along n) or n-major [BN][BK+4]
// Requirements (checked by the host): both operands FP64, 16-byte aligned
// bases, even leading dimensions and even contraction offsets.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int bytes) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

template <int BM, int BN, bool AK, bool BKM>
struct CpCfg {
    static constexpr int BK = 16;
    static constexpr int PK = BK + 4;
    static constexpr int A_ELEMS = AK ? BK * (BM + 4) : BM * PK;
    static constexpr int B_ELEMS = BKM ? BK * (BN + 4) : BN * PK;
    static constexpr int STAGE = A_ELEMS + B_ELEMS;
};

template <int BM, int BN, int WM, int WN, bool AK, bool BKM, int STAGES>
constexpr int mma_cp_smem_bytes() {
    return (int)sizeof(double) * STAGES * CpCfg<BM, BN, AK, BKM>::STAGE;
}

// one k-slice [k0, k0 + 16) of A and B into one stage
template <int BM, int BN, bool AK, bool BKM>
__device__ __forceinline__ void cp_stage(const GemmDesc& d, int m0, int n0, int k0, double* As, double* Bs) {
    using C = CpCfg<BM, BN, AK, BKM>;
    const double* A = (const double*)d.A.ptr;
    const double* B = (const double*)d.B.ptr;
    const int64_t lda = d.A.ld, ldb = d.B.ld;
    const int M = d.M, N = d.N, K = d.K;
    if (AK) {  // BK rows of BM doubles, pieces of two along m
        constexpr int PIECES = C::BK * BM / 2;
        for (int e = threadIdx.x; e < PIECES; e += 256) {
            const int kk = e / (BM / 2), mm = (e % (BM / 2)) * 2;
            const int k = k0 + kk, m = m0 + mm;
            const int bytes = (k < K) ? (m + 1 < M ? 16 : (m < M ? 8 : 0)) : 0;
            cp_async16(As + kk * (BM + 4) + mm, bytes ? A + (int64_t)k * lda + m : A, bytes);
        }
    } else {  // BM rows of BK doubles, pieces of two along k
        constexpr int PIECES = BM * C::BK / 2;
        for (int e = threadIdx.x; e < PIECES; e += 256) {
            const int mm = e / (C::BK / 2), kk = (e % (C::BK / 2)) * 2;
            const int k = k0 + kk, m = m0 + mm;
            const int bytes = (m < M) ? (k + 1 < K ? 16 : (k < K ? 8 : 0)) : 0;
            cp_async16(As + mm * C::PK + kk, bytes ? A + (int64_t)m * lda + k : A, bytes);
        }
    }
    if (BKM) {
        constexpr int PIECES = C::BK * BN / 2;
        for (int e = threadIdx.x; e < PIECES; e += 256) {
            const int kk = e / (BN / 2), nn = (e % (BN / 2)) * 2;
            const int k = k0 + kk, n = n0 + nn;
            const int bytes = (k < K) ? (n + 1 < N ? 16 : (n < N ? 8 : 0)) : 0;
            cp_async16(Bs + kk * (BN + 4) + nn, bytes ? B + (int64_t)k * ldb + n : B, bytes);
        }
    } else {
        constexpr int PIECES = BN * C::BK / 2;
        for (int e = threadIdx.x; e < PIECES; e += 256) {
            const int nn = e / (C::BK / 2), kk = (e % (C::BK / 2)) * 2;
            const int k = k0 + kk, n = n0 + nn;
            const int bytes = (n < N) ? (k + 1 < K ? 16 : (k < K ? 8 : 0)) : 0;
            cp_async16(Bs + nn * C::PK + kk, bytes ? B + (int64_t)n * ldb + k : B, bytes);
        }
    }
}

// The first STAGES-1 stages of a tile's operands, in flight on return.  Issued
// by every thread; the shared memory of those stages must be free (after the
// previous tile's body, which ends with all copies landed and a barrier).
template <int BM, int BN, bool AK, bool BKM, int STAGES>
__device__ __forceinline__ void mma_cp_prologue(const GemmDesc& d, int m0, int n0, double* smem) {
    using C = CpCfg<BM, BN, AK, BKM>;
    const int nk = (d.K + C::BK - 1) / C::BK;
#pragma unroll
    for (int st = 0; st < STAGES - 1; ++st) {
        if (st < nk) cp_stage<BM, BN, AK, BKM>(d, m0, n0, st * C::BK, smem + st * C::STAGE, smem + st * C::STAGE + C::A_ELEMS);
        cp_async_commit();
    }
}

// The k loop of one tile whose prologue is in flight; returns with every copy
// landed and the shared memory free.
template <int BM, int BN, int WM, int WN, bool AK, bool BKM, int STAGES>
__device__ __forceinline__ void mma_cp_body(const GemmDesc& d, int m0, int n0, double* smem,
                                            double (&acc)[MmaCfg<BM, BN, WM, WN>::MT][MmaCfg<BM, BN, WM, WN>::NT][2]) {
    using M_ = MmaCfg<BM, BN, WM, WN>;
    using C = CpCfg<BM, BN, AK, BKM>;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    const int wm0 = (warp / WN) * (8 * M_::MT), wn0 = (warp % WN) * (8 * M_::NT);
#pragma unroll
    for (int i = 0; i < M_::MT; ++i)
#pragma unroll
        for (int j = 0; j < M_::NT; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
    const int nk = (d.K + C::BK - 1) / C::BK;
    for (int kt = 0; kt < nk; ++kt) {
        cp_async_wait<STAGES - 2>();
        __syncthreads();
        {
            const int nx = kt + STAGES - 1;
            if (nx < nk) {
                double* s = smem + (nx % STAGES) * C::STAGE;
                cp_stage<BM, BN, AK, BKM>(d, m0, n0, nx * C::BK, s, s + C::A_ELEMS);
            }
            cp_async_commit();
        }
        const double* as = smem + (kt % STAGES) * C::STAGE;
        const double* bs = as + C::A_ELEMS;
#pragma unroll
        for (int kq = 0; kq < C::BK / 4; ++kq) {
            double a[M_::MT], b[M_::NT];
            const int kr = kq * 4 + t;
#pragma unroll
            for (int i = 0; i < M_::MT; ++i) {
                const int m = wm0 + i * 8 + g;
                a[i] = AK ? as[kr * (BM + 4) + m] : as[m * C::PK + kr];
            }
#pragma unroll
            for (int j = 0; j < M_::NT; ++j) {
                const int n = wn0 + j * 8 + g;
                b[j] = BKM ? bs[kr * (BN + 4) + n] : bs[n * C::PK + kr];
            }
#pragma unroll
            for (int i = 0; i < M_::MT; ++i)
#pragma unroll
                for (int j = 0; j < M_::NT; ++j) mma_f64(acc[i][j][0], acc[i][j][1], a[i], b[j]);
        }
    }
    cp_async_wait<0>();
    __syncthreads();
}

template <int BM, int BN, int WM, int WN, bool AK, bool BKM, int STAGES>
__device__ __forceinline__ void mma_mainloop_cp(const GemmDesc& d, int m0, int n0, double* smem,
                                                double (&acc)[MmaCfg<BM, BN, WM, WN>::MT][MmaCfg<BM, BN, WM, WN>::NT][2]) {
    mma_cp_prologue<BM, BN, AK, BKM, STAGES>(d, m0, n0, smem);
    mma_cp_body<BM, BN, WM, WN, AK, BKM, STAGES>(d, m0, n0, smem, acc);
}

}  // namespace bdc
