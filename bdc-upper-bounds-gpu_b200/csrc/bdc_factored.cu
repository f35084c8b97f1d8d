// bdc_factored.cu -- the factored engine: one BA iteration as FP64 matrix
// products over the half tables, with the BA update fused into the largest one.
//
// Reference path replaced (Pintz45/BDC-Upper-Bounds-GPU): the same iteration
// as backend/BAA.cu:590-639 (q pass 429-485, D pass 487-530, normalisation
// 590-639, max deviation 916-946).  The reference evaluates N(x,y) pair by
// pair through the split identity (total_transitions, BAA.cu:340-395):
//     N(x, y) = sum_j A_j[x_hi][y_hi] * B_{k-j}[x_lo][y_lo],
// A_j = cache_{n1,j}, B_m = cache_{n2,m}.  For fixed j this is a Kronecker
// product, so with the iterate laid out as a 2^{n1} x 2^{n2} matrix P:
//   q-side:  Q_j = A_j^T P B_{k-j}                    (2^j x 2^{k-j} block of q)
//   D-side:  G   = sum_j A_j Lq_j B_{k-j}^T,  D(x) = h(x) - G(x) / C(n,k)
// with Lq_j = ln q reshaped to 2^j x 2^{k-j} and h(x) = sum_y W ln W (from
// the count path, once per handle).  Each term is evaluated in the cheaper
// association: "L" terms (2^j <= 2^{k-j}) contract x_hi first, "R" terms
// contract x_lo first.  Per iteration:
//   1. UL = AL^T Pw, VR = Pw BR        (Pw = |O(x)| p(x) at representatives,
//                                        0 elsewhere; AL, BR = the L / R tables)
//   2. Q_t = U_t B_m (L), A_j^T V_t (R) -> q parts; fold orbits -> ln q
//   3. M_t = Lq_t B_m^T (L), N_t = A_j Lq_t (R) -> operands of step 4
//   4. G = [AL | NR] [ML ; BR^T] with the BA update as epilogue: D, logW,
//      exp(logW - shift), the new iterate (in place) and block partials of
//      max D, sum |O| e, max logW, sum |O| p D
//   5. one-block finalize: ln Z, mx, upper bound, stop test, next shift.
// Counts are exact (integers <= 2^16 widened to FP64); all sums are FP64.
#include <cfloat>
#include <cmath>
#include <vector>

#include "bdc_engine.cuh"
#include "bdc_gemm.cuh"

namespace bdc {

constexpr int kErrShift = 1;  // DevState::error: exp shift out of range, re-scale

struct Term {
    int j, m;       // split point and the low sub-length k - j
    int left;       // 1: L term (contract x_hi first), 0: R term
    int off;        // column offset inside AL (L) or BR (R)
    int idA, idB;   // A_j / B_m is the identity (j == n1 / m == n2)
};

}  // namespace bdc

struct FactoredState {
    int H1 = 0, H2 = 0, KL = 0, KR = 0, Kp = 0, T = 0;
    std::vector<bdc::Term> terms;
    double* Pw = nullptr;     // [2^n]  |O(x)| e(x) at representatives, 0 elsewhere
    double* Lt = nullptr;     // [2^n]  ln e(x) (p = e / Z)
    double* hx = nullptr;     // [2^n]  h(x) at representatives
    double* LA = nullptr;     // [H1][Kp]  = [AL | NR]
    double* RB = nullptr;     // [Kp][H2]  = [ML ; BR^T]
    double* UL = nullptr;     // [KL][H2]
    double* VR = nullptr;     // [H1][KR]
    double* ulpart = nullptr; // [S1][KL][H2]
    double* vrpart = nullptr; // [S2][H1][KR]
    int S1 = 1, S2 = 1;
    double* qparts = nullptr; // [T][2^k]
    double* lnq_full = nullptr;  // [2^k]
    double* epart = nullptr;  // [ctas][4]
    int ctas_g = 0;
    // launch plans
    bdc::GemmDesc* d_big = nullptr;  int n_big = 0, tiles_big = 0;     // UL, VR partials
    bdc::GemmDesc* d_qrows = nullptr; int n_qrows = 0, tiles_qrows = 0;
    bdc::GemmDesc* d_qtile = nullptr; int n_qtile = 0, tiles_qtile = 0;
    bdc::GemmDesc* d_drows = nullptr; int n_drows = 0, tiles_drows = 0;
    bdc::GemmDesc* d_dtile = nullptr; int n_dtile = 0, tiles_dtile = 0;
    bdc::GemmDesc* d_g = nullptr;
    int launches_per_iter = 0;
};

namespace bdc {

// ---------------------------------------------------------------- helpers
__device__ __forceinline__ double op_load(const Operand& o, int64_t r, int64_t c) {
    if (o.kind == OP_EYE) return r == c ? 1.0 : 0.0;
    const int64_t idx = o.trans ? c * o.ld + r : r * o.ld + c;
    if (o.kind == OP_U16) return (double)__ldg((const uint16_t*)o.ptr + idx);
    return __ldg((const double*)o.ptr + idx);
}

// element (r, c) is contiguous along c (row-major storage) unless transposed
__device__ __forceinline__ bool contiguous_in_rows(const Operand& o) { return o.trans != 0; }

__device__ __forceinline__ int find_desc(const GemmDesc* d, int nd, int t) {
    int i = 0;
    while (i + 1 < nd && d[i + 1].tile_begin <= t) ++i;
    return i;
}

__device__ __forceinline__ bool gated(const DevState* st) { return st && (st->done || st->error); }

// ------------------------------------------------------------ tiled GEMM
// 256 threads = WARPS_M x WARPS_N warps; a warp is 4 (m) x 8 (n) lanes; a
// thread owns rows mbase + q*8 + {0,1} (q < TM/2) and columns
// nbase + q*16 + {0,1} (q < TN/2), so that each shared-memory fragment load
// is one 16-byte access per lane with broadcast (A) or contiguous (B) lanes.
template <int BM, int BN, int BK, int WARPS_M, int WARPS_N, int EPI>
__global__ void __launch_bounds__(256) k_gemm_tile(const GemmDesc* __restrict__ descs, int ndesc,
                                                   BaEpilogue ep, const DevState* st) {
    constexpr int TM = BM / (WARPS_M * 4);
    constexpr int TN = BN / (WARPS_N * 8);
    static_assert(WARPS_M * WARPS_N == 8, "256 threads");
    static_assert(TM % 2 == 0 && TN % 2 == 0, "pairs");
    constexpr int A_PER = BK * BM / 256;
    constexpr int B_PER = BK * BN / 256;
    if (gated(st)) return;
    const int di = find_desc(descs, ndesc, blockIdx.x);
    const GemmDesc& d = descs[di];
    const Operand A = d.A, B = d.B;
    const int M = d.M, N = d.N, K = d.K;
    const int t = blockIdx.x - d.tile_begin;
    const int m0 = (t / d.tiles_n) * BM, n0 = (t % d.tiles_n) * BN;

    __shared__ __align__(16) double As[2][BK][BM];
    __shared__ __align__(16) double Bs[2][BK][BN];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int wm = warp / WARPS_N, wn = warp % WARPS_N;
    const int mbase = wm * (BM / WARPS_M) + (lane >> 3) * 2;
    const int nbase = wn * (BN / WARPS_N) + (lane & 7) * 2;
    const bool a_rows = contiguous_in_rows(A);   // A(m,k) contiguous along m
    const bool b_cols = !contiguous_in_rows(B);  // B(k,n) contiguous along n

    double ra[A_PER], rb[B_PER];
    auto gload = [&](int k0) {
#pragma unroll
        for (int i = 0; i < A_PER; ++i) {
            const int e = tid + i * 256;
            const int kk = a_rows ? e / BM : e % BK;
            const int mm = a_rows ? e % BM : e / BK;
            const int m = m0 + mm, k = k0 + kk;
            ra[i] = (m < M && k < K) ? op_load(A, m, k) : 0.0;
        }
#pragma unroll
        for (int i = 0; i < B_PER; ++i) {
            const int e = tid + i * 256;
            const int kk = b_cols ? e / BN : e % BK;
            const int nn = b_cols ? e % BN : e / BK;
            const int n = n0 + nn, k = k0 + kk;
            rb[i] = (n < N && k < K) ? op_load(B, k, n) : 0.0;
        }
    };
    auto sstore = [&](int buf) {
#pragma unroll
        for (int i = 0; i < A_PER; ++i) {
            const int e = tid + i * 256;
            const int kk = a_rows ? e / BM : e % BK;
            const int mm = a_rows ? e % BM : e / BK;
            As[buf][kk][mm] = ra[i];
        }
#pragma unroll
        for (int i = 0; i < B_PER; ++i) {
            const int e = tid + i * 256;
            const int kk = b_cols ? e / BN : e % BK;
            const int nn = b_cols ? e % BN : e / BK;
            Bs[buf][kk][nn] = rb[i];
        }
    };

    double acc[TM][TN];
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) acc[i][j] = 0.0;

    const int nk = (K + BK - 1) / BK;
    gload(0);
    sstore(0);
    __syncthreads();
    for (int s = 0; s < nk; ++s) {
        const int cur = s & 1;
        if (s + 1 < nk) gload((s + 1) * BK);
#pragma unroll
        for (int kk = 0; kk < BK; ++kk) {
            double a[TM], b[TN];
#pragma unroll
            for (int q = 0; q < TM / 2; ++q) {
                const double2 v = *reinterpret_cast<const double2*>(&As[cur][kk][mbase + q * 8]);
                a[2 * q] = v.x;
                a[2 * q + 1] = v.y;
            }
#pragma unroll
            for (int q = 0; q < TN / 2; ++q) {
                const double2 v = *reinterpret_cast<const double2*>(&Bs[cur][kk][nbase + q * 16]);
                b[2 * q] = v.x;
                b[2 * q + 1] = v.y;
            }
#pragma unroll
            for (int i = 0; i < TM; ++i)
#pragma unroll
                for (int j = 0; j < TN; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
        }
        if (s + 1 < nk) sstore(cur ^ 1);
        __syncthreads();
    }

    if (EPI == 0) {
#pragma unroll
        for (int i = 0; i < TM; ++i) {
            const int m = m0 + mbase + (i >> 1) * 8 + (i & 1);
            if (m >= M) continue;
#pragma unroll
            for (int j = 0; j < TN; ++j) {
                const int n = n0 + nbase + (j >> 1) * 16 + (j & 1);
                if (n >= N) continue;
                double* c = d.C + (int64_t)m * d.ldc_m + (int64_t)n * d.ldc_n;
                const double v = d.alpha * acc[i][j];
                *c = d.accumulate ? *c + v : v;
            }
        }
        return;
    }

    // ---- BA epilogue: rows are x_hi, columns x_lo, x = (x_hi << n2) | x_lo
    const double shift = st->shift;
    const double lnz = st->log_z;
    double mD = -DBL_MAX, sE = 0.0, mL = -DBL_MAX, sR = 0.0;
#pragma unroll
    for (int i = 0; i < TM; ++i) {
        const int m = m0 + mbase + (i >> 1) * 8 + (i & 1);
        if (m >= M) continue;
#pragma unroll
        for (int j = 0; j < TN; ++j) {
            const int n = n0 + nbase + (j >> 1) * 16 + (j & 1);
            if (n >= N) continue;
            const uint32_t x = ((uint32_t)m << ep.n2) | (uint32_t)n;
            if (!is_rep(x, ep.n)) continue;
            const double o = (double)orbit_size(x, ep.n);
            const double D = __ldg(ep.hx + x) - acc[i][j] * ep.inv_c;
            const double lnp = ep.Lt[x] - lnz;
            const double lw = lnp + D - shift;
            const double e = exp(lw);
            ep.Lt[x] = lw;
            ep.Pw[x] = o * e;
            mD = fmax(mD, D);
            mL = fmax(mL, lw);
            sE = fma(o, e, sE);
            sR = fma(o * exp(lnp), D, sR);
        }
    }
    // CTA reduction of the four partials
    __shared__ double red[4][8];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        mD = fmax(mD, __shfl_xor_sync(0xFFFFFFFFu, mD, off));
        mL = fmax(mL, __shfl_xor_sync(0xFFFFFFFFu, mL, off));
        sE += __shfl_xor_sync(0xFFFFFFFFu, sE, off);
        sR += __shfl_xor_sync(0xFFFFFFFFu, sR, off);
    }
    if (lane == 0) {
        red[0][warp] = mD;
        red[1][warp] = sE;
        red[2][warp] = mL;
        red[3][warp] = sR;
    }
    __syncthreads();
    if (tid == 0) {
        double a0 = red[0][0], a1 = red[1][0], a2 = red[2][0], a3 = red[3][0];
        for (int w = 1; w < 8; ++w) {
            a0 = fmax(a0, red[0][w]);
            a1 += red[1][w];
            a2 = fmax(a2, red[2][w]);
            a3 += red[3][w];
        }
        double* p = ep.part + (size_t)blockIdx.x * 4;
        p[0] = a0;
        p[1] = a1;
        p[2] = a2;
        p[3] = a3;
    }
}

// --------------------------------------------------------- few-row GEMM
// Output rows M <= 8.  CTA = 64 columns x 4 K-slices; the chunk of B is
// staged in shared memory whatever its storage order; A is broadcast.
constexpr int kRowsMax = 8;
constexpr int kRowsCols = 64;
constexpr int kRowsKC = 32;

__global__ void __launch_bounds__(256) k_gemm_rows(const GemmDesc* __restrict__ descs, int ndesc,
                                                   const DevState* st) {
    if (gated(st)) return;
    const int di = find_desc(descs, ndesc, blockIdx.x);
    const GemmDesc& d = descs[di];
    const Operand A = d.A, B = d.B;
    const int M = d.M, N = d.N, K = d.K;
    const int t = blockIdx.x - d.tile_begin;
    const int n0 = t * kRowsCols;
    __shared__ double As[kRowsMax][kRowsKC];
    __shared__ double Bs[kRowsKC][kRowsCols + 1];
    __shared__ double red[4][kRowsMax][kRowsCols];
    const int tid = threadIdx.x;
    const int col = tid & (kRowsCols - 1);
    const int ks = tid >> 6;  // 0..3
    const bool b_cols = !contiguous_in_rows(B);
    double acc[kRowsMax];
#pragma unroll
    for (int r = 0; r < kRowsMax; ++r) acc[r] = 0.0;
    for (int k0 = 0; k0 < K; k0 += kRowsKC) {
        for (int e = tid; e < kRowsMax * kRowsKC; e += 256) {
            const int r = e / kRowsKC, kk = e % kRowsKC;
            As[r][kk] = (r < M && k0 + kk < K) ? op_load(A, r, k0 + kk) : 0.0;
        }
        for (int e = tid; e < kRowsKC * kRowsCols; e += 256) {
            const int kk = b_cols ? e / kRowsCols : e % kRowsKC;
            const int nn = b_cols ? e % kRowsCols : e / kRowsKC;
            const int n = n0 + nn, k = k0 + kk;
            Bs[kk][nn] = (n < N && k < K) ? op_load(B, k, n) : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int kk = ks; kk < kRowsKC; kk += 4) {
            const double b = Bs[kk][col];
#pragma unroll
            for (int r = 0; r < kRowsMax; ++r) acc[r] = fma(As[r][kk], b, acc[r]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int r = 0; r < kRowsMax; ++r) red[ks][r][col] = acc[r];
    __syncthreads();
    for (int e = tid; e < kRowsMax * kRowsCols; e += 256) {
        const int r = e / kRowsCols, c = e % kRowsCols;
        const int n = n0 + c;
        if (r >= M || n >= N) continue;
        const double v = d.alpha * (red[0][r][c] + red[1][r][c] + red[2][r][c] + red[3][r][c]);
        double* cp = d.C + (int64_t)r * d.ldc_m + (int64_t)n * d.ldc_n;
        *cp = d.accumulate ? *cp + v : v;
    }
}

// ------------------------------------------------------------ small kernels
// out[i] = sum_s part[s * stride + i] for the UL and VR split-K partials
__global__ void k_sum_parts(const double* __restrict__ a, int sa, int64_t na, double* __restrict__ oa,
                            const double* __restrict__ b, int sb, int64_t nb, double* __restrict__ ob,
                            const DevState* st) {
    if (gated(st)) return;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < na + nb;
         i += (int64_t)gridDim.x * blockDim.x) {
        if (i < na) {
            double s = 0.0;
            for (int p = 0; p < sa; ++p) s += a[(int64_t)p * na + i];
            oa[i] = s;
        } else {
            const int64_t j = i - na;
            double s = 0.0;
            for (int p = 0; p < sb; ++p) s += b[(int64_t)p * nb + j];
            ob[j] = s;
        }
    }
}

// acc[y] = sum_t qparts[t][y]; q(rep r) = sum_{y in O(r)} acc[y] / (|O(r)| C Z);
// ln q with the reference's 0 for q == 0; expanded to every y.
__global__ void k_fold_q(const double* __restrict__ qparts, int T, int k, double inv_c,
                         double* __restrict__ lnq_full, double* __restrict__ lnq, const DevState* st) {
    if (gated(st)) return;
    const int ny = 1 << k;
    const double inv_z = exp(-st->log_z);
    for (int y = blockIdx.x * blockDim.x + threadIdx.x; y < ny; y += gridDim.x * blockDim.x) {
        const uint32_t r = orbit_rep((uint32_t)y, k);
        const uint32_t rv = reverse_bits(r, k), cv = complement_bits(r, k), rcv = reverse_bits(cv, k);
        uint32_t mem[4];
        int nm = 0;
        mem[nm++] = r;
        if (rv != r) mem[nm++] = rv;
        if (cv != r && cv != rv) mem[nm++] = cv;
        if (rcv != r && rcv != rv && rcv != cv) mem[nm++] = rcv;
        double acc = 0.0;
        for (int e = 0; e < nm; ++e)
            for (int t = 0; t < T; ++t) acc += qparts[(size_t)t * ny + mem[e]];
        const double q = acc * inv_c * inv_z / (double)nm;
        const double lq = (q != 0.0) ? log(q) : 0.0;
        lnq_full[y] = lq;
        if ((uint32_t)y == r) lnq[y] = lq;  // representatives are < 2^{k-1}
    }
}

__global__ void __launch_bounds__(256)
k_fac_finalize(const double* __restrict__ part, int nb, double a, DevState* st) {
    if (gated(st)) return;
    __shared__ double red[4][256];
    double mD = -DBL_MAX, sE = 0.0, mL = -DBL_MAX, sR = 0.0;
    for (int b = threadIdx.x; b < nb; b += 256) {
        mD = fmax(mD, part[(size_t)b * 4 + 0]);
        sE += part[(size_t)b * 4 + 1];
        mL = fmax(mL, part[(size_t)b * 4 + 2]);
        sR += part[(size_t)b * 4 + 3];
    }
    red[0][threadIdx.x] = mD;
    red[1][threadIdx.x] = sE;
    red[2][threadIdx.x] = mL;
    red[3][threadIdx.x] = sR;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            red[0][threadIdx.x] = fmax(red[0][threadIdx.x], red[0][threadIdx.x + s]);
            red[1][threadIdx.x] += red[1][threadIdx.x + s];
            red[2][threadIdx.x] = fmax(red[2][threadIdx.x], red[2][threadIdx.x + s]);
            red[3][threadIdx.x] += red[3][threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x != 0) return;
    mD = red[0][0];
    sE = red[1][0];
    mL = red[2][0];
    sR = red[3][0];
    if (!(sE > 0.0) || !isfinite(sE) || mL > 600.0 || mL < -600.0) {
        st->error = kErrShift;  // e over/underflowed: re-scale from Lt, then finish
        st->max_logw = mL;      // relative to shift; k_fac_rescale subtracts it
        st->max_d = mD;
        st->rate = sR;
        return;
    }
    // Lt holds logW - shift, so ln p' - ln p = D - shift - ln Z
    const double lnz = log(sE);
    const double ln2 = 0.69314718055994530942;
    const double mx = st->zero_p ? INFINITY : (mD - st->shift - lnz) / ln2;
    st->max_d = mD;
    st->rate = sR;
    st->lse = st->shift + lnz;
    st->mx = mx;
    st->max_logw = mL + st->shift;
    st->log_z = lnz;
    // next shift: the largest new ln p plus the current bound on D
    st->shift = (mL - lnz) + mD;
    st->zero_p = 0;
    st->iter += 1;
    st->done = !(mx >= a);
}

// re-scale after an exp over/underflow: Lt -= s, Pw = |O| exp(Lt), sum
__global__ void __launch_bounds__(256)
k_fac_rescale(const uint32_t* __restrict__ reps, int64_t R, int n, double* Lt, double* Pw,
              double* part, DevState* st) {
    const double s = st->max_logw;  // max of Lt after the failed epilogue
    double sum = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < R; i += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t x = reps[i];
        const double l = Lt[x] - s;
        const double o = (double)orbit_size(x, n);
        Lt[x] = l;
        const double e = exp(l);
        Pw[x] = o * e;
        sum = fma(o, e, sum);
    }
    __shared__ double red[256];
    red[threadIdx.x] = sum;
    __syncthreads();
    for (int t = 128; t > 0; t >>= 1) {
        if (threadIdx.x < t) red[threadIdx.x] += red[threadIdx.x + t];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

__global__ void k_fac_rescale_finish(const double* part, int nb, double a, DevState* st) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double sE = 0.0;
    for (int b = 0; b < nb; ++b) sE += part[b];
    // Lt now holds logW - (shift + s) with maximum 0
    const double shift_eff = st->shift + st->max_logw;
    const double lnz = log(sE);
    const double ln2 = 0.69314718055994530942;
    const double mx = st->zero_p ? INFINITY : (st->max_d - shift_eff - lnz) / ln2;
    st->lse = shift_eff + lnz;
    st->mx = mx;
    st->max_logw = shift_eff;
    st->log_z = lnz;
    st->shift = -lnz + st->max_d;
    st->zero_p = 0;
    st->error = 0;
    st->iter += 1;
    st->done = !(mx >= a);
}

// p -> (Pw, Lt) at representatives; block max of ln p for the first shift
__global__ void __launch_bounds__(256)
k_fac_load(const uint32_t* __restrict__ reps, int64_t R, int n, const double* __restrict__ p,
           double* Pw, double* Lt, double* part, DevState* st) {
    double mx = -DBL_MAX;
    int zero = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < R; i += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t x = reps[i];
        const double v = p[i];
        Pw[x] = (double)orbit_size(x, n) * v;
        const double l = (v != 0.0) ? log(v) : 0.0;  // ln 0 = 0 (backend/BAA.cu:573-580)
        Lt[x] = l;
        mx = fmax(mx, l);
        if (v == 0.0) zero = 1;
    }
    __shared__ double red[256];
    __shared__ int zr[256];
    red[threadIdx.x] = mx;
    zr[threadIdx.x] = zero;
    __syncthreads();
    for (int t = 128; t > 0; t >>= 1) {
        if (threadIdx.x < t) {
            red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + t]);
            zr[threadIdx.x] |= zr[threadIdx.x + t];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = red[0];
        part[2 * blockIdx.x + 1] = (double)zr[0];
    }
}

__global__ void k_fac_load_finish(const double* part, int nb, int k, DevState* st) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double mx = -DBL_MAX, z = 0.0;
    for (int b = 0; b < nb; ++b) {
        mx = fmax(mx, part[2 * b]);
        z = fmax(z, part[2 * b + 1]);
    }
    st->log_z = 0.0;
    st->shift = mx + (double)k * 0.69314718055994530942;  // first guess; re-scaled if off
    st->zero_p = (z != 0.0);
}

// p per representative from the dense state: p = Pw / (|O| Z)
__global__ void k_fac_store(const uint32_t* __restrict__ reps, int64_t R, int n,
                            const double* __restrict__ Pw, double* __restrict__ p, const DevState* st) {
    const double inv_z = exp(-st->log_z);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < R; i += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t x = reps[i];
        p[i] = Pw[x] * inv_z / (double)orbit_size(x, n);
    }
}

// scatter h per representative into the dense layout
__global__ void k_scatter(const uint32_t* __restrict__ reps, int64_t R, const double* __restrict__ v,
                          double* __restrict__ dense) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < R; i += (int64_t)gridDim.x * blockDim.x)
        dense[reps[i]] = v[i];
}

// constant parts of LA (AL columns) and RB (BR^T rows) from the bundles
__global__ void k_fill_tables(int H1, int H2, int Kp, const uint16_t* __restrict__ bhi, int strideA,
                              const uint16_t* __restrict__ blo, int strideB, const int* __restrict__ colmap,
                              int KL, int KR, double* LA, double* RB) {
    // colmap[c] for c < KL: bundle offset (of A_j) of AL column c;
    // colmap[KL + c] for c < KR: bundle offset (of B_m) of BR column c
    const int64_t nA = (int64_t)H1 * KL, nB = (int64_t)KR * H2;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nA + nB;
         e += (int64_t)gridDim.x * blockDim.x) {
        if (e < nA) {
            const int64_t xh = e / KL;
            const int c = (int)(e % KL);
            LA[xh * Kp + c] = (double)bhi[xh * strideA + colmap[c]];
        } else {
            const int64_t f = e - nA;
            const int c = (int)(f / H2);
            const int64_t xl = f % H2;
            RB[(int64_t)(KL + c) * H2 + xl] = (double)blo[xl * strideB + colmap[KL + c]];
        }
    }
}

// ------------------------------------------------------------ planning
using TileBig = void (*)(const GemmDesc*, int, BaEpilogue, const DevState*);

static Operand op_f64(const double* p, int64_t ld, int trans) {
    Operand o;
    o.ptr = p;
    o.ld = ld;
    o.kind = OP_F64;
    o.trans = trans;
    return o;
}
static Operand op_u16(const uint16_t* p, int64_t ld, int trans) {
    Operand o;
    o.ptr = p;
    o.ld = ld;
    o.kind = OP_U16;
    o.trans = trans;
    return o;
}
static Operand op_eye() {
    Operand o;
    o.kind = OP_EYE;
    return o;
}
static Operand op_t(Operand o) {
    if (o.kind != OP_EYE) o.trans ^= 1;
    return o;
}

static GemmDesc make_desc(Operand A, Operand B, double* C, int64_t ldc_m, int64_t ldc_n, int M, int N, int K) {
    GemmDesc d{};
    d.A = A;
    d.B = B;
    d.C = C;
    d.ldc_m = ldc_m;
    d.ldc_n = ldc_n;
    d.M = M;
    d.N = N;
    d.K = K;
    d.alpha = 1.0;
    d.accumulate = 0;
    return d;
}

// C^T = B^T A^T: the same product with the roles of rows and columns swapped
static GemmDesc transposed(const GemmDesc& d) {
    GemmDesc t = make_desc(op_t(d.B), op_t(d.A), d.C, d.ldc_n, d.ldc_m, d.N, d.M, d.K);
    t.alpha = d.alpha;
    t.accumulate = d.accumulate;
    return t;
}

struct Plan {
    std::vector<GemmDesc> rows, tiles;
};

// route one small product to the few-row kernel (after transposing if it is
// the column count that is small) or to the 64x64 tile kernel
static void route(Plan& P, const GemmDesc& d) {
    if (d.M <= kRowsMax) P.rows.push_back(d);
    else if (d.N <= kRowsMax) P.rows.push_back(transposed(d));
    else P.tiles.push_back(d);
}

static int assign_tiles(std::vector<GemmDesc>& v, int bm, int bn) {
    int t = 0;
    for (auto& d : v) {
        d.tiles_m = (d.M + bm - 1) / bm;
        d.tiles_n = (d.N + bn - 1) / bn;
        d.tile_begin = t;
        t += d.tiles_m * d.tiles_n;
    }
    return t;
}

static int assign_rows(std::vector<GemmDesc>& v) {
    int t = 0;
    for (auto& d : v) {
        d.tiles_m = 1;
        d.tiles_n = (d.N + kRowsCols - 1) / kRowsCols;
        d.tile_begin = t;
        t += d.tiles_n;
    }
    return t;
}

static cudaError_t upload(std::vector<GemmDesc>& v, GemmDesc** dst) {
    if (v.empty()) return cudaSuccess;
    cudaError_t e = cudaMalloc(dst, sizeof(GemmDesc) * v.size());
    if (e != cudaSuccess) return e;
    return cudaMemcpy(*dst, v.data(), sizeof(GemmDesc) * v.size(), cudaMemcpyHostToDevice);
}

bool factored_supports(int n, int k) {
    // needs k < n (W is not the identity), half lengths that fit the uint16
    // bundles, and a dense 2^n state that fits comfortably in device memory
    return k >= 1 && k < n && n >= 4 && n <= 28 && k <= 14;
}

bdc_status factored_init(bdc_handle* H) {
    FactoredState* F = new FactoredState();
    H->fac = F;
    const Split& s = H->s;
    F->H1 = 1 << s.n1;
    F->H2 = 1 << s.n2;
    const int k = H->k;
    // terms and their association
    int KL = 0, KR = 0;
    for (int j = s.jlo; j <= s.jhi; ++j) {
        Term t{};
        t.j = j;
        t.m = k - j;
        t.idA = (j == s.n1);
        t.idB = (t.m == s.n2);
        if (t.idA && t.idB) return fail(BDC_ERR_UNSUPPORTED, "factored engine: k == n");
        t.left = t.idB ? 1 : (t.idA ? 0 : (j <= t.m));
        F->terms.push_back(t);
    }
    for (auto& t : F->terms) {
        if (t.left) { t.off = KL; KL += 1 << t.j; }
    }
    for (auto& t : F->terms) {
        if (!t.left) { t.off = KR; KR += 1 << t.m; }
    }
    F->KL = KL;
    F->KR = KR;
    F->Kp = (KL + KR + 7) / 8 * 8;
    F->T = (int)F->terms.size();
    const int64_t NX = (int64_t)1 << H->n;
    const int ny = 1 << k;
    const int H1 = F->H1, H2 = F->H2, Kp = F->Kp;

    // device buffers
    auto al = [&](double** p, size_t cnt) -> cudaError_t {
        H->bytes += cnt * sizeof(double);
        return cudaMalloc(p, cnt * sizeof(double) + 16);
    };
    BDC_CUDA_TRY(al(&F->Pw, NX));
    BDC_CUDA_TRY(al(&F->Lt, NX));
    BDC_CUDA_TRY(al(&F->hx, NX));
    BDC_CUDA_TRY(al(&F->LA, (size_t)H1 * Kp));
    BDC_CUDA_TRY(al(&F->RB, (size_t)Kp * H2));
    BDC_CUDA_TRY(al(&F->UL, (size_t)(KL > 0 ? KL : 1) * H2));
    BDC_CUDA_TRY(al(&F->VR, (size_t)H1 * (KR > 0 ? KR : 1)));
    // split-K so that the two thin products fill the GPU
    F->S1 = KL > 0 ? std::max(1, std::min(32, (H->num_sms * 4) / std::max(1, ((KL + 127) / 128) * ((H2 + 127) / 128)))) : 1;
    F->S2 = KR > 0 ? std::max(1, std::min(32, (H->num_sms * 4) / std::max(1, ((H1 + 127) / 128) * ((KR + 127) / 128)))) : 1;
    while (F->S1 > 1 && H1 % F->S1) --F->S1;
    while (F->S2 > 1 && H2 % F->S2) --F->S2;
    BDC_CUDA_TRY(al(&F->ulpart, (size_t)F->S1 * (KL > 0 ? KL : 1) * H2));
    BDC_CUDA_TRY(al(&F->vrpart, (size_t)F->S2 * H1 * (KR > 0 ? KR : 1)));
    BDC_CUDA_TRY(al(&F->qparts, (size_t)F->T * ny));
    BDC_CUDA_TRY(al(&F->lnq_full, (size_t)ny));
    F->ctas_g = ((H1 + 127) / 128) * ((H2 + 127) / 128);
    BDC_CUDA_TRY(al(&F->epart, (size_t)std::max(F->ctas_g, 2 * H->nb_upd) * 4));
    BDC_CUDA_TRY(cudaMemsetAsync(F->LA, 0, sizeof(double) * H1 * Kp, H->stream));
    BDC_CUDA_TRY(cudaMemsetAsync(F->RB, 0, sizeof(double) * Kp * H2, H->stream));
    BDC_CUDA_TRY(cudaMemsetAsync(F->hx, 0, sizeof(double) * NX, H->stream));
    BDC_CUDA_TRY(cudaMemsetAsync(F->Pw, 0, sizeof(double) * NX, H->stream));
    BDC_CUDA_TRY(cudaMemsetAsync(F->Lt, 0, sizeof(double) * NX, H->stream));

    // constant table columns
    {
        std::vector<int> colmap(KL + KR);
        for (auto& t : F->terms) {
            if (t.left) for (int c = 0; c < (1 << t.j); ++c) colmap[t.off + c] = bundle_offset(t.j) + c;
            else for (int c = 0; c < (1 << t.m); ++c) colmap[KL + t.off + c] = bundle_offset(t.m) + c;
        }
        int* d_cm = nullptr;
        BDC_CUDA_TRY(cudaMalloc(&d_cm, sizeof(int) * (colmap.size() + 1)));
        BDC_CUDA_TRY(cudaMemcpy(d_cm, colmap.data(), sizeof(int) * colmap.size(), cudaMemcpyHostToDevice));
        k_fill_tables<<<H->num_sms * 8, 256, 0, H->stream>>>(H1, H2, Kp, H->A.rows, H->A.stride, H->B.rows,
                                                            H->B.stride, d_cm, KL, KR, F->LA, F->RB);
        BDC_CUDA_TRY(cudaGetLastError());
        BDC_CUDA_TRY(cudaStreamSynchronize(H->stream));
        cudaFree(d_cm);
    }
    k_scatter<<<H->num_sms * 8, 256, 0, H->stream>>>(H->d_reps, H->R, H->d_h, F->hx);
    BDC_CUDA_TRY(cudaGetLastError());

    // ---- plan 1: UL = AL^T Pw and VR = Pw BR, split over the contraction
    std::vector<GemmDesc> big;
    if (KL > 0) {
        const int kc = H1 / F->S1;
        for (int sidx = 0; sidx < F->S1; ++sidx) {
            // A(m = col c, kk = x_hi) = LA[x_hi * Kp + c]; B(kk = x_hi, n = x_lo) = Pw
            Operand A = op_f64(F->LA + (int64_t)sidx * kc * Kp, Kp, 1);
            Operand B = op_f64(F->Pw + (int64_t)sidx * kc * H2, H2, 0);
            big.push_back(make_desc(A, B, F->ulpart + (size_t)sidx * KL * H2, H2, 1, KL, H2, kc));
        }
    }
    if (KR > 0) {
        const int kc = H2 / F->S2;
        for (int sidx = 0; sidx < F->S2; ++sidx) {
            // A(m = x_hi, kk = x_lo) = Pw; B(kk = x_lo, n = c) = RB[(KL + c) * H2 + x_lo]
            Operand A = op_f64(F->Pw + (int64_t)sidx * kc, H2, 0);
            Operand B = op_f64(F->RB + (int64_t)KL * H2 + (int64_t)sidx * kc, H2, 1);
            big.push_back(make_desc(A, B, F->vrpart + (size_t)sidx * H1 * KR, KR, 1, H1, KR, kc));
        }
    }
    F->n_big = (int)big.size();
    F->tiles_big = assign_tiles(big, 128, 128);
    BDC_CUDA_TRY(upload(big, &F->d_big));

    // ---- plan 2: q parts Q_t (2^j x 2^m, row-major = flat y order)
    Plan pq, pd;
    for (int ti = 0; ti < F->T; ++ti) {
        const Term& t = F->terms[ti];
        const int nj = 1 << t.j, nm = 1 << t.m;
        double* C = F->qparts + (size_t)ti * ny;
        if (t.left) {
            Operand A = op_f64(F->UL + (int64_t)t.off * H2, H2, 0);  // U_t(yh, x_lo)
            Operand B = t.idB ? op_eye() : op_u16(H->B.rows + bundle_offset(t.m), H->B.stride, 0);
            route(pq, make_desc(A, B, C, nm, 1, nj, nm, H2));
        } else {
            Operand A = t.idA ? op_eye() : op_u16(H->A.rows + bundle_offset(t.j), H->A.stride, 1);
            Operand B = op_f64(F->VR + t.off, KR, 0);  // V_t(x_hi, yl)
            route(pq, make_desc(A, B, C, nm, 1, nj, nm, H1));
        }
        // D-side operands
        Operand Lq = op_f64(F->lnq_full, nm, 0);  // Lq_t(yh, yl)
        if (t.left) {
            // M_t (2^j x H2) = Lq_t B_m^T -> RB rows [off, off + 2^j)
            Operand B = t.idB ? op_eye() : op_u16(H->B.rows + bundle_offset(t.m), H->B.stride, 1);
            route(pd, make_desc(Lq, B, F->RB + (int64_t)t.off * H2, H2, 1, nj, H2, nm));
        } else {
            // N_t (H1 x 2^m) = A_j Lq_t -> LA columns [KL + off, + 2^m)
            Operand A = t.idA ? op_eye() : op_u16(H->A.rows + bundle_offset(t.j), H->A.stride, 0);
            route(pd, make_desc(A, Lq, F->LA + KL + t.off, Kp, 1, H1, nm, nj));
        }
    }
    F->n_qrows = (int)pq.rows.size();
    F->tiles_qrows = assign_rows(pq.rows);
    F->n_qtile = (int)pq.tiles.size();
    F->tiles_qtile = assign_tiles(pq.tiles, 64, 64);
    F->n_drows = (int)pd.rows.size();
    F->tiles_drows = assign_rows(pd.rows);
    F->n_dtile = (int)pd.tiles.size();
    F->tiles_dtile = assign_tiles(pd.tiles, 64, 64);
    BDC_CUDA_TRY(upload(pq.rows, &F->d_qrows));
    BDC_CUDA_TRY(upload(pq.tiles, &F->d_qtile));
    BDC_CUDA_TRY(upload(pd.rows, &F->d_drows));
    BDC_CUDA_TRY(upload(pd.tiles, &F->d_dtile));

    // ---- plan 3: G = LA RB with the BA epilogue
    {
        std::vector<GemmDesc> g;
        g.push_back(make_desc(op_f64(F->LA, Kp, 0), op_f64(F->RB, H2, 0), nullptr, 0, 0, H1, H2, Kp));
        assign_tiles(g, 128, 128);
        BDC_CUDA_TRY(upload(g, &F->d_g));
    }
    F->launches_per_iter = 1 + 1 + (F->n_qrows > 0) + (F->n_qtile > 0) + 1 + (F->n_drows > 0) +
                           (F->n_dtile > 0) + 1 + 1;
    BDC_CUDA_TRY(cudaStreamSynchronize(H->stream));
    return BDC_OK;
}

void factored_free(bdc_handle* H) {
    FactoredState* F = H->fac;
    if (!F) return;
    for (double* p : {F->Pw, F->Lt, F->hx, F->LA, F->RB, F->UL, F->VR, F->ulpart, F->vrpart, F->qparts,
                      F->lnq_full, F->epart})
        cudaFree(p);
    for (GemmDesc* p : {F->d_big, F->d_qrows, F->d_qtile, F->d_drows, F->d_dtile, F->d_g}) cudaFree(p);
    delete F;
    H->fac = nullptr;
}

static BaEpilogue make_epilogue(bdc_handle* H) {
    FactoredState* F = H->fac;
    BaEpilogue ep;
    ep.n = H->n;
    ep.n2 = H->s.n2;
    ep.hx = F->hx;
    ep.Lt = F->Lt;
    ep.Pw = F->Pw;
    ep.inv_c = H->inv_c;
    ep.part = F->epart;
    ep.st = H->d_st;
    return ep;
}

// the stages of one iteration, each gated by DevState::done / error
enum Stage { ST_QBIG = 0, ST_QSMALL, ST_FOLD, ST_DSMALL, ST_G, ST_FIN, ST_COUNT };

static cudaError_t enqueue_stage(bdc_handle* H, int stage, double a) {
    FactoredState* F = H->fac;
    cudaStream_t s = H->stream;
    const BaEpilogue ep = make_epilogue(H);
    switch (stage) {
        case ST_QBIG: {
            if (F->n_big > 0)
                k_gemm_tile<128, 128, 8, 4, 2, 0><<<F->tiles_big, 256, 0, s>>>(F->d_big, F->n_big, ep, H->d_st);
            const int64_t na = (int64_t)F->KL * F->H2, nb = (int64_t)F->H1 * F->KR;
            k_sum_parts<<<H->num_sms * 4, 256, 0, s>>>(F->ulpart, F->S1, F->KL > 0 ? na : 0, F->UL, F->vrpart,
                                                       F->S2, F->KR > 0 ? nb : 0, F->VR, H->d_st);
            break;
        }
        case ST_QSMALL:
            if (F->n_qrows > 0) k_gemm_rows<<<F->tiles_qrows, 256, 0, s>>>(F->d_qrows, F->n_qrows, H->d_st);
            if (F->n_qtile > 0)
                k_gemm_tile<64, 64, 16, 4, 2, 0><<<F->tiles_qtile, 256, 0, s>>>(F->d_qtile, F->n_qtile, ep, H->d_st);
            break;
        case ST_FOLD: {
            const int ny = 1 << H->k;
            k_fold_q<<<(ny + 255) / 256, 256, 0, s>>>(F->qparts, F->T, H->k, H->inv_c, F->lnq_full, H->d_lnq,
                                                     H->d_st);
            break;
        }
        case ST_DSMALL:
            if (F->n_drows > 0) k_gemm_rows<<<F->tiles_drows, 256, 0, s>>>(F->d_drows, F->n_drows, H->d_st);
            if (F->n_dtile > 0)
                k_gemm_tile<64, 64, 16, 4, 2, 0><<<F->tiles_dtile, 256, 0, s>>>(F->d_dtile, F->n_dtile, ep, H->d_st);
            break;
        case ST_G:
            k_gemm_tile<128, 128, 8, 4, 2, 1><<<F->ctas_g, 256, 0, s>>>(F->d_g, 1, ep, H->d_st);
            break;
        case ST_FIN:
            k_fac_finalize<<<1, 256, 0, s>>>(F->epart, F->ctas_g, a, H->d_st);
            break;
    }
    return cudaGetLastError();
}

static cudaError_t enqueue_iteration(bdc_handle* H, double a) {
    for (int st = 0; st < ST_COUNT; ++st) {
        cudaError_t e = enqueue_stage(H, st, a);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

bdc_status factored_load_p(bdc_handle* H) {
    FactoredState* F = H->fac;
    const int64_t NX = (int64_t)1 << H->n;
    BDC_CUDA_TRY(cudaMemsetAsync(F->Pw, 0, sizeof(double) * NX, H->stream));
    const int nb = H->nb_upd;
    k_fac_load<<<nb, 256, 0, H->stream>>>(H->d_reps, H->R, H->n, H->d_p[0], F->Pw, F->Lt, F->epart, H->d_st);
    k_fac_load_finish<<<1, 32, 0, H->stream>>>(F->epart, nb, H->k, H->d_st);
    BDC_CUDA_TRY(cudaGetLastError());
    return BDC_OK;
}

bdc_status factored_store_p(bdc_handle* H, double* p_out) {
    FactoredState* F = H->fac;
    k_fac_store<<<H->nb_upd, 256, 0, H->stream>>>(H->d_reps, H->R, H->n, F->Pw, p_out, H->d_st);
    BDC_CUDA_TRY(cudaGetLastError());
    return BDC_OK;
}

static bdc_status rescale(bdc_handle* H, double a) {
    FactoredState* F = H->fac;
    k_fac_rescale<<<H->nb_upd, 256, 0, H->stream>>>(H->d_reps, H->R, H->n, F->Lt, F->Pw, F->epart, H->d_st);
    k_fac_rescale_finish<<<1, 32, 0, H->stream>>>(F->epart, H->nb_upd, a, H->d_st);
    BDC_CUDA_TRY(cudaGetLastError());
    return BDC_OK;
}

static void fill_stats(bdc_handle* H, long long it0, bdc_stats* stats) {
    if (!stats) return;
    const double ln2 = 0.69314718055994530942;
    stats->iters = H->h_st->iter - it0;
    stats->total_iters = H->h_st->iter;
    stats->mx = H->h_st->mx;
    stats->upper_bound = H->h_st->max_d / ln2;
    stats->rate = H->h_st->rate / ln2;
    stats->lse = H->h_st->lse / ln2;
    stats->converged = H->h_st->done;
}

bdc_status factored_iterate(bdc_handle* H, int64_t max_iters, double a, bdc_stats* stats) {
    BDC_CUDA_TRY(cudaMemsetAsync(&H->d_st->done, 0, sizeof(int), H->stream));
    const long long it0 = H->h_st->iter;
    long long target = it0 + max_iters;
    int64_t chunk = 1;
    for (int guard = 0; guard < 1000000; ++guard) {
        const long long done_iters = H->h_st->iter;
        const int64_t remaining = target - done_iters;
        if (remaining <= 0) break;
        const int64_t c = chunk < remaining ? chunk : remaining;
        for (int64_t i = 0; i < c; ++i) BDC_CUDA_TRY(enqueue_iteration(H, a));
        BDC_CUDA_TRY(cudaMemcpyAsync(H->h_st, H->d_st, sizeof(DevState), cudaMemcpyDeviceToHost, H->stream));
        BDC_CUDA_TRY(cudaStreamSynchronize(H->stream));
        if (H->h_st->error == kErrShift) {
            bdc_status rc = rescale(H, a);
            if (rc != BDC_OK) return rc;
            BDC_CUDA_TRY(cudaMemcpyAsync(H->h_st, H->d_st, sizeof(DevState), cudaMemcpyDeviceToHost, H->stream));
            BDC_CUDA_TRY(cudaStreamSynchronize(H->stream));
        } else if (H->h_st->error) {
            return fail(BDC_ERR_NUMERIC, "factored engine: device error %d", H->h_st->error);
        }
        if (H->h_st->done) break;
        if (chunk < 64) chunk *= 2;
    }
    fill_stats(H, it0, stats);
    return BDC_OK;
}

bdc_status factored_profile(bdc_handle* H, int iters, bdc_profile_t* out) {
    FactoredState* F = H->fac;
    BDC_CUDA_TRY(cudaMemsetAsync(&H->d_st->done, 0, sizeof(int), H->stream));
    cudaEvent_t ev[ST_COUNT + 1];
    for (auto& e : ev) BDC_CUDA_TRY(cudaEventCreate(&e));
    double acc[ST_COUNT] = {0}, tot = 0;
    for (int it = 0; it < iters; ++it) {
        BDC_CUDA_TRY(cudaEventRecord(ev[0], H->stream));
        for (int st = 0; st < ST_COUNT; ++st) {
            BDC_CUDA_TRY(enqueue_stage(H, st, -INFINITY));
            BDC_CUDA_TRY(cudaEventRecord(ev[st + 1], H->stream));
        }
        BDC_CUDA_TRY(cudaEventSynchronize(ev[ST_COUNT]));
        BDC_CUDA_TRY(cudaMemcpy(H->h_st, H->d_st, sizeof(DevState), cudaMemcpyDeviceToHost));
        if (H->h_st->error == kErrShift) {
            bdc_status rc = rescale(H, -INFINITY);
            if (rc != BDC_OK) return rc;
        }
        float ms;
        for (int st = 0; st < ST_COUNT; ++st) {
            cudaEventElapsedTime(&ms, ev[st], ev[st + 1]);
            acc[st] += ms;
        }
        cudaEventElapsedTime(&ms, ev[0], ev[ST_COUNT]);
        tot += ms;
    }
    for (auto& e : ev) cudaEventDestroy(e);
    BDC_CUDA_TRY(cudaMemcpyAsync(H->h_st, H->d_st, sizeof(DevState), cudaMemcpyDeviceToHost, H->stream));
    BDC_CUDA_TRY(cudaStreamSynchronize(H->stream));
    out->ms_q = (acc[ST_QBIG] + acc[ST_QSMALL]) / iters;
    out->ms_fold = acc[ST_FOLD] / iters;
    out->ms_d = (acc[ST_DSMALL] + acc[ST_G]) / iters;
    out->ms_update = acc[ST_FIN] / iters;
    out->ms_iter = tot / iters;
    out->ms_main = acc[ST_G] / iters;
    out->work_main = 2.0 * (double)F->H1 * (double)F->H2 * (double)(F->KL + F->KR);
    out->launches = F->launches_per_iter;
    out->iters = iters;
    return BDC_OK;
}

}  // namespace bdc
