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

// q-side small product of one term: Q_t = sum_s a(s) (x) b(s), the outer
// products of a(s) = a + s*a_stride (2^j entries) and b(s) = b + s*b_stride
// (2^m entries), s over the contracted half (L terms: a = column of U_t,
// b = row of B_m; R terms: a = row of A_j, b = row of V_t).
struct OuterDesc {
    const void* a;
    const void* b;
    int64_t a_stride, b_stride;
    int a_u16, b_u16;
    int j, m;
    int S;           // length of the contracted range
    int term;        // slice of qparts
};

// D-side small product of one term, one s at a time (Lq_t = ln q as 2^j x 2^m):
//   L: out_s[yh] = sum_yl Lq_t[yh][yl] B_m[s][yl]   (column s of M_t -> RB)
//   R: out_s[yl] = sum_yh A_j[s][yh] Lq_t[yh][yl]   (row s of N_t -> LA)
struct MatvecDesc {
    const uint16_t* v;  // bundle rows: v(s) = v + s * v_stride
    int64_t v_stride;
    double* out;        // element i of s at out[s * s_stride + i * i_stride]
    int64_t s_stride, i_stride;
    int j, m, left;
    int S;
    int cta_begin;
};

// how the fold reads Q_t: 0 = split slices in qparts, 1 = U^T rows (the
// identity B of an L term), 2 = V rows (the identity A of an R term); the
// identity terms of the D side are written by the fold as copies of ln q.
struct FoldTerm {
    int kind;
    int j, m, off;
    int idB_left;   // L term with identity B_m: RB rows [off, off+2^j) = Lq_t
    int idA_right;  // R term with identity A_j: LA columns [KL+off, +2^m) = Lq_t
};

struct Term {
    int j, m;       // split point and the low sub-length k - j
    int left;       // 1: L term (contract x_hi first), 0: R term
    int off;        // column offset inside AL (L) or BR (R)
    int idA, idB;   // A_j / B_m is the identity (j == n1 / m == n2)
};

}  // namespace bdc

struct FactoredState {
    int H1 = 0, H2 = 0, KL = 0, KR = 0, Kp = 0, T = 0;
    int H1h = 0;              // rows that hold representatives: x_hi < H1 / 2
    std::vector<bdc::Term> terms;
    double* Pw = nullptr;     // [2^{n-1}]  |O(x)| e(x) at representatives, 0 elsewhere
    double* Lt = nullptr;     // [2^{n-1}]  ln e(x) (p = e / Z)
    double* hx = nullptr;     // [2^{n-1}]  h(x) at representatives
    double* LA = nullptr;     // [H1h][Kp]  = [AL | NR]
    double* RB = nullptr;     // [Kp][H2]  = [ML ; BR^T]
    double* UL = nullptr;     // [H2][KL]  (U^T: column c of AL^T Pw is row-contiguous)
    double* VR = nullptr;     // [H1h][KR]
    double* ulpart = nullptr; // [S1][H2][KL]
    double* vrpart = nullptr; // [S2][H1h][KR]
    int S1 = 1, S2 = 1;
    double* qparts = nullptr; // [T][QS][2^k]
    double* qsum = nullptr;   // [T][2^k]  qparts summed over the splits
    int QS = 1;               // split of the s range of the small q products
    double* lnq_full = nullptr;  // [2^k]
    double* epart = nullptr;  // [ctas][4]
    int ctas_g = 0;
    // launch plans
    bdc::GemmDesc* d_big = nullptr;  int n_big = 0, tiles_big = 0;     // UL, VR partials
    bdc::OuterDesc* d_qsmall = nullptr; int n_qsmall = 0;   // q-side small products
    bdc::MatvecDesc* d_dsmall = nullptr; int n_dsmall = 0;  // D-side small products
    int dsmall_chunk = 64;                                  // s values per CTA
    int ctas_dsmall = 0, smem_dsmall = 0;
    bdc::FoldTerm* d_fold = nullptr;                        // per term: how the fold reads Q_t
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
    const double inv_z = exp(-lnz);
    double mD = -DBL_MAX, sE = 0.0, mL = -DBL_MAX, sR = 0.0, zero = 0.0;
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
            // an entry that is exactly 0 in the caller's distribution (Lt holds
            // NaN) takes ln p = 0, as the reference's apply_log_kernel leaves
            // ln 0 at 0 (backend/BAA.cu:573-580); later iterates keep exact logs
            const double pw = ep.Pw[x];
            const double lt = ep.Lt[x];
            const bool zero_in = (lt != lt);
            const double lnp = zero_in ? 0.0 : lt - lnz;
            const double lw = lnp + D - shift;
            const double e = exp(lw);
            ep.Lt[x] = lw;
            ep.Pw[x] = o * e;
            mD = fmax(mD, D);
            mL = fmax(mL, lw);
            sE = fma(o, e, sE);
            sR = fma(pw * inv_z, D, sR);
            if (zero_in) zero = 1.0;
        }
    }
    // CTA reduction of the five partials
    __shared__ double red[5][8];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        mD = fmax(mD, __shfl_xor_sync(0xFFFFFFFFu, mD, off));
        mL = fmax(mL, __shfl_xor_sync(0xFFFFFFFFu, mL, off));
        sE += __shfl_xor_sync(0xFFFFFFFFu, sE, off);
        sR += __shfl_xor_sync(0xFFFFFFFFu, sR, off);
        zero = fmax(zero, __shfl_xor_sync(0xFFFFFFFFu, zero, off));
    }
    if (lane == 0) {
        red[0][warp] = mD;
        red[1][warp] = sE;
        red[2][warp] = mL;
        red[3][warp] = sR;
        red[4][warp] = zero;
    }
    __syncthreads();
    if (tid == 0) {
        double a0 = red[0][0], a1 = red[1][0], a2 = red[2][0], a3 = red[3][0], a4 = red[4][0];
        for (int w = 1; w < 8; ++w) {
            a0 = fmax(a0, red[0][w]);
            a1 += red[1][w];
            a2 = fmax(a2, red[2][w]);
            a3 += red[3][w];
            a4 = fmax(a4, red[4][w]);
        }
        double* p = ep.part + (size_t)blockIdx.x * 8;
        p[0] = a0;
        p[1] = a1;
        p[2] = a2;
        p[3] = a3;
        p[4] = a4;
    }
}

// ------------------------------------------------- q-side small products
// CTA = one (term, split of the s range); thread t owns OPT consecutive
// outputs o = y = yh * 2^m + yl of Q_t and accumulates a(s)[yh] * b(s)[yl].
__device__ __forceinline__ double ld_any(const void* p, int u16, int64_t i) {
    return u16 ? (double)__ldg((const uint16_t*)p + i) : __ldg((const double*)p + i);
}

template <int OPT>
__global__ void __launch_bounds__(256) k_qsmall(const OuterDesc* __restrict__ descs, int QS, int k,
                                                double* __restrict__ qparts, const DevState* st) {
    if (gated(st)) return;
    const OuterDesc& d = descs[blockIdx.x / QS];
    const int split = blockIdx.x % QS;
    const int ny = 1 << k;
    const int s0 = (int)((int64_t)d.S * split / QS), s1 = (int)((int64_t)d.S * (split + 1) / QS);
    const int o0 = threadIdx.x * OPT;
    if (o0 >= ny) return;
    const int m = d.m;
    const int mask = (1 << m) - 1;
    double acc[OPT];
#pragma unroll
    for (int i = 0; i < OPT; ++i) acc[i] = 0.0;
    if ((1 << m) >= OPT) {
        // one yh, OPT consecutive yl
        const int yh = o0 >> m, yl0 = o0 & mask;
        for (int s = s0; s < s1; ++s) {
            const double av = ld_any(d.a, d.a_u16, (int64_t)s * d.a_stride + yh);
            const int64_t bb = (int64_t)s * d.b_stride + yl0;
#pragma unroll
            for (int i = 0; i < OPT; ++i) acc[i] = fma(av, ld_any(d.b, d.b_u16, bb + i), acc[i]);
        }
    } else {
        // OPT / 2^m consecutive yh, all 2^m yl
        const int yh0 = o0 >> m;
        for (int s = s0; s < s1; ++s) {
            const int64_t ab = (int64_t)s * d.a_stride + yh0, bb = (int64_t)s * d.b_stride;
#pragma unroll
            for (int i = 0; i < OPT; ++i)
                acc[i] = fma(ld_any(d.a, d.a_u16, ab + (i >> m)), ld_any(d.b, d.b_u16, bb + (i & mask)),
                             acc[i]);
        }
    }
    double* out = qparts + ((size_t)d.term * QS + split) * ny + o0;
#pragma unroll
    for (int i = 0; i < OPT; ++i) out[i] = acc[i];
}

// ------------------------------------------------- D-side small products
// CTA = one term and a chunk of s; Lq_t staged in shared memory with row
// stride 2^m + 1; one warp per s.
__global__ void __launch_bounds__(256) k_dsmall(const MatvecDesc* __restrict__ descs, int nd, int chunk,
                                                const double* __restrict__ lnq_full, const DevState* st) {
    if (gated(st)) return;
    int di = 0;
    while (di + 1 < nd && descs[di + 1].cta_begin <= (int)blockIdx.x) ++di;
    const MatvecDesc& d = descs[di];
    const int c = blockIdx.x - d.cta_begin;
    const int nj = 1 << d.j, nm = 1 << d.m;
    const int rs = nm + 1;
    extern __shared__ double lq[];  // [nj][nm + 1]
    for (int e = threadIdx.x; e < nj * nm; e += blockDim.x) lq[(e >> d.m) * rs + (e & (nm - 1))] = lnq_full[e];
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int sb = c * chunk, se = min(sb + chunk, d.S);
    for (int s = sb + warp; s < se; s += 8) {
        const uint16_t* v = d.v + (int64_t)s * d.v_stride;
        double* out = d.out + (int64_t)s * d.s_stride;
        if (d.left) {
            // out[yh] = sum_yl Lq[yh][yl] v[yl]
            if (nj >= 32) {
                for (int yh = lane; yh < nj; yh += 32) {
                    double acc = 0.0;
                    const double* row = lq + yh * rs;
                    for (int yl = 0; yl < nm; ++yl) acc = fma(row[yl], (double)__ldg(v + yl), acc);
                    out[(int64_t)yh * d.i_stride] = acc;
                }
            } else {
                for (int yh = 0; yh < nj; ++yh) {
                    double acc = 0.0;
                    const double* row = lq + yh * rs;
                    for (int yl = lane; yl < nm; yl += 32) acc = fma(row[yl], (double)__ldg(v + yl), acc);
#pragma unroll
                    for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xFFFFFFFFu, acc, off);
                    if (lane == 0) out[(int64_t)yh * d.i_stride] = acc;
                }
            }
        } else {
            // out[yl] = sum_yh v[yh] Lq[yh][yl]
            if (nm >= 32) {
                for (int yl = lane; yl < nm; yl += 32) {
                    double acc = 0.0;
                    for (int yh = 0; yh < nj; ++yh) acc = fma((double)__ldg(v + yh), lq[yh * rs + yl], acc);
                    out[(int64_t)yl * d.i_stride] = acc;
                }
            } else {
                double acc[32];
#pragma unroll
                for (int yl = 0; yl < 32; ++yl) acc[yl] = 0.0;
                for (int yh = lane; yh < nj; yh += 32) {
                    const double vv = (double)__ldg(v + yh);
                    const double* row = lq + yh * rs;
#pragma unroll
                    for (int yl = 0; yl < 32; ++yl)
                        if (yl < nm) acc[yl] = fma(vv, row[yl], acc[yl]);
                }
#pragma unroll
                for (int yl = 0; yl < 32; ++yl) {
                    if (yl >= nm) break;
                    double a = acc[yl];
#pragma unroll
                    for (int off = 16; off > 0; off >>= 1) a += __shfl_xor_sync(0xFFFFFFFFu, a, off);
                    if (lane == 0) out[(int64_t)yl * d.i_stride] = a;
                }
            }
        }
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

// q(rep r) = sum_{y in O(r)} acc[y] / (|O(r)| C Z) with acc[y] = sum over
// terms of Q_t[y] (split slices, or U^T / V rows for identity terms); ln q
// with the reference's 0 for q == 0 (backend/BAA.cu:573-580), expanded to
// every y, and copied into RB / LA where a D-side product is the identity.
// phase 1: qsum[t][y] = sum over the splits of qparts[t][split][y]
__global__ void k_qsum(const FoldTerm* __restrict__ terms, int T, const double* __restrict__ qparts, int QS, int k,
                       double* __restrict__ qsum, const DevState* st) {
    if (gated(st)) return;
    const int ny = 1 << k;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < T * ny; e += gridDim.x * blockDim.x) {
        const int t = e / ny, y = e % ny;
        if (terms[t].kind != 0) continue;
        const double* q = qparts + (size_t)t * QS * ny + y;
        double a = 0.0;
        for (int sp = 0; sp < QS; ++sp) a += q[(size_t)sp * ny];
        qsum[e] = a;
    }
}

// Q_t[y] from the split sums, or from U^T / V for identity terms (V holds
// only the rows x_hi < H1h; the rows above are zero)
__device__ __forceinline__ double term_value(const FoldTerm& f, const double* qsum, int t, int ny,
                                             const double* ULt, int KL, const double* VR, int KR, int H1h,
                                             uint32_t y) {
    if (f.kind == 0) return qsum[(size_t)t * ny + y];
    const uint32_t yh = y >> f.m, yl = y & ((1u << f.m) - 1u);
    if (f.kind == 1) return ULt[(size_t)yl * KL + f.off + yh];  // Q_t = U_t
    return yh < (uint32_t)H1h ? VR[(size_t)yh * KR + f.off + yl] : 0.0;  // Q_t = V_t
}

// phase 2: q(rep r) = sum_{y in O(r)} sum_t Q_t[y] / (|O(r)| C Z); ln q with
// the reference's 0 for q == 0 (backend/BAA.cu:573-580), expanded to every
// y, and copied into RB / LA where a D-side product is the identity.
__global__ void k_fold_q(const FoldTerm* __restrict__ terms, int T, const double* __restrict__ qsum,
                         const double* __restrict__ ULt, int KL, const double* __restrict__ VR, int KR, int H1h,
                         int k, double inv_c, double* __restrict__ lnq_full, double* __restrict__ lnq,
                         double* __restrict__ RB, int H2, double* __restrict__ LA, int Kp, const DevState* st) {
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
            for (int t = 0; t < T; ++t) acc += term_value(terms[t], qsum, t, ny, ULt, KL, VR, KR, H1h, mem[e]);
        const double q = acc * inv_c * inv_z / (double)nm;
        const double lq = (q != 0.0) ? log(q) : 0.0;
        lnq_full[y] = lq;
        if ((uint32_t)y == r) lnq[y] = lq;  // representatives are < 2^{k-1}
        for (int t = 0; t < T; ++t) {
            const FoldTerm& f = terms[t];
            const uint32_t yh = (uint32_t)y >> f.m, yl = (uint32_t)y & ((1u << f.m) - 1u);
            if (f.idB_left) RB[(size_t)(f.off + yh) * H2 + yl] = lq;  // M_t = Lq_t
            if (f.idA_right && yh < (uint32_t)H1h) LA[(size_t)yh * Kp + KL + f.off + yl] = lq;  // N_t = Lq_t
        }
    }
}

__global__ void __launch_bounds__(256)
k_fac_finalize(const double* __restrict__ part, int nb, double a, DevState* st) {
    if (gated(st)) return;
    __shared__ double red[5][256];
    double mD = -DBL_MAX, sE = 0.0, mL = -DBL_MAX, sR = 0.0, zero = 0.0;
    for (int b = threadIdx.x; b < nb; b += 256) {
        mD = fmax(mD, part[(size_t)b * 8 + 0]);
        sE += part[(size_t)b * 8 + 1];
        mL = fmax(mL, part[(size_t)b * 8 + 2]);
        sR += part[(size_t)b * 8 + 3];
        zero = fmax(zero, part[(size_t)b * 8 + 4]);
    }
    red[0][threadIdx.x] = mD;
    red[1][threadIdx.x] = sE;
    red[2][threadIdx.x] = mL;
    red[3][threadIdx.x] = sR;
    red[4][threadIdx.x] = zero;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            red[0][threadIdx.x] = fmax(red[0][threadIdx.x], red[0][threadIdx.x + s]);
            red[1][threadIdx.x] += red[1][threadIdx.x + s];
            red[2][threadIdx.x] = fmax(red[2][threadIdx.x], red[2][threadIdx.x + s]);
            red[3][threadIdx.x] += red[3][threadIdx.x + s];
            red[4][threadIdx.x] = fmax(red[4][threadIdx.x], red[4][threadIdx.x + s]);
        }
        __syncthreads();
    }
    if (threadIdx.x != 0) return;
    mD = red[0][0];
    sE = red[1][0];
    mL = red[2][0];
    sR = red[3][0];
    st->zero_p = (red[4][0] != 0.0);
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
        // ln 0 = 0 (backend/BAA.cu:573-580): marked with NaN for the epilogue
        const double l = (v != 0.0) ? log(v) : 0.0;
        Lt[x] = (v != 0.0) ? l : __longlong_as_double(0x7ff8000000000000ll);
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
static Operand op_f64(const double* p, int64_t ld, int trans) {
    Operand o;
    o.ptr = p;
    o.ld = ld;
    o.kind = OP_F64;
    o.trans = trans;
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

template <typename T>
static cudaError_t upload(const std::vector<T>& v, T** dst) {
    if (v.empty()) return cudaSuccess;
    cudaError_t e = cudaMalloc(dst, sizeof(T) * v.size());
    if (e != cudaSuccess) return e;
    return cudaMemcpy(*dst, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice);
}

bool factored_supports(int n, int k) {
    // needs k < n (W is not the identity), half tables that fit the uint16
    // bundles, and a dense 2^n state that fits comfortably in device memory
    return k >= 1 && k < n && n >= 2 && n <= 28 && k <= 14;
}

static int qsmall_opt(int k) {
    const int ny = 1 << k;
    return ny >= 256 ? ny / 256 : 1;
}

bdc_status factored_init(bdc_handle* H) {
    FactoredState* F = new FactoredState();
    H->fac = F;
    const Split& s = H->s;
    F->H1 = 1 << s.n1;
    F->H2 = 1 << s.n2;
    // every representative is <= its complement, so its top bit is 0 and
    // x_hi < H1 / 2: only those rows of the iterate and of G are needed
    F->H1h = F->H1 / 2;
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
    for (auto& t : F->terms)
        if (t.left) { t.off = KL; KL += 1 << t.j; }
    for (auto& t : F->terms)
        if (!t.left) { t.off = KR; KR += 1 << t.m; }
    F->KL = KL;
    F->KR = KR;
    F->Kp = (KL + KR + 7) / 8 * 8;
    F->T = (int)F->terms.size();
    const int64_t NX = (int64_t)1 << (H->n - 1);
    const int ny = 1 << k;
    const int H1 = F->H1h, H2 = F->H2, Kp = F->Kp;  // H1: the rows kept
    const int KLa = KL > 0 ? KL : 1, KRa = KR > 0 ? KR : 1;

    // small q products: split the contracted range so the launch fills the GPU
    int n_outer = 0;
    for (auto& t : F->terms) n_outer += (t.left ? !t.idB : !t.idA);
    F->QS = n_outer > 0 ? std::max(1, std::min(64, (H->num_sms * 4) / n_outer)) : 1;
    while (F->QS > 1 && (std::min(H1, H2) / F->QS) < 16) F->QS /= 2;

    auto al = [&](double** p, size_t cnt) -> cudaError_t {
        H->bytes += cnt * sizeof(double);
        return cudaMalloc(p, cnt * sizeof(double) + 16);
    };
    BDC_CUDA_TRY(al(&F->Pw, NX));
    BDC_CUDA_TRY(al(&F->Lt, NX));
    BDC_CUDA_TRY(al(&F->hx, NX));
    BDC_CUDA_TRY(al(&F->LA, (size_t)H1 * Kp));
    BDC_CUDA_TRY(al(&F->RB, (size_t)Kp * H2));
    BDC_CUDA_TRY(al(&F->UL, (size_t)H2 * KLa));
    BDC_CUDA_TRY(al(&F->VR, (size_t)H1 * KRa));
    // split-K of the two thin products so that they fill the GPU
    const int tiles_ul = ((KL + 127) / 128) * ((H2 + 127) / 128);
    const int tiles_vr = ((H1 + 127) / 128) * ((KR + 127) / 128);
    F->S1 = KL > 0 ? std::max(1, std::min(32, (H->num_sms * 4) / std::max(1, tiles_ul))) : 1;
    F->S2 = KR > 0 ? std::max(1, std::min(32, (H->num_sms * 4) / std::max(1, tiles_vr))) : 1;
    while (F->S1 > 1 && (H1 % F->S1 || H1 / F->S1 < 8)) --F->S1;
    while (F->S2 > 1 && (H2 % F->S2 || H2 / F->S2 < 8)) --F->S2;
    BDC_CUDA_TRY(al(&F->ulpart, (size_t)F->S1 * H2 * KLa));
    BDC_CUDA_TRY(al(&F->vrpart, (size_t)F->S2 * H1 * KRa));
    BDC_CUDA_TRY(al(&F->qparts, (size_t)F->T * F->QS * ny));
    BDC_CUDA_TRY(al(&F->qsum, (size_t)F->T * ny));
    BDC_CUDA_TRY(al(&F->lnq_full, (size_t)ny));
    F->ctas_g = ((H1 + 127) / 128) * ((H2 + 127) / 128);
    BDC_CUDA_TRY(al(&F->epart, (size_t)std::max(F->ctas_g * 2, 2 * H->nb_upd) * 4));
    BDC_CUDA_TRY(cudaMemsetAsync(F->LA, 0, sizeof(double) * H1 * Kp, H->stream));
    BDC_CUDA_TRY(cudaMemsetAsync(F->RB, 0, sizeof(double) * Kp * H2, H->stream));
    BDC_CUDA_TRY(cudaMemsetAsync(F->hx, 0, sizeof(double) * NX, H->stream));
    BDC_CUDA_TRY(cudaMemsetAsync(F->Pw, 0, sizeof(double) * NX, H->stream));
    BDC_CUDA_TRY(cudaMemsetAsync(F->Lt, 0, sizeof(double) * NX, H->stream));
    BDC_CUDA_TRY(cudaMemsetAsync(F->qparts, 0, sizeof(double) * F->T * F->QS * ny, H->stream));

    // constant table columns of LA (AL) and rows of RB (BR^T)
    {
        std::vector<int> colmap(KL + KR + 1);
        for (auto& t : F->terms) {
            if (t.left) for (int c = 0; c < (1 << t.j); ++c) colmap[t.off + c] = bundle_offset(t.j) + c;
            else for (int c = 0; c < (1 << t.m); ++c) colmap[KL + t.off + c] = bundle_offset(t.m) + c;
        }
        int* d_cm = nullptr;
        BDC_CUDA_TRY(cudaMalloc(&d_cm, sizeof(int) * colmap.size()));
        BDC_CUDA_TRY(cudaMemcpy(d_cm, colmap.data(), sizeof(int) * colmap.size(), cudaMemcpyHostToDevice));
        // a left term's A_j or a right term's B_m is never the identity
        k_fill_tables<<<H->num_sms * 8, 256, 0, H->stream>>>(H1, H2, Kp, H->A.rows, H->A.stride, H->B.rows,
                                                            H->B.stride, d_cm, KL, KR, F->LA, F->RB);
        BDC_CUDA_TRY(cudaGetLastError());
        BDC_CUDA_TRY(cudaStreamSynchronize(H->stream));
        cudaFree(d_cm);
    }
    k_scatter<<<H->num_sms * 8, 256, 0, H->stream>>>(H->d_reps, H->R, H->d_h, F->hx);
    BDC_CUDA_TRY(cudaGetLastError());

    // ---- the two thin products, split over the contraction:
    //   U^T (H2 x KL) = (AL^T Pw)^T and V (H1h x KR) = Pw BR
    std::vector<GemmDesc> big;
    if (KL > 0) {
        const int kc = H1 / F->S1;
        for (int sidx = 0; sidx < F->S1; ++sidx) {
            // A(m = c, kk = x_hi) = LA[x_hi * Kp + c]; B(kk = x_hi, n = x_lo) = Pw; C(c, x_lo) -> U^T[x_lo][c]
            Operand A = op_f64(F->LA + (int64_t)sidx * kc * Kp, Kp, 1);
            Operand B = op_f64(F->Pw + (int64_t)sidx * kc * H2, H2, 0);
            big.push_back(make_desc(A, B, F->ulpart + (size_t)sidx * H2 * KL, 1, KL, KL, H2, kc));
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

    // ---- per-term small products and the fold plan
    std::vector<OuterDesc> outer;
    std::vector<MatvecDesc> mv;
    std::vector<FoldTerm> fold;
    int cta = 0;
    for (int ti = 0; ti < F->T; ++ti) {
        const Term& t = F->terms[ti];
        FoldTerm f{};
        f.j = t.j;
        f.m = t.m;
        f.off = t.off;
        if (t.left) {
            if (t.idB) {
                f.kind = 1;       // Q_t = U_t
                f.idB_left = 1;   // M_t = Lq_t
            } else {
                OuterDesc o{};
                o.a = F->UL + t.off;                       // a(s)[yh] = U^T[s][off + yh]
                o.a_stride = KL;
                o.a_u16 = 0;
                o.b = H->B.rows + bundle_offset(t.m);      // b(s)[yl] = B_m[s][yl]
                o.b_stride = H->B.stride;
                o.b_u16 = 1;
                o.j = t.j;
                o.m = t.m;
                o.S = H2;
                o.term = ti;
                outer.push_back(o);
                MatvecDesc d{};
                d.v = H->B.rows + bundle_offset(t.m);
                d.v_stride = H->B.stride;
                d.out = F->RB + (int64_t)t.off * H2;       // M_t[yh][s] -> RB[off + yh][s]
                d.s_stride = 1;
                d.i_stride = H2;
                d.j = t.j;
                d.m = t.m;
                d.left = 1;
                d.S = H2;
                d.cta_begin = cta;
                cta += (H2 + F->dsmall_chunk - 1) / F->dsmall_chunk;
                mv.push_back(d);
            }
        } else {
            if (t.idA) {
                f.kind = 2;        // Q_t = V_t
                f.idA_right = 1;   // N_t = Lq_t
            } else {
                OuterDesc o{};
                o.a = H->A.rows + bundle_offset(t.j);      // a(s)[yh] = A_j[s][yh]
                o.a_stride = H->A.stride;
                o.a_u16 = 1;
                o.b = F->VR + t.off;                       // b(s)[yl] = V[s][off + yl]
                o.b_stride = KR;
                o.b_u16 = 0;
                o.j = t.j;
                o.m = t.m;
                o.S = H1;
                o.term = ti;
                outer.push_back(o);
                MatvecDesc d{};
                d.v = H->A.rows + bundle_offset(t.j);
                d.v_stride = H->A.stride;
                d.out = F->LA + KL + t.off;                // N_t[s][yl] -> LA[s][KL + off + yl]
                d.s_stride = Kp;
                d.i_stride = 1;
                d.j = t.j;
                d.m = t.m;
                d.left = 0;
                d.S = H1;
                d.cta_begin = cta;
                cta += (H1 + F->dsmall_chunk - 1) / F->dsmall_chunk;
                mv.push_back(d);
            }
        }
        fold.push_back(f);
    }
    F->n_qsmall = (int)outer.size();
    F->n_dsmall = (int)mv.size();
    F->ctas_dsmall = cta;
    int max_smem = 0;
    for (auto& d : mv) max_smem = std::max(max_smem, (int)(sizeof(double) * (1 << d.j) * ((1 << d.m) + 1)));
    F->smem_dsmall = max_smem;
    if (max_smem > 48 * 1024)
        BDC_CUDA_TRY(cudaFuncSetAttribute(k_dsmall, cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem));
    BDC_CUDA_TRY(upload(outer, &F->d_qsmall));
    BDC_CUDA_TRY(upload(mv, &F->d_dsmall));
    BDC_CUDA_TRY(upload(fold, &F->d_fold));

    // ---- G = LA RB with the BA epilogue
    {
        std::vector<GemmDesc> g;
        g.push_back(make_desc(op_f64(F->LA, Kp, 0), op_f64(F->RB, H2, 0), nullptr, 0, 0, H1, H2, Kp));
        assign_tiles(g, 128, 128);
        BDC_CUDA_TRY(upload(g, &F->d_g));
    }
    F->launches_per_iter = (F->n_big > 0 ? 2 : 0) + (F->n_qsmall > 0) + 2 + (F->n_dsmall > 0) + 1 + 1;
    BDC_CUDA_TRY(cudaStreamSynchronize(H->stream));
    return BDC_OK;
}

void factored_free(bdc_handle* H) {
    FactoredState* F = H->fac;
    if (!F) return;
    for (double* p : {F->Pw, F->Lt, F->hx, F->LA, F->RB, F->UL, F->VR, F->ulpart, F->vrpart, F->qparts,
                      F->qsum, F->lnq_full, F->epart})
        cudaFree(p);
    cudaFree(F->d_big);
    cudaFree(F->d_g);
    cudaFree(F->d_qsmall);
    cudaFree(F->d_dsmall);
    cudaFree(F->d_fold);
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

static cudaError_t launch_qsmall(bdc_handle* H) {
    FactoredState* F = H->fac;
    const int grid = F->n_qsmall * F->QS;
    switch (qsmall_opt(H->k)) {
        case 1: k_qsmall<1><<<grid, 256, 0, H->stream>>>(F->d_qsmall, F->QS, H->k, F->qparts, H->d_st); break;
        case 2: k_qsmall<2><<<grid, 256, 0, H->stream>>>(F->d_qsmall, F->QS, H->k, F->qparts, H->d_st); break;
        case 4: k_qsmall<4><<<grid, 256, 0, H->stream>>>(F->d_qsmall, F->QS, H->k, F->qparts, H->d_st); break;
        case 8: k_qsmall<8><<<grid, 256, 0, H->stream>>>(F->d_qsmall, F->QS, H->k, F->qparts, H->d_st); break;
        case 16: k_qsmall<16><<<grid, 256, 0, H->stream>>>(F->d_qsmall, F->QS, H->k, F->qparts, H->d_st); break;
        case 32: k_qsmall<32><<<grid, 256, 0, H->stream>>>(F->d_qsmall, F->QS, H->k, F->qparts, H->d_st); break;
        case 64: k_qsmall<64><<<grid, 256, 0, H->stream>>>(F->d_qsmall, F->QS, H->k, F->qparts, H->d_st); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

static cudaError_t enqueue_stage(bdc_handle* H, int stage, double a) {
    FactoredState* F = H->fac;
    cudaStream_t s = H->stream;
    const BaEpilogue ep = make_epilogue(H);
    switch (stage) {
        case ST_QBIG: {
            if (F->n_big > 0) {
                k_gemm_tile<128, 128, 8, 4, 2, 0><<<F->tiles_big, 256, 0, s>>>(F->d_big, F->n_big, ep, H->d_st);
                const int64_t na = (int64_t)F->KL * F->H2, nb = (int64_t)F->H1h * F->KR;
                k_sum_parts<<<H->num_sms * 4, 256, 0, s>>>(F->ulpart, F->S1, F->KL > 0 ? na : 0, F->UL, F->vrpart,
                                                           F->S2, F->KR > 0 ? nb : 0, F->VR, H->d_st);
            }
            break;
        }
        case ST_QSMALL:
            if (F->n_qsmall > 0) return launch_qsmall(H);
            break;
        case ST_FOLD: {
            const int ny = 1 << H->k;
            const int nqs = (F->T * ny + 255) / 256;
            k_qsum<<<nqs < 4096 ? nqs : 4096, 256, 0, s>>>(F->d_fold, F->T, F->qparts, F->QS, H->k, F->qsum, H->d_st);
            k_fold_q<<<(ny + 63) / 64, 64, 0, s>>>(F->d_fold, F->T, F->qsum, F->UL, F->KL, F->VR, F->KR, F->H1h, H->k,
                                                  H->inv_c, F->lnq_full, H->d_lnq, F->RB, F->H2, F->LA, F->Kp,
                                                  H->d_st);
            break;
        }
        case ST_DSMALL:
            if (F->n_dsmall > 0)
                k_dsmall<<<F->ctas_dsmall, 256, F->smem_dsmall, s>>>(F->d_dsmall, F->n_dsmall, F->dsmall_chunk,
                                                                     F->lnq_full, H->d_st);
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
    const int64_t NX = (int64_t)1 << (H->n - 1);  // representatives have x < 2^{n-1}
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
    out->work_main = 2.0 * (double)F->H1h * (double)F->H2 * (double)(F->KL + F->KR);
    out->launches = F->launches_per_iter;
    out->iters = iters;
    return BDC_OK;
}

}  // namespace bdc
