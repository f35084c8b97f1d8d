// bdc_solve.cu -- a certified solver for C_{n,k} on the factored engine.
//
// For every input distribution p the Blahut-Arimoto bracket
//     I(p;W) <= C <= max_x D(W(.|x) || q_p)
// holds (the right side is the bound the reference prints as its stopping
// statistic, backend/BAA.cu:413-425 and 820-913), so a solver may move p by
// any rule as long as each reported number is evaluated exactly at the point
// it belongs to.  No counterpart in the reference, which runs plain BA until
// max_x log2 p'/p < a (backend/main_BAA.cu:73).  Three phases:
//
//  1. Anderson-accelerated BA on the whole input space: the last m
//     differences of the BA map F are mixed in p (orbit-weighted least
//     squares), negative entries are clipped to 0, and a mixed point is kept
//     only when the rate at it is at least the rate of the plain step.
//  2. Support: the inputs with positive mass or with D(x) near the bound form
//     a set S.  BA restricted to S runs with the same acceleration on rows
//     N(x, .) of S held in device memory (exact integers in FP32).
//  3. Certification: one full evaluation at p_S gives D(x) for every x, the
//     bound and the rate.  Inputs outside S whose D(x) exceeds the rate join
//     S and phase 2 repeats; otherwise the bracket is final.
//
// Slowly vanishing inputs (D(x) just below C) make plain BA converge
// sublinearly; removing them in phase 2 leaves a problem that converges fast,
// and phase 3 proves that nothing outside S could carry mass.
#include <algorithm>
#include <cfloat>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <vector>

#include "bdc_engine.cuh"

namespace bdc {

constexpr int kAAMax = 10;  // history of the Anderson mixing
// the restricted problem runs accelerated BA to this bracket (bits), then
// Newton on the support (Newton from 1e-5 or 1e-6 bits stops short at 16/8 to
// 26/13 and costs more than the BA steps it saves)
constexpr double kRestrictedSwitchBits = 1e-7;

// ------------------------------------------------------------ vector kernels
// out = sum_i w_i u_i v_i over blocks (w = orbit sizes, 2 or 4)
__device__ __forceinline__ double block_reduce_sum(double v, double* sh) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r += sh[w];
    return r;  // valid in thread 0
}

// f = g - x; with have_last: dF = f - f_last, dG = g - g_last into the ring
// slot; then f_last = f, g_last = g
__global__ void k_aa_push(int64_t L, const double* __restrict__ x, const double* __restrict__ g,
                          double* __restrict__ f_last, double* __restrict__ g_last, double* __restrict__ dF,
                          double* __restrict__ dG, int have_last) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < L; i += (int64_t)gridDim.x * blockDim.x) {
        const double gi = g[i], fi = gi - x[i];
        if (have_last) {
            dF[i] = fi - f_last[i];
            dG[i] = gi - g_last[i];
        }
        f_last[i] = fi;
        g_last[i] = gi;
    }
}

struct AAPtrs {
    const double* dF[kAAMax];
    const double* dG[kAAMax];
    double gamma[kAAMax];
    int m;
};

// partial sums of w dF_a . dF_new and w dF_a . f_last for the m active slots
__global__ void __launch_bounds__(256) k_aa_dots(int64_t L, const uint8_t* __restrict__ wts, AAPtrs P,
                                                 const double* __restrict__ dF_new, const double* __restrict__ f,
                                                 double* __restrict__ part) {
    __shared__ double sh[8];
    double a1[kAAMax], a2[kAAMax];
    for (int a = 0; a < kAAMax; ++a) a1[a] = a2[a] = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < L; i += (int64_t)gridDim.x * blockDim.x) {
        const double w = (double)wts[i];
        const double dn = w * dF_new[i], fn = w * f[i];
#pragma unroll
        for (int a = 0; a < kAAMax; ++a)
            if (a < P.m) {
                const double d = P.dF[a][i];
                a1[a] = fma(d, dn, a1[a]);
                a2[a] = fma(d, fn, a2[a]);
            }
    }
    for (int a = 0; a < P.m; ++a) {
        const double r1 = block_reduce_sum(a1[a], sh);
        const double r2 = block_reduce_sum(a2[a], sh);
        if (threadIdx.x == 0) {
            part[(size_t)blockIdx.x * 2 * kAAMax + a] = r1;
            part[(size_t)blockIdx.x * 2 * kAAMax + kAAMax + a] = r2;
        }
    }
}

// one warp per output a (blockIdx.x)
__global__ void k_aa_dots_finish(const double* __restrict__ part, int nb, int m, double* __restrict__ out) {
    const int a = blockIdx.x;
    if (a >= 2 * kAAMax || (a % kAAMax) >= m) return;
    const double s = warp_parts<false>(part + a, nb, 2 * kAAMax);
    if (threadIdx.x == 0) out[a] = s;
}

// x = g_last - sum_a gamma_a dG_a, clipped at 0; partial sums of w x
__global__ void __launch_bounds__(256) k_aa_mix(int64_t L, const uint8_t* __restrict__ wts, AAPtrs P,
                                                const double* __restrict__ g_last, double* __restrict__ x,
                                                double* __restrict__ part) {
    __shared__ double sh[8];
    double s = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < L; i += (int64_t)gridDim.x * blockDim.x) {
        double v = g_last[i];
#pragma unroll
        for (int a = 0; a < kAAMax; ++a)
            if (a < P.m) v -= P.gamma[a] * P.dG[a][i];
        v = v > 0.0 ? v : 0.0;
        x[i] = v;
        s = fma((double)wts[i], v, s);
    }
    const double r = block_reduce_sum(s, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = r;
}

// x /= sum of the partials (every block re-adds them: nb is small)
__global__ void k_scale_by_sum(int64_t L, double* __restrict__ x, const double* __restrict__ part, int nb) {
    __shared__ double inv;
    if (threadIdx.x < 32) {
        const double s = warp_parts<false>(part, nb, 1);
        if (threadIdx.x == 0) inv = s > 0.0 ? 1.0 / s : 0.0;
    }
    __syncthreads();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < L; i += (int64_t)gridDim.x * blockDim.x)
        x[i] *= inv;
}

// ------------------------------------------------------------- support set
// appends i to idx (capacity cap) when it is not yet in S and either carries
// mass (p > pmin) or has D(x) > dmin; in_s marks members
__global__ void k_select(int64_t R, const double* __restrict__ p, const double* __restrict__ D, double pmin,
                         double dmin, uint8_t* __restrict__ in_s, int* __restrict__ count, uint32_t* __restrict__ idx,
                         int cap) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < R; i += (int64_t)gridDim.x * blockDim.x) {
        if (in_s[i]) continue;
        if ((p && p[i] > pmin) || D[i] > dmin) {
            const int slot = atomicAdd(count, 1);
            if (slot < cap) idx[slot] = (uint32_t)i;
        }
    }
}

__global__ void k_max_vec(int64_t L, const double* __restrict__ v, double* __restrict__ part) {
    __shared__ double sh[8];
    double m = -DBL_MAX;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < L; i += (int64_t)gridDim.x * blockDim.x)
        m = fmax(m, v[i]);
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xFFFFFFFFu, m, o));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, sh[w]);
        part[blockIdx.x] = fmax(m, sh[0]);
    }
}

// N(x_s, y) for the members of S, as FP32 (exact: N <= C(n,k) < 2^24 for n <= 26)
__global__ void k_rows(Split sp, HalfTables A, HalfTables B, const uint32_t* __restrict__ reps,
                       const uint32_t* __restrict__ idx, int S, float* __restrict__ rows) {
    const int ny = 1 << sp.k;
    const int64_t tot = (int64_t)S * ny;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
        const int s = (int)(e / ny), y = (int)(e % ny);
        rows[e] = (float)split_count(sp, A, B, reps[idx[s]], (uint32_t)y);
    }
}

__global__ void k_gather_u8(int S, const uint32_t* __restrict__ idx, const uint32_t* __restrict__ reps, int n,
                            uint8_t* __restrict__ w) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < S; s += gridDim.x * blockDim.x)
        w[s] = (uint8_t)orbit_size(reps[idx[s]], n);
}

__global__ void k_gather_f64(int S, const uint32_t* __restrict__ idx, const double* __restrict__ src,
                             double* __restrict__ dst) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < S; s += gridDim.x * blockDim.x) dst[s] = src[idx[s]];
}

__global__ void k_scatter_f64(int S, const uint32_t* __restrict__ idx, const double* __restrict__ src,
                              double* __restrict__ dst) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < S; s += gridDim.x * blockDim.x) dst[idx[s]] = src[s];
}

__global__ void k_orbit_weights(int64_t R, const uint32_t* __restrict__ reps, int n, uint8_t* __restrict__ w) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < R; i += (int64_t)gridDim.x * blockDim.x)
        w[i] = (uint8_t)orbit_size(reps[i], n);
}

// ---------------------------------------------------- the restricted BA map

// Device state of the restricted problem's accelerated loop (rs_accelerated):
// the Anderson Gram matrix by physical history slot, the mixing weights, the
// bracket of all evaluated points and the flags that gate every kernel of a
// captured step, so that a CUDA graph of several steps runs without the host.
struct RsAAState {
    double A[kAAMax][kAAMax];  // w dF_a . dF_b for physical slots a, b
    double b[kAAMax];          // w dF_a . f_last, by physical slot
    double gamma[kAAMax];      // mixing weights of this step, oldest difference first
    double ub, rate;           // bracket over every evaluated point (nats)
    double u, r, ua, ra;       // this step's plain and mixed evaluations (nats)
    double target;             // stop once ub - rate < target (nats)
    long long evals;
    int npush;                 // differences pushed since the last clear
    int have_last;             // f_last / g_last hold the previous pair
    int solve_ok;              // this step has mixing weights
    int stop_plain;            // the bracket reached the target at the plain point
    int stop_mixed;            // ... at the mixed point
    int fin;                   // finished: every later kernel returns at once
};

// gate 0: always run; 1: not finished; 2: and the plain point did not stop
// the loop; 3: and this step has mixing weights
__device__ __forceinline__ bool rs_skip(const RsAAState* st, int gate) {
    if (!st || gate == 0) return false;
    if (st->fin) return true;
    if (gate >= 2 && st->stop_plain) return true;
    return gate >= 3 && !st->solve_ok;
}

// acc(y) = sum_s |O_s| p_s N(x_s, y) for a slab of 32 outputs per block: lane
// = output, warp w = members w, w + 32, ... (kRsQLoads loads in flight, the
// multiply-adds in member order), the 32 warps' sums added in warp order.
// The last block to finish then forms ln q(y) with q(y) = (1/(4C)) sum over
// the group {id, rev, comp, rev comp} of acc(g y) (ln 0 = 0) and re-arms the
// ticket.
constexpr int kRsQThreads = 1024;
constexpr int kRsQLoads = 12;
__global__ void __launch_bounds__(kRsQThreads) k_rs_q(int S, int k, const float* __restrict__ rows,
                                                      const uint8_t* __restrict__ w, const double* __restrict__ p,
                                                      double inv_c, double* __restrict__ acc,
                                                      double* __restrict__ lnq, unsigned* __restrict__ ticket,
                                                      const RsAAState* st, int gate) {
    if (rs_skip(st, gate)) return;
    __shared__ double sh[kRsQThreads / 32][33];
    __shared__ bool last;
    const int ny = 1 << k;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int y = blockIdx.x * 32 + lane;
    double a = 0.0;
    if (y < ny) {
        for (int s = warp; s < S; s += kRsQLoads * 32) {
            float r[kRsQLoads];
            double wp[kRsQLoads];
#pragma unroll
            for (int u = 0; u < kRsQLoads; ++u) {
                const int t = s + 32 * u;
                r[u] = t < S ? rows[(int64_t)t * ny + y] : 0.0f;
                wp[u] = t < S ? (double)w[t] * p[t] : 0.0;
            }
#pragma unroll
            for (int u = 0; u < kRsQLoads; ++u) a = fma(wp[u], (double)r[u], a);
        }
    }
    sh[warp][lane] = a;
    __syncthreads();
    if (warp == 0) {
        double t = 0.0;
#pragma unroll 8
        for (int i = 0; i < kRsQThreads / 32; ++i) t += sh[i][lane];
        if (y < ny) acc[y] = t;
        __threadfence();
    }
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    for (int yy = threadIdx.x; yy < ny; yy += blockDim.x) {
        const uint32_t r = reverse_bits((uint32_t)yy, k), c = complement_bits((uint32_t)yy, k),
                       rc = reverse_bits(c, k);
        const double q = 0.25 * inv_c * (__ldcg(acc + yy) + __ldcg(acc + r) + __ldcg(acc + c) + __ldcg(acc + rc));
        lnq[yy] = q > 0.0 ? log(q) : 0.0;
    }
    if (threadIdx.x == 0) *ticket = 0u;
}

// D_s = h_s - (1/C) sum_y N(x_s, y) ln q(y): one block per member, each thread
// V consecutive outputs per vector load and up to eight vectors in flight,
// summed in order; the block's threads added as a warp tree, then the warps
// in order
template <int V>
__global__ void __launch_bounds__(256) k_rs_div(int ny, const float* __restrict__ rows,
                                                const double* __restrict__ lnq, const double* __restrict__ h,
                                                double inv_c, double* __restrict__ D, const RsAAState* st,
                                                int gate) {
    if (rs_skip(st, gate)) return;
    __shared__ double sh[8];
    const int s = blockIdx.x;
    const float* __restrict__ row = rows + (int64_t)s * ny;
    const int step = blockDim.x * V;
    double a = 0.0;
    for (int y0 = threadIdx.x * V; y0 < ny; y0 += 8 * step) {
        float r[8][V];
        double l[8][V];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int yy = y0 + u * step;
            if (yy < ny) {
                if constexpr (V == 4) {
                    const float4 f = *reinterpret_cast<const float4*>(row + yy);
                    const double2 l0 = *reinterpret_cast<const double2*>(lnq + yy);
                    const double2 l1 = *reinterpret_cast<const double2*>(lnq + yy + 2);
                    r[u][0] = f.x;
                    r[u][1] = f.y;
                    r[u][2] = f.z;
                    r[u][3] = f.w;
                    l[u][0] = l0.x;
                    l[u][1] = l0.y;
                    l[u][2] = l1.x;
                    l[u][3] = l1.y;
                } else {
#pragma unroll
                    for (int v = 0; v < V; ++v) {
                        r[u][v] = row[yy + v];
                        l[u][v] = lnq[yy + v];
                    }
                }
            } else {
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    r[u][v] = 0.0f;
                    l[u][v] = 0.0;
                }
            }
        }
#pragma unroll
        for (int u = 0; u < 8; ++u)
#pragma unroll
            for (int v = 0; v < V; ++v) a = fma((double)r[u][v], l[u][v], a);
    }
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xFFFFFFFFu, a, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = sh[0];
        for (int i = 1; i < (int)(blockDim.x >> 5); ++i) t += sh[i];
        D[s] = h[s] - t * inv_c;
    }
}

// p'_s = p_s e^{D_s - max D} / Z (one block: S is small); out[0] = max D,
// out[1] = rate of p (nats).  rec 1 / 2 records them in st as the step's
// plain / mixed evaluation, adds them to the bracket and sets the stop flag
// when the bracket is below the target.
__device__ __forceinline__ void rs_update_body(int S, const double* __restrict__ D, const uint8_t* __restrict__ w,
                                               const double* __restrict__ p, double* __restrict__ pn,
                                               double* __restrict__ out, RsAAState* st, int gate, int rec) {
    if (rs_skip(st, gate)) return;
    __shared__ double sh[32], shm[32];
    __shared__ double mD, Zs;
    {  // max D and sum |O| p D: each thread's members in order, a warp tree, the warps in order
        double m = -DBL_MAX, r = 0.0;
        for (int s = threadIdx.x; s < S; s += blockDim.x) {
            const double d = D[s];
            m = fmax(m, d);
            r += (double)w[s] * p[s] * d;
        }
        for (int o = 16; o > 0; o >>= 1) {
            m = fmax(m, __shfl_xor_sync(0xFFFFFFFFu, m, o));
            r += __shfl_xor_sync(0xFFFFFFFFu, r, o);
        }
        if ((threadIdx.x & 31) == 0) {
            shm[threadIdx.x >> 5] = m;
            sh[threadIdx.x >> 5] = r;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = shm[0], r = sh[0];
        for (int i = 1; i < (int)(blockDim.x >> 5); ++i) {
            m = fmax(m, shm[i]);
            r += sh[i];
        }
        mD = m;
        out[0] = m;
        out[1] = r;
        if (rec) {
            if (rec == 1) {
                st->u = m;
                st->r = r;
            } else {
                st->ua = m;
                st->ra = r;
            }
            if (isfinite(m)) st->ub = fmin(st->ub, m);
            if (isfinite(r)) st->rate = fmax(st->rate, r);
            st->evals += 1;
            if (st->ub - st->rate < st->target) {
                if (rec == 1) st->stop_plain = 1;
                else st->stop_mixed = 1;
            }
        }
    }
    __syncthreads();
    double z = 0.0;
    for (int s = threadIdx.x; s < S; s += blockDim.x) {
        const double v = p[s] * exp(D[s] - mD);
        pn[s] = v;
        z = fma((double)w[s], v, z);
    }
    for (int o = 16; o > 0; o >>= 1) z += __shfl_xor_sync(0xFFFFFFFFu, z, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = z;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += sh[i];
        Zs = t;
    }
    __syncthreads();
    const double inv = 1.0 / Zs;
    for (int s = threadIdx.x; s < S; s += blockDim.x) pn[s] *= inv;
}

__global__ void __launch_bounds__(1024) k_rs_update(int S, const double* __restrict__ D,
                                                    const uint8_t* __restrict__ w, const double* __restrict__ p,
                                                    double* __restrict__ pn, double* __restrict__ out,
                                                    RsAAState* st, int gate, int rec) {
    rs_update_body(S, D, w, p, pn, out, st, gate, rec);
}

// ------------------------------------------------- Newton on the support
// The support equations D_s(p) = c (s in F), sum_s |O_s| p_s = 1.  With
// q(y) = (1/4C) sum_g acc(g y) invariant under the group G = {id, rev, comp,
// rev comp}, dD_s/dp_t = -(|O_t| / C^2) M_st where M = Nbar diag(1/q) Nbar^T
// and Nbar_s(y) = (1/4) sum_g N(x_s, g y) (symmetric positive semidefinite).
// Rows of Nbar / sqrt(q) for the members F of S:
__global__ void k_nt_rows(int nF, int k, const int* __restrict__ F, const float* __restrict__ rows,
                          const double* __restrict__ acc, double inv_c, double* __restrict__ out) {
    const int ny = 1 << k;
    const int64_t tot = (int64_t)nF * ny;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
        const int f = (int)(e / ny);
        const uint32_t y = (uint32_t)(e % ny);
        const uint32_t r = reverse_bits(y, k), c = complement_bits(y, k), rc = reverse_bits(c, k);
        const float* row = rows + (int64_t)F[f] * ny;
        const double nb = 0.25 * ((double)row[y] + (double)row[r] + (double)row[c] + (double)row[rc]);
        const double q = 0.25 * inv_c * (acc[y] + acc[r] + acc[c] + acc[rc]);
        out[e] = q > 0.0 ? nb / sqrt(q) : 0.0;
    }
}

// one panel [j0, j1) of a right-looking Cholesky of the lower triangle of M
// (row-major, stride ld), one CTA; the trailing block is updated afterwards
// by a matrix product.  bad[0] is set when a pivot is not positive.
__global__ void __launch_bounds__(1024) k_chol_panel(double* __restrict__ M, int n, int ld, int j0, int j1,
                                                     int* __restrict__ bad) {
    __shared__ double piv;
    for (int c = j0; c < j1; ++c) {
        if (threadIdx.x == 0) {
            const double d = M[(int64_t)c * ld + c];
            if (!(d > 0.0)) bad[0] = 1;
            piv = d > 0.0 ? sqrt(d) : 1.0;
            M[(int64_t)c * ld + c] = piv;
        }
        __syncthreads();
        for (int i = c + 1 + threadIdx.x; i < n; i += blockDim.x) M[(int64_t)i * ld + c] /= piv;
        __syncthreads();
        const int w = j1 - c - 1;  // panel columns right of c
        if (w > 0) {
            const int64_t tot = (int64_t)(n - c - 1) * w;
            for (int64_t e = threadIdx.x; e < tot; e += blockDim.x) {
                const int i = c + 1 + (int)(e / w), cc = c + 1 + (int)(e % w);
                if (cc <= i) M[(int64_t)i * ld + cc] -= M[(int64_t)i * ld + c] * M[(int64_t)cc * ld + c];
            }
        }
        __syncthreads();
    }
}

// With M = L L^T: z1 = M^-1 D_F, z2 = M^-1 1, c = sum z1 / sum z2,
// u = z1 - c z2, d_t = C^2 u_t / |O_t|, pn = p_F + d.  out = [c, number of
// pn <= 0, max |d|, max p_F].  One CTA; b1, b2 are scratch of length n.
__global__ void __launch_bounds__(1024) k_newton_solve(const double* __restrict__ L, int n, int ld,
                                                       const double* __restrict__ Dv, const int* __restrict__ F,
                                                       const uint8_t* __restrict__ w, const double* __restrict__ p,
                                                       double C2, double* __restrict__ b1, double* __restrict__ b2,
                                                       double* __restrict__ pn, double* __restrict__ out) {
    __shared__ double sh[32], sh2[32];
    __shared__ double y1, y2;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        b1[i] = Dv[F[i]];
        b2[i] = 1.0;
    }
    __syncthreads();
    for (int i = 0; i < n; ++i) {  // forward: L y = b
        if (threadIdx.x == 0) {
            const double d = L[(int64_t)i * ld + i];
            y1 = b1[i] / d;
            y2 = b2[i] / d;
            b1[i] = y1;
            b2[i] = y2;
        }
        __syncthreads();
        for (int t = i + 1 + threadIdx.x; t < n; t += blockDim.x) {
            const double l = L[(int64_t)t * ld + i];
            b1[t] -= l * y1;
            b2[t] -= l * y2;
        }
        __syncthreads();
    }
    for (int i = n - 1; i >= 0; --i) {  // back: L^T x = y
        if (threadIdx.x == 0) {
            const double d = L[(int64_t)i * ld + i];
            y1 = b1[i] / d;
            y2 = b2[i] / d;
            b1[i] = y1;
            b2[i] = y2;
        }
        __syncthreads();
        for (int t = threadIdx.x; t < i; t += blockDim.x) {
            const double l = L[(int64_t)i * ld + t];
            b1[t] -= l * y1;
            b2[t] -= l * y2;
        }
        __syncthreads();
    }
    double s1 = 0.0, s2 = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        s1 += b1[i];
        s2 += b2[i];
    }
    for (int o = 16; o > 0; o >>= 1) {
        s1 += __shfl_xor_sync(0xFFFFFFFFu, s1, o);
        s2 += __shfl_xor_sync(0xFFFFFFFFu, s2, o);
    }
    if ((threadIdx.x & 31) == 0) {
        sh[threadIdx.x >> 5] = s1;
        sh2[threadIdx.x >> 5] = s2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
            a += sh[i];
            b += sh2[i];
        }
        y1 = a / b;
    }
    __syncthreads();
    const double c = y1;
    double neg = 0.0, md = 0.0, mp = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int s = F[i];
        const double d = C2 * (b1[i] - c * b2[i]) / (double)w[s];
        const double v = p[s] + d;
        pn[i] = v;
        if (!(v > 0.0)) neg += 1.0;
        md = fmax(md, fabs(d));
        mp = fmax(mp, p[s]);
    }
    for (int o = 16; o > 0; o >>= 1) {
        neg += __shfl_xor_sync(0xFFFFFFFFu, neg, o);
        md = fmax(md, __shfl_xor_sync(0xFFFFFFFFu, md, o));
        mp = fmax(mp, __shfl_xor_sync(0xFFFFFFFFu, mp, o));
    }
    __syncthreads();
    if ((threadIdx.x & 31) == 0) {
        sh[threadIdx.x >> 5] = neg;
        sh2[threadIdx.x >> 5] = md;
        b1[threadIdx.x >> 5] = mp;  // b1 is no longer needed
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0, m = 0.0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
            a += sh[i];
            b = fmax(b, sh2[i]);
            m = fmax(m, b1[i]);
        }
        out[0] = c;
        out[1] = a;
        out[2] = b;
        out[3] = m;
    }
}

// p_S <- 0 outside F, pn on F, then sum |O| p = 1 (one CTA)
__global__ void __launch_bounds__(1024) k_newton_apply(int S, int nF, const int* __restrict__ F,
                                                       const double* __restrict__ pn, const uint8_t* __restrict__ w,
                                                       double* __restrict__ p, int keep_outside) {
    __shared__ double sh[32];
    __shared__ double tot;
    if (!keep_outside)
        for (int s = threadIdx.x; s < S; s += blockDim.x) p[s] = 0.0;
    __syncthreads();
    for (int i = threadIdx.x; i < nF; i += blockDim.x) p[F[i]] = pn[i] > 0.0 ? pn[i] : 0.0;
    __syncthreads();
    double z = 0.0;
    for (int s = threadIdx.x; s < S; s += blockDim.x) z = fma((double)w[s], p[s], z);
    for (int o = 16; o > 0; o >>= 1) z += __shfl_xor_sync(0xFFFFFFFFu, z, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = z;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += sh[i];
        tot = t;
    }
    __syncthreads();
    const double inv = 1.0 / tot;
    for (int s = threadIdx.x; s < S; s += blockDim.x) p[s] *= inv;
}

// ------------------------------------------------------------ host side
// Scratch of the solver, kept per handle: a block released by a DevBuf goes
// back to the handle's pool and the next request of the same size takes it,
// so repeated solves neither allocate nor free (cudaMalloc / cudaFree of
// hundreds of MB per solve stalled the host for up to seconds) and the
// solver's vectors keep their addresses, which keeps the captured BA-map
// graphs valid.  All of the solver's work is ordered on the handle's
// stream, so a block handed out again is never still in use.
struct SolvePool {
    std::multimap<size_t, void*> free_blocks;
    ~SolvePool() {
        for (auto& kv : free_blocks) cudaFree(kv.second);
    }
};

static thread_local SolvePool* t_pool = nullptr;  // the pool of the solve running on this thread

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    SolvePool* pool = nullptr;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    void release() {
        if (p && pool) pool->free_blocks.emplace(bytes, p);
        else if (p) cudaFree(p);
        p = nullptr;
    }
    ~DevBuf() { release(); }
    template <typename T>
    T* get() const { return (T*)p; }
};

static cudaError_t dalloc(DevBuf& b, size_t bytes) {
    b.release();
    bytes = bytes > 0 ? bytes : 16;
    b.bytes = bytes;
    b.pool = t_pool;
    if (t_pool) {
        auto it = t_pool->free_blocks.find(bytes);
        if (it != t_pool->free_blocks.end()) {
            b.p = it->second;
            t_pool->free_blocks.erase(it);
            return cudaSuccess;
        }
    }
    return cudaMalloc(&b.p, bytes);
}

// sets the thread's pool for the duration of one solve
struct PoolScope {
    explicit PoolScope(SolvePool* p) { t_pool = p; }
    ~PoolScope() { t_pool = nullptr; }
};

// Anderson mixing on vectors of length L with orbit weights w; the Gram
// matrix of the stored differences lives on the host (m <= kAAMax numbers a
// row), the vectors on the device.
struct Anderson {
    int64_t L = 0;
    int m = 0, count = 0, head = 0, nb = 0;
    DevBuf f_last, g_last, part, dots;
    DevBuf dF[kAAMax], dG[kAAMax];
    int slot[kAAMax];              // ring order: slot[0] oldest
    double A[kAAMax][kAAMax];      // w dF_a . dF_b for ring positions a, b
    double b[kAAMax];              // w dF_a . f_last
    bool have_last = false;

    cudaError_t init(int64_t len, int mem, int sms) {
        L = len;
        m = mem;
        nb = (int)std::min<int64_t>(sms * 4, (L + 255) / 256);
        nb = std::max(nb, 1);
        cudaError_t e = dalloc(f_last, sizeof(double) * L);
        if (e == cudaSuccess) e = dalloc(g_last, sizeof(double) * L);
        if (e == cudaSuccess) e = dalloc(part, sizeof(double) * nb * 2 * kAAMax);
        if (e == cudaSuccess) e = dalloc(dots, sizeof(double) * 2 * kAAMax);
        for (int i = 0; i < m && e == cudaSuccess; ++i) {
            e = dalloc(dF[i], sizeof(double) * L);
            if (e == cudaSuccess) e = dalloc(dG[i], sizeof(double) * L);
        }
        clear();
        return e;
    }
    void clear() {
        count = 0;
        head = 0;
        have_last = false;
    }
    AAPtrs ptrs() const {
        AAPtrs P{};
        P.m = count;
        for (int a = 0; a < count; ++a) {
            P.dF[a] = dF[slot[a]].get<double>();
            P.dG[a] = dG[slot[a]].get<double>();
        }
        return P;
    }
    // records the pair (x, g = F(x)); updates the Gram rows on the host
    bdc_status push(const double* x, const double* g, const uint8_t* w, cudaStream_t s) {
        if (!have_last) {
            k_aa_push<<<nb, 256, 0, s>>>(L, x, g, f_last.get<double>(), g_last.get<double>(), nullptr, nullptr, 0);
            BDC_CUDA_TRY(cudaGetLastError());
            have_last = true;
            return BDC_OK;
        }
        // the new difference goes to the next free slot (dropping the oldest)
        int sl;
        if (count < m) {
            sl = count;
            slot[count++] = sl;
        } else {
            sl = slot[0];
            for (int a = 1; a < m; ++a) slot[a - 1] = slot[a];
            slot[m - 1] = sl;
            for (int a = 1; a < m; ++a)
                for (int c = 1; c < m; ++c) A[a - 1][c - 1] = A[a][c];
        }
        k_aa_push<<<nb, 256, 0, s>>>(L, x, g, f_last.get<double>(), g_last.get<double>(), dF[sl].get<double>(),
                                     dG[sl].get<double>(), 1);
        BDC_CUDA_TRY(cudaGetLastError());
        AAPtrs P = ptrs();
        k_aa_dots<<<nb, 256, 0, s>>>(L, w, P, dF[sl].get<double>(), f_last.get<double>(), part.get<double>());
        k_aa_dots_finish<<<2 * kAAMax, 32, 0, s>>>(part.get<double>(), nb, count, dots.get<double>());
        BDC_CUDA_TRY(cudaGetLastError());
        double hd[2 * kAAMax];
        BDC_CUDA_TRY(cudaMemcpyAsync(hd, dots.get<double>(), sizeof(hd), cudaMemcpyDeviceToHost, s));
        BDC_CUDA_TRY(cudaStreamSynchronize(s));
        const int nw = count - 1;  // ring position of the new difference
        for (int a = 0; a < count; ++a) {
            A[nw][a] = A[a][nw] = hd[a];
            b[a] = hd[kAAMax + a];
        }
        return BDC_OK;
    }
    // least-squares weights: (A + lambda I) gamma = b, by Cholesky with a
    // small ridge; false when the system is degenerate
    bool solve(double* gamma) const {
        const int c = count;
        if (c < 1) return false;
        double M[kAAMax][kAAMax];
        double tr = 0.0;
        for (int a = 0; a < c; ++a) tr += A[a][a];
        if (!(tr > 0.0) || !std::isfinite(tr)) return false;
        const double lam = 1e-12 * tr / c;
        for (int a = 0; a < c; ++a)
            for (int d = 0; d < c; ++d) M[a][d] = A[a][d] + (a == d ? lam : 0.0);
        for (int j = 0; j < c; ++j) {
            double dsum = M[j][j];
            for (int t = 0; t < j; ++t) dsum -= M[j][t] * M[j][t];
            if (!(dsum > 0.0)) return false;
            M[j][j] = std::sqrt(dsum);
            for (int i = j + 1; i < c; ++i) {
                double v = M[i][j];
                for (int t = 0; t < j; ++t) v -= M[i][t] * M[j][t];
                M[i][j] = v / M[j][j];
            }
        }
        double y[kAAMax];
        for (int i = 0; i < c; ++i) {
            double v = b[i];
            for (int t = 0; t < i; ++t) v -= M[i][t] * y[t];
            y[i] = v / M[i][i];
        }
        for (int i = c - 1; i >= 0; --i) {
            double v = y[i];
            for (int t = i + 1; t < c; ++t) v -= M[t][i] * gamma[t];
            gamma[i] = v / M[i][i];
        }
        for (int i = 0; i < c; ++i)
            if (!std::isfinite(gamma[i])) return false;
        return true;
    }
    // x = g_last - sum gamma dG, clipped and normalised (sum w x = 1)
    bdc_status mix(const double* gamma, const uint8_t* w, double* x, cudaStream_t s) {
        AAPtrs P = ptrs();
        for (int a = 0; a < P.m; ++a) P.gamma[a] = gamma[a];
        k_aa_mix<<<nb, 256, 0, s>>>(L, w, P, g_last.get<double>(), x, part.get<double>());
        k_scale_by_sum<<<nb, 256, 0, s>>>(L, x, part.get<double>(), nb);
        BDC_CUDA_TRY(cudaGetLastError());
        return BDC_OK;
    }
};

struct Bracket {
    double ub = DBL_MAX, rate = -DBL_MAX;
    void add(double u, double r) {
        if (std::isfinite(u)) ub = std::min(ub, u);
        if (std::isfinite(r)) rate = std::max(rate, r);
    }
    double gap_bits() const { return (ub - rate) / 0.69314718055994530942; }
};

// The restricted problem on S: rows, weights, h, and its BA map
struct Restricted {
    int S = 0, ny = 0;
    DevBuf idx, rows, w, h, acc, lnq, D, out, ticket;

    bdc_status build(bdc_handle* H, const std::vector<uint32_t>& members) {
        S = (int)members.size();
        ny = 1 << H->k;
        BDC_CUDA_TRY(dalloc(idx, sizeof(uint32_t) * S));
        BDC_CUDA_TRY(dalloc(rows, sizeof(float) * (size_t)S * ny));
        BDC_CUDA_TRY(dalloc(w, S));
        BDC_CUDA_TRY(dalloc(h, sizeof(double) * S));
        BDC_CUDA_TRY(dalloc(acc, sizeof(double) * ny));
        BDC_CUDA_TRY(dalloc(lnq, sizeof(double) * ny));
        BDC_CUDA_TRY(dalloc(D, sizeof(double) * S));
        BDC_CUDA_TRY(dalloc(out, sizeof(double) * 2));
        BDC_CUDA_TRY(dalloc(ticket, sizeof(unsigned)));
        BDC_CUDA_TRY(cudaMemsetAsync(ticket.p, 0, sizeof(unsigned), H->stream));
        BDC_CUDA_TRY(cudaMemcpyAsync(idx.p, members.data(), sizeof(uint32_t) * S, cudaMemcpyHostToDevice, H->stream));
        const int g = std::max(1, std::min(H->num_sms * 8, (int)(((int64_t)S * ny + 255) / 256)));
        k_rows<<<g, 256, 0, H->stream>>>(H->s, H->A, H->B, H->d_reps, idx.get<uint32_t>(), S, rows.get<float>());
        k_gather_u8<<<(S + 255) / 256, 256, 0, H->stream>>>(S, idx.get<uint32_t>(), H->d_reps, H->n, w.get<uint8_t>());
        k_gather_f64<<<(S + 255) / 256, 256, 0, H->stream>>>(S, idx.get<uint32_t>(), H->d_h, h.get<double>());
        BDC_CUDA_TRY(cudaGetLastError());
        return BDC_OK;
    }
    // queues p -> pn (three kernels, gated by st / gate, recorded by rec; see
    // k_rs_update)
    // queues acc, ln q and D of p (two kernels, gated by st / gate)
    cudaError_t enqueue_qd(bdc_handle* H, const double* p, RsAAState* st, int gate) {
        cudaStream_t s = H->stream;
        k_rs_q<<<(ny + 31) / 32, kRsQThreads, 0, s>>>(S, H->k, rows.get<float>(), w.get<uint8_t>(), p, H->inv_c,
                                                      acc.get<double>(), lnq.get<double>(), ticket.get<unsigned>(),
                                                      st, gate);
        if (ny >= 128)
            k_rs_div<4><<<S, std::max(32, std::min(256, ny / 32)), 0, s>>>(ny, rows.get<float>(), lnq.get<double>(),
                                                               h.get<double>(), H->inv_c, D.get<double>(), st, gate);
        else
            k_rs_div<1><<<S, 32, 0, s>>>(ny, rows.get<float>(), lnq.get<double>(), h.get<double>(), H->inv_c,
                                         D.get<double>(), st, gate);
        return cudaGetLastError();
    }
    cudaError_t enqueue_map(bdc_handle* H, const double* p, double* pn, RsAAState* st, int gate, int rec) {
        cudaStream_t s = H->stream;
        const cudaError_t e = enqueue_qd(H, p, st, gate);
        if (e != cudaSuccess) return e;
        k_rs_update<<<1, 1024, 0, s>>>(S, D.get<double>(), w.get<uint8_t>(), p, pn, out.get<double>(), st, gate,
                                       rec);
        return cudaGetLastError();
    }
    // p -> pn; ub / rate (nats) of p
    bdc_status map(bdc_handle* H, const double* p, double* pn, double* ub, double* rate) {
        cudaStream_t s = H->stream;
        BDC_CUDA_TRY(enqueue_map(H, p, pn, nullptr, 0, 0));
        double o[2];
        BDC_CUDA_TRY(cudaMemcpyAsync(o, out.p, sizeof(o), cudaMemcpyDeviceToHost, s));
        BDC_CUDA_TRY(cudaStreamSynchronize(s));
        *ub = o[0];
        *rate = o[1];
        return BDC_OK;
    }
};

// ------------------------------- the restricted loop, resident on the device
// The same Anderson-accelerated BA with the rate guard as accelerated_ba, for
// the restricted problem, with every decision taken on the device from
// RsAAState: one step is the plain map, the push of the new differences with
// their Gram products, the least-squares weights, the mixed point, its map and
// the choice of the next iterate -- six kernels (per map the member sums
// and D, then one block that updates and, after the plain map, pushes,
// solves and mixes, after the mixed map accepts), captured kRsGraphSteps
// steps to a CUDA graph; the host reads the state once per graph.
constexpr int kRsGraphSteps = 16;

struct RsSlots {
    double* dF[kAAMax];
    double* dG[kAAMax];
};

// the rate guard: the mixed point is kept when it has weights, a finite
// bound and a rate at least the plain step's
__device__ __forceinline__ bool rs_mixed_kept(const RsAAState* st) {
    return st->solve_ok && isfinite(st->ua) && st->ra >= st->r;
}

// ---- the step's small kernels merged, one block each (L = |S| is small):
// push + dot products + the Anderson solve, mix + normalise, accept + state.
constexpr int kRsBlock = 1024;

// f = g - x; with a last pair, dF = f - f_last and dG = g - g_last go to the
// ring slot sl = npush % m, with the dot products w dF_a . dF_sl and
// w dF_a . f over the slots in use; then f_last = f, g_last = g.  Thread 0
// then writes the new Gram row and right side and solves (A + lambda I)
// gamma = b by Cholesky with the ridge lambda = 1e-12 tr(A) / c over the c
// slots in use; solve_ok = 0 when the system is degenerate or this was the
// first pair after a clear.
__device__ __forceinline__ void rs_push_solve_body(int L, int m, const uint8_t* __restrict__ wts,
                                                   const double* __restrict__ x, const double* __restrict__ g,
                                                   double* __restrict__ f_last, double* __restrict__ g_last,
                                                   RsSlots P, RsAAState* st) {
    if (rs_skip(st, 2)) return;
    const bool diff = st->have_last != 0;
    const int sl = st->npush % m;
    const int act = min(st->npush + 1, m);
    double a1[kAAMax], a2[kAAMax];
#pragma unroll
    for (int a = 0; a < kAAMax; ++a) a1[a] = a2[a] = 0.0;
    for (int i = threadIdx.x; i < L; i += kRsBlock) {
        const double gi = g[i], fi = gi - x[i];
        if (diff) {
            const double dn = fi - f_last[i];
            P.dF[sl][i] = dn;
            P.dG[sl][i] = gi - g_last[i];
            const double w = (double)wts[i];
#pragma unroll
            for (int a = 0; a < kAAMax; ++a)
                if (a < act) {
                    const double d = (a == sl) ? dn : P.dF[a][i];
                    a1[a] = fma(d, w * dn, a1[a]);
                    a2[a] = fma(d, w * fi, a2[a]);
                }
        }
        f_last[i] = fi;
        g_last[i] = gi;
    }
    // the dot products: a warp tree per warp, then thread a (a < act) adds
    // the warps' w dF_a . dF_sl in warp order and thread kAAMax + a the
    // w dF_a . f; the Gram matrix comes to shared memory at the same time
    __shared__ double wp[kRsBlock / 32][2 * kAAMax];
    __shared__ double sA[kAAMax][kAAMax], sb[kAAMax];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (diff) {
#pragma unroll
        for (int a = 0; a < kAAMax; ++a)
            if (a < act) {
                double v1 = a1[a], v2 = a2[a];
                for (int o = 16; o > 0; o >>= 1) {
                    v1 += __shfl_xor_sync(0xFFFFFFFFu, v1, o);
                    v2 += __shfl_xor_sync(0xFFFFFFFFu, v2, o);
                }
                if (lane == 0) {
                    wp[warp][a] = v1;
                    wp[warp][kAAMax + a] = v2;
                }
            }
    }
    if (threadIdx.x < kAAMax * kAAMax) {
        const int i = threadIdx.x / kAAMax, j = threadIdx.x % kAAMax;
        sA[i][j] = st->A[i][j];
    } else if (threadIdx.x < kAAMax * kAAMax + kAAMax) {
        sb[threadIdx.x - kAAMax * kAAMax] = st->b[threadIdx.x - kAAMax * kAAMax];
    }
    __syncthreads();  // every thread has read st
    if (diff && threadIdx.x < 2 * kAAMax && threadIdx.x % kAAMax < act) {
        const int a = threadIdx.x % kAAMax;
        double t = 0.0;
        for (int i = 0; i < kRsBlock / 32; ++i) t += wp[i][threadIdx.x];
        if (threadIdx.x < kAAMax) {
            sA[sl][a] = t;
            sA[a][sl] = t;
            st->A[sl][a] = t;
            st->A[a][sl] = t;
        } else {
            sb[a] = t;
            st->b[a] = t;
        }
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    st->solve_ok = 0;
    if (!st->have_last) {
        st->have_last = 1;
        return;
    }
    const int c = act;
    st->npush += 1;
    // the system in ring order, oldest difference first: position j holds
    // physical slot (npush - c + j) % m.  Products and differences are
    // rounded separately (no FMA contraction), as in the host-side solve of
    // the full-space loop.
    int ph[kAAMax];
    for (int j = 0; j < c; ++j) ph[j] = (st->npush - c + j) % m;
    double M[kAAMax][kAAMax], y[kAAMax], gam[kAAMax];
    double tr = 0.0;
    for (int a = 0; a < c; ++a) tr += sA[ph[a]][ph[a]];
    if (!(tr > 0.0) || !isfinite(tr)) return;
    const double lam = 1e-12 * tr / c;
    for (int a = 0; a < c; ++a)
        for (int d = 0; d < c; ++d) M[a][d] = sA[ph[a]][ph[d]] + (a == d ? lam : 0.0);
    for (int j = 0; j < c; ++j) {
        double dsum = M[j][j];
        for (int t = 0; t < j; ++t) dsum = __dsub_rn(dsum, __dmul_rn(M[j][t], M[j][t]));
        if (!(dsum > 0.0)) return;
        M[j][j] = sqrt(dsum);
        for (int i = j + 1; i < c; ++i) {
            double v = M[i][j];
            for (int t = 0; t < j; ++t) v = __dsub_rn(v, __dmul_rn(M[i][t], M[j][t]));
            M[i][j] = v / M[j][j];
        }
    }
    for (int i = 0; i < c; ++i) {
        double v = sb[ph[i]];
        for (int t = 0; t < i; ++t) v = __dsub_rn(v, __dmul_rn(M[i][t], y[t]));
        y[i] = v / M[i][i];
    }
    for (int i = c - 1; i >= 0; --i) {
        double v = y[i];
        for (int t = i + 1; t < c; ++t) v = __dsub_rn(v, __dmul_rn(M[t][i], gam[t]));
        gam[i] = v / M[i][i];
    }
    for (int i = 0; i < c; ++i)
        if (!isfinite(gam[i])) return;
    for (int i = 0; i < c; ++i) st->gamma[i] = gam[i];  // ring order
    st->solve_ok = 1;
}

// xa = g_last - sum_a gamma_a dG_a, clipped at 0, normalised to sum w xa = 1
__device__ __forceinline__ void rs_mix_scale_body(int L, int m, const uint8_t* __restrict__ wts, RsSlots P,
                                                  const double* __restrict__ g_last, double* __restrict__ xa,
                                                  const RsAAState* st) {
    if (rs_skip(st, 3)) return;
    __shared__ double sh[kRsBlock / 32];
    __shared__ double inv;
    const int c = min(st->npush, m);
    double gam[kAAMax];
    const double* dg[kAAMax];
#pragma unroll
    for (int a = 0; a < kAAMax; ++a) {
        gam[a] = (a < c) ? st->gamma[a] : 0.0;
        dg[a] = P.dG[(a < c) ? (st->npush - c + a) % m : 0];
    }
    double sum = 0.0;
    for (int i = threadIdx.x; i < L; i += kRsBlock) {
        double v = g_last[i];
#pragma unroll
        for (int a = 0; a < kAAMax; ++a)
            if (a < c) v -= gam[a] * dg[a][i];
        v = v > 0.0 ? v : 0.0;
        xa[i] = v;
        sum = fma((double)wts[i], v, sum);
    }
    const double t = block_reduce_sum(sum, sh);
    if (threadIdx.x == 0) inv = t > 0.0 ? 1.0 / t : 0.0;
    __syncthreads();
    for (int i = threadIdx.x; i < L; i += kRsBlock) xa[i] *= inv;
}

// the next iterate (the mixed image when kept, else the plain one); then a
// rejected mixed point clears the history (when it holds a difference) and a
// stop flag ends the loop
__device__ __forceinline__ void rs_accept_body(int L, int m, double* __restrict__ x, const double* __restrict__ g,
                                               const double* __restrict__ ga, RsAAState* st) {
    if (rs_skip(st, 1)) return;
    const double* __restrict__ src = (!st->stop_plain && rs_mixed_kept(st)) ? ga : g;
    for (int i = threadIdx.x; i < L; i += kRsBlock) x[i] = src[i];
    __syncthreads();  // every thread has read st
    if (threadIdx.x != 0) return;
    if (st->stop_plain) {
        st->fin = 1;
        return;
    }
    if (!rs_mixed_kept(st) && min(st->npush, m) >= 1) {
        st->npush = 0;
        st->have_last = 0;
    }
    if (st->stop_mixed) st->fin = 1;
    st->solve_ok = 0;
}

// the plain map's update (gate 1), then push + solve (gate 2), then the
// mixed point (gate 3), one block: each part reads what the one before it
// left in st and in the vectors after a block barrier
__global__ void __launch_bounds__(kRsBlock) k_rs_step_plain(int L, int m, const double* __restrict__ D,
                                                           const uint8_t* __restrict__ w, const double* __restrict__ x,
                                                           double* __restrict__ g, double* __restrict__ out,
                                                           double* __restrict__ f_last, double* __restrict__ g_last,
                                                           RsSlots P, double* __restrict__ xa, RsAAState* st) {
    rs_update_body(L, D, w, x, g, out, st, 1, 1);
    __syncthreads();
    rs_push_solve_body(L, m, w, x, g, f_last, g_last, P, st);
    __syncthreads();
    rs_mix_scale_body(L, m, w, P, g_last, xa, st);
}

// the mixed map's update (gate 3), then the next iterate (gate 1)
__global__ void __launch_bounds__(kRsBlock) k_rs_step_mixed(int L, int m, const double* __restrict__ D,
                                                           const uint8_t* __restrict__ w, const double* __restrict__ xa,
                                                           double* __restrict__ ga, double* __restrict__ out,
                                                           double* __restrict__ x, const double* __restrict__ g,
                                                           RsAAState* st) {
    rs_update_body(L, D, w, xa, ga, out, st, 3, 2);
    __syncthreads();
    rs_accept_body(L, m, x, g, ga, st);
}

struct RsAA {
    int L = 0, m = 0;
    DevBuf f_last, g_last, st;
    DevBuf dF[kAAMax], dG[kAAMax];
    RsAAState* host[2] = {nullptr, nullptr};  // pinned copies of the state, one per graph in flight
    cudaEvent_t copied[2] = {nullptr, nullptr};

    ~RsAA() {
        for (int i = 0; i < 2; ++i) {
            if (host[i]) cudaFreeHost(host[i]);
            if (copied[i]) cudaEventDestroy(copied[i]);
        }
    }
    cudaError_t init(int len, int mem) {
        L = len;
        m = mem;
        cudaError_t e = cudaSuccess;
        for (int i = 0; i < 2 && e == cudaSuccess; ++i) {
            e = cudaMallocHost(&host[i], sizeof(RsAAState));
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&copied[i], cudaEventDisableTiming);
        }
        if (e == cudaSuccess) e = dalloc(f_last, sizeof(double) * L);
        if (e == cudaSuccess) e = dalloc(g_last, sizeof(double) * L);
        if (e == cudaSuccess) e = dalloc(st, sizeof(RsAAState));
        for (int i = 0; i < m && e == cudaSuccess; ++i) {
            e = dalloc(dF[i], sizeof(double) * L);
            if (e == cudaSuccess) e = dalloc(dG[i], sizeof(double) * L);
        }
        return e;
    }
    RsSlots slots() const {
        RsSlots P{};
        for (int i = 0; i < m; ++i) {
            P.dF[i] = dF[i].get<double>();
            P.dG[i] = dG[i].get<double>();
        }
        return P;
    }
};

static cudaError_t rs_enqueue_step(bdc_handle* H, Restricted& rs, RsAA& aa, double* x, double* g, double* xa,
                                   double* ga) {
    cudaStream_t s = H->stream;
    RsAAState* st = aa.st.get<RsAAState>();
    const uint8_t* w = rs.w.get<uint8_t>();
    cudaError_t e = rs.enqueue_qd(H, x, st, 1);
    if (e != cudaSuccess) return e;
    k_rs_step_plain<<<1, kRsBlock, 0, s>>>(aa.L, aa.m, rs.D.get<double>(), w, x, g, rs.out.get<double>(),
                                           aa.f_last.get<double>(), aa.g_last.get<double>(), aa.slots(), xa, st);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    e = rs.enqueue_qd(H, xa, st, 3);
    if (e != cudaSuccess) return e;
    k_rs_step_mixed<<<1, kRsBlock, 0, s>>>(aa.L, aa.m, rs.D.get<double>(), w, xa, ga, rs.out.get<double>(), x, g,
                                           st);
    return cudaGetLastError();
}

// accelerated_ba on the restricted problem, resident on the device: runs
// until the bracket (started from br) is below gap_bits or about max_evals
// evaluations (checked once per graph of kRsGraphSteps steps); x holds the
// start and receives the last accepted point
static bdc_status rs_accelerated(bdc_handle* H, Restricted& rs, RsAA& aa, double* x, double* g, double* xa,
                                 double* ga, double gap_bits, int64_t max_evals, Bracket& br, int64_t* evals) {
    cudaStream_t s = H->stream;
    RsAAState hs;
    memset(&hs, 0, sizeof(hs));
    hs.ub = br.ub;
    hs.rate = br.rate;
    hs.target = gap_bits * 0.69314718055994530942;
    BDC_CUDA_TRY(cudaMemcpyAsync(aa.st.p, &hs, sizeof(hs), cudaMemcpyHostToDevice, s));
    BDC_CUDA_TRY(cudaStreamSynchronize(s));
    // captured on the handle's own stream (the caller's may be the legacy
    // default stream, which cannot be captured), launched on the caller's
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    H->stream = H->own_stream;
    cudaError_t e = cudaStreamBeginCapture(H->own_stream, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        for (int k = 0; k < kRsGraphSteps && e == cudaSuccess; ++k) e = rs_enqueue_step(H, rs, aa, x, g, xa, ga);
        const cudaError_t e2 = cudaStreamEndCapture(H->own_stream, &graph);
        if (e == cudaSuccess) e = e2;
    }
    H->stream = s;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
    // two graphs in flight: while the host reads the state after one, the
    // next already runs (after the loop finishes every kernel returns at
    // once, so a graph queued past the end changes nothing)
    auto queue = [&](int i) -> cudaError_t {
        cudaError_t r = cudaGraphLaunch(exec, s);
        if (r == cudaSuccess) r = cudaMemcpyAsync(aa.host[i], aa.st.p, sizeof(RsAAState), cudaMemcpyDeviceToHost, s);
        if (r == cudaSuccess) r = cudaEventRecord(aa.copied[i], s);
        return r;
    };
    int next = 0;
    if (e == cudaSuccess) e = queue(0);
    if (e == cudaSuccess) e = queue(1);
    while (e == cudaSuccess) {
        e = cudaEventSynchronize(aa.copied[next]);
        if (e != cudaSuccess) break;
        const RsAAState& h = *aa.host[next];
        if (h.fin || h.evals >= max_evals) break;
        e = queue(next);
        next ^= 1;
    }
    // the last queued graph wrote the other copy
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess) hs = *aa.host[next ^ 1];
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (e != cudaSuccess) return fail(BDC_ERR_CUDA, "bdc_solve: restricted loop: %s", cudaGetErrorString(e));
    br.ub = hs.ub;
    br.rate = hs.rate;
    *evals += hs.evals;
    return BDC_OK;
}

__global__ void __launch_bounds__(1024) k_ridge(double* __restrict__ M, int n, int ld, double rel) {
    __shared__ double sh[32];
    double m = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) m = fmax(m, M[(int64_t)i * ld + i]);
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xFFFFFFFFu, m, o));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
    __syncthreads();
    double mm = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) mm = fmax(mm, sh[i]);
    for (int i = threadIdx.x; i < n; i += blockDim.x) M[(int64_t)i * ld + i] += rel * mm;
}

// Active-set Newton on the support equations of the restricted problem,
// started from p (device, |S|): F = members with D_s within `margin` of the
// rate; each step solves the linearised equations on F (Cholesky of M on
// the device), members that the step would make non-positive leave F, and
// members outside F whose D_s exceeds the rate join it.  *ok = false when
// the factorisation breaks down (p is then left at a valid point).
static bdc_status newton_polish(bdc_handle* H, Restricted& rs, double* p, double* scratch, double margin, Bracket& rb,
                                bool* ok) {
    cudaStream_t s = H->stream;
    const int S = rs.S, ny = rs.ny;
    *ok = true;
    if (S > 8192) {
        *ok = false;
        return BDC_OK;
    }
    DevBuf dF, Bq, M, b1, b2, pn, out, bad;
    BDC_CUDA_TRY(dalloc(dF, sizeof(int) * S));
    BDC_CUDA_TRY(dalloc(Bq, sizeof(double) * (size_t)S * ny));
    BDC_CUDA_TRY(dalloc(M, sizeof(double) * (size_t)S * S));
    BDC_CUDA_TRY(dalloc(b1, sizeof(double) * std::max(S, 64)));
    BDC_CUDA_TRY(dalloc(b2, sizeof(double) * S));
    BDC_CUDA_TRY(dalloc(pn, sizeof(double) * S));
    BDC_CUDA_TRY(dalloc(out, sizeof(double) * 4));
    BDC_CUDA_TRY(dalloc(bad, sizeof(int)));
    // one descriptor and tile map for every product below (at most S x S)
    struct ScratchHolder {
        DgemmScratch sc;
        ~ScratchHolder() { dgemm_scratch_free(sc); }
    } gh;
    BDC_CUDA_TRY(dgemm_scratch_alloc(gh.sc, ((S + 63) / 64) * ((S + 63) / 64), s));
    const DgemmScratch& gsc = gh.sc;
    std::vector<double> hD(S), hp(S);
    auto fetch = [&]() -> bdc_status {
        BDC_CUDA_TRY(cudaMemcpyAsync(hD.data(), rs.D.p, sizeof(double) * S, cudaMemcpyDeviceToHost, s));
        BDC_CUDA_TRY(cudaMemcpyAsync(hp.data(), p, sizeof(double) * S, cudaMemcpyDeviceToHost, s));
        BDC_CUDA_TRY(cudaStreamSynchronize(s));
        return BDC_OK;
    };
    // sets p to vals on F, 0 elsewhere, normalised
    auto apply = [&](const std::vector<int>& F, const double* vals_dev) -> bdc_status {
        BDC_CUDA_TRY(cudaMemcpyAsync(dF.p, F.data(), sizeof(int) * F.size(), cudaMemcpyHostToDevice, s));
        k_newton_apply<<<1, 1024, 0, s>>>(S, (int)F.size(), dF.get<int>(), vals_dev, rs.w.get<uint8_t>(), p, 0);
        BDC_CUDA_TRY(cudaGetLastError());
        return BDC_OK;
    };
    double ub, c;
    bdc_status rc = rs.map(H, p, scratch, &ub, &c);
    if (rc != BDC_OK) return rc;
    rb.add(ub, c);
    rc = fetch();
    if (rc != BDC_OK) return rc;
    std::vector<int> F;
    for (int i = 0; i < S; ++i)
        if (hD[i] > c - margin) F.push_back(i);
    const double C2 = H->C * H->C;
    for (int outer = 0; outer < 10; ++outer) {
        for (int inner = 0; inner < 40 && !F.empty(); ++inner) {
            const int nF = (int)F.size();
            BDC_CUDA_TRY(cudaMemcpyAsync(dF.p, F.data(), sizeof(int) * nF, cudaMemcpyHostToDevice, s));
            const int g = std::max(1, std::min(H->num_sms * 8, (int)(((int64_t)nF * ny + 255) / 256)));
            k_nt_rows<<<g, 256, 0, s>>>(nF, H->k, dF.get<int>(), rs.rows.get<float>(), rs.acc.get<double>(), H->inv_c,
                                        Bq.get<double>());
            BDC_CUDA_TRY(cudaGetLastError());
            BDC_CUDA_TRY(dgemm_nt(gsc, Bq.get<double>(), ny, Bq.get<double>(), ny, M.get<double>(), nF, nF, nF, ny, 1.0,
                                  0, s));
            k_ridge<<<1, 1024, 0, s>>>(M.get<double>(), nF, nF, 1e-15);
            BDC_CUDA_TRY(cudaMemsetAsync(bad.p, 0, sizeof(int), s));
            for (int j0 = 0; j0 < nF; j0 += 32) {
                const int j1 = std::min(nF, j0 + 32);
                k_chol_panel<<<1, 1024, 0, s>>>(M.get<double>(), nF, nF, j0, j1, bad.get<int>());
                BDC_CUDA_TRY(cudaGetLastError());
                if (j1 < nF)
                    BDC_CUDA_TRY(dgemm_nt(gsc, M.get<double>() + (int64_t)j1 * nF + j0, nF, M.get<double>() + (int64_t)j1 * nF + j0,
                                          nF, M.get<double>() + (int64_t)j1 * nF + j1, nF, nF - j1, nF - j1, j1 - j0, -1.0,
                                          1, s));
            }
            int hbad = 0;
            BDC_CUDA_TRY(cudaMemcpyAsync(&hbad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, s));
            BDC_CUDA_TRY(cudaStreamSynchronize(s));
            if (hbad) {
                *ok = false;
                return BDC_OK;
            }
            k_newton_solve<<<1, 1024, 0, s>>>(M.get<double>(), nF, nF, rs.D.get<double>(), dF.get<int>(),
                                              rs.w.get<uint8_t>(), p, C2, b1.get<double>(), b2.get<double>(),
                                              pn.get<double>(), out.get<double>());
            BDC_CUDA_TRY(cudaGetLastError());
            double ho[4];
            BDC_CUDA_TRY(cudaMemcpyAsync(ho, out.p, sizeof(ho), cudaMemcpyDeviceToHost, s));
            BDC_CUDA_TRY(cudaStreamSynchronize(s));
            if (ho[1] > 0.0) {
                // members that the step sends to zero or below leave F
                std::vector<double> hpn(nF);
                BDC_CUDA_TRY(cudaMemcpyAsync(hpn.data(), pn.p, sizeof(double) * nF, cudaMemcpyDeviceToHost, s));
                BDC_CUDA_TRY(cudaStreamSynchronize(s));
                std::vector<int> keep;
                std::vector<double> kv;
                for (int i = 0; i < nF; ++i)
                    if (hpn[i] > 0.0) {
                        keep.push_back(F[i]);
                        kv.push_back(hp[F[i]]);
                    }
                F.swap(keep);
                BDC_CUDA_TRY(cudaMemcpyAsync(pn.p, kv.data(), sizeof(double) * kv.size(), cudaMemcpyHostToDevice, s));
                rc = apply(F, pn.get<double>());
                if (rc != BDC_OK) return rc;
            } else {
                rc = apply(F, pn.get<double>());
                if (rc != BDC_OK) return rc;
            }
            rc = rs.map(H, p, scratch, &ub, &c);
            if (rc != BDC_OK) return rc;
            rb.add(ub, c);
            rc = fetch();
            if (rc != BDC_OK) return rc;
            if (ho[1] == 0.0 && (ub - c <= 1e-15 * std::fabs(c) || ho[2] <= 1e-16 * ho[3])) break;
        }
        // members outside F that beat the rate join it with a small mass
        std::vector<int> add;
        double mp = 0.0;
        for (int i = 0; i < S; ++i) mp = std::max(mp, hp[i]);
        std::vector<char> inF(S, 0);
        for (int f : F) inF[f] = 1;
        for (int i = 0; i < S; ++i)
            if (!inF[i] && hD[i] > c + 1e-14 * std::fabs(c)) add.push_back(i);
        if (add.empty()) break;
        std::vector<int> F2 = F;
        F2.insert(F2.end(), add.begin(), add.end());
        std::sort(F2.begin(), F2.end());
        std::vector<double> vals(F2.size());
        for (size_t i = 0; i < F2.size(); ++i) vals[i] = inF[F2[i]] ? hp[F2[i]] : 1e-3 * mp;
        F.swap(F2);
        BDC_CUDA_TRY(cudaMemcpyAsync(pn.p, vals.data(), sizeof(double) * vals.size(), cudaMemcpyHostToDevice, s));
        rc = apply(F, pn.get<double>());
        if (rc != BDC_OK) return rc;
        rc = rs.map(H, p, scratch, &ub, &c);
        if (rc != BDC_OK) return rc;
        rb.add(ub, c);
        rc = fetch();
        if (rc != BDC_OK) return rc;
    }
    return BDC_OK;
}

// Anderson-accelerated BA with the rate guard on an abstract map; stops when
// the bracket of the evaluated points is below gap_bits or after max_evals
// evaluations.  x holds the start and receives the last accepted point.
template <typename Map>
static bdc_status accelerated_ba(bdc_handle* H, Anderson& aa, const uint8_t* w, Map&& F, double* x, double* g,
                                 double* xa, double* ga, int64_t L, double gap_bits, int64_t max_evals,
                                 Bracket& br, int64_t* evals) {
    cudaStream_t s = H->stream;
    aa.clear();
    int64_t ev = 0;
    while (ev < max_evals) {
        double u, r;
        bdc_status rc = F(x, g, &u, &r);
        if (rc != BDC_OK) return rc;
        ++ev;
        br.add(u, r);
        if (br.gap_bits() < gap_bits) {
            BDC_CUDA_TRY(cudaMemcpyAsync(x, g, sizeof(double) * L, cudaMemcpyDeviceToDevice, s));
            break;
        }
        rc = aa.push(x, g, w, s);
        if (rc != BDC_OK) return rc;
        double gamma[kAAMax];
        bool mixed = false;
        if (aa.count >= 1 && aa.solve(gamma)) {
            rc = aa.mix(gamma, w, xa, s);
            if (rc != BDC_OK) return rc;
            double ua, ra;
            rc = F(xa, ga, &ua, &ra);
            if (rc != BDC_OK) return rc;
            ++ev;
            br.add(ua, ra);
            if (std::isfinite(ua) && ra >= r) {
                BDC_CUDA_TRY(cudaMemcpyAsync(x, ga, sizeof(double) * L, cudaMemcpyDeviceToDevice, s));
                mixed = true;
            }
        }
        if (!mixed) {
            if (aa.count >= 1) aa.clear();
            BDC_CUDA_TRY(cudaMemcpyAsync(x, g, sizeof(double) * L, cudaMemcpyDeviceToDevice, s));
        }
        if (br.gap_bits() < gap_bits) break;
    }
    *evals += ev;
    return BDC_OK;
}

}  // namespace bdc

using namespace bdc;

namespace bdc {

// The solver with a choice of its first phase: SOLVE_ANDERSON (bdc_solve),
// SOLVE_MOMENTUM (the accelerated loop of factored_accelerate, run on the
// handle's own iterate to the switch bracket) or SOLVE_FROM_POINT (the caller
// has brought the handle's iterate near the optimum already: only the
// support phases run, starting from the best bounds the handle has seen).
enum SolvePhase1 { SOLVE_ANDERSON = 0, SOLVE_MOMENTUM = 1, SOLVE_FROM_POINT = 2 };

bdc_status solve_impl(bdc_handle_t H, double gap_bits, int64_t max_evals, bdc_stats* stats, int phase1) {
    if (!H) return fail(BDC_ERR_ARG, "bdc_solve: NULL handle");
    if (!H->p_set) return fail(BDC_ERR_STATE, "bdc_solve: no distribution set");
    if (H->engine != BDC_ENGINE_FACTORED) return fail(BDC_ERR_UNSUPPORTED, "bdc_solve: needs the factored engine (k < n)");
    if (H->shard_world > 1) return fail(BDC_ERR_STATE, "bdc_solve: this handle holds a shard of the rows");
    if (!(gap_bits > 0.0) || max_evals < 1) return fail(BDC_ERR_ARG, "bdc_solve: need gap_bits > 0 and max_evals >= 1");
    if (H->n > 26) return fail(BDC_ERR_UNSUPPORTED, "bdc_solve: counts of n > 26 do not fit FP32 exactly");
    BDC_CUDA_TRY(cudaSetDevice(H->device));
    if (!H->solve_pool) H->solve_pool = new SolvePool();
    // declared before every DevBuf of this call, so it outlives them
    PoolScope pool_scope((SolvePool*)H->solve_pool);
    cudaStream_t s = H->stream;
    const int64_t R = H->R;
    const int sms = H->num_sms;
    const int nbR = (int)std::min<int64_t>(sms * 8, (R + 255) / 256);
    const auto t_start = std::chrono::steady_clock::now();
    auto elapsed = [&] { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count(); };

    Bracket br;
    int64_t evals = 0;
    const double switch_bits = std::max(gap_bits, kSupportSwitchBits);
    bdc_status rc = BDC_OK;
    if (phase1 == SOLVE_MOMENTUM) {
        // the momentum phase on the handle's dense state, then its point
        bdc_stats s1{};
        rc = factored_accelerate(H, max_evals, switch_bits, &s1);
        if (rc != BDC_OK) return rc;
        evals += s1.iters;
    }
    if (phase1 != SOLVE_ANDERSON) {
        BDC_CUDA_TRY(cudaMemcpyAsync(H->h_st, H->d_st, sizeof(DevState), cudaMemcpyDeviceToHost, s));
        BDC_CUDA_TRY(cudaStreamSynchronize(s));
        br.add(H->h_st->best_ub, H->h_st->best_rate);
        if (H->verbose)
            printf("bdc: solve phase 1 (momentum): %lld full evaluations, gap %.3e bits (%.3f s)\n", (long long)evals,
                   br.gap_bits(), elapsed());
    }
    // start: the handle's current iterate
    const double* cur = nullptr;
    rc = engine_current_p(H, &cur);
    if (rc != BDC_OK) return rc;
    DevBuf x, g, xa, ga, D, wts, in_s, cnt, sel, mpart;
    BDC_CUDA_TRY(dalloc(x, sizeof(double) * R));
    BDC_CUDA_TRY(dalloc(g, sizeof(double) * R));
    BDC_CUDA_TRY(dalloc(xa, sizeof(double) * R));
    BDC_CUDA_TRY(dalloc(ga, sizeof(double) * R));
    BDC_CUDA_TRY(dalloc(D, sizeof(double) * R));
    BDC_CUDA_TRY(dalloc(wts, R));
    BDC_CUDA_TRY(dalloc(in_s, R));
    BDC_CUDA_TRY(dalloc(cnt, sizeof(int)));
    BDC_CUDA_TRY(dalloc(mpart, sizeof(double) * nbR));
    const int cap = (int)std::min<int64_t>(R, 1 << 20);
    BDC_CUDA_TRY(dalloc(sel, sizeof(uint32_t) * cap));
    BDC_CUDA_TRY(cudaMemcpyAsync(x.p, cur, sizeof(double) * R, cudaMemcpyDeviceToDevice, s));
    k_orbit_weights<<<nbR, 256, 0, s>>>(R, H->d_reps, H->n, wts.get<uint8_t>());
    BDC_CUDA_TRY(cudaMemsetAsync(in_s.p, 0, R, s));
    BDC_CUDA_TRY(cudaGetLastError());

    auto full_map = [&](const double* pin, double* pout, double* u, double* r) -> bdc_status {
        bdc_status e = factored_map(H, pin, pout, nullptr);
        *u = H->h_st->max_d;
        *r = H->h_st->rate;
        return e;
    };
    // ---- phase 1
    if (phase1 == SOLVE_ANDERSON) {
        Anderson aa;
        BDC_CUDA_TRY(aa.init(R, 8, sms));
        rc = accelerated_ba(H, aa, wts.get<uint8_t>(), full_map, x.get<double>(), g.get<double>(), xa.get<double>(),
                            ga.get<double>(), R, switch_bits, max_evals, br, &evals);
        if (rc != BDC_OK) return rc;
    }
    if (H->verbose && phase1 == SOLVE_ANDERSON)
        printf("bdc: solve phase 1: %lld full evaluations, gap %.3e bits (%.3f s)\n", (long long)evals, br.gap_bits(),
               elapsed());

    // ---- phases 2 and 3
    std::vector<uint32_t> members;
    bool certified = br.gap_bits() < gap_bits;
    double cert_ub = br.ub, cert_rate = br.rate;
    for (int round = 0; round < 32 && !certified && evals < max_evals; ++round) {
        // full evaluation at x with D for every representative
        rc = factored_map(H, x.get<double>(), g.get<double>(), D.get<double>());
        if (rc != BDC_OK) return rc;
        ++evals;
        const double ub = H->h_st->max_d, rate = H->h_st->rate;
        br.add(ub, rate);
        cert_ub = ub;
        cert_rate = rate;
        if (H->verbose)
            printf("bdc: solve round %d: full evaluation with D, bracket %.3e bits (%.3f s)\n", round,
                   (ub - rate) / 0.69314718055994530942, elapsed());
        if ((ub - rate) / 0.69314718055994530942 < gap_bits) {
            certified = true;
            break;
        }
        // candidates: mass above 1e-12 of the largest (first round only), or
        // D(x) within max(10 gap, 1e-3 nats) of the bound (first round) / above
        // the rate (later rounds: the inputs that violate optimality of p_S)
        double pmax = 0.0;
        if (round == 0) {
            k_max_vec<<<nbR, 256, 0, s>>>(R, x.get<double>(), mpart.get<double>());
            std::vector<double> hp(nbR);
            BDC_CUDA_TRY(cudaMemcpyAsync(hp.data(), mpart.p, sizeof(double) * nbR, cudaMemcpyDeviceToHost, s));
            BDC_CUDA_TRY(cudaStreamSynchronize(s));
            for (double v : hp) pmax = std::max(pmax, v);
        }
        const double dmin = round == 0 ? ub - std::max(10.0 * (ub - rate), 1e-3) : rate + 1e-13 * std::fabs(rate);
        BDC_CUDA_TRY(cudaMemsetAsync(cnt.p, 0, sizeof(int), s));
        k_select<<<nbR, 256, 0, s>>>(R, round == 0 ? x.get<double>() : nullptr, D.get<double>(), 1e-12 * pmax, dmin,
                                     in_s.get<uint8_t>(), cnt.get<int>(), sel.get<uint32_t>(), cap);
        BDC_CUDA_TRY(cudaGetLastError());
        int nnew = 0;
        BDC_CUDA_TRY(cudaMemcpyAsync(&nnew, cnt.p, sizeof(int), cudaMemcpyDeviceToHost, s));
        BDC_CUDA_TRY(cudaStreamSynchronize(s));
        if (nnew == 0 && round > 0) {
            certified = true;  // p_S is optimal: no input outside S beats the rate
            break;
        }
        if (nnew > cap || (int64_t)members.size() + nnew > (1 << 18))
            return fail(BDC_ERR_UNSUPPORTED, "bdc_solve: support candidates exceed %d", 1 << 18);
        std::vector<uint32_t> add(nnew);
        BDC_CUDA_TRY(cudaMemcpyAsync(add.data(), sel.p, sizeof(uint32_t) * nnew, cudaMemcpyDeviceToHost, s));
        BDC_CUDA_TRY(cudaStreamSynchronize(s));
        members.insert(members.end(), add.begin(), add.end());
        std::sort(members.begin(), members.end());
        members.erase(std::unique(members.begin(), members.end()), members.end());
        {
            std::vector<uint8_t> flags(R, 0);
            for (uint32_t i : members) flags[i] = 1;
            BDC_CUDA_TRY(cudaMemcpyAsync(in_s.p, flags.data(), R, cudaMemcpyHostToDevice, s));
            BDC_CUDA_TRY(cudaStreamSynchronize(s));
        }
        // restricted problem, started from x on S (new members get a small
        // share of the largest entry so that they can grow)
        Restricted rs;
        rc = rs.build(H, members);
        if (rc != BDC_OK) return rc;
        if (H->verbose)
            printf("bdc: solve round %d: %zu members, rows built (%.3f s)\n", round, members.size(), elapsed());
        const int Sn = rs.S;
        DevBuf ps, pg, psa, pga;
        BDC_CUDA_TRY(dalloc(ps, sizeof(double) * Sn));
        BDC_CUDA_TRY(dalloc(pg, sizeof(double) * Sn));
        BDC_CUDA_TRY(dalloc(psa, sizeof(double) * Sn));
        BDC_CUDA_TRY(dalloc(pga, sizeof(double) * Sn));
        {
            std::vector<double> hx(Sn);
            k_gather_f64<<<(Sn + 255) / 256, 256, 0, s>>>(Sn, rs.idx.get<uint32_t>(), x.get<double>(), ps.get<double>());
            BDC_CUDA_TRY(cudaMemcpyAsync(hx.data(), ps.p, sizeof(double) * Sn, cudaMemcpyDeviceToHost, s));
            std::vector<uint8_t> hw(Sn);
            BDC_CUDA_TRY(cudaMemcpyAsync(hw.data(), rs.w.p, Sn, cudaMemcpyDeviceToHost, s));
            BDC_CUDA_TRY(cudaStreamSynchronize(s));
            double mx = 0.0;
            for (double v : hx) mx = std::max(mx, v);
            double z = 0.0;
            for (int i = 0; i < Sn; ++i) {
                if (!(hx[i] > 1e-6 * mx)) hx[i] = 1e-6 * mx;
                z += hw[i] * hx[i];
            }
            for (double& v : hx) v /= z;
            BDC_CUDA_TRY(cudaMemcpyAsync(ps.p, hx.data(), sizeof(double) * Sn, cudaMemcpyHostToDevice, s));
        }
        RsAA aa;
        BDC_CUDA_TRY(aa.init(Sn, kAAMax));
        DevBuf pbak;
        BDC_CUDA_TRY(dalloc(pbak, sizeof(double) * Sn));
        Bracket rb;
        int64_t revals = 0;
        // accelerated restricted BA to a moderate gap, then Newton on the
        // support to the precision of FP64.  Newton starts from a copy of the
        // BA iterate: when its systems break down or it stops short of the
        // target, the copy comes back (its steps set members to zero for
        // good, which BA could not undo) and BA alone runs to the target.
        const double target = std::min(gap_bits * 1e-2, 1e-11);
        rc = rs_accelerated(H, rs, aa, ps.get<double>(), pg.get<double>(), psa.get<double>(), pga.get<double>(),
                            std::max(target, kRestrictedSwitchBits), 400000, rb, &revals);
        if (rc != BDC_OK) return rc;
        if (H->verbose)
            printf("bdc: solve round %d: restricted BA, %lld evaluations, restricted gap %.3e bits (%.3f s)\n", round,
                   (long long)revals, rb.gap_bits(), elapsed());
        if (rb.gap_bits() >= target) {
            BDC_CUDA_TRY(cudaMemcpyAsync(pbak.p, ps.p, sizeof(double) * Sn, cudaMemcpyDeviceToDevice, s));
            Bracket nb;
            bool newton_ok = false;
            rc = newton_polish(H, rs, ps.get<double>(), pg.get<double>(),
                               std::max(1e-5, 100.0 * rb.gap_bits() * 0.69314718055994530942), nb, &newton_ok);
            if (rc != BDC_OK) return rc;
            const bool done = newton_ok && nb.gap_bits() < target;
            if (H->verbose)
                printf("bdc: solve round %d: Newton on the support %s, restricted gap %.3e bits (%.3f s)\n", round,
                       done ? "done" : "stopped short", nb.gap_bits(), elapsed());
            if (done) {
                rb.add(nb.ub, nb.rate);
            } else {
                BDC_CUDA_TRY(cudaMemcpyAsync(ps.p, pbak.p, sizeof(double) * Sn, cudaMemcpyDeviceToDevice, s));
                rc = rs_accelerated(H, rs, aa, ps.get<double>(), pg.get<double>(), psa.get<double>(),
                                    pga.get<double>(), target, 400000, rb, &revals);
                if (rc != BDC_OK) return rc;
            }
        }
        if (H->verbose)
            printf("bdc: solve round %d: |S| = %d, %lld restricted evaluations, restricted gap %.3e bits (%.3f s)\n",
                   round, Sn, (long long)revals, rb.gap_bits(), elapsed());
        // expand p_S into the full space
        BDC_CUDA_TRY(cudaMemsetAsync(x.p, 0, sizeof(double) * R, s));
        k_scatter_f64<<<(Sn + 255) / 256, 256, 0, s>>>(Sn, rs.idx.get<uint32_t>(), ps.get<double>(), x.get<double>());
        BDC_CUDA_TRY(cudaGetLastError());
    }
    // leave the handle at the final point; its zero entries stay zero under
    // later BA iterations
    BDC_CUDA_TRY(cudaMemcpyAsync(H->d_p[0], x.p, sizeof(double) * R, cudaMemcpyDeviceToDevice, s));
    rc = engine_after_set_p(H, 1);
    if (rc != BDC_OK) return rc;
    if (stats) {
        const double ln2 = 0.69314718055994530942;
        stats->iters = evals;
        stats->total_iters = evals;
        stats->mx = br.gap_bits();
        stats->upper_bound = cert_ub / ln2;
        stats->rate = cert_rate / ln2;
        stats->lse = NAN;
        stats->best_upper_bound = br.ub / ln2;
        stats->best_rate = br.rate / ln2;
        stats->converged = br.gap_bits() < gap_bits;
    }
    (void)certified;
    return BDC_OK;
}

}  // namespace bdc

extern "C" bdc_status bdc_solve(bdc_handle_t H, double gap_bits, int64_t max_evals, bdc_stats* stats) {
    return solve_impl(H, gap_bits, max_evals, stats, SOLVE_ANDERSON);
}

namespace bdc {
void solve_pool_release(bdc_handle* H) {
    delete (SolvePool*)H->solve_pool;
    H->solve_pool = nullptr;
}
}  // namespace bdc
