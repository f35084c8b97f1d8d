// bdc_count.cu -- the exact subsequence-count path and the two passes of one BA
// iteration that are built on it.
//
// Reference path (Pintz45/BDC-Upper-Bounds-GPU, backend/BAA.cu):
//   total_transitions   340-395  N(x,y) by the split identity
//   compute_den_kernel  429-485  q(y) = sum_x p(x) W(y|x)  (atomics per pair)
//   compute_log_W_gpu   487-530  ln p(x) + D(x)
//   compute_KL_kernel   533-571  D(x) = sum_y W ln(W/q)
//
// B200 design (differs from the reference on purpose):
//   * no per-x DP + unranking: every thread owns a fixed structured set of
//     2^{TB+BB} output words y (TB top bits x BB bottom bits, the middle bits
//     are the thread's index in its x-group) and evaluates the DENSE row
//     N(x, y) for its y's.  For split point j the distinct half-table entries
//     of those y's are loaded once and reused by all products (register
//     tiling of the Kronecker-sum structure N = sum_j A_j (x) B_{k-j});
//   * the q pass accumulates sum_x |O(x)| p(x) N(x,y) per raw y in registers
//     (no atomics) and folds orbits once at the end:
//         q(rep r) = sum_{y in O(r)} acc[y] / (|O(r)| C(n,k));
//   * the D pass uses the p-independent entropy term h(x) = sum_y W ln W,
//     computed once per handle, so that each pair costs one multiply-add:
//         D(x) = h(x) - (1/C) sum_y N(x,y) ln q(y).
#include <utility>

#include "bdc_common.cuh"
#include "bdc_engine.cuh"
#include "bdc_kernels.cuh"

namespace bdc {

// ------------------------------------------------------------ pair counts
__global__ void k_count_pairs(Split s, HalfTables A, HalfTables B, const uint32_t* __restrict__ xs,
                              const uint32_t* __restrict__ ys, int64_t npairs,
                              uint32_t* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < npairs;
         i += (int64_t)gridDim.x * blockDim.x)
        out[i] = split_count(s, A, B, xs[i], ys[i]);
}

// ------------------------------------------------------- dense count tiles
// Thread-owned y set: y(t, b) = (t << (K - TB)) | (g << BB) | b with
// t < 2^TB, b < 2^BB and g the thread's index inside its x-group of
// 2^{K-TB-BB} threads.
template <int K, int TB, int BB>
struct Tile {
    static constexpr int T = 1 << TB;
    static constexpr int NB = 1 << BB;
    static constexpr int YPT = T * NB;
    static constexpr int MID = K - TB - BB;
    static constexpr int GROUP = 1 << MID;  // threads per x
    static_assert(MID >= 0, "tile larger than the output alphabet");

    __device__ __forceinline__ static uint32_t y_of(uint32_t g, int t, int b) {
        return ((uint32_t)t << (K - TB)) | (g << BB) | (uint32_t)b;
    }
};

// N consecutive uint16 entries (N <= 8) from an address aligned to 2N bytes,
// in one load
template <int N, bool SH = false>
__device__ __forceinline__ void ld_u16(const uint16_t* __restrict__ p, uint32_t (&o)[N]) {
    if constexpr (SH) {
        // a row staged in shared memory
        if constexpr (N == 8) {
            const uint4 v = *(const uint4*)p;
            const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                o[2 * i] = w[i] & 0xFFFFu;
                o[2 * i + 1] = w[i] >> 16;
            }
        } else if constexpr (N == 4) {
            const uint2 v = *(const uint2*)p;
            o[0] = v.x & 0xFFFFu;
            o[1] = v.x >> 16;
            o[2] = v.y & 0xFFFFu;
            o[3] = v.y >> 16;
        } else if constexpr (N == 2) {
            const uint32_t v = *(const uint32_t*)p;
            o[0] = v & 0xFFFFu;
            o[1] = v >> 16;
        } else {
            o[0] = *p;
        }
    } else if constexpr (N == 8) {
        const uint4 v = __ldg((const uint4*)p);
        const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            o[2 * i] = w[i] & 0xFFFFu;
            o[2 * i + 1] = w[i] >> 16;
        }
    } else if constexpr (N == 4) {
        const uint2 v = __ldg((const uint2*)p);
        o[0] = v.x & 0xFFFFu;
        o[1] = v.x >> 16;
        o[2] = v.y & 0xFFFFu;
        o[3] = v.y >> 16;
    } else if constexpr (N == 2) {
        const uint32_t v = __ldg((const unsigned int*)p);
        o[0] = v & 0xFFFFu;
        o[1] = v >> 16;
    } else {
        o[0] = __ldg(p);
    }
}

// One split point J of the dense row: N[t][b] += A_J[xh][y >> M] * B_M[xl][y & (2^M-1)].
template <int K, int TB, int BB, int J, bool SH>
__device__ __forceinline__ void tile_term(const Split& s, const uint16_t* __restrict__ ar,
                                          const uint16_t* __restrict__ br, uint32_t xh, uint32_t xl,
                                          uint32_t g, uint32_t (&N)[1 << TB][1 << BB]) {
    constexpr int M = K - J;
    constexpr int T = 1 << TB, NB = 1 << BB;
    // distinct entries along t and b for the A (high) and B (low) halves
    constexpr int AT = (J >= TB) ? T : (1 << J);
    constexpr int AB = (M >= BB) ? 1 : (1 << (BB - M));
    constexpr int BT = (J >= TB) ? 1 : (1 << (TB - J));
    constexpr int BN = (M >= BB) ? NB : (1 << M);
    if (J < s.jlo || J > s.jhi) return;  // uniform across the grid
    // y = (t << (K-TB)) + (g << BB) + b with disjoint bit fields, so y >> M and
    // y & (2^M - 1) split into the same fields without carries: a per-thread
    // part (from g) and a compile-time part (from t, b) that becomes the
    // load's immediate offset.
    constexpr uint32_t mlo = (1u << M) - 1u;
    const uint32_t gA = (g << BB) >> M;
    const uint32_t gB = (g << BB) & mlo;
    // The identity halves (j = n1: A_j[xh][yh] = [xh == yh]; k-j = n2 likewise
    // for B) are uniform branches, so the table terms carry no compare/select.
    uint32_t av[AT][AB], bv[BT][BN];
    if (J == s.n1) {
#pragma unroll
        for (int ta = 0; ta < AT; ++ta)
#pragma unroll
            for (int ba = 0; ba < AB; ++ba) {
                const uint32_t t = (J >= TB) ? ta : (ta << (TB - J));
                const uint32_t b = (M >= BB) ? 0 : (ba << M);
                av[ta][ba] = (uint32_t)(xh == gA + ((t << (K - TB)) >> M) + (b >> M));
            }
    } else if constexpr (J >= TB) {
        // the A row is stored rotated (rotate_bundle): the T entries of one
        // thread, y_hi = (t << (J - TB)) | low, sit at (low << TB) | t, one
        // vector load for all t
#pragma unroll
        for (int ba = 0; ba < AB; ++ba) {
            const uint32_t low = gA + ((M >= BB) ? 0u : (uint32_t)ba);
            uint32_t v[T];
            ld_u16<T, SH>(ar + bundle_offset(J) + (low << TB), v);
#pragma unroll
            for (int ta = 0; ta < AT; ++ta) av[ta][ba] = v[ta];
        }
    } else {
        // J < TB: the 2^J entries y_hi = 0 .. 2^J - 1 are contiguous (gA = 0)
        uint32_t v[AT];
        ld_u16<AT, SH>(ar + bundle_offset(J), v);
#pragma unroll
        for (int ta = 0; ta < AT; ++ta)
#pragma unroll
            for (int ba = 0; ba < AB; ++ba) av[ta][ba] = v[ta];
    }
    if (M == s.n2) {
#pragma unroll
        for (int tb = 0; tb < BT; ++tb)
#pragma unroll
            for (int bb = 0; bb < BN; ++bb) {
                const uint32_t t = (J >= TB) ? 0 : tb;
                bv[tb][bb] = (uint32_t)(xl == gB + ((t << (K - TB)) & mlo) + ((uint32_t)bb & mlo));
            }
    } else {
        // the BN entries of one t are contiguous and aligned to BN: one vector load
        const uint16_t* __restrict__ pb = br + bundle_offset(M) + gB;
#pragma unroll
        for (int tb = 0; tb < BT; ++tb) {
            const uint32_t t = (J >= TB) ? 0 : tb;
            uint32_t v[BN];
            ld_u16<BN, SH>(pb + ((t << (K - TB)) & mlo), v);
#pragma unroll
            for (int bb = 0; bb < BN; ++bb) bv[tb][bb] = v[bb];
        }
    }
#pragma unroll
    for (int t = 0; t < T; ++t)
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            const int ai = (J >= TB) ? t : (t >> (TB - J));
            const int aj = (M >= BB) ? 0 : (b >> M);
            const int bi = (J >= TB) ? 0 : (t & (BT - 1));
            const int bj = (M >= BB) ? b : (b & (BN - 1));
            N[t][b] += av[ai][aj] * bv[bi][bj];
        }
}

template <int K, int TB, int BB, bool SH, int... Js>
__device__ __forceinline__ void tile_row_impl(const Split& s, const uint16_t* ar, const uint16_t* br,
                                              uint32_t xh, uint32_t xl, uint32_t g,
                                              uint32_t (&N)[1 << TB][1 << BB],
                                              std::integer_sequence<int, Js...>) {
    (tile_term<K, TB, BB, Js, SH>(s, ar, br, xh, xl, g, N), ...);
}

// the same from the two rows of x already staged in shared memory
template <int K, int TB, int BB>
__device__ __forceinline__ void tile_row_staged(const Split& s, const uint16_t* ar, const uint16_t* br, uint32_t x,
                                                uint32_t g, uint32_t (&N)[1 << TB][1 << BB]) {
#pragma unroll
    for (int t = 0; t < (1 << TB); ++t)
#pragma unroll
        for (int b = 0; b < (1 << BB); ++b) N[t][b] = 0u;
    const uint32_t xh = x >> s.n2, xl = x & low_mask(s.n2);
    tile_row_impl<K, TB, BB, true>(s, ar, br, xh, xl, g, N, std::make_integer_sequence<int, K + 1>{});
}

// Dense counts N(x, y(t,b)) for all of this thread's y.
template <int K, int TB, int BB>
__device__ __forceinline__ void tile_row(const Split& s, const HalfTables& A, const HalfTables& B,
                                         uint32_t x, uint32_t g, uint32_t (&N)[1 << TB][1 << BB]) {
#pragma unroll
    for (int t = 0; t < (1 << TB); ++t)
#pragma unroll
        for (int b = 0; b < (1 << BB); ++b) N[t][b] = 0u;
    const uint32_t xh = x >> s.n2, xl = x & low_mask(s.n2);
    const uint16_t* ar = A.rows + (size_t)xh * A.stride;
    const uint16_t* br = B.rows + (size_t)xl * B.stride;
    tile_row_impl<K, TB, BB, false>(s, ar, br, xh, xl, g, N, std::make_integer_sequence<int, K + 1>{});
}

// ------------------------------------------------ rows staged in shared memory
// For k >= 12 a whole CTA (256 threads) works on one x at a time, and every
// entry of the x's A row and B row is read by some thread.  One thread copies
// the next x's two rows into shared memory (cp.async.bulk, completion on an
// mbarrier) while the CTA computes the current x from the previous copy;
// the table reads then come from shared memory instead of waiting on L2.
constexpr uint32_t kStageSpin = 1u << 22;  // polls of a bounded mbarrier wait
constexpr int kErrCountStage = 5;          // DevState::error: a staging wait ran out

__device__ __forceinline__ uint32_t cnt_smem(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void cnt_mbar_init(uint32_t bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ bool cnt_mbar_wait(uint32_t bar, uint32_t parity) {
    for (uint32_t i = 0; i < kStageSpin; ++i) {
        uint32_t ok = 0;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

// the A row (rotated bundle) and the B row of x into buffer dst, bytes
// counted on bar; rows start 16-byte aligned and are multiples of 16 bytes
__device__ __forceinline__ void stage_rows(const Split& s, const HalfTables& A, const HalfTables& B, uint32_t x,
                                           uint16_t* dst, uint32_t bar) {
    const uint32_t xh = x >> s.n2, xl = x & low_mask(s.n2);
    const uint32_t ba = (uint32_t)A.stride * 2u, bb = (uint32_t)B.stride * 2u;
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(ba + bb) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     cnt_smem(dst)),
                 "l"(A.rows + (size_t)xh * A.stride), "r"(ba), "r"(bar)
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     cnt_smem(dst + A.stride)),
                 "l"(B.rows + (size_t)xl * B.stride), "r"(bb), "r"(bar)
                 : "memory");
}

__host__ __device__ constexpr bool staged_rows(int group) { return group == 256; }

// Residency of the two passes.  They wait on L1/L2 table loads, so
// occupancy pays: tiles of 16 words per thread are compiled for 4 CTAs of 256
// threads per SM (64 registers; 829 -> 918 iterations/s at 20/10, 10.7 ->
// 13.5 at 24/12 over 2 CTAs) and launched with 4 CTAs per SM; larger tiles
// keep their registers and 2 CTAs per SM in the grid.
template <int TB, int BB>
struct CountOcc {
    static constexpr bool small = (1 << (TB + BB)) <= 16;
    static constexpr int min_blocks = small ? 4 : 1;
    static constexpr int grid_per_sm = small ? 4 : 2;
};

// ------------------------------------------------------- compensated FP32
// Sums of FP32 products carried as an unevaluated pair (hi, lo) of floats.
// A double operand enters as its two-float split v = vh + vl (48 bits); a
// count N < 2^24 is exact as a float.  The product's rounding error comes
// from an FMA, the sum's from Knuth's two-sum, and both go into lo:
//     pr = vh N;  err = fma(vh, N, -pr);  tail = fma(vl, N, err)
//     s = hi + pr;  e = two-sum error;  hi = s;  lo += e + tail
// The _rn intrinsics keep the compiler from contracting the additions into
// FMAs, which would break the error terms.
struct F32Pair {
    float hi = 0.0f, lo = 0.0f;
    __device__ __forceinline__ void add_prod(float vh, float vl, float nf) {
        const float pr = __fmul_rn(vh, nf);
        const float err = fmaf(vh, nf, -pr);
        const float tail = fmaf(vl, nf, err);
        const float s = __fadd_rn(hi, pr);
        const float bv = __fsub_rn(s, hi);
        const float e = __fadd_rn(__fsub_rn(hi, __fsub_rn(s, bv)), __fsub_rn(pr, bv));
        hi = s;
        lo = __fadd_rn(lo, __fadd_rn(e, tail));
    }
    __device__ __forceinline__ double value() const { return (double)hi + (double)lo; }
};

__device__ __forceinline__ void split_f32(double v, float& vh, float& vl) {
    vh = __double2float_rn(v);
    vl = __double2float_rn(v - (double)vh);
}

// ------------------------------------------------------------- q pass
// acc[y] = sum over this CTA's x of |O(x)| p(x) N(x,y), written per CTA to
// part[blockIdx.x][y]; k_qfold reduces over CTAs.  C32: the per-thread sums
// run in compensated FP32 (F32Pair) and leave the thread as doubles.
template <int K, int TB, int BB, bool C32>
__global__ void __launch_bounds__(256, CountOcc<TB, BB>::min_blocks) k_qpass(Split s, HalfTables A, HalfTables B,
                                               const uint32_t* __restrict__ reps,
                                               const double* __restrict__ p_buf0,
                                               const double* __restrict__ p_buf1, int64_t R,
                                               double* __restrict__ part, const DevState* st,
                                               int use_state) {
    using TL = Tile<K, TB, BB>;
    if (use_state && st->done) return;
    const double* __restrict__ p = (use_state && st->cur) ? p_buf1 : p_buf0;
    const int groups_per_cta = blockDim.x / TL::GROUP;
    const int grp = threadIdx.x / TL::GROUP;
    const uint32_t g = threadIdx.x % TL::GROUP;
    const int64_t ngroups = (int64_t)gridDim.x * groups_per_cta;
    const int64_t gid = (int64_t)blockIdx.x * groups_per_cta + grp;
    const int64_t chunk = (R + ngroups - 1) / ngroups;
    const int64_t i0 = gid * chunk;
    const int64_t i1 = (i0 + chunk < R) ? i0 + chunk : R;

    double acc[TL::T][TL::NB];
#pragma unroll
    for (int t = 0; t < TL::T; ++t)
#pragma unroll
        for (int b = 0; b < TL::NB; ++b) acc[t][b] = 0.0;

    if constexpr (C32) {
        // runs of kRun x's in compensated FP32, each run's sums added to the
        // FP64 totals: the run length bounds the growth of the lo words'
        // own rounding (at most kRun^2 u^2 of the run's sum, u = 2^-24)
        constexpr int kRun = 32;
        for (int64_t r0 = i0; r0 < i1; r0 += kRun) {
            const int64_t r1 = (r0 + kRun < i1) ? r0 + kRun : i1;
            F32Pair acc32[TL::T][TL::NB];
            for (int64_t i = r0; i < r1; ++i) {
                const uint32_t x = __ldg(reps + i);
                const double w = (double)orbit_size(x, s.n) * __ldg(p + i);
                uint32_t N[TL::T][TL::NB];
                tile_row<K, TB, BB>(s, A, B, x, g, N);
                float wh, wl;
                split_f32(w, wh, wl);
#pragma unroll
                for (int t = 0; t < TL::T; ++t)
#pragma unroll
                    for (int b = 0; b < TL::NB; ++b) acc32[t][b].add_prod(wh, wl, (float)N[t][b]);
            }
#pragma unroll
            for (int t = 0; t < TL::T; ++t)
#pragma unroll
                for (int b = 0; b < TL::NB; ++b) acc[t][b] += acc32[t][b].value();
        }
    } else if constexpr (staged_rows(TL::GROUP)) {
        // the CTA is one x-group: rows staged through shared memory, after sh_acc
        extern __shared__ __align__(16) double sh_dyn[];
        uint16_t* rows = (uint16_t*)(sh_dyn + (1 << K));  // [2][A.stride + B.stride]
        __shared__ __align__(8) uint64_t rbar[2];
        const int rs = A.stride + B.stride;
        if (threadIdx.x == 0) {
            cnt_mbar_init(cnt_smem(&rbar[0]));
            cnt_mbar_init(cnt_smem(&rbar[1]));
        }
        __syncthreads();
        int bad = 0, failed = 0;  // this thread's wait ran out; some thread's did (uniform)
        const int64_t nx = i1 - i0;
        if (threadIdx.x == 0 && nx > 0) stage_rows(s, A, B, __ldg(reps + i0), rows, cnt_smem(&rbar[0]));
        int64_t ix = 0;
        for (; ix < nx; ++ix) {
            const int b = (int)(ix & 1);
            if (threadIdx.x == 0 && ix + 1 < nx)
                stage_rows(s, A, B, __ldg(reps + i0 + ix + 1), rows + (b ^ 1) * rs, cnt_smem(&rbar[b ^ 1]));
            if (!cnt_mbar_wait(cnt_smem(&rbar[b]), (uint32_t)(ix >> 1) & 1u)) bad = 1;
            const uint32_t x = __ldg(reps + i0 + ix);
            const double w = (double)orbit_size(x, s.n) * __ldg(p + i0 + ix);
            uint32_t N[TL::T][TL::NB];
            tile_row_staged<K, TB, BB>(s, rows + b * rs, rows + b * rs + A.stride, x, g, N);
#pragma unroll
            for (int t = 0; t < TL::T; ++t)
#pragma unroll
                for (int bb = 0; bb < TL::NB; ++bb) acc[t][bb] = fma(w, (double)N[t][bb], acc[t][bb]);
            failed = __syncthreads_or(bad);  // buffer b is free for x_{ix+2}
            if (failed) break;
        }
        if (failed) {
            // a copy that never completed: wait (bounded) for the one still in
            // flight, record the error, and leave NaN sums behind
            if (threadIdx.x == 0) {
                if (ix + 1 < nx) (void)cnt_mbar_wait(cnt_smem(&rbar[(ix + 1) & 1]), (uint32_t)((ix + 1) >> 1) & 1u);
                if (st) ((DevState*)st)->error = kErrCountStage;
            }
#pragma unroll
            for (int t = 0; t < TL::T; ++t)
#pragma unroll
                for (int bb = 0; bb < TL::NB; ++bb) acc[t][bb] = __longlong_as_double(0x7ff8000000000000ll);
        }
    } else {
        for (int64_t i = i0; i < i1; ++i) {
            const uint32_t x = __ldg(reps + i);
            const double w = (double)orbit_size(x, s.n) * __ldg(p + i);
            uint32_t N[TL::T][TL::NB];
            tile_row<K, TB, BB>(s, A, B, x, g, N);
#pragma unroll
            for (int t = 0; t < TL::T; ++t)
#pragma unroll
                for (int b = 0; b < TL::NB; ++b) acc[t][b] = fma(w, (double)N[t][b], acc[t][b]);
        }
    }

    // reduce the CTA's groups (same g => same y set) in shared memory
    extern __shared__ double sh_acc[];  // [1 << K]
    for (int y = threadIdx.x; y < (1 << K); y += blockDim.x) sh_acc[y] = 0.0;
    __syncthreads();
    for (int gg = 0; gg < groups_per_cta; ++gg) {
        if (grp == gg) {
#pragma unroll
            for (int t = 0; t < TL::T; ++t)
#pragma unroll
                for (int b = 0; b < TL::NB; ++b) sh_acc[TL::y_of(g, t, b)] += acc[t][b];
        }
        __syncthreads();
    }
    double* out = part + (size_t)blockIdx.x * (1 << K);
    for (int y = threadIdx.x; y < (1 << K); y += blockDim.x) out[y] = sh_acc[y];
}

// ------------------------------------------------------------- D / h pass
// MODE 0: D(x) = h(x) - (1/C) sum_y N(x,y) ln q(rep y)       -> out_d[i]
// MODE 1: h(x) = (1/C) sum_y N ln N - ln C                    -> out_d[i]
// C32 (MODE 0 only): each thread's share of sum_y N ln q runs in
// compensated FP32 (F32Pair); the group reduction and h - v/C stay FP64.
template <int K, int TB, int BB, int MODE, bool C32 = false>
__global__ void __launch_bounds__(256, CountOcc<TB, BB>::min_blocks) k_dpass(Split s, HalfTables A, HalfTables B,
                                               const uint32_t* __restrict__ reps, int64_t R,
                                               const double* __restrict__ lnq,
                                               const double* __restrict__ h,
                                               double inv_c, double log_c,
                                               double* __restrict__ out_d, uint32_t* __restrict__ out_nnz,
                                               const DevState* st, int use_state) {
    using TL = Tile<K, TB, BB>;
    if (use_state && st->done) return;
    const int groups_per_cta = blockDim.x / TL::GROUP;
    const int grp = threadIdx.x / TL::GROUP;
    const uint32_t g = threadIdx.x % TL::GROUP;
    const int64_t ngroups = (int64_t)gridDim.x * groups_per_cta;
    const int64_t gid = (int64_t)blockIdx.x * groups_per_cta + grp;
    const int64_t chunk = (R + ngroups - 1) / ngroups;
    const int64_t i0 = gid * chunk;
    const int64_t i1 = (i0 + chunk < R) ? i0 + chunk : R;
    const int lane = threadIdx.x & 31;

    static_assert(!C32 || MODE == 0, "compensated FP32 is for the D pass");
    double lq[TL::T][TL::NB];
    float lqh[C32 ? TL::T : 1][C32 ? TL::NB : 1], lql[C32 ? TL::T : 1][C32 ? TL::NB : 1];
    if (MODE == 0) {
#pragma unroll
        for (int t = 0; t < TL::T; ++t)
#pragma unroll
            for (int b = 0; b < TL::NB; ++b) {
                lq[t][b] = __ldg(lnq + orbit_rep(TL::y_of(g, t, b), K));
                if constexpr (C32) split_f32(lq[t][b], lqh[t][b], lql[t][b]);
            }
    }

    // per-warp partial sums of the group's x, folded every XC rows
    constexpr int XC = 32;
    constexpr int WPG = (TL::GROUP + 31) / 32;  // warps per group
    __shared__ double sh_part[XC][8];            // [x slot][warp of the CTA]
    __shared__ uint32_t sh_nz[XC][8];
    const int warp = threadIdx.x >> 5;
    // this thread's share of one x: sum_y N ln q (MODE 0) or sum N ln N and
    // the nonzero count (MODE 1)
    auto per_x = [&](const uint32_t (&N)[TL::T][TL::NB], double& v, uint32_t& nz) {
        if constexpr (C32) {
            F32Pair sv;
#pragma unroll
            for (int t = 0; t < TL::T; ++t)
#pragma unroll
                for (int b = 0; b < TL::NB; ++b) sv.add_prod(lqh[t][b], lql[t][b], (float)N[t][b]);
            v = sv.value();
        } else {
#pragma unroll
            for (int t = 0; t < TL::T; ++t)
#pragma unroll
                for (int b = 0; b < TL::NB; ++b) {
                    if (MODE == 0) {
                        v = fma((double)N[t][b], lq[t][b], v);
                    } else {
                        const uint32_t c = N[t][b];
                        if (c) {
                            v = fma((double)c, log((double)c), v);
                            ++nz;
                        }
                    }
                }
        }
    };
    auto finish_x = [&](int64_t i, double v, uint32_t nz) {
        out_d[i] = (MODE == 0) ? (__ldg(h + i) - v * inv_c) : (v * inv_c - log_c);
        if (MODE == 1) out_nnz[i] = nz;
    };
    if constexpr (staged_rows(TL::GROUP)) {
        // the CTA is one x-group: each x's two rows staged through shared memory
        extern __shared__ __align__(16) uint16_t rows[];  // [2][A.stride + B.stride]
        __shared__ __align__(8) uint64_t rbar[2];
        const int rs = A.stride + B.stride;
        if (threadIdx.x == 0) {
            cnt_mbar_init(cnt_smem(&rbar[0]));
            cnt_mbar_init(cnt_smem(&rbar[1]));
        }
        __syncthreads();
        int bad = 0, failed = 0;  // this thread's wait ran out; some thread's did (uniform)
        const int64_t nx = i1 - i0;
        if (threadIdx.x == 0 && nx > 0) stage_rows(s, A, B, __ldg(reps + i0), rows, cnt_smem(&rbar[0]));
        int64_t ix = 0;
        for (; ix < nx; ++ix) {
            const int b = (int)(ix & 1);
            if (threadIdx.x == 0 && ix + 1 < nx)
                stage_rows(s, A, B, __ldg(reps + i0 + ix + 1), rows + (b ^ 1) * rs, cnt_smem(&rbar[b ^ 1]));
            if (!cnt_mbar_wait(cnt_smem(&rbar[b]), (uint32_t)(ix >> 1) & 1u)) bad = 1;
            const uint32_t x = __ldg(reps + i0 + ix);
            uint32_t N[TL::T][TL::NB];
            tile_row_staged<K, TB, BB>(s, rows + b * rs, rows + b * rs + A.stride, x, g, N);
            double v = 0.0;
            uint32_t nz = 0;
            per_x(N, v, nz);
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                v += __shfl_xor_sync(0xFFFFFFFFu, v, off);
                if (MODE == 1) nz += __shfl_xor_sync(0xFFFFFFFFu, nz, off);
            }
            const int slot = (int)(ix % XC);
            if (lane == 0) {
                sh_part[slot][warp] = v;
                sh_nz[slot][warp] = nz;
            }
            failed = __syncthreads_or(bad);  // buffer b is free for x_{ix+2}; the slot is written
            if (slot == XC - 1 || ix == nx - 1) {
                if (threadIdx.x <= slot) {
                    const int xs = threadIdx.x;
                    double vv = 0.0;
                    uint32_t nn = 0;
                    for (int w = 0; w < WPG; ++w) {
                        vv += sh_part[xs][w];
                        nn += sh_nz[xs][w];
                    }
                    finish_x(i0 + ix - slot + xs, vv, nn);
                }
                __syncthreads();
            }
            if (failed) break;
        }
        if (failed && threadIdx.x == 0) {
            // a copy that never completed: wait (bounded) for the one still in
            // flight and record the error (the D values of this CTA are stale)
            if (ix + 1 < nx) (void)cnt_mbar_wait(cnt_smem(&rbar[(ix + 1) & 1]), (uint32_t)((ix + 1) >> 1) & 1u);
            if (st) ((DevState*)st)->error = kErrCountStage;
        }
    } else {
    // All groups of a CTA run the same number of rounds so that the
    // barriers below are uniform.
    for (int64_t r0 = 0; r0 < chunk; r0 += XC) {
        for (int xs = 0; xs < XC; ++xs) {
            const int64_t i = i0 + r0 + xs;
            double v = 0.0;
            uint32_t nz = 0;
            if (i < i1) {
                const uint32_t x = __ldg(reps + i);
                uint32_t N[TL::T][TL::NB];
                tile_row<K, TB, BB>(s, A, B, x, g, N);
                per_x(N, v, nz);
            }
            if (TL::GROUP <= 32) {
                // the group is a lane-aligned slice of one warp
#pragma unroll
                for (int off = TL::GROUP / 2; off > 0; off >>= 1) {
                    v += __shfl_xor_sync(0xFFFFFFFFu, v, off);
                    if (MODE == 1) nz += __shfl_xor_sync(0xFFFFFFFFu, nz, off);
                }
                if (g == 0 && i < i1) finish_x(i, v, nz);
            } else {
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) {
                    v += __shfl_xor_sync(0xFFFFFFFFu, v, off);
                    if (MODE == 1) nz += __shfl_xor_sync(0xFFFFFFFFu, nz, off);
                }
                if (lane == 0) {
                    sh_part[xs][warp] = v;
                    sh_nz[xs][warp] = nz;
                }
            }
        }
        if (TL::GROUP > 32) {
            __syncthreads();
            if (threadIdx.x < XC * groups_per_cta) {
                const int gg = threadIdx.x / XC, xs = threadIdx.x % XC;
                const int64_t gi0 = ((int64_t)blockIdx.x * groups_per_cta + gg) * chunk;
                const int64_t gi1 = (gi0 + chunk < R) ? gi0 + chunk : R;
                const int64_t i = gi0 + r0 + xs;
                if (i < gi1) {
                    double v = 0.0;
                    uint32_t nz = 0;
                    for (int w = 0; w < WPG; ++w) {
                        v += sh_part[xs][gg * WPG + w];
                        nz += sh_nz[xs][gg * WPG + w];
                    }
                    finish_x(i, v, nz);
                }
            }
            __syncthreads();
        }
    }
    }
}

// -------------------------------------------------------------- q fold
// lnq[r] = ln( sum_{y in O(r)} sum_c part[c][y] / (|O(r)| C) ) for
// representative slots r < 2^{k-1}; 0 for other slots and for q == 0.
// One warp per slot; fixed lane-strided order, so the result is deterministic.
__global__ void k_qfold(const double* __restrict__ part, int nparts, int k, double inv_c,
                        double* __restrict__ lnq, double* __restrict__ q_out, const DevState* st,
                        int use_state) {
    if (use_state && st->done) return;
    const int nq = (k >= 1) ? (1 << (k - 1)) : 1;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const int ny = 1 << k;
    for (int r = warp; r < nq; r += nwarps) {
        if (!is_rep((uint32_t)r, k)) {
            if (lane == 0) { lnq[r] = 0.0; if (q_out) q_out[r] = 0.0; }
            continue;
        }
        uint32_t mem[4];
        int nm = 0;
        const uint32_t rv = reverse_bits((uint32_t)r, k);
        const uint32_t cv = complement_bits((uint32_t)r, k);
        const uint32_t rcv = reverse_bits(cv, k);
        mem[nm++] = (uint32_t)r;
        if (rv != (uint32_t)r) mem[nm++] = rv;
        if (cv != (uint32_t)r && cv != rv) mem[nm++] = cv;
        if (rcv != (uint32_t)r && rcv != rv && rcv != cv) mem[nm++] = rcv;
        double acc = 0.0;
        for (int c = lane; c < nparts; c += 32) {
            const double* row = part + (size_t)c * ny;
            for (int e = 0; e < nm; ++e) acc += row[mem[e]];
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xFFFFFFFFu, acc, off);
        if (lane == 0) {
            const double q = acc * inv_c / (double)orbit_size((uint32_t)r, k);
            lnq[r] = (q != 0.0) ? log(q) : 0.0;
            if (q_out) q_out[r] = q;
        }
    }
}

// ------------------------------------------------------- rotated A bundle
// Copy of a high-half bundle in which each segment j >= tb stores entry y at
// ((y mod 2^{j-tb}) << tb) | (y >> (j - tb)): the top tb bits of y become the
// bottom ones, so the entries a dense tile reads together (its t values, the
// top bits of y) are adjacent.  Segments j < tb are copied as they are.
__global__ void k_rotate_bundle(const uint16_t* __restrict__ src, int64_t rows, int stride, int mmax, int tb,
                                uint16_t* __restrict__ dst) {
    const int64_t total = rows * stride;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t row = e / stride;
        const int i = (int)(e % stride);
        uint32_t dpos = (uint32_t)i;
        if (i >= 1) {
            const int j = 31 - __clz(i);  // segment: 2^j <= i < 2^{j+1}
            const uint32_t y = (uint32_t)i - (1u << j);
            if (j <= mmax && j >= tb) {
                const int lo = j - tb;
                dpos = (1u << j) + (((y & ((1u << lo) - 1u)) << tb) | (y >> lo));
            }
        }
        dst[row * stride + dpos] = src[e];
    }
}

cudaError_t launch_rotate_bundle(const HalfTables& A, int tb, uint16_t* dst, cudaStream_t stream) {
    const int64_t total = ((int64_t)A.stride) << A.h;
    int64_t blocks = (total + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_rotate_bundle<<<(int)blocks, 256, 0, stream>>>(A.rows, (int64_t)1 << A.h, A.stride, A.mmax, tb, dst);
    return cudaGetLastError();
}

// ------------------------------------------------------------ dispatch
// (TB, BB) per output length K: 16 words per thread for K >= 4.
// (TB, BB) per output length K: 16 words per thread for 4 <= K <= 12, and
// larger tiles above so that an x-group never exceeds 256 threads.
template <int K>
struct TileChoice {
    static constexpr int TB = (K >= 13) ? 3 : (K >= 4) ? 2 : (K >= 2 ? 1 : 0);
    static constexpr int BB = (K >= 14) ? 3 : (K >= 4) ? 2 : (K >= 2 ? 1 : 0);
};

template <int K>
static int cta_threads() {
    constexpr int G = Tile<K, TileChoice<K>::TB, TileChoice<K>::BB>::GROUP;
    return G >= 256 ? G : 256;
}

template <int K>
static cudaError_t launch_qpass_k(const CountLaunch& L, const double* p0, const double* p1,
                                  double* part, const DevState* st, int use_state) {
    constexpr int TB = TileChoice<K>::TB, BB = TileChoice<K>::BB;
    const int threads = cta_threads<K>();
    // the partial sums, then (staged rows, FP64 sums) two buffers of the A and B rows
    constexpr bool staged = staged_rows(Tile<K, TB, BB>::GROUP);
    const size_t rows_b = (staged && !L.c32) ? 2 * (size_t)(L.A.stride + L.B.stride) * sizeof(uint16_t) : 0;
    const size_t shm = (sizeof(double) << K) + rows_b;
    auto kern = L.c32 ? k_qpass<K, TB, BB, true> : k_qpass<K, TB, BB, false>;
    if (shm > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
        if (e != cudaSuccess) return e;
    }
    kern<<<L.grid, threads, shm, L.stream>>>(L.s, L.A, L.B, L.reps, p0, p1, L.R, part, st, use_state);
    return cudaGetLastError();
}

template <int K, int MODE>
static cudaError_t launch_dpass_k(const CountLaunch& L, const double* lnq, const double* h,
                                  double inv_c, double log_c, double* out, uint32_t* nnz,
                                  const DevState* st, int use_state) {
    constexpr int TB = TileChoice<K>::TB, BB = TileChoice<K>::BB;
    const int threads = cta_threads<K>();
    auto kern = (MODE == 0 && L.c32) ? k_dpass<K, TB, BB, MODE, MODE == 0> : k_dpass<K, TB, BB, MODE, false>;
    // staged rows: two buffers of the A and B rows
    constexpr bool staged = staged_rows(Tile<K, TB, BB>::GROUP);
    const size_t shm = staged ? 2 * (size_t)(L.A.stride + L.B.stride) * sizeof(uint16_t) : 0;
    if (shm > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
        if (e != cudaSuccess) return e;
    }
    kern<<<L.grid, threads, shm, L.stream>>>(L.s, L.A, L.B, L.reps, L.R, lnq, h, inv_c, log_c, out, nnz, st,
                                             use_state);
    return cudaGetLastError();
}

#define BDC_K_CASES(X) X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14)

int count_group_size(int k) {
    switch (k) {
#define C_(K) case K: return Tile<K, TileChoice<K>::TB, TileChoice<K>::BB>::GROUP;
        BDC_K_CASES(C_)
#undef C_
        default: return 0;
    }
}

int count_tile_tb(int k) {
    switch (k) {
#define C_(K) case K: return TileChoice<K>::TB;
        BDC_K_CASES(C_)
#undef C_
        default: return 0;
    }
}

int count_ctas_per_sm(int k) {
    switch (k) {
#define C_(K) case K: return CountOcc<TileChoice<K>::TB, TileChoice<K>::BB>::grid_per_sm;
        BDC_K_CASES(C_)
#undef C_
        default: return 1;
    }
}

int count_cta_threads(int k) {
    switch (k) {
#define C_(K) case K: return cta_threads<K>();
        BDC_K_CASES(C_)
#undef C_
        default: return 0;
    }
}

cudaError_t launch_qpass(const CountLaunch& L, const double* p0, const double* p1, double* part,
                         const DevState* st, int use_state) {
    switch (L.s.k) {
#define C_(K) case K: return launch_qpass_k<K>(L, p0, p1, part, st, use_state);
        BDC_K_CASES(C_)
#undef C_
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_dpass(const CountLaunch& L, const double* lnq, const double* h, double inv_c,
                         double log_c, double* out, const DevState* st, int use_state) {
    switch (L.s.k) {
#define C_(K) case K: return launch_dpass_k<K, 0>(L, lnq, h, inv_c, log_c, out, nullptr, st, use_state);
        BDC_K_CASES(C_)
#undef C_
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_hpass(const CountLaunch& L, double inv_c, double log_c, double* out, uint32_t* nnz) {
    switch (L.s.k) {
#define C_(K) case K: return launch_dpass_k<K, 1>(L, nullptr, nullptr, inv_c, log_c, out, nnz, nullptr, 0);
        BDC_K_CASES(C_)
#undef C_
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_qfold(const double* part, int nparts, int k, double inv_c, double* lnq,
                         double* q_out, const DevState* st, int use_state, cudaStream_t stream) {
    const int nq = (k >= 1) ? (1 << (k - 1)) : 1;
    const int warps = nq;
    const int threads = 256;
    int blocks = (warps * 32 + threads - 1) / threads;
    if (blocks > 4096) blocks = 4096;
    k_qfold<<<blocks, threads, 0, stream>>>(part, nparts, k, inv_c, lnq, q_out, st, use_state);
    return cudaGetLastError();
}

cudaError_t launch_count_pairs(const Split& s, const HalfTables& A, const HalfTables& B,
                               const uint32_t* xs, const uint32_t* ys, int64_t npairs,
                               uint32_t* out, cudaStream_t stream) {
    if (npairs <= 0) return cudaSuccess;
    int64_t blocks = (npairs + 255) / 256;
    if (blocks > 148 * 32) blocks = 148 * 32;
    k_count_pairs<<<(int)blocks, 256, 0, stream>>>(s, A, B, xs, ys, npairs, out);
    return cudaGetLastError();
}

}  // namespace bdc
