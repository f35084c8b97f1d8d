// bdc_factored.cu -- the factored engine: one BA iteration as FP64 matrix
// products over the half tables, with the BA update fused into the largest one.
//
// Reference path replaced (Pintz45/BDC-Upper-Bounds-GPU): the iteration of
// backend/BAA.cu:590-639 (q pass 429-485, D pass 487-530, normalisation
// 590-639, max deviation 916-946).  The reference evaluates N(x,y) pair by
// pair through the split identity (total_transitions, BAA.cu:340-395):
//     N(x, y) = sum_j A_j[x_hi][y_hi] * B_{k-j}[x_lo][y_lo],
// A_j = cache_{n1,j}, B_m = cache_{n2,m}.  For a fixed j this is a Kronecker
// product, so with the iterate laid out as a 2^{n1} x 2^{n2} matrix P:
//   q side:  Q_j = A_j^T P B_{k-j}                (the 2^j x 2^{k-j} block of q)
//   D side:  G   = sum_j A_j Lq_j B_{k-j}^T,  D(x) = h(x) - G(x) / C(n,k)
// with Lq_j = ln q reshaped to 2^j x 2^{k-j} and h(x) = sum_y W ln W (from
// the count path, once per handle).  Each term uses the cheaper association:
// "L" terms (2^j <= 2^{k-j}) contract x_hi first, "R" terms contract x_lo
// first.  Every representative is <= its complement, so its top bit is 0 and
// only the rows x_hi < H1/2 of the iterate and of G exist.  Per iteration:
//   1. U^T = (AL^T Pw)^T, V = Pw BR      (Pw = |O(x)| p(x) at representatives,
//                                          0 elsewhere; AL, BR: L / R tables)
//   2. Q_t = U_t B_m (L), A_j^T V_t (R) -> q parts; fold orbits -> ln q
//   3. M_t = Lq_t B_m^T (L), N_t = A_j Lq_t (R) -> operands of step 4
//   4. G = [AL | NR] [ML ; BR^T] with the BA update as epilogue: D, logW,
//      exp(logW - shift), the new iterate (in place) and block partials of
//      max D, sum |O| e, max logW, sum |O| p D
//   5. one-block finalize: ln Z, mx, upper bound, stop test, next shift.
// All products run on the FP64 tensor-core path (bdc_mma.cuh).  Counts are
// exact integers < 2^16 widened to FP64; all sums are FP64.  The tile shape
// and split of the large products are picked at set-up by timing candidates.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <map>
#include <string>
#include <type_traits>
#include <vector>

#include <cstring>

#include "bdc_engine.cuh"
#include "bdc_gemm.cuh"
#include "bdc_mma.cuh"
#include "bdc_ozaki.cuh"

namespace bdc {

constexpr int kErrShift = 1;  // DevState::error: exp shift out of range, re-scale

// how the fold reads Q_t: 0 = split slices in qparts, 1 = U^T rows (the
// identity B of an L term), 2 = V rows (the identity A of an R term); the
// identity terms of the D side are written by the fold as copies of ln q.
struct FoldTerm {
    int kind;
    int j, m, off;
    int64_t qoff;   // kind 0: first split slice of Q_t in qparts
    int qs;         // kind 0: number of split slices
    int idB_left;   // L term with identity B_m: RB rows [off, off+2^j) = Lq_t
    int idA_right;  // R term with identity A_j: LA columns [KL+off, +2^m) = Lq_t
};

struct Term {
    int j, m;       // split point and the low sub-length k - j
    int left;       // 1: L term (contract x_hi first), 0: R term
    int off;        // column offset inside AL (L) or BR (R)
    int idA, idB;   // A_j / B_m is the identity (j == n1 / m == n2)
};

// tile configurations of the FP64 tensor-core products (BM x BN, warps WM x WN)
enum MmaConfig { CFG_128x128 = 0, CFG_128x64, CFG_64x128, CFG_64x64, CFG_128x16, CFG_16x128, CFG_128x32, CFG_COUNT };
static const int kCfgBM[CFG_COUNT] = {128, 128, 64, 64, 128, 16, 128};
static const int kCfgBN[CFG_COUNT] = {128, 64, 128, 64, 16, 128, 32};

struct Launch {
    GemmDesc* d = nullptr;   // device descriptors
    int* map = nullptr;      // CTA -> descriptor index
    int n = 0, tiles = 0, cfg = CFG_64x64;
    int layout = -1;         // -1: register-staged mainloop; else the cp.async one (see k_mma_store)
    int grid = 0;            // G only: CTAs launched (0: one per tile; fewer: each loops over tiles)
};

// q side thin product of one term over a slice [s0, s1) of its contraction:
//   out[i][w] += sum_s small(s)[i] * wide(s)[w]   (i < SMALL, w < WIDE)
// with small(s) = small + s * small_stride, wide(s) = wide + s * wide_stride;
// out element (i, w) at out[i * WIDE + w] (L terms: i = yh, w = yl) or
// out[w * SMALL + i] (R terms: i = yl, w = yh), i.e. Q_t in flat y order.
struct ThinQ {
    const void* small;
    const void* wide;
    int64_t small_stride, wide_stride;
    int small_u16, wide_u16;
    int SMALL, WIDE;
    int s0, s1;
    double* out;
    int out_trans;
};

// D side thin product of one term, one output row per table row s:
//   out[s][i] = sum_w wide(s)[w] * Lq'[w][i]      (i < SMALL, w < WIDE)
// wide(s) = a half-table row (uint16); Lq'[w][i] = ln q at y = i * WIDE + w
// (L terms, i = yh) or y = w * SMALL + i (R terms, i = yl); out at
// out[s * out_s + i * out_i] (RB rows or LA columns).
struct ThinD {
    const uint16_t* wide;
    int64_t wide_stride;
    int SMALL, WIDE;
    int rows;
    int lq_trans;
    double* out;
    int64_t out_s, out_i;
    int cta_begin;
};

// D side, fused over all terms: one entry per CTA, rows [row0, row0 + the
// CTA's row count) of one term; IT outputs x RT rows per thread, LPR lanes
// splitting the contraction
struct ThinDF {
    const uint16_t* wide;
    int64_t wide_stride;
    int SMALL, WIDE, rows, row0;
    int lq_trans;
    double* out;
    int64_t out_s, out_i;
    int IT, LPR;
};

}  // namespace bdc

struct FactoredState {
    int H1 = 0, H2 = 0, KL = 0, KR = 0, Kp = 0, T = 0;
    int H1h = 0;              // rows held: x_hi in [row0, row0 + H1h) (all x_hi < H1 / 2 on one GPU)
    int row0 = 0;             // first row held (a shard of the rows over several GPUs; 0 on one GPU)
    int64_t i0 = 0, Rl = 0;   // the representatives in those rows: [i0, i0 + Rl) of the ascending list
    int64_t* d_rowstart = nullptr;  // [H1h + 1]: held row r's representatives are [i0 + rowstart[r], i0 + rowstart[r + 1])
    double* rpart = nullptr;        // [2 H1h]: per-row partials of the load
    int rows_smem = 0;              // dynamic shared memory of the row kernels
    std::vector<bdc::Term> terms;
    double* Pw = nullptr;     // [2^{n-1}]  |O(x)| e(x) at representatives, 0 elsewhere
    double* Lt = nullptr;     // [2^{n-1}]  ln e(x) (p = e / Z)
    double* hx = nullptr;     // [2^{n-1}]  h(x) at representatives
    uint16_t* Bp = nullptr;   // low-half tables, row c = table row rev(c) (dense column order)
    double* Ddense = nullptr; // [2^{n-1}] D(x) of a map with D output (allocated on first use)
    double* dout = nullptr;   // where the G epilogue writes D (nullptr: nowhere)
    double eta = 1.0;         // step of the update in the G epilogue (1: the BA map)
    std::vector<int> colmax;  // per dense column: largest x_hi of a representative, -1 if none
    double* LA = nullptr;     // [H1h][Kp]  = [AL | NR]
    double* RB = nullptr;     // [Kp][H2]  = [ML ; BR^T]
    double* UL = nullptr;     // [H2][KL]  (U^T)
    double* VR = nullptr;     // [H1h][KR]
    double* ulpart = nullptr; // [S1][H2][KL]
    double* vrpart = nullptr; // [S2][H1h][KR]
    int S1 = 1, S2 = 1;
    double* qparts = nullptr; // split slices of the small q products (FoldTerm::qoff)
    double* qsum = nullptr;   // [T][2^k]  qparts summed over the splits
    double* qacc = nullptr;   // [2^k]     sum over the terms
    // thin per-term products, grouped by the small size (index log2 SMALL)
    bdc::ThinQ* d_thinq[8] = {};
    int n_thinq[8] = {};
    bdc::ThinD* d_thind[8] = {};
    int n_thind[8] = {}, ctas_thind[8] = {};
    // the same products on the FP64 tensor-core path, used for the size
    // classes where the tuner found them faster
    bdc::Launch mq[8], md[8];
    bool use_mq[8] = {}, use_md[8] = {};
    // all per-term products of a side in one launch (used when faster)
    bdc::ThinQ* d_qf = nullptr;
    int n_qf = 0, qf_stage = 0;
    // the fused q side split: terms of fewer than 8 small outputs on k_qthin,
    // 8 to 64 on the FP64 tensor path (k_qthin_mma), where that times faster
    bdc::ThinQ *d_ql = nullptr, *d_qm = nullptr;
    int n_ql = 0, n_qm = 0, ql_stage = 0, qm_stage = 0;
    bool use_qm = false;
    bdc::ThinDF* d_df[4] = {};  // by log2 IT
    int n_df[4] = {};
    // the terms of 2 to 64 outputs on the FP64 tensor path (k_dthin_mma), in
    // place of a class of d_df where that times faster
    bdc::ThinDF* d_dm[4] = {};  // by the class of d_df
    int n_dm[4] = {}, dm_smem[4] = {};
    bool use_dm[4] = {};
    bool use_qf = false, use_df = false;
    double* lnq_full = nullptr;  // [2^k]
    double* epart = nullptr;  // [ctas][8]
    int ctas_g = 0;
    bdc::OzakiG* oz = nullptr;  // G on the int8 tensor cores (when set up and chosen)
    bool use_oz = false;
    bdc::Launch ul, vr, g;
    bdc::FoldTerm* d_fold = nullptr;
    int launches_per_iter = 0;
    // independent thin products run as parallel branches
    cudaStream_t side[8] = {};
    cudaEvent_t ev_fork = nullptr, ev_join[8] = {};
    // a captured chunk of kGraphIters iterations for the threshold graph_a
    cudaGraphExec_t graph = nullptr;
    double graph_a = 0.0;
    // accelerated loop: the normalised log iterates x_t and x_{t-1}, and the
    // graph of kAccSteps steps
    double* snap0 = nullptr;
    double* snap1 = nullptr;
    cudaGraphExec_t cycle = nullptr;
    double cycle_eta = 0.0;
    // captured single BA maps (factored_map), by their vectors
    struct MapGraph {
        const double* pin = nullptr;
        double* pout = nullptr;
        double* dout = nullptr;
        cudaGraphExec_t exec = nullptr;
    };
    MapGraph maps[4];
    int maps_next = 0;
};

namespace bdc {

__device__ __forceinline__ bool gated(const DevState* st) { return st && (st->done || st->error); }

enum Stage { ST_QBIG = 0, ST_QSMALL, ST_FOLD, ST_DSMALL, ST_G, ST_FIN, ST_COUNT };
static cudaError_t enqueue_stage(bdc_handle* H, int stage, double a);
static cudaError_t enqueue_qthin_split(bdc_handle* H, cudaStream_t s, const DevState* st);

// Dense layout of the iterate: row x_hi, column rev(x_lo) (the low half
// bit-reversed).  A representative x satisfies x <= rev(x) and x <=
// rev(comp(x)), so x_hi is at most a bound that rises and then falls along
// the columns; whole tiles of the dense matrices then hold no
// representative and are skipped.  The map is its own inverse.
__host__ __device__ __forceinline__ uint32_t fac_pos(uint32_t x, int n2) {
    const uint32_t m = low_mask(n2);
    return (x & ~m) | reverse_bits(x & m, n2);
}

// the index of representative x in a dense buffer that holds the rows
// x_hi >= row0 (a shard of the rows; row0 = 0 on one GPU)
__host__ __device__ __forceinline__ uint32_t fac_loc(uint32_t x, int n, int row0) {
    return fac_pos(x, n >> 1) - ((uint32_t)row0 << (n >> 1));
}

// the string at dense position xd of the held rows (fac_pos is an
// involution), and whether it is a representative: kernels that touch every
// representative walk the dense arrays in memory order this way, coalesced,
// instead of the ascending list (whose positions are bit-reversed in a row)
__device__ __forceinline__ uint32_t fac_str(uint32_t xd, int n, int row0) {
    return fac_pos(xd + ((uint32_t)row0 << (n >> 1)), n >> 1);
}


// ------------------------------------------------ products: plain store
// LAYOUT < 0: register-staged mainloop (any operand kind); otherwise the
// cp.async mainloop with A k-major when bit 0 is set and B k-major when bit 1
// is set (FP64 operands only)
template <int BM, int BN, int WM, int WN, int LAYOUT>
__global__ void __launch_bounds__(256) k_mma_store(const GemmDesc* __restrict__ descs, const int* __restrict__ map,
                                                   const DevState* st) {
    using C = MmaCfg<BM, BN, WM, WN>;
    if (gated(st)) return;
    extern __shared__ __align__(16) double smem[];
    const GemmDesc& d = descs[map[blockIdx.x]];
    const int t = blockIdx.x - d.tile_begin;
    const int m0 = (t / d.tiles_n) * BM, n0 = (t % d.tiles_n) * BN;
    double acc[C::MT][C::NT][2];
    if constexpr (LAYOUT < 0) mma_mainloop<BM, BN, WM, WN>(d, m0, n0, smem, acc);
    else mma_mainloop_cp<BM, BN, WM, WN, (LAYOUT & 1) != 0, (LAYOUT & 2) != 0, 3>(d, m0, n0, smem, acc);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, tq = lane & 3;
    const int wm0 = (warp / WN) * (8 * C::MT), wn0 = (warp % WN) * (8 * C::NT);
#pragma unroll
    for (int i = 0; i < C::MT; ++i) {
        const int m = m0 + wm0 + i * 8 + g;
        if (m >= d.M) continue;
#pragma unroll
        for (int j = 0; j < C::NT; ++j)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int n = n0 + wn0 + j * 8 + 2 * tq + h;
                if (n >= d.N) continue;
                double* c = d.C + (int64_t)m * d.ldc_m + (int64_t)n * d.ldc_n;
                const double v = d.alpha * acc[i][j][h];
                *c = d.accumulate ? *c + v : v;
            }
    }
}

// ------------------------------------------- the G product + BA update
// rows are x_hi, columns x_lo, x = (x_hi << n2) | x_lo; only representatives
// are updated; block partials [max D, sum |O| e, max (logW - shift),
// sum |O| p D, input-zero flag] go to ep.part[blockIdx.x * 8 + 0..4].
// CTA b takes the tiles b, b + gridDim.x, ... of the ntiles that hold
// representatives (one each when the grid covers them all); with the cp.async
// mainloop the next tile's first stages are in flight during this tile's
// epilogue.
template <int BM, int BN, int WM, int WN, bool WITH_D, bool CP>
__global__ void __launch_bounds__(256, (BM * BN <= 4096) ? 3 : 2) k_mma_ba(const GemmDesc* __restrict__ descs, const int* __restrict__ tiles,
                                                   int ntiles, BaEpilogue ep, const DevState* st) {
    using C = MmaCfg<BM, BN, WM, WN>;
    if (gated(st)) return;
    extern __shared__ __align__(16) double smem[];
    const GemmDesc& d = descs[0];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, tq = lane & 3;
    const int wm0 = (warp / WN) * (8 * C::MT), wn0 = (warp % WN) * (8 * C::NT);
    const double shift = st->shift;
    const double lnz = st->log_z;
    const double inv_z = exp(-lnz);
    double mD = -DBL_MAX, sE = 0.0, mL = -DBL_MAX, sR = 0.0, zero = 0.0;
    int ti = blockIdx.x;
    if constexpr (CP) {
        if (ti < ntiles) {
            const int t = tiles[ti];
            mma_cp_prologue<BM, BN, false, true, 3>(d, (t / d.tiles_n) * BM, (t % d.tiles_n) * BN, smem);
        }
    }
    for (; ti < ntiles; ti += gridDim.x) {
    const int t = tiles[ti];
    const int m0 = (t / d.tiles_n) * BM, n0 = (t % d.tiles_n) * BN;
    double acc[C::MT][C::NT][2];
    if constexpr (CP) {
        mma_cp_body<BM, BN, WM, WN, false, true, 3>(d, m0, n0, smem, acc);
        if (ti + (int)gridDim.x < ntiles) {
            const int tn = tiles[ti + gridDim.x];
            mma_cp_prologue<BM, BN, false, true, 3>(d, (tn / d.tiles_n) * BM, (tn % d.tiles_n) * BN, smem);
        }
    } else {
        mma_mainloop<BM, BN, WM, WN>(d, m0, n0, smem, acc);
    }
#pragma unroll
    for (int i = 0; i < C::MT; ++i) {
        const int m = m0 + wm0 + i * 8 + g;
        if (m >= d.M) continue;
#pragma unroll
        for (int j = 0; j < C::NT; ++j)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int n = n0 + wn0 + j * 8 + 2 * tq + h;
                if (n >= d.N) continue;
                const uint32_t xd = ((uint32_t)m << ep.n2) | (uint32_t)n;
                const uint32_t x = fac_pos(xd + ((uint32_t)ep.row0 << ep.n2), ep.n2);
                if (!is_rep(x, ep.n)) continue;
                const double o = (double)orbit_size(x, ep.n);
                const double D = __ldg(ep.hx + xd) - acc[i][j][h] * ep.inv_c;
                if (WITH_D) ep.Dout[xd] = D;
                // an entry that is exactly 0 in the caller's distribution (Lt
                // holds NaN) takes ln p = 0, as the reference's apply_log_kernel
                // leaves ln 0 at 0 (backend/BAA.cu:573-580); later iterates keep
                // exact logarithms
                const double pw = ep.Pw[xd];
                const double lt = ep.Lt[xd];
                const bool zero_in = (lt != lt);
                const double lnp = zero_in ? 0.0 : lt - lnz;
                const double lw = lnp + ep.eta * D - shift;
                const double e = exp(lw);
                ep.Lt[xd] = lw;
                ep.Pw[xd] = o * e;
                mD = fmax(mD, D);
                mL = fmax(mL, lw);
                sE = fma(o, e, sE);
                sR = fma(pw * inv_z, D, sR);
                if (zero_in) zero = 1.0;
            }
    }
    }
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
    if (threadIdx.x == 0) {
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

#define BDC_CFG_ARGS_128x128 128, 128, 2, 4
#define BDC_CFG_ARGS_128x64 128, 64, 4, 2
#define BDC_CFG_ARGS_64x128 64, 128, 2, 4
#define BDC_CFG_ARGS_64x64 64, 64, 2, 4
#define BDC_CFG_ARGS_128x16 128, 16, 8, 1
#define BDC_CFG_ARGS_16x128 16, 128, 1, 8
#define BDC_CFG_ARGS_128x32 128, 32, 4, 2

static int cfg_smem(int cfg, int layout = -1) {
#define CASE_(C, ARGS)                                                                          \
    case C:                                                                                     \
        switch (layout) {                                                                       \
            case 0: return mma_cp_smem_bytes<ARGS, false, false, 3>();                          \
            case 1: return mma_cp_smem_bytes<ARGS, true, false, 3>();                           \
            case 2: return mma_cp_smem_bytes<ARGS, false, true, 3>();                           \
            case 3: return mma_cp_smem_bytes<ARGS, true, true, 3>();                            \
            default: return mma_smem_bytes<ARGS>();                                             \
        }
    switch (cfg) {
        CASE_(CFG_128x128, BDC_CFG_ARGS_128x128)
        CASE_(CFG_128x64, BDC_CFG_ARGS_128x64)
        CASE_(CFG_64x128, BDC_CFG_ARGS_64x128)
        CASE_(CFG_64x64, BDC_CFG_ARGS_64x64)
        CASE_(CFG_128x16, BDC_CFG_ARGS_128x16)
        CASE_(CFG_16x128, BDC_CFG_ARGS_16x128)
        CASE_(CFG_128x32, BDC_CFG_ARGS_128x32)
    }
#undef CASE_
    return 0;
}

// the cp.async mainloop is instantiated for the layouts the products use:
// 3 (U: both k-major), 0 (V and the solver's A B^T: both contraction-major)
static bool cp_instantiated(int cfg, int layout) {
    const bool big = cfg == CFG_128x128 || cfg == CFG_128x64 || cfg == CFG_64x128 || cfg == CFG_64x64;
    return big && (layout == 0 || layout == 3);
}

static cudaError_t set_smem_attrs() {
    static bool done = false;
    if (done) return cudaSuccess;
#define SET_K(KERNEL, BYTES)                                                                     \
    {                                                                                            \
        cudaError_t e = cudaFuncSetAttribute(KERNEL, cudaFuncAttributeMaxDynamicSharedMemorySize, BYTES); \
        if (e != cudaSuccess) return e;                                                          \
    }
#define SET_STORE(ARGS)                                                                          \
    SET_K((k_mma_store<ARGS, -1>), (mma_smem_bytes<ARGS>()))
#define SET_STORE_CP(ARGS)                                                                       \
    SET_K((k_mma_store<ARGS, 0>), (mma_cp_smem_bytes<ARGS, false, false, 3>()))                 \
    SET_K((k_mma_store<ARGS, 3>), (mma_cp_smem_bytes<ARGS, true, true, 3>()))
#define SET_BA(ARGS)                                                                             \
    SET_K((k_mma_ba<ARGS, false, false>), (mma_smem_bytes<ARGS>()))                              \
    SET_K((k_mma_ba<ARGS, true, false>), (mma_smem_bytes<ARGS>()))                               \
    SET_K((k_mma_ba<ARGS, false, true>), (mma_cp_smem_bytes<ARGS, false, true, 3>()))            \
    SET_K((k_mma_ba<ARGS, true, true>), (mma_cp_smem_bytes<ARGS, false, true, 3>()))
    SET_STORE(BDC_CFG_ARGS_128x128)
    SET_STORE(BDC_CFG_ARGS_128x64)
    SET_STORE(BDC_CFG_ARGS_64x128)
    SET_STORE(BDC_CFG_ARGS_64x64)
    SET_STORE(BDC_CFG_ARGS_128x16)
    SET_STORE(BDC_CFG_ARGS_16x128)
    SET_STORE(BDC_CFG_ARGS_128x32)
    SET_STORE_CP(BDC_CFG_ARGS_128x128)
    SET_STORE_CP(BDC_CFG_ARGS_128x64)
    SET_STORE_CP(BDC_CFG_ARGS_64x128)
    SET_STORE_CP(BDC_CFG_ARGS_64x64)
    SET_BA(BDC_CFG_ARGS_128x128)
    SET_BA(BDC_CFG_ARGS_128x64)
    SET_BA(BDC_CFG_ARGS_64x128)
    SET_BA(BDC_CFG_ARGS_64x64)
#undef SET_BA
#undef SET_STORE_CP
#undef SET_STORE
#undef SET_K
    done = true;
    return cudaSuccess;
}

static cudaError_t launch_store(const Launch& L, cudaStream_t s, const DevState* st) {
    if (L.n == 0 || L.tiles == 0) return cudaSuccess;
    const int lay = cp_instantiated(L.cfg, L.layout) ? L.layout : -1;
    const int sm = cfg_smem(L.cfg, lay);
#define GO_(ARGS)                                                                                          \
    if (lay == 0) k_mma_store<ARGS, 0><<<L.tiles, 256, sm, s>>>(L.d, L.map, st);                           \
    else if (lay == 3) k_mma_store<ARGS, 3><<<L.tiles, 256, sm, s>>>(L.d, L.map, st);                      \
    else k_mma_store<ARGS, -1><<<L.tiles, 256, sm, s>>>(L.d, L.map, st);
    switch (L.cfg) {
        case CFG_128x128: GO_(BDC_CFG_ARGS_128x128) break;
        case CFG_128x64: GO_(BDC_CFG_ARGS_128x64) break;
        case CFG_64x128: GO_(BDC_CFG_ARGS_64x128) break;
        case CFG_64x64: GO_(BDC_CFG_ARGS_64x64) break;
        case CFG_128x16: k_mma_store<BDC_CFG_ARGS_128x16, -1><<<L.tiles, 256, sm, s>>>(L.d, L.map, st); break;
        case CFG_16x128: k_mma_store<BDC_CFG_ARGS_16x128, -1><<<L.tiles, 256, sm, s>>>(L.d, L.map, st); break;
        case CFG_128x32: k_mma_store<BDC_CFG_ARGS_128x32, -1><<<L.tiles, 256, sm, s>>>(L.d, L.map, st); break;
        default: return cudaErrorInvalidValue;
    }
#undef GO_
    return cudaGetLastError();
}

// G: A = [A_L | N_R] contiguous along the contraction, B = [M_L ; B_R^T]
// contiguous along the output columns: the cp.async mainloop with layout 2
static cudaError_t launch_ba(const Launch& L, const BaEpilogue& ep, cudaStream_t s, const DevState* st) {
    const bool wd = ep.Dout != nullptr, cp = L.layout == 2;
    const int sm = cfg_smem(L.cfg, cp ? 2 : -1);
    const int grid = (L.grid > 0 && L.grid < L.tiles) ? L.grid : L.tiles;
#define GO_(ARGS)                                                                                        \
    if (wd && cp) k_mma_ba<ARGS, true, true><<<grid, 256, sm, s>>>(L.d, L.map, L.tiles, ep, st);         \
    else if (wd) k_mma_ba<ARGS, true, false><<<grid, 256, sm, s>>>(L.d, L.map, L.tiles, ep, st);         \
    else if (cp) k_mma_ba<ARGS, false, true><<<grid, 256, sm, s>>>(L.d, L.map, L.tiles, ep, st);         \
    else k_mma_ba<ARGS, false, false><<<grid, 256, sm, s>>>(L.d, L.map, L.tiles, ep, st);
    switch (L.cfg) {
        case CFG_128x128: GO_(BDC_CFG_ARGS_128x128) break;
        case CFG_128x64: GO_(BDC_CFG_ARGS_128x64) break;
        case CFG_64x128: GO_(BDC_CFG_ARGS_64x128) break;
        case CFG_64x64: GO_(BDC_CFG_ARGS_64x64) break;
        default: return cudaErrorInvalidValue;
    }
#undef GO_
    return cudaGetLastError();
}

// ------------------------------------------------------ thin products
__device__ __forceinline__ double ld_val(const void* p, int u16, int64_t i) {
    return u16 ? (double)__ldg((const uint16_t*)p + i) : __ldg((const double*)p + i);
}

// q side: CTA = (descriptor, block of 256 wide indices); blockDim 256.  The
// small side of a chunk of 64 rows is staged in shared memory and broadcast;
// each thread streams its wide column (coalesced across the warp) with 8 row
// loads in flight.  When WIDE < 256 the spare threads take every
// (256 / WIDE)-th row and the partial sums are added in shared memory.
template <int SMALL>
__global__ void __launch_bounds__(256) k_thin_q(const ThinQ* __restrict__ descs, int nblk, const DevState* st) {
    if (gated(st)) return;
    const ThinQ& d = descs[blockIdx.x / nblk];
    const int wb = blockIdx.x % nblk;
    const int lanes_w = d.WIDE < 256 ? d.WIDE : 256;  // threads along w
    const int rows_par = 256 / lanes_w;               // threads along s
    const int tw = threadIdx.x % lanes_w, ts = threadIdx.x / lanes_w;
    const int w = wb * 256 + tw;
    const bool active = (w < d.WIDE) && (ts < rows_par);
    constexpr int CH = 64, U = 8;
    __shared__ double sm[CH][SMALL];
    double acc[SMALL];
#pragma unroll
    for (int i = 0; i < SMALL; ++i) acc[i] = 0.0;
    for (int c0 = d.s0; c0 < d.s1; c0 += CH) {
        const int nrow = min(CH, d.s1 - c0);
        __syncthreads();
        for (int e = threadIdx.x; e < CH * SMALL; e += 256) {
            const int r = e / SMALL, i = e % SMALL;
            sm[r][i] = (r < nrow) ? ld_val(d.small, d.small_u16, (int64_t)(c0 + r) * d.small_stride + i) : 0.0;
        }
        __syncthreads();
        if (active) {
            for (int r0 = ts; r0 < nrow; r0 += rows_par * U) {
                double wv[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int r = r0 + u * rows_par;
                    wv[u] = (r < nrow) ? ld_val(d.wide, d.wide_u16, (int64_t)(c0 + r) * d.wide_stride + w) : 0.0;
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int r = min(r0 + u * rows_par, CH - 1);  // rows past nrow carry weight 0
#pragma unroll
                    for (int i = 0; i < SMALL; ++i) acc[i] = fma(sm[r][i], wv[u], acc[i]);
                }
            }
        }
    }
    if (rows_par > 1) {
        // add the rows_par partial sums of each w (fixed order)
        __shared__ double red[256];
        for (int i = 0; i < SMALL; ++i) {
            __syncthreads();
            red[threadIdx.x] = active ? acc[i] : 0.0;
            __syncthreads();
            if (ts == 0 && w < d.WIDE) {
                double a = 0.0;
                for (int q = 0; q < rows_par; ++q) a += red[q * lanes_w + tw];
                acc[i] = a;
            }
        }
        if (ts != 0) return;
    }
    if (w >= d.WIDE) return;
#pragma unroll
    for (int i = 0; i < SMALL; ++i) {
        if (d.out_trans) d.out[(int64_t)w * SMALL + i] = acc[i];
        else d.out[(int64_t)i * d.WIDE + w] = acc[i];
    }
}

// D side: CTA = 16 table rows of one descriptor (64 threads, 4 lanes per
// row); ln q of the term is staged in shared memory as Lq'[w][i] and read
// with broadcasts while each lane walks a quarter of its row in 16-byte
// pieces, two in flight; the 4 partial sums of a row are added by shuffles.
constexpr int kThinDRows = 16;

template <int SMALL>
__global__ void __launch_bounds__(64) k_thin_d(const ThinD* __restrict__ descs, int nd,
                                               const double* __restrict__ lnq_full, const DevState* st) {
    if (gated(st)) return;
    int lo = 0, hi = nd - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (descs[mid].cta_begin <= (int)blockIdx.x) lo = mid;
        else hi = mid - 1;
    }
    const ThinD& d = descs[lo];
    const int q = threadIdx.x & 3;
    const int row = (blockIdx.x - d.cta_begin) * kThinDRows + (threadIdx.x >> 2);
    extern __shared__ double lqs[];  // [WIDE][SMALL]
    const int ny = SMALL * d.WIDE;
    for (int e = threadIdx.x; e < ny; e += 64) {
        const int w = e / SMALL, i = e % SMALL;
        lqs[e] = d.lq_trans ? lnq_full[w * SMALL + i] : lnq_full[i * d.WIDE + w];
    }
    __syncthreads();
    const bool live = row < d.rows;
    double acc[SMALL];
#pragma unroll
    for (int i = 0; i < SMALL; ++i) acc[i] = 0.0;
    const uint16_t* v = d.wide + (int64_t)(live ? row : 0) * d.wide_stride;
    if (live && (d.WIDE & 31) == 0 && ((uintptr_t)v & 15) == 0) {
        // lane q takes the 8-entry pieces q, q + 4, q + 8, ...
        for (int w0 = q * 8; w0 < d.WIDE; w0 += 64) {
            uint4 pc[2];
            pc[0] = __ldg(reinterpret_cast<const uint4*>(v + w0));
            pc[1] = (w0 + 32 < d.WIDE) ? __ldg(reinterpret_cast<const uint4*>(v + w0 + 32)) : make_uint4(0, 0, 0, 0);
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const uint32_t pk[4] = {pc[h].x, pc[h].y, pc[h].z, pc[h].w};
                const int wb = w0 + 32 * h;
                if (wb >= d.WIDE) break;
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const double wv = (double)((pk[u >> 1] >> (16 * (u & 1))) & 0xFFFFu);
                    const double* lr = lqs + (wb + u) * SMALL;
#pragma unroll
                    for (int i = 0; i < SMALL; ++i) acc[i] = fma(wv, lr[i], acc[i]);
                }
            }
        }
    } else if (live) {
        for (int w = q; w < d.WIDE; w += 4) {
            const double wv = (double)(__ldg(v + w));
            const double* lr = lqs + w * SMALL;
#pragma unroll
            for (int i = 0; i < SMALL; ++i) acc[i] = fma(wv, lr[i], acc[i]);
        }
    }
#pragma unroll
    for (int i = 0; i < SMALL; ++i) {
        acc[i] += __shfl_xor_sync(0xFFFFFFFFu, acc[i], 1);
        acc[i] += __shfl_xor_sync(0xFFFFFFFFu, acc[i], 2);
    }
    if (!live || q != 0) return;
    double* o = d.out + (int64_t)row * d.out_s;
#pragma unroll
    for (int i = 0; i < SMALL; ++i) o[(int64_t)i * d.out_i] = acc[i];
}

static cudaError_t launch_thin_q(int lg, const ThinQ* d, int n, int ny, cudaStream_t s, const DevState* st) {
    const int small = 1 << lg, wide = ny / small;
    const int nblk = (wide + 255) / 256;
    const int grid = n * nblk;
    switch (lg) {
        case 0: k_thin_q<1><<<grid, 256, 0, s>>>(d, nblk, st); break;
        case 1: k_thin_q<2><<<grid, 256, 0, s>>>(d, nblk, st); break;
        case 2: k_thin_q<4><<<grid, 256, 0, s>>>(d, nblk, st); break;
        case 3: k_thin_q<8><<<grid, 256, 0, s>>>(d, nblk, st); break;
        case 4: k_thin_q<16><<<grid, 256, 0, s>>>(d, nblk, st); break;
        case 5: k_thin_q<32><<<grid, 256, 0, s>>>(d, nblk, st); break;
        case 6: k_thin_q<64><<<grid, 256, 0, s>>>(d, nblk, st); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

static cudaError_t launch_thin_d(int lg, const ThinD* d, int n, int ctas, int ny, const double* lnq_full,
                                 cudaStream_t s, const DevState* st) {
    const size_t sm = sizeof(double) * ny;
    switch (lg) {
        case 0: k_thin_d<1><<<ctas, 64, sm, s>>>(d, n, lnq_full, st); break;
        case 1: k_thin_d<2><<<ctas, 64, sm, s>>>(d, n, lnq_full, st); break;
        case 2: k_thin_d<4><<<ctas, 64, sm, s>>>(d, n, lnq_full, st); break;
        case 3: k_thin_d<8><<<ctas, 64, sm, s>>>(d, n, lnq_full, st); break;
        case 4: k_thin_d<16><<<ctas, 64, sm, s>>>(d, n, lnq_full, st); break;
        case 5: k_thin_d<32><<<ctas, 64, sm, s>>>(d, n, lnq_full, st); break;
        case 6: k_thin_d<64><<<ctas, 64, sm, s>>>(d, n, lnq_full, st); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

// q side, every term and slice in one launch: CTA = one ThinQ entry (a term
// and a slice [s0, s1) of its contraction), 2^k / 16 threads, each owning IT
// (1 or 2) small indices x 16 / IT consecutive wide indices, the latter read
// as 16-byte pieces of the table row; 16 FP64 FMAs per row and thread.
__device__ __forceinline__ void unpack2(const uint32_t p, double* v) {
    v[0] = (double)(p & 0xFFFFu);
    v[1] = (double)(p >> 16);
}

__device__ __forceinline__ void unpack8(const uint4 p, double* v) {
    unpack2(p.x, v);
    unpack2(p.y, v + 2);
    unpack2(p.z, v + 4);
    unpack2(p.w, v + 6);
}

// The slice's rows stream through shared memory with cp.async, kQtRows rows a
// stage and kQtStages stages in flight (the table rows are 16-byte pieces,
// the small rows 8-byte ones since their stride is odd), so that the CTA keeps
// tens of kilobytes of loads outstanding without holding them in registers.
constexpr int kQtRows = 8;
constexpr int kQtStages = 3;

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem));
}

// small indices a thread covers: up to 8, so that each table entry it
// converts feeds up to 8 FMAs; the thread's 16 outputs are IT small x 16 / IT
// wide indices
__host__ __device__ constexpr int qthin_it(int SMALL) { return SMALL < 8 ? SMALL : 8; }

// the WT = 16 / IT table entries of a thread in one staged row
template <int WT>
__device__ __forceinline__ void qthin_entries(const uint8_t* p, double (&v)[WT]) {
    if constexpr (WT == 16) {
        const uint4* q = reinterpret_cast<const uint4*>(p);
        unpack8(q[0], v);
        unpack8(q[1], v + 8);
    } else if constexpr (WT == 8) {
        unpack8(*reinterpret_cast<const uint4*>(p), v);
    } else if constexpr (WT == 4) {
        const uint2 q = *reinterpret_cast<const uint2*>(p);
        unpack2(q.x, v);
        unpack2(q.y, v + 2);
    } else {
        unpack2(*reinterpret_cast<const uint32_t*>(p), v);
    }
}

template <int IT>
__device__ __forceinline__ void qthin_run(const ThinQ& q, int stage_bytes, uint8_t* qsm) {
    constexpr int WT = 16 / IT;
    const int nwb = q.WIDE / WT;
    const int tid = threadIdx.x;
    const int wb = tid % nwb, ib = tid / nwb;
    const int i0 = ib * IT, w0 = wb * WT;
    const uint16_t* wide = (const uint16_t*)q.wide;
    const double* small = (const double*)q.small;
    const int wpieces = q.WIDE / 8;              // 16-byte pieces per table row
    const int wbytes = q.WIDE * 2, sbytes = q.SMALL * 8;
    const int rows = q.s1 - q.s0;
    const int nst = (rows + kQtRows - 1) / kQtRows;
    auto issue = [&](int stg) {
        uint8_t* base = qsm + (stg % kQtStages) * stage_bytes;
        const int r0 = q.s0 + stg * kQtRows;
        const int nr = min(kQtRows, q.s1 - r0);
        for (int e = tid; e < nr * wpieces; e += blockDim.x) {
            const int r = e / wpieces, c = e % wpieces;
            cp_async16(base + r * wbytes + c * 16, wide + (int64_t)(r0 + r) * q.wide_stride + c * 8, 16);
        }
        uint8_t* sb = base + kQtRows * wbytes;
        for (int e = tid; e < nr * q.SMALL; e += blockDim.x) {
            const int r = e / q.SMALL, c = e % q.SMALL;
            cp_async8(sb + r * sbytes + c * 8, small + (int64_t)(r0 + r) * q.small_stride + c);
        }
    };
    double acc[16];
#pragma unroll
    for (int e = 0; e < 16; ++e) acc[e] = 0.0;
#pragma unroll
    for (int p = 0; p < kQtStages - 1; ++p) {
        if (p < nst) issue(p);
        cp_async_commit();
    }
    for (int stg = 0; stg < nst; ++stg) {
        cp_async_wait<kQtStages - 2>();
        __syncthreads();
        if (stg + kQtStages - 1 < nst) issue(stg + kQtStages - 1);
        cp_async_commit();
        const uint8_t* base = qsm + (stg % kQtStages) * stage_bytes;
        const double* sb = reinterpret_cast<const double*>(base + kQtRows * wbytes);
        const int nr = min(kQtRows, q.s1 - (q.s0 + stg * kQtRows));
        if (i0 < q.SMALL) {
            for (int r = 0; r < nr; ++r) {
                double v[WT], av[IT];
                qthin_entries<WT>(base + r * wbytes + w0 * 2, v);
                // the IT small values in 16-byte pieces (i0 is a multiple of IT)
                if constexpr (IT >= 2) {
#pragma unroll
                    for (int t = 0; t < IT; t += 2) {
                        const double2 a2 = *reinterpret_cast<const double2*>(sb + r * q.SMALL + i0 + t);
                        av[t] = a2.x;
                        av[t + 1] = a2.y;
                    }
                } else {
                    av[0] = sb[r * q.SMALL + i0];
                }
#pragma unroll
                for (int t = 0; t < IT; ++t)
#pragma unroll
                    for (int e = 0; e < WT; ++e) acc[t * WT + e] = fma(av[t], v[e], acc[t * WT + e]);
            }
        }
    }
    cp_async_wait<0>();
    if (i0 >= q.SMALL) return;
#pragma unroll
    for (int e = 0; e < 16; ++e) {
        const int i = i0 + e / WT, w = w0 + e % WT;
        if (q.out_trans) q.out[(int64_t)w * q.SMALL + i] = acc[e];
        else q.out[(int64_t)i * q.WIDE + w] = acc[e];
    }
}

__global__ void __launch_bounds__(256) k_qthin(const ThinQ* __restrict__ descs, int stage_bytes, const DevState* st) {
    if (gated(st)) return;
    extern __shared__ __align__(16) uint8_t qsm[];
    const ThinQ& q = descs[blockIdx.x];
    switch (qthin_it(q.SMALL)) {
        case 1: qthin_run<1>(q, stage_bytes, qsm); break;
        case 2: qthin_run<2>(q, stage_bytes, qsm); break;
        case 4: qthin_run<4>(q, stage_bytes, qsm); break;
        default: qthin_run<8>(q, stage_bytes, qsm); break;
    }
}

// D side, every term in one launch: CTA = one ThinDF entry.  Lq' of the term
// is staged in shared memory in chunks of 8 contraction indices padded by
// one double (so that lanes 8 indices apart fall on different banks); each
// thread accumulates RT rows x IT outputs over its lane's share of the
// contraction, reading 8 table entries per row at a time, and the LPR lanes
// of a row group add their partial sums by shuffles.
constexpr int kDfRT = 4;

template <int IT>
__global__ void __launch_bounds__(256) k_dthin(const ThinDF* __restrict__ descs, const double* __restrict__ lnq_full,
                                               const DevState* st) {
    if (gated(st)) return;
    extern __shared__ double lq[];
    const ThinDF& t = descs[blockIdx.x];
    const int SMALL = t.SMALL, WIDE = t.WIDE;
    const int cs = 8 * SMALL + 1;  // padded chunk of 8 contraction indices
    // eight loads per thread in flight, then their stores
    for (int e0 = threadIdx.x; e0 < SMALL * WIDE; e0 += 8 * blockDim.x) {
        double v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int e = e0 + u * (int)blockDim.x, w = e / SMALL, i = e % SMALL;
            v[u] = (e < SMALL * WIDE) ? (t.lq_trans ? __ldg(lnq_full + w * SMALL + i) : __ldg(lnq_full + i * WIDE + w))
                                      : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int e = e0 + u * (int)blockDim.x, w = e / SMALL, i = e % SMALL;
            if (e < SMALL * WIDE) lq[(w >> 3) * cs + (w & 7) * SMALL + i] = v[u];
        }
    }
    __syncthreads();
    const int LPR = t.LPR;
    const int lane = threadIdx.x % LPR, rest = threadIdx.x / LPR;
    const int ng = SMALL / IT;
    const int ig = rest % ng, rg = rest / ng;
    const int r0 = t.row0 + rg * kDfRT;
    const int i0 = ig * IT;
    double acc[kDfRT][IT];
#pragma unroll
    for (int r = 0; r < kDfRT; ++r)
#pragma unroll
        for (int i = 0; i < IT; ++i) acc[r][i] = 0.0;
    const uint16_t* rowp[kDfRT];
#pragma unroll
    for (int r = 0; r < kDfRT; ++r) rowp[r] = t.wide + (int64_t)min(r0 + r, t.rows - 1) * t.wide_stride;
    // two chunks of 8 contraction indices per step: both chunks' table loads
    // are issued before either is used
    const int step = LPR * 8;
    for (int w8 = lane * 8; w8 < WIDE; w8 += 2 * step) {
        const bool two = w8 + step < WIDE;
        uint32_t pk[2][kDfRT][4];
#pragma unroll
        for (int c = 0; c < 2; ++c)
#pragma unroll
            for (int r = 0; r < kDfRT; ++r) {
                const uint4 q = (c == 0 || two) ? __ldg(reinterpret_cast<const uint4*>(rowp[r] + w8 + c * step))
                                                : make_uint4(0u, 0u, 0u, 0u);
                pk[c][r][0] = q.x;
                pk[c][r][1] = q.y;
                pk[c][r][2] = q.z;
                pk[c][r][3] = q.w;
            }
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            if (c == 1 && !two) break;
            const double* lc = lq + ((w8 + c * step) >> 3) * cs + i0;
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                double v[kDfRT];
#pragma unroll
                for (int r = 0; r < kDfRT; ++r) v[r] = (double)((pk[c][r][u >> 1] >> (16 * (u & 1))) & 0xFFFFu);
#pragma unroll
                for (int i = 0; i < IT; ++i) {
                    const double l = lc[u * SMALL + i];
#pragma unroll
                    for (int r = 0; r < kDfRT; ++r) acc[r][i] = fma(v[r], l, acc[r][i]);
                }
            }
        }
    }
    for (int o = LPR >> 1; o > 0; o >>= 1)
#pragma unroll
        for (int r = 0; r < kDfRT; ++r)
#pragma unroll
            for (int i = 0; i < IT; ++i) acc[r][i] += __shfl_xor_sync(0xFFFFFFFFu, acc[r][i], o);
    if (lane != 0) return;
#pragma unroll
    for (int r = 0; r < kDfRT; ++r) {
        if (r0 + r >= t.rows) break;
#pragma unroll
        for (int i = 0; i < IT; ++i) t.out[(int64_t)(r0 + r) * t.out_s + (int64_t)(i0 + i) * t.out_i] = acc[r][i];
    }
}

// D side on the FP64 tensor path, for the terms of 2 to 64 outputs: CTA =
// one ThinDF entry of kDmRows table rows, warp w = rows 8w .. 8w + 7, all
// SMALL outputs as SMALL / 8 mma.sync m8n8k4 tiles (one tile, zero-padded,
// below 8).  Lq' of the term sits in
// shared memory at row pitch SMALL + 2 (the four row groups of a B fragment
// land 8 doubles apart: two wavefronts, the minimum for 256 bytes); the
// table rows stream through two buffers of kDmChunk entries with cp.async
// (row pitch kDmPitch entries: 16-byte aligned, rows 4 banks apart).  Within
// each 16 contraction indices, k-step j of lane column q takes index 4q + j,
// so that a lane's four A entries are one 8-byte load (A and B use the same
// order, and the sum does not depend on it).
constexpr int kDmRows = 64;
constexpr int kDmChunk = 64;
constexpr int kDmPitch = 72;

// Lq' row pitch; terms of 2 or 4 outputs use one 8-wide tile, zero-padded
__host__ __device__ constexpr int dmma_ld(int SMALL) { return (SMALL < 8 ? 8 : SMALL) + 2; }
static int dthin_mma_smem(int SMALL, int WIDE) {
    return (int)sizeof(double) * WIDE * dmma_ld(SMALL) + 2 * kDmRows * kDmPitch * (int)sizeof(uint16_t);
}

template <int NB>
__device__ __forceinline__ void dthin_mma_run(const ThinDF& t, const double* __restrict__ lnq_full, double* dsm) {
    const int SMALL = t.SMALL, WIDE = t.WIDE, ld = dmma_ld(SMALL);
    double* L = dsm;                                         // [WIDE][ld]
    uint16_t* T = reinterpret_cast<uint16_t*>(dsm + WIDE * ld);  // [2][kDmRows][kDmPitch]
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int gr = lane >> 2, q = lane & 3;
    auto issue = [&](int c) {
        uint16_t* buf = T + (c & 1) * kDmRows * kDmPitch;
        for (int e = tid; e < kDmRows * (kDmChunk / 8); e += 256) {
            const int r = e / (kDmChunk / 8), piece = e % (kDmChunk / 8);
            const int row = min(t.row0 + r, t.rows - 1);
            cp_async16(buf + r * kDmPitch + piece * 8, t.wide + (int64_t)row * t.wide_stride + c * kDmChunk + piece * 8,
                       16);
        }
    };
    const int nch = WIDE / kDmChunk;
    // Lq' by 8-byte asynchronous copies in the first chunk's group (all of a
    // thread's copies in flight at once), zeros past SMALL by plain stores
    const int SP = NB * 8;  // outputs of the tiles: SMALL, or 8 with zeros past SMALL
    for (int e = tid; e < SP * WIDE; e += 256) {
        const int w = e / SP, i = e % SP;
        if (i >= SMALL) L[w * ld + i] = 0.0;
        else cp_async8(L + w * ld + i, t.lq_trans ? lnq_full + w * SMALL + i : lnq_full + i * WIDE + w);
    }
    issue(0);
    cp_async_commit();
    double acc[NB][2];
#pragma unroll
    for (int nb = 0; nb < NB; ++nb) acc[nb][0] = acc[nb][1] = 0.0;
    for (int c = 0; c < nch; ++c) {
        if (c + 1 < nch) issue(c + 1);
        cp_async_commit();
        cp_async_wait<1>();
        __syncthreads();
        const uint16_t* arow = T + (c & 1) * kDmRows * kDmPitch + (warp * 8 + gr) * kDmPitch;
#pragma unroll
        for (int ks = 0; ks < kDmChunk / 16; ++ks) {
            const uint2 pk = *reinterpret_cast<const uint2*>(arow + ks * 16 + 4 * q);
            const double av[4] = {(double)(pk.x & 0xFFFFu), (double)(pk.x >> 16), (double)(pk.y & 0xFFFFu),
                                  (double)(pk.y >> 16)};
            const double* lrow = L + (c * kDmChunk + ks * 16 + 4 * q) * ld + gr;
#pragma unroll
            for (int j = 0; j < 4; ++j)
#pragma unroll
                for (int nb = 0; nb < NB; ++nb) mma_f64(acc[nb][0], acc[nb][1], av[j], lrow[j * ld + nb * 8]);
        }
        __syncthreads();  // the buffer is free for chunk c + 2
    }
    const int row = t.row0 + warp * 8 + gr;
    if (row >= t.rows) return;
#pragma unroll
    for (int nb = 0; nb < NB; ++nb)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int i = nb * 8 + 2 * q + h;
            if (i < SMALL) t.out[(int64_t)row * t.out_s + (int64_t)i * t.out_i] = acc[nb][h];
        }
}

__global__ void __launch_bounds__(256) k_dthin_mma(const ThinDF* __restrict__ descs, const double* __restrict__ lnq_full,
                                                   const DevState* st) {
    if (gated(st)) return;
    extern __shared__ __align__(16) double dmsm[];
    const ThinDF& t = descs[blockIdx.x];
    switch (t.SMALL) {
        case 2:
        case 4:
        case 8: dthin_mma_run<1>(t, lnq_full, dmsm); break;
        case 16: dthin_mma_run<2>(t, lnq_full, dmsm); break;
        case 32: dthin_mma_run<4>(t, lnq_full, dmsm); break;
        default: dthin_mma_run<8>(t, lnq_full, dmsm); break;
    }
}

// q side on the FP64 tensor path, for the terms of 8 to 64 small outputs
// at 2^k = 4096 outputs per term: CTA = one ThinQ slice [s0, s1) of the
// contraction, producing the term's SMALL x WIDE partial product.  Warp w
// owns small tile ti (8 outputs i) and 64 wide outputs from c0 as eight
// mma.sync m8n8k4 tiles; tile u's column n stands for w = c0 + 8n + u, so a
// lane's B entries of one row (n = lane / 4, all u) are 8 adjacent table
// entries, one 16-byte load.  Rows stream through two buffers of kQmRows
// (table rows at pitch WIDE, small rows at pitch SMALL + 8: two wavefronts
// for the four rows of an A fragment); rows past s1 read zero small values.
constexpr int kQmRows = 32;

__host__ __device__ constexpr int qmma_ld(int SMALL) { return SMALL >= 16 ? SMALL + 8 : SMALL; }
__host__ __device__ constexpr int qmma_stage(int SMALL, int WIDE) {
    return kQmRows * (qmma_ld(SMALL) * 8 + WIDE * 2);
}

__global__ void __launch_bounds__(256) k_qthin_mma(const ThinQ* __restrict__ descs, int stage_bytes,
                                                   const DevState* st) {
    if (gated(st)) return;
    extern __shared__ __align__(16) uint8_t qmsm[];
    const ThinQ& q = descs[blockIdx.x];
    const int SMALL = q.SMALL, WIDE = q.WIDE, lds = qmma_ld(SMALL);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int gr = lane >> 2, qq = lane & 3;
    const int groups = WIDE / 64;  // 64-column groups
    const int ti = warp / groups, c0 = (warp % groups) * 64;
    const uint16_t* wide = (const uint16_t*)q.wide;
    const double* small = (const double*)q.small;
    const int rows = q.s1 - q.s0;
    const int nst = (rows + kQmRows - 1) / kQmRows;
    auto issue = [&](int stg) {
        uint8_t* base = qmsm + (stg & 1) * stage_bytes;
        const int r0 = q.s0 + stg * kQmRows;
        const int nr = min(kQmRows, q.s1 - r0);
        const int wpieces = WIDE / 8;
        for (int e = tid; e < nr * wpieces; e += 256) {
            const int r = e / wpieces, c = e % wpieces;
            cp_async16(base + r * WIDE * 2 + c * 16, wide + (int64_t)(r0 + r) * q.wide_stride + c * 8, 16);
        }
        double* sb = reinterpret_cast<double*>(base + kQmRows * WIDE * 2);
        for (int e = tid; e < kQmRows * SMALL; e += 256) {
            const int r = e / SMALL, c = e % SMALL;
            if (r < nr) cp_async8(sb + r * lds + c, small + (int64_t)(r0 + r) * q.small_stride + c);
            else sb[r * lds + c] = 0.0;  // rows past the slice contribute nothing
        }
    };
    double acc[8][2];
#pragma unroll
    for (int u = 0; u < 8; ++u) acc[u][0] = acc[u][1] = 0.0;
    issue(0);
    cp_async_commit();
    for (int stg = 0; stg < nst; ++stg) {
        if (stg + 1 < nst) issue(stg + 1);
        cp_async_commit();
        cp_async_wait<1>();
        __syncthreads();
        const uint8_t* base = qmsm + (stg & 1) * stage_bytes;
        const uint16_t* tb = reinterpret_cast<const uint16_t*>(base);
        const double* sb = reinterpret_cast<const double*>(base + kQmRows * WIDE * 2);
#pragma unroll 2
        for (int ks = 0; ks < kQmRows / 4; ++ks) {
            const int r = ks * 4 + qq;  // the contraction row of this lane's k index
            const double a = sb[r * lds + ti * 8 + gr];
            const uint4 pk = *reinterpret_cast<const uint4*>(tb + r * WIDE + c0 + 8 * gr);
            const uint32_t pw[4] = {pk.x, pk.y, pk.z, pk.w};
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const double b = (double)((pw[u >> 1] >> (16 * (u & 1))) & 0xFFFFu);
                mma_f64(acc[u][0], acc[u][1], a, b);
            }
        }
        __syncthreads();  // the buffer is free for stage stg + 2
    }
    const int i = ti * 8 + gr;
#pragma unroll
    for (int u = 0; u < 8; ++u)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int w = c0 + 8 * (2 * qq + h) + u;
            if (q.out_trans) q.out[(int64_t)w * SMALL + i] = acc[u][h];
            else q.out[(int64_t)i * WIDE + w] = acc[u][h];
        }
}

static cudaError_t launch_qthin_mma(const ThinQ* d, int n, int stage_bytes, cudaStream_t s, const DevState* st) {
    k_qthin_mma<<<n, 256, 2 * stage_bytes, s>>>(d, stage_bytes, st);
    return cudaGetLastError();
}

// shared memory of k_qthin: the largest term's stage (table rows + small rows)
static int qthin_stage_bytes(const std::vector<ThinQ>& v) {
    int m = 0;
    for (const auto& q : v) m = std::max(m, kQtRows * (q.WIDE * 2 + q.SMALL * 8));
    return (m + 15) & ~15;
}

static cudaError_t launch_qthin(const ThinQ* d, int n, int stage_bytes, cudaStream_t s, const DevState* st) {
    k_qthin<<<n, 256, stage_bytes * kQtStages, s>>>(d, stage_bytes, st);
    return cudaGetLastError();
}

static int dthin_smem(int k) { return (int)sizeof(double) * ((1 << k) + (1 << k) / 8 + 8); }

static cudaError_t launch_dthin(const ThinDF* d, int n, int it, int k, const double* lnq_full, cudaStream_t s,
                                const DevState* st) {
    const int sm = dthin_smem(k);
    switch (it) {
        case 1: k_dthin<1><<<n, 256, sm, s>>>(d, lnq_full, st); break;
        case 2: k_dthin<2><<<n, 256, sm, s>>>(d, lnq_full, st); break;
        case 4: k_dthin<4><<<n, 256, sm, s>>>(d, lnq_full, st); break;
        case 8: k_dthin<8><<<n, 256, sm, s>>>(d, lnq_full, st); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

static cudaError_t launch_dthin_mma(const ThinDF* d, int n, int smem, const double* lnq_full, cudaStream_t s,
                                    const DevState* st) {
    k_dthin_mma<<<n, 256, smem, s>>>(d, lnq_full, st);
    return cudaGetLastError();
}

static cudaError_t set_thin_smem(int ny) {
    const int sm = (int)sizeof(double) * ny;
    if (sm <= 48 * 1024) return cudaSuccess;
    cudaError_t e = cudaSuccess;
#define SET_(S) if (e == cudaSuccess) e = cudaFuncSetAttribute(k_thin_d<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    SET_(1) SET_(2) SET_(4) SET_(8) SET_(16) SET_(32) SET_(64)
#undef SET_
    return e;
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
// phase 1: qsum[t][y] = sum over the split slices of Q_t
__global__ void k_qsum(const FoldTerm* __restrict__ terms, int T, const double* __restrict__ qparts, int k,
                       double* __restrict__ qsum, const DevState* st) {
    if (gated(st)) return;
    const int ny = 1 << k;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < T * ny; e += gridDim.x * blockDim.x) {
        const int t = e / ny, y = e % ny;
        const FoldTerm& f = terms[t];
        if (f.kind != 0) continue;
        const double* q = qparts + f.qoff + y;
        double a = 0.0;
        for (int sp = 0; sp < f.qs; ++sp) a += q[(size_t)sp * ny];
        qsum[e] = a;
    }
}

// Q_t[y] from the split sums, or from U^T / V for identity terms (V holds
// only the rows x_hi < H1h; the rows above are zero)
__device__ __forceinline__ double term_value(const FoldTerm& f, const double* qsum, int t, int ny,
                                             const double* ULt, int KL, const double* VR, int KR, int H1h,
                                             int row0, uint32_t y) {
    if (f.kind == 0) return qsum[(size_t)t * ny + y];
    const uint32_t yh = y >> f.m, yl = y & ((1u << f.m) - 1u);
    if (f.kind == 1) return ULt[(size_t)reverse_bits(yl, f.m) * KL + f.off + yh];  // Q_t = U_t (rows: rev x_lo)
    // Q_t = V_t at row x_hi = yh: held rows only (the others are another shard's)
    const uint32_t r = yh - (uint32_t)row0;
    return (yh >= (uint32_t)row0 && r < (uint32_t)H1h) ? VR[(size_t)r * KR + f.off + yl] : 0.0;
}

// phase 2: acc[y] = sum_t Q_t[y]: CTA = 32 consecutive y, warp w reads the
// terms w, w + 8, ... (coalesced along y), and the 8 partial sums are added
// in a fixed order
__global__ void __launch_bounds__(256) k_fold_acc(const FoldTerm* __restrict__ terms, int T,
                                                  const double* __restrict__ qsum, const double* __restrict__ ULt,
                                                  int KL, const double* __restrict__ VR, int KR, int H1h, int row0,
                                                  int k, double* __restrict__ acc, const DevState* st) {
    if (gated(st)) return;
    __shared__ double part[8][33];
    const int ny = 1 << k;
    const int yy = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int y = blockIdx.x * 32 + yy;
    double a = 0.0;
    if (y < ny)
        for (int t = w; t < T; t += 8) a += term_value(terms[t], qsum, t, ny, ULt, KL, VR, KR, H1h, row0, (uint32_t)y);
    part[w][yy] = a;
    __syncthreads();
    if (w == 0 && y < ny) {
        double s = part[0][yy];
        for (int j = 1; j < 8; ++j) s += part[j][yy];
        acc[y] = s;
    }
}

// phase 3: q(rep r) = sum_{y in O(r)} acc[y] / (|O(r)| C Z); ln q with the
// reference's 0 for q == 0 (backend/BAA.cu:573-580), expanded to every y,
// and copied into RB / LA where a D-side product is the identity.
__global__ void k_fold_q(const FoldTerm* __restrict__ terms, int T, const double* __restrict__ accv, int k,
                         double inv_c, double* __restrict__ lnq_full, double* __restrict__ lnq, double* __restrict__ RB,
                         int H2, double* __restrict__ LA, int Kp, int KL, int H1h, int row0, const DevState* st) {
    if (gated(st)) return;
    const int ny = 1 << k;
    const int y = blockIdx.x * blockDim.x + threadIdx.x;
    if (y >= ny) return;
    const double inv_z = exp(-st->log_z);
    const uint32_t r = orbit_rep((uint32_t)y, k);
    const uint32_t rv = reverse_bits(r, k), cv = complement_bits(r, k), rcv = reverse_bits(cv, k);
    double acc = accv[r];
    int nm = 1;
    if (rv != r) {
        acc += accv[rv];
        ++nm;
    }
    if (cv != r && cv != rv) {
        acc += accv[cv];
        ++nm;
    }
    if (rcv != r && rcv != rv && rcv != cv) {
        acc += accv[rcv];
        ++nm;
    }
    const double q = acc * inv_c * inv_z / (double)nm;
    const double lq = (q != 0.0) ? log(q) : 0.0;
    lnq_full[y] = lq;
    if ((uint32_t)y == r) lnq[y] = lq;  // representatives are < 2^{k-1}
    for (int t = 0; t < T; ++t) {
        const FoldTerm& f = terms[t];
        const uint32_t yh = (uint32_t)y >> f.m, yl = (uint32_t)y & ((1u << f.m) - 1u);
        if (f.idB_left) RB[(size_t)(f.off + yh) * H2 + reverse_bits(yl, f.m)] = lq;  // M_t = Lq_t
        const uint32_t r = yh - (uint32_t)row0;  // the held rows of N_t = Lq_t
        if (f.idA_right && yh >= (uint32_t)row0 && r < (uint32_t)H1h) LA[(size_t)r * Kp + KL + f.off + yl] = lq;
    }
}

__global__ void __launch_bounds__(256)
k_fac_finalize(const double* __restrict__ part, int nb, double a, double eta, DevState* st) {
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
    // Lt holds ln p + eta D - shift, so ln p' - ln p = eta D - shift - ln Z
    const double lnz = log(sE);
    const double ln2 = 0.69314718055994530942;
    const double mx = st->zero_p ? INFINITY : (eta * mD - st->shift - lnz) / ln2;
    st->max_d = mD;
    st->rate = sR;
    st->best_ub = fmin(st->best_ub, mD);
    st->best_rate = fmax(st->best_rate, sR);
    st->lse = st->shift + lnz;
    st->mx = mx;
    st->max_logw = mL + st->shift;
    st->log_z = lnz;
    // next shift: the largest new ln p plus eta times the current bound on D
    st->shift = (mL - lnz) + eta * mD;
    st->zero_p = 0;
    st->iter += 1;
    st->done = !(mx >= a);
}

// re-scale after an exp over/underflow: Lt -= s, Pw = |O| exp(Lt), sum
__global__ void __launch_bounds__(256)
k_fac_rescale(const uint32_t* __restrict__ reps, int64_t R, int n, int row0, double* Lt, double* Pw,
              double* part, DevState* st, int on_shift_error) {
    if (on_shift_error && st->error != kErrShift) return;  // queued unconditionally in a captured map
    const double s = st->max_logw;  // max of Lt after the failed epilogue
    double sum = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < R; i += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t x = reps[i], xd = fac_loc(x, n, row0);
        const double l = Lt[xd] - s;
        const double o = (double)orbit_size(x, n);
        Lt[xd] = l;
        const double e = exp(l);
        Pw[xd] = o * e;
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

__global__ void k_fac_rescale_finish(const double* part, int nb, double a, DevState* st, int on_shift_error) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    if (on_shift_error && st->error != kErrShift) return;
    double sE = 0.0;
    for (int b = 0; b < nb; ++b) sE += part[b];
    // Lt now holds logW - (shift + s) with maximum 0
    const double shift_eff = st->shift + st->max_logw;
    const double lnz = log(sE);
    const double ln2 = 0.69314718055994530942;
    const double mx = st->zero_p ? INFINITY : (st->max_d - shift_eff - lnz) / ln2;
    st->best_ub = fmin(st->best_ub, st->max_d);
    st->best_rate = fmax(st->best_rate, st->rate);
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

// one warp
__global__ void k_fac_load_finish(const double* part, int nb, int k, DevState* st) {
    if (blockIdx.x != 0) return;
    const double mx = warp_parts<true>(part, nb, 2);
    const double z = warp_parts<true>(part + 1, nb, 2);
    if (threadIdx.x != 0) return;
    st->log_z = 0.0;
    st->shift = mx + (double)k * 0.69314718055994530942;  // first guess; re-scaled if off
    st->zero_p = (z != 0.0);
}

// ---- per-representative vectors <-> dense rows, one CTA per held row.
// The representatives of row x_hi are a contiguous run of the ascending list
// in ascending x_lo, while the dense row stores column rev(x_lo): the CTA
// ranks the row's representatives by a block scan of the flags in x_lo order
// and moves the run through shared memory, so that both sides are read and
// written in memory order.  Shared memory: the run (8 bytes per column) and
// the ranks (2 bytes per column, 0xFFFF where no representative).
constexpr uint16_t kNoRank = 0xFFFF;

__host__ __device__ constexpr int rows_smem_bytes(int n2) { return (8 + 2) << n2; }

// ranks of the representatives of row xh in x_lo order into rk; returns their
// number (every thread)
__device__ __forceinline__ int row_ranks(uint32_t xh, int n, int n2, uint16_t* rk) {
    __shared__ int wsum[8];
    const int H2 = 1 << n2, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int C = H2 >= 256 ? H2 / 256 : 1;  // consecutive x_lo per thread
    const int lo0 = tid * C;
    int cnt = 0;
    for (int j = 0; j < C && lo0 + j < H2; ++j) cnt += is_rep((xh << n2) | (uint32_t)(lo0 + j), n) ? 1 : 0;
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += v;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    int base = incl - cnt, total = 0;
#pragma unroll
    for (int w = 0; w < 8; ++w) {
        if (w < warp) base += wsum[w];
        total += wsum[w];
    }
    for (int j = 0; j < C && lo0 + j < H2; ++j) {
        const bool rep = is_rep((xh << n2) | (uint32_t)(lo0 + j), n);
        rk[lo0 + j] = rep ? (uint16_t)base : kNoRank;
        base += rep ? 1 : 0;
    }
    __syncthreads();
    return total;
}

// p -> (Pw, Lt) on the held rows, per-row partials [max ln p, zero flag]
// (k_fac_load's per-element rules)
__global__ void __launch_bounds__(256) k_fac_load_rows(const int64_t* __restrict__ rs, int n, int row0,
                                                       const double* __restrict__ p, double* __restrict__ Pw,
                                                       double* __restrict__ Lt, double* __restrict__ part,
                                                       int strict_zero) {
    extern __shared__ double rsm[];
    const int n2 = n >> 1, H2 = 1 << n2, r = blockIdx.x;
    uint16_t* rk = reinterpret_cast<uint16_t*>(rsm + H2);
    const uint32_t xh = (uint32_t)(row0 + r);
    const int cnt = row_ranks(xh, n, n2, rk);
    const int64_t b0 = rs[r];
    for (int j = threadIdx.x; j < cnt; j += 256) rsm[j] = p[b0 + j];
    __syncthreads();
    double mx = -DBL_MAX;
    int zero = 0;
    double* pw = Pw + ((int64_t)r << n2);
    double* lt = Lt + ((int64_t)r << n2);
    for (int c = threadIdx.x; c < H2; c += 256) {
        const uint32_t xl = reverse_bits((uint32_t)c, n2);
        const uint16_t k = rk[xl];
        if (k == kNoRank) continue;
        const double v = rsm[k];
        pw[c] = (double)orbit_size((xh << n2) | xl, n) * v;
        if (strict_zero) {
            lt[c] = (v > 0.0) ? log(v) : -INFINITY;
            if (v > 0.0) mx = fmax(mx, log(v));
            continue;
        }
        const double l = (v != 0.0) ? log(v) : 0.0;
        lt[c] = (v != 0.0) ? l : __longlong_as_double(0x7ff8000000000000ll);
        mx = fmax(mx, l);
        if (v == 0.0) zero = 1;
    }
    __shared__ double red[8];
    __shared__ int zr[8];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mx = fmax(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, o));
        zero |= __shfl_xor_sync(0xFFFFFFFFu, zero, o);
    }
    if ((threadIdx.x & 31) == 0) {
        red[threadIdx.x >> 5] = mx;
        zr[threadIdx.x >> 5] = zero;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < 8; ++w) {
            red[0] = fmax(red[0], red[w]);
            zr[0] |= zr[w];
        }
        part[2 * r] = red[0];
        part[2 * r + 1] = (double)zr[0];
    }
}

// MODE 0: p = Pw / (|O| Z) (k_fac_store's rule); MODE 1: out = dense (a
// gather of D); MODE 2: dense = v (a scatter of h), on the held rows
template <int MODE>
__global__ void __launch_bounds__(256) k_fac_rows(const int64_t* __restrict__ rs, int n, int row0,
                                                  const double* __restrict__ src, double* __restrict__ dst,
                                                  const DevState* st) {
    extern __shared__ double rsm[];
    const int n2 = n >> 1, H2 = 1 << n2, r = blockIdx.x;
    uint16_t* rk = reinterpret_cast<uint16_t*>(rsm + H2);
    const uint32_t xh = (uint32_t)(row0 + r);
    const int cnt = row_ranks(xh, n, n2, rk);
    const int64_t b0 = rs[r];
    const double inv_z = (MODE == 0) ? exp(-st->log_z) : 1.0;
    if (MODE == 2) {
        for (int j = threadIdx.x; j < cnt; j += 256) rsm[j] = src[b0 + j];
        __syncthreads();
        double* d = dst + ((int64_t)r << n2);
        for (int c = threadIdx.x; c < H2; c += 256) {
            const uint16_t k = rk[reverse_bits((uint32_t)c, n2)];
            if (k != kNoRank) d[c] = rsm[k];
        }
        return;
    }
    const double* d = src + ((int64_t)r << n2);
    for (int c = threadIdx.x; c < H2; c += 256) {
        const uint32_t xl = reverse_bits((uint32_t)c, n2);
        const uint16_t k = rk[xl];
        if (k == kNoRank) continue;
        rsm[k] = (MODE == 0) ? d[c] * inv_z / (double)orbit_size((xh << n2) | xl, n) : d[c];
    }
    __syncthreads();
    for (int j = threadIdx.x; j < cnt; j += 256) dst[b0 + j] = rsm[j];
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

// the low-half tables in dense-column order: row c = table row rev(c)
__global__ void k_permute_rows(const uint16_t* __restrict__ src, int64_t stride, int rows, int n2,
                               uint16_t* __restrict__ dst) {
    const int64_t total = (int64_t)rows * stride;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = e / stride, w = e % stride;
        dst[e] = src[(int64_t)reverse_bits((uint32_t)c, n2) * stride + w];
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

// the operand restricted to contraction indices >= k0
static Operand k_offset(Operand o, bool is_a, int64_t k0) {
    if (o.kind == OP_EYE || k0 == 0) return o;
    const int64_t step = is_a ? (o.trans ? k0 * o.ld : k0) : (o.trans ? k0 : k0 * o.ld);
    if (o.kind == OP_U16) o.ptr = (const uint16_t*)o.ptr + step;
    else o.ptr = (const double*)o.ptr + step;
    return o;
}

// S products over consecutive slices of the contraction, output s at C + s * cstride;
// slice boundaries are multiples of 16 (whole k-slices, aligned operands)
static void split_k(std::vector<GemmDesc>& out, const GemmDesc& d, int S, int64_t cstride) {
    for (int s = 0; s < S; ++s) {
        const int64_t k0 = ((int64_t)d.K * s / S) & ~(int64_t)15;
        const int64_t k1 = (s + 1 == S) ? d.K : (((int64_t)d.K * (s + 1) / S) & ~(int64_t)15);
        GemmDesc e = d;
        e.A = k_offset(d.A, true, k0);
        e.B = k_offset(d.B, false, k0);
        e.K = (int)(k1 - k0);
        e.C = d.C + s * cstride;
        out.push_back(e);
    }
}

static int assign_tiles(std::vector<GemmDesc>& v, int cfg) {
    int t = 0;
    for (auto& d : v) {
        d.tiles_m = (d.M + kCfgBM[cfg] - 1) / kCfgBM[cfg];
        d.tiles_n = (d.N + kCfgBN[cfg] - 1) / kCfgBN[cfg];
        d.tile_begin = t;
        t += d.tiles_m * d.tiles_n;
    }
    return t;
}

static void free_launch(Launch& L) {
    cudaFree(L.d);
    cudaFree(L.map);
    L.d = nullptr;
    L.map = nullptr;
}

// the cp.async layout of a list of products, or -1 when a product does not
// qualify (an operand that is not FP64, an odd leading dimension or a base
// that is not 16-byte aligned) or the layouts differ
static int cp_layout(const std::vector<GemmDesc>& v) {
    int lay = -2;
    for (const auto& d : v) {
        if (d.A.kind != OP_F64 || d.B.kind != OP_F64) return -1;
        if ((d.A.ld & 1) || (d.B.ld & 1)) return -1;
        if (((uintptr_t)d.A.ptr & 15) || ((uintptr_t)d.B.ptr & 15)) return -1;
        const int l = (d.A.trans ? 1 : 0) | (d.B.trans ? 0 : 2);
        if (lay == -2) lay = l;
        else if (lay != l) return -1;
    }
    return lay < 0 ? -1 : lay;
}

static cudaError_t make_launch(Launch& L, std::vector<GemmDesc> v, int cfg) {
    free_launch(L);
    L.cfg = cfg;
    L.layout = cp_layout(v);
    L.n = (int)v.size();
    L.tiles = assign_tiles(v, cfg);
    if (v.empty()) return cudaSuccess;
    std::vector<int> map(L.tiles);
    for (int i = 0; i < (int)v.size(); ++i)
        for (int t = 0; t < v[i].tiles_m * v[i].tiles_n; ++t) map[v[i].tile_begin + t] = i;
    cudaError_t e = cudaMalloc(&L.d, sizeof(GemmDesc) * v.size());
    if (e == cudaSuccess) e = cudaMemcpy(L.d, v.data(), sizeof(GemmDesc) * v.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&L.map, sizeof(int) * map.size());
    if (e == cudaSuccess) e = cudaMemcpy(L.map, map.data(), sizeof(int) * map.size(), cudaMemcpyHostToDevice);
    return e;
}

template <typename F>
static float time_ms(bdc_handle* H, F&& launch, cudaError_t* err = nullptr) {
    // the best of three rounds of three launches, after a warm-up launch; a
    // launch that returns an error (or leaves one) makes the time 1e30 and
    // the error is passed out through err
    cudaError_t first = cudaSuccess;
    auto run = [&] {
        if constexpr (std::is_same_v<decltype(launch()), cudaError_t>) {
            const cudaError_t e = launch();
            if (first == cudaSuccess) first = e;
        } else {
            launch();
        }
    };
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    run();
    float best = 1e30f;
    for (int round = 0; round < 3; ++round) {
        cudaEventRecord(a, H->stream);
        for (int r = 0; r < 3; ++r) run();
        cudaEventRecord(b, H->stream);
        cudaEventSynchronize(b);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        best = std::min(best, ms / 3.f);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    const cudaError_t last = cudaGetLastError();
    if (first == cudaSuccess) first = last;
    if (err) *err = first;
    return first == cudaSuccess ? best : 1e30f;
}

// G with only the tiles that hold representatives (colmax: per dense column
// the largest row of a representative); CTA i runs tile map[i]
static cudaError_t make_tile_launch(Launch& L, GemmDesc d, int cfg, const std::vector<int>& colmax) {
    free_launch(L);
    L.cfg = cfg;
    L.layout = cp_layout({d});
    L.n = 1;
    const int BM = kCfgBM[cfg], BN = kCfgBN[cfg];
    d.tiles_m = (d.M + BM - 1) / BM;
    d.tiles_n = (d.N + BN - 1) / BN;
    d.tile_begin = 0;
    std::vector<int> ids;
    for (int tm = 0; tm < d.tiles_m; ++tm)
        for (int tn = 0; tn < d.tiles_n; ++tn) {
            int mx = -1;
            for (int c = tn * BN; c < std::min(d.N, (tn + 1) * BN); ++c) mx = std::max(mx, colmax[c]);
            if (mx >= tm * BM) ids.push_back(tm * d.tiles_n + tn);
        }
    L.tiles = (int)ids.size();
    if (ids.empty()) return cudaSuccess;
    cudaError_t e = cudaMalloc(&L.d, sizeof(GemmDesc));
    if (e == cudaSuccess) e = cudaMemcpy(L.d, &d, sizeof(GemmDesc), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&L.map, sizeof(int) * ids.size());
    if (e == cudaSuccess) e = cudaMemcpy(L.map, ids.data(), sizeof(int) * ids.size(), cudaMemcpyHostToDevice);
    return e;
}

// Tuning choices pinned in a text file named by the environment variable
// BDC_TUNE_FILE (lines "n k key a b"): a choice found there is used without
// timing, new choices are appended, so that repeated runs (a profiler's, for
// instance) execute the same kernels.
struct TuneFile {
    std::string path;
    std::map<std::string, std::pair<int, int>> m;
    std::vector<std::string> fresh;
    int n = 0, k = 0;
    void load(int n_, int k_) {
        n = n_;
        k = k_;
        const char* e = getenv("BDC_TUNE_FILE");
        if (!e || !*e) return;
        path = e;
        FILE* f = fopen(path.c_str(), "r");
        if (!f) return;
        int a, b, nn, kk;
        char key[64];
        while (fscanf(f, "%d %d %63s %d %d", &nn, &kk, key, &a, &b) == 5)
            if (nn == n && kk == k) m[key] = {a, b};
        fclose(f);
    }
    bool get(const char* key, int* a, int* b) const {
        auto it = m.find(key);
        if (it == m.end()) return false;
        *a = it->second.first;
        *b = it->second.second;
        return true;
    }
    void put(const char* key, int a, int b) {
        if (path.empty()) return;
        m[key] = {a, b};
        char line[128];
        snprintf(line, sizeof(line), "%d %d %s %d %d\n", n, k, key, a, b);
        fresh.push_back(line);
    }
    void save() {
        if (path.empty() || fresh.empty()) return;
        FILE* f = fopen(path.c_str(), "a");
        if (!f) return;
        for (auto& l : fresh) fputs(l.c_str(), f);
        fclose(f);
        fresh.clear();
    }
};

// chooses tile shape and split of one of the wide q-side products by timing
// them; gen(cfg, S) lists the descriptors of a candidate (S: the split of
// the longest contraction, kfull its length)
template <typename Gen, typename Post>
static bdc_status tune_thin(bdc_handle* H, TuneFile& tf, const char* key, Launch& L, Gen&& gen, Post&& post,
                            int kfull, int max_split, int kmin, const char* what, int* split_out) {
    const int cfgs[4] = {CFG_128x128, CFG_128x64, CFG_64x128, CFG_64x64};
    float best = 1e30f;
    int best_cfg = CFG_64x64, best_s = 1;
    const bool pinned = tf.get(key, &best_cfg, &best_s);
    for (int ci = 0; ci < 4 && !pinned; ++ci) {
        for (int S = 1; S <= max_split; S *= 2) {
            if (kfull / S < kmin) break;
            std::vector<GemmDesc> v = gen(cfgs[ci], S);
            Launch T;
            BDC_CUDA_TRY(make_launch(T, v, cfgs[ci]));
            if (T.tiles > 64 * H->num_sms) {
                free_launch(T);
                continue;
            }
            // the product and the sum of its S split slices
            const float ms = time_ms(H, [&] {
                const cudaError_t e = launch_store(T, H->stream, nullptr);
                post(S);
                return e;
            });
            free_launch(T);
            if (ms < best) {
                best = ms;
                best_cfg = cfgs[ci];
                best_s = S;
            }
        }
    }
    if (!pinned) tf.put(key, best_cfg, best_s);
    BDC_CUDA_TRY(make_launch(L, gen(best_cfg, best_s), best_cfg));
    *split_out = best_s;
    if (H->verbose)
        printf("bdc: tuned %s: tile %dx%d, split %d, %.1f us\n", what, kCfgBM[best_cfg], kCfgBN[best_cfg], best_s,
               best * 1e3f);
    return BDC_OK;
}

// A thin q-side product as a matrix product on the tensor-core path, in the
// orientation whose long side (the wide index w) is M:
//   C(w, i) = sum_s wide(s)[w] small(s)[i] over s in [s0, s1)
static GemmDesc thin_q_desc(const ThinQ& q) {
    Operand A, B;
    A.ptr = q.wide;
    A.ld = q.wide_stride;
    A.kind = q.wide_u16 ? OP_U16 : OP_F64;
    A.trans = 1;
    B.ptr = q.small;
    B.ld = q.small_stride;
    B.kind = q.small_u16 ? OP_U16 : OP_F64;
    B.trans = 0;
    GemmDesc d = make_desc(k_offset(A, true, q.s0), k_offset(B, false, q.s0), q.out, q.out_trans ? q.SMALL : 1,
                           q.out_trans ? 1 : q.WIDE, q.WIDE, q.SMALL, q.s1 - q.s0);
    return d;
}

// A thin D-side product: C(s, i) = sum_w wide(s)[w] Lq'[w][i]
static GemmDesc thin_d_desc(const ThinD& t, const double* lnq_full) {
    Operand A, B;
    A.ptr = t.wide;
    A.ld = t.wide_stride;
    A.kind = OP_U16;
    A.trans = 0;
    B.ptr = lnq_full;
    B.kind = OP_F64;
    B.trans = t.lq_trans ? 0 : 1;
    B.ld = t.lq_trans ? t.SMALL : t.WIDE;
    return make_desc(A, B, t.out, t.out_s, t.out_i, t.rows, t.SMALL, t.WIDE);
}

// times the CUDA-core kernel of one size class against the tensor-core
// launch in a few tile shapes and keeps the fastest
template <typename Core>
static bdc_status tune_class(bdc_handle* H, TuneFile& tf, const char* key, const std::vector<GemmDesc>& descs,
                             Launch& L, bool& use_mma, Core&& core_launch, const char* what, int lg) {
    const int cfgs[5] = {CFG_128x16, CFG_128x32, CFG_64x64, CFG_128x64, CFG_64x128};
    int best_cfg = -1, unused = 0;
    const bool pinned = tf.get(key, &best_cfg, &unused);
    // the CUDA-core kernels hold one accumulator per small output in
    // registers, up to 64; wider terms always take a tensor-core tile
    const bool core_ok = lg <= 6;
    const float core_ms = (pinned || !core_ok) ? 0.f : time_ms(H, core_launch);
    float best = core_ok ? core_ms : 1e30f;
    if (pinned && !core_ok && best_cfg < 0) best_cfg = CFG_64x64;
    for (int c : cfgs) {
        if (pinned) break;
        Launch T;
        BDC_CUDA_TRY(make_launch(T, descs, c));
        const float ms = time_ms(H, [&] { return launch_store(T, H->stream, nullptr); });
        free_launch(T);
        if (ms < best) {
            best = ms;
            best_cfg = c;
        }
    }
    if (!pinned) tf.put(key, best_cfg, 0);
    use_mma = best_cfg >= 0;
    if (use_mma) BDC_CUDA_TRY(make_launch(L, descs, best_cfg));
    if (H->verbose)
        printf("bdc: tuned %s, %d outputs per term: %s %.1f us (CUDA cores %.1f us)\n", what, 1 << lg,
               use_mma ? (best_cfg == CFG_128x16 ? "mma 128x16" : best_cfg == CFG_128x32 ? "mma 128x32"
                          : best_cfg == CFG_64x64 ? "mma 64x64" : best_cfg == CFG_128x64 ? "mma 128x64" : "mma 64x128")
                       : "CUDA cores",
               best * 1e3f, core_ms * 1e3f);
    return BDC_OK;
}

cudaError_t dgemm_scratch_alloc(DgemmScratch& sc, int max_tiles, cudaStream_t s) {
    dgemm_scratch_free(sc);
    cudaError_t e = cudaMalloc(&sc.desc, sizeof(GemmDesc));
    if (e == cudaSuccess) e = cudaMalloc(&sc.map, sizeof(int) * (size_t)std::max(1, max_tiles));
    if (e == cudaSuccess) e = cudaMemsetAsync(sc.map, 0, sizeof(int) * (size_t)std::max(1, max_tiles), s);
    if (e == cudaSuccess) sc.tiles = max_tiles;
    return e;
}

void dgemm_scratch_free(DgemmScratch& sc) {
    cudaFree(sc.desc);
    cudaFree(sc.map);
    sc = DgemmScratch{};
}

// C (M x N, row stride ldc) = alpha A B^T (+ C when accumulate) for row-major
// A (M x K, stride lda) and B (N x K, stride ldb) on the FP64 tensor-core
// path; a helper for small dense work outside the iteration (the certified
// solver's Newton systems).  The descriptor goes to sc.desc on the same
// stream, so a call does not overwrite it under the previous call's kernel.
cudaError_t dgemm_nt(const DgemmScratch& sc, const double* A, int lda, const double* B, int ldb, double* C, int ldc,
                     int M, int N, int K, double alpha, int accumulate, cudaStream_t s) {
    static bool attrs = false;
    if (!attrs) {
        cudaError_t e = set_smem_attrs();
        if (e != cudaSuccess) return e;
        attrs = true;
    }
    std::vector<GemmDesc> v{make_desc(op_f64(A, lda, 0), op_f64(B, ldb, 1), C, ldc, 1, M, N, K)};
    v[0].alpha = alpha;
    v[0].accumulate = accumulate;
    Launch L;
    L.cfg = CFG_64x64;
    L.layout = cp_layout(v);
    L.n = 1;
    L.tiles = assign_tiles(v, CFG_64x64);
    if (L.tiles > sc.tiles || !sc.desc) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemcpyAsync(sc.desc, v.data(), sizeof(GemmDesc), cudaMemcpyHostToDevice, s);
    L.d = (GemmDesc*)sc.desc;
    L.map = sc.map;
    if (e == cudaSuccess) e = launch_store(L, s, nullptr);
    L.d = nullptr;  // owned by the scratch
    L.map = nullptr;
    return e;
}

bool factored_supports(int n, int k) {
    // needs k < n (W is not the identity), half tables that fit the uint16
    // bundles, a dense 2^{n-1} state that fits comfortably in device memory,
    // and per-term products of at most 128 small outputs (a term's small side
    // is 2^min(j, k - j), up to 2^floor(k/2))
    return k >= 1 && k < n && n >= 2 && n <= 28 && k <= 14;
}

static BaEpilogue make_epilogue(bdc_handle* H);

bdc_status factored_init(bdc_handle* H) {
    BDC_CUDA_TRY(set_smem_attrs());
    FactoredState* F = new FactoredState();
    H->fac = F;
    TuneFile tf;
    tf.load(H->n, H->k);
    const Split& s = H->s;
    F->H1 = 1 << s.n1;
    F->H2 = 1 << s.n2;
    // every representative is <= its complement, so its top bit is 0 and
    // x_hi < H1 / 2: only those rows of the iterate and of G are needed
    F->H1h = F->H1 / 2;
    // the rows this handle holds: all of them on one GPU; a window of whole
    // rows, balanced by the number of representatives, for shard rank r of w
    // (representatives ascend, and x_hi = x >> n2, so a row window is one
    // contiguous range of them)
    std::vector<uint32_t> hr((size_t)H->R);
    BDC_CUDA_TRY(cudaMemcpyAsync(hr.data(), H->d_reps, sizeof(uint32_t) * hr.size(), cudaMemcpyDeviceToHost,
                                 H->stream));
    BDC_CUDA_TRY(cudaStreamSynchronize(H->stream));
    {
        const int w = H->shard_world, r = H->shard_rank;
        if (w < 1 || r < 0 || r >= w || w > F->H1h)
            return fail(BDC_ERR_ARG, "factored engine: shard %d of %d over %d rows", r, w, F->H1h);
        auto below = [&](int row) {  // representatives with x_hi < row
            return (int64_t)(std::lower_bound(hr.begin(), hr.end(), (uint32_t)row << s.n2) - hr.begin());
        };
        auto cut = [&](int q) {  // first row of shard q
            if (q <= 0) return 0;
            if (q >= w) return F->H1h;
            const int64_t target = H->R * q / w;
            int lo = 0, hi = F->H1h;
            while (lo < hi) {
                const int mid = (lo + hi) / 2;
                if (below(mid) >= target) hi = mid;
                else lo = mid + 1;
            }
            return std::max(lo, q);  // at least one row per shard
        };
        const int c0 = std::min(cut(r), F->H1h - (w - r)), c1 = (r + 1 == w) ? F->H1h : std::min(cut(r + 1), F->H1h - (w - r - 1));
        F->row0 = c0;
        F->H1h = c1 - c0;
        F->i0 = below(c0);
        F->Rl = below(c1) - F->i0;
        // where each held row's run of representatives starts (k_fac_rows)
        std::vector<int64_t> rs((size_t)F->H1h + 1);
        for (int q = 0; q <= F->H1h; ++q) rs[(size_t)q] = below(c0 + q) - F->i0;
        BDC_CUDA_TRY(cudaMalloc(&F->d_rowstart, sizeof(int64_t) * rs.size()));
        BDC_CUDA_TRY(cudaMemcpy(F->d_rowstart, rs.data(), sizeof(int64_t) * rs.size(), cudaMemcpyHostToDevice));
        BDC_CUDA_TRY(cudaMalloc(&F->rpart, sizeof(double) * 2 * (size_t)F->H1h));
        F->rows_smem = rows_smem_bytes(s.n2);
        if (F->rows_smem > 48 * 1024) {
            BDC_CUDA_TRY(cudaFuncSetAttribute(k_fac_load_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, F->rows_smem));
            BDC_CUDA_TRY(cudaFuncSetAttribute(k_fac_rows<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, F->rows_smem));
            BDC_CUDA_TRY(cudaFuncSetAttribute(k_fac_rows<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, F->rows_smem));
            BDC_CUDA_TRY(cudaFuncSetAttribute(k_fac_rows<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, F->rows_smem));
        }
    }
    const int k = H->k;
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
    const int64_t NX = (int64_t)F->H1h * F->H2;  // the dense rows held
    const int ny = 1 << k;
    const int H1 = F->H1h, H2 = F->H2, Kp = F->Kp;  // H1: the rows kept
    const int KLa = KL > 0 ? KL : 1, KRa = KR > 0 ? KR : 1;
    const int max_split = 16;

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
    BDC_CUDA_TRY(al(&F->ulpart, (size_t)max_split * H2 * KLa));
    BDC_CUDA_TRY(al(&F->vrpart, (size_t)max_split * H1 * KRa));
    BDC_CUDA_TRY(al(&F->lnq_full, (size_t)ny));
    BDC_CUDA_TRY(cudaMemsetAsync(F->LA, 0, sizeof(double) * H1 * Kp, H->stream));
    BDC_CUDA_TRY(cudaMemsetAsync(F->RB, 0, sizeof(double) * Kp * H2, H->stream));
    BDC_CUDA_TRY(cudaMemsetAsync(F->hx, 0, sizeof(double) * NX, H->stream));
    BDC_CUDA_TRY(cudaMemsetAsync(F->Pw, 0, sizeof(double) * NX, H->stream));
    BDC_CUDA_TRY(cudaMemsetAsync(F->Lt, 0, sizeof(double) * NX, H->stream));
    BDC_CUDA_TRY(cudaMemsetAsync(F->lnq_full, 0, sizeof(double) * ny, H->stream));

    // low-half tables in dense-column order, and the largest row of a
    // representative in each dense column (for skipping empty tiles)
    {
        const size_t cnt = (size_t)H2 * H->B.stride;
        BDC_CUDA_TRY(cudaMalloc(&F->Bp, cnt * sizeof(uint16_t) + 16));
        H->bytes += cnt * sizeof(uint16_t);
        k_permute_rows<<<H->num_sms * 8, 256, 0, H->stream>>>(H->B.rows, H->B.stride, H2, s.n2, F->Bp);
        BDC_CUDA_TRY(cudaGetLastError());
        F->colmax.assign(H2, -1);
        for (int64_t i = F->i0; i < F->i0 + F->Rl; ++i) {
            const uint32_t xd = fac_pos(hr[i], s.n2);
            const int c = (int)(xd & low_mask(s.n2)), xh = (int)(xd >> s.n2) - F->row0;
            if (xh > F->colmax[c]) F->colmax[c] = xh;
        }
    }

    // constant table columns of LA (AL) and rows of RB (BR^T); a left term's
    // A_j or a right term's B_m is never the identity
    {
        std::vector<int> colmap(KL + KR + 1);
        for (auto& t : F->terms) {
            if (t.left) for (int c = 0; c < (1 << t.j); ++c) colmap[t.off + c] = bundle_offset(t.j) + c;
            else for (int c = 0; c < (1 << t.m); ++c) colmap[KL + t.off + c] = bundle_offset(t.m) + c;
        }
        int* d_cm = nullptr;
        BDC_CUDA_TRY(cudaMalloc(&d_cm, sizeof(int) * colmap.size()));
        BDC_CUDA_TRY(cudaMemcpy(d_cm, colmap.data(), sizeof(int) * colmap.size(), cudaMemcpyHostToDevice));
        k_fill_tables<<<H->num_sms * 8, 256, 0, H->stream>>>(H1, H2, Kp, H->A.rows + (size_t)F->row0 * H->A.stride,
                                                            H->A.stride, F->Bp,
                                                            H->B.stride, d_cm, KL, KR, F->LA, F->RB);
        BDC_CUDA_TRY(cudaGetLastError());
        BDC_CUDA_TRY(cudaStreamSynchronize(H->stream));
        cudaFree(d_cm);
    }
    k_fac_rows<2><<<F->H1h, 256, F->rows_smem, H->stream>>>(F->d_rowstart, H->n, F->row0, H->d_h + F->i0, F->hx,
                                                            nullptr);
    BDC_CUDA_TRY(cudaGetLastError());

    // ---- the two thin products: U^T (H2 x KL) = (AL^T Pw)^T, V (H1h x KR) = Pw BR
    // Only the rows x_hi <= colmax[c] of a dense column c hold
    // representatives: U^T contracts each block of columns over those rows
    // only, V each block of rows over the columns that reach it.  The split
    // of a block is proportional to its contraction; split slices that no
    // block writes stay zero.
    if (KL > 0) {
        // A(m = c, kk = x_hi) = LA[x_hi * Kp + c]; B(kk = x_hi, n = col) = Pw; C(c, col) -> U^T[col][c]
        auto gen = [&](int cfg, int S) {
            std::vector<GemmDesc> v;
            const int BN = kCfgBN[cfg];
            for (int n0 = 0; n0 < H2; n0 += BN) {
                const int nb = std::min(BN, H2 - n0);
                int kb = 0;
                for (int c = n0; c < n0 + nb; ++c) kb = std::max(kb, F->colmax[c] + 1);
                if (kb == 0) continue;
                kb = std::min(H1, (kb + 15) & ~15);  // rows past the last representative are zero
                GemmDesc d = make_desc(op_f64(F->LA, Kp, 1), op_f64(F->Pw + n0, H2, 0), F->ulpart + (int64_t)n0 * KL,
                                       1, KL, KL, nb, kb);
                split_k(v, d, std::max(1, (int)(((int64_t)S * kb + H1 - 1) / H1)), (int64_t)H2 * KL);
            }
            return v;
        };
        auto post = [&](int S) {
            k_sum_parts<<<H->num_sms * 4, 256, 0, H->stream>>>(F->ulpart, S, (int64_t)KL * H2, F->UL, F->vrpart, 1, 0,
                                                               F->VR, nullptr);
        };
        bdc_status rc = tune_thin(H, tf, "ul", F->ul, gen, post, H1, max_split, 16, "U = AL^T Pw", &F->S1);
        if (rc != BDC_OK) return rc;
    }
    if (KR > 0) {
        // A(m = x_hi, kk = col) = Pw; B(kk = col, n = c) = RB[(KL + c) * H2 + col]
        auto gen = [&](int cfg, int S) {
            std::vector<GemmDesc> v;
            const int BM = kCfgBM[cfg];
            for (int m0 = 0; m0 < H1; m0 += BM) {
                const int mb = std::min(BM, H1 - m0);
                int clo = H2, chi = -1;
                for (int c = 0; c < H2; ++c)
                    if (F->colmax[c] >= m0) {
                        clo = std::min(clo, c);
                        chi = c;
                    }
                if (chi < 0) continue;
                // whole k-slices; the columns added at either end are zero in these rows
                clo &= ~15;
                const int kb = std::min(H2, (chi + 1 + 15) & ~15) - clo;
                const Operand A = k_offset(op_f64(F->Pw + (int64_t)m0 * H2, H2, 0), true, clo);
                const Operand B = k_offset(op_f64(F->RB + (int64_t)KL * H2, H2, 1), false, clo);
                GemmDesc d = make_desc(A, B, F->vrpart + (int64_t)m0 * KR, KR, 1, mb, KR, kb);
                split_k(v, d, std::max(1, (int)(((int64_t)S * kb + H2 - 1) / H2)), (int64_t)H1 * KR);
            }
            return v;
        };
        auto post = [&](int S) {
            k_sum_parts<<<H->num_sms * 4, 256, 0, H->stream>>>(F->ulpart, 1, 0, F->UL, F->vrpart, S,
                                                               (int64_t)H1 * KR, F->VR, nullptr);
        };
        bdc_status rc = tune_thin(H, tf, "vr", F->vr, gen, post, H2, max_split, 16, "V = Pw BR", &F->S2);
        if (rc != BDC_OK) return rc;
    }

    // ---- per-term thin products and the fold plan.  q side: Q_t as a sum of
    // outer products over the contracted half, split into slices so that the
    // launch fills the GPU (the fold sums the slices); D side: one row-dot
    // per half-table row.  Terms whose A_j or B_m is the identity are read or
    // written directly by the fold.
    std::vector<ThinQ> tq[8];
    std::vector<ThinD> td[8];
    std::vector<FoldTerm> fold;
    struct QPlan { int term, lg; ThinQ d; int S; };
    std::vector<QPlan> qplan;
    int qctas_one = 0;
    for (int ti = 0; ti < F->T; ++ti) {
        const Term& t = F->terms[ti];
        FoldTerm f{};
        f.j = t.j;
        f.m = t.m;
        f.off = t.off;
        if (t.left && t.idB) {
            f.kind = 1;       // Q_t = U_t
            f.idB_left = 1;   // M_t = Lq_t
        } else if (!t.left && t.idA) {
            f.kind = 2;        // Q_t = V_t
            f.idA_right = 1;   // N_t = Lq_t
        } else {
            ThinQ q{};
            ThinD d{};
            if (t.left) {
                // Q_t[yh][yl] = sum_{x_lo} U^T[x_lo][off + yh] B_m[x_lo][yl]
                q.small = F->UL + t.off;
                q.small_stride = KL;
                q.small_u16 = 0;
                q.wide = F->Bp + bundle_offset(t.m);
                q.wide_stride = H->B.stride;
                q.wide_u16 = 1;
                q.SMALL = 1 << t.j;
                q.WIDE = 1 << t.m;
                q.s1 = H2;
                q.out_trans = 0;
                // M_t[yh][x_lo] = sum_yl B_m[x_lo][yl] Lq[yh][yl] -> RB[off + yh][x_lo]
                d.wide = F->Bp + bundle_offset(t.m);
                d.wide_stride = H->B.stride;
                d.SMALL = 1 << t.j;
                d.WIDE = 1 << t.m;
                d.rows = H2;
                d.lq_trans = 0;
                d.out = F->RB + (int64_t)t.off * H2;
                d.out_s = 1;
                d.out_i = H2;
            } else {
                // Q_t[yh][yl] = sum_{x_hi} A_j[x_hi][yh] V[x_hi][off + yl]
                q.small = F->VR + t.off;
                q.small_stride = KR;
                q.small_u16 = 0;
                q.wide = H->A.rows + (size_t)F->row0 * H->A.stride + bundle_offset(t.j);
                q.wide_stride = H->A.stride;
                q.wide_u16 = 1;
                q.SMALL = 1 << t.m;
                q.WIDE = 1 << t.j;
                q.s1 = H1;
                q.out_trans = 1;
                // N_t[x_hi][yl] = sum_yh A_j[x_hi][yh] Lq[yh][yl] -> LA[x_hi][KL + off + yl]
                d.wide = H->A.rows + (size_t)F->row0 * H->A.stride + bundle_offset(t.j);
                d.wide_stride = H->A.stride;
                d.SMALL = 1 << t.m;
                d.WIDE = 1 << t.j;
                d.rows = H1;
                d.lq_trans = 1;
                d.out = F->LA + KL + t.off;
                d.out_s = Kp;
                d.out_i = 1;
            }
            int lg = 0;
            while ((1 << lg) < q.SMALL) ++lg;
            if (lg > 7) return fail(BDC_ERR_UNSUPPORTED, "factored engine: term with more than 128 small outputs");
            qplan.push_back({ti, lg, q, 1});
            qctas_one += (q.WIDE + 255) / 256;
            td[lg].push_back(d);
        }
        fold.push_back(f);
    }
    // one split count for every q-side product: about 8 CTAs per SM, >= 64 rows a slice
    int QS = 1;
    while (qctas_one > 0 && QS < 64 && qctas_one * QS * 2 <= 8 * H->num_sms && std::min(H1, H2) / (QS * 2) >= 64)
        QS *= 2;
    int64_t qelems = 0;
    for (auto& qp : qplan) qelems += (int64_t)QS * ny;
    BDC_CUDA_TRY(al(&F->qparts, (size_t)std::max<int64_t>(qelems, 1)));
    BDC_CUDA_TRY(al(&F->qsum, (size_t)F->T * ny));
    BDC_CUDA_TRY(al(&F->qacc, (size_t)ny));
    BDC_CUDA_TRY(cudaMemsetAsync(F->qparts, 0, sizeof(double) * std::max<int64_t>(qelems, 1), H->stream));
    int64_t qo = 0;
    for (auto& qp : qplan) {
        fold[qp.term].qoff = qo;
        fold[qp.term].qs = QS;
        const int S = qp.d.s1;
        for (int sp = 0; sp < QS; ++sp) {
            ThinQ q = qp.d;
            q.s0 = (int)((int64_t)S * sp / QS);
            q.s1 = (int)((int64_t)S * (sp + 1) / QS);
            q.out = F->qparts + qo + (int64_t)sp * ny;
            tq[qp.lg].push_back(q);
        }
        qo += (int64_t)QS * ny;
    }
    for (int lg = 0; lg < 8; ++lg) {
        if (!tq[lg].empty()) {
            BDC_CUDA_TRY(cudaMalloc(&F->d_thinq[lg], sizeof(ThinQ) * tq[lg].size()));
            BDC_CUDA_TRY(cudaMemcpy(F->d_thinq[lg], tq[lg].data(), sizeof(ThinQ) * tq[lg].size(), cudaMemcpyHostToDevice));
            F->n_thinq[lg] = (int)tq[lg].size();
        }
        if (!td[lg].empty()) {
            int cta = 0;
            for (auto& d : td[lg]) {
                d.cta_begin = cta;
                cta += (d.rows + kThinDRows - 1) / kThinDRows;
            }
            BDC_CUDA_TRY(cudaMalloc(&F->d_thind[lg], sizeof(ThinD) * td[lg].size()));
            BDC_CUDA_TRY(cudaMemcpy(F->d_thind[lg], td[lg].data(), sizeof(ThinD) * td[lg].size(), cudaMemcpyHostToDevice));
            F->n_thind[lg] = (int)td[lg].size();
            F->ctas_thind[lg] = cta;
        }
    }
    BDC_CUDA_TRY(set_thin_smem(ny));
    for (int lg = 0; lg < 8; ++lg) {
        if (F->n_thinq[lg]) {
            std::vector<GemmDesc> v;
            for (auto& q : tq[lg]) v.push_back(thin_q_desc(q));
            char key[16];
            snprintf(key, sizeof(key), "q%d", lg);
            bdc_status rc = tune_class(
                H, tf, key, v, F->mq[lg], F->use_mq[lg],
                [&] { launch_thin_q(lg, F->d_thinq[lg], F->n_thinq[lg], ny, H->stream, nullptr); },
                "q-side term products", lg);
            if (rc != BDC_OK) return rc;
        }
        if (F->n_thind[lg]) {
            std::vector<GemmDesc> v;
            for (auto& d : td[lg]) v.push_back(thin_d_desc(d, F->lnq_full));
            char key[16];
            snprintf(key, sizeof(key), "d%d", lg);
            bdc_status rc = tune_class(
                H, tf, key, v, F->md[lg], F->use_md[lg],
                [&] {
                    launch_thin_d(lg, F->d_thind[lg], F->n_thind[lg], F->ctas_thind[lg], ny, F->lnq_full, H->stream,
                                  nullptr);
                },
                "D-side term products", lg);
            if (rc != BDC_OK) return rc;
        }
    }
    for (int lg = 0; lg < 8; ++lg) {
        BDC_CUDA_TRY(cudaStreamCreateWithFlags(&F->side[lg], cudaStreamNonBlocking));
        BDC_CUDA_TRY(cudaEventCreateWithFlags(&F->ev_join[lg], cudaEventDisableTiming));
    }
    BDC_CUDA_TRY(cudaEventCreateWithFlags(&F->ev_fork, cudaEventDisableTiming));
    {
        BDC_CUDA_TRY(cudaMalloc(&F->d_fold, sizeof(FoldTerm) * fold.size()));
        BDC_CUDA_TRY(cudaMemcpy(F->d_fold, fold.data(), sizeof(FoldTerm) * fold.size(), cudaMemcpyHostToDevice));
    }

    // ---- the per-term products of each side fused into one launch (per
    // side, and per output-tile width on the D side), used where the tuner
    // times them faster than the per-class launches.  They need 16-byte
    // aligned table rows of >= 16 entries and 2^k / 16 >= 32 threads.
    {
        // (the q kernel runs 256 threads, one per 16 outputs at k = 12 and
        // fewer busy ones below)
        bool qok = k >= 9 && k <= 12, dok = k >= 9 && k <= 14;
        std::vector<ThinQ> all_q;
        for (int lg = 0; lg < 8; ++lg)
            for (auto& q : tq[lg]) {
                const int IT = qthin_it(q.SMALL);
                const int WT = 16 / IT;
                if ((q.SMALL & (q.SMALL - 1)) != 0 || q.WIDE % WT != 0 || (q.WIDE / WT) * (q.SMALL / IT) != ny / 16 ||
                    ((uintptr_t)q.wide & 15) != 0 || (q.wide_stride % 8) != 0 || q.wide_u16 != 1 || q.small_u16 != 0)
                    qok = false;
                all_q.push_back(q);
            }
        std::vector<ThinDF> all_d[4];
        for (int lg = 0; lg < 8; ++lg)
            for (auto& d : td[lg]) {
                if (d.WIDE < 8 || ((uintptr_t)d.wide & 15) != 0 || (d.wide_stride % 8) != 0) dok = false;
                ThinDF f{};
                f.wide = d.wide;
                f.wide_stride = d.wide_stride;
                f.SMALL = d.SMALL;
                f.WIDE = d.WIDE;
                f.rows = d.rows;
                f.lq_trans = d.lq_trans;
                f.out = d.out;
                f.out_s = d.out_s;
                f.out_i = d.out_i;
                f.IT = std::min(d.SMALL, 8);
                f.LPR = std::max(1, std::min(32, d.WIDE / 32));
                const int ng = d.SMALL / f.IT;
                if (f.LPR * ng > 256) dok = false;
                const int rows_per_cta = (256 / (f.LPR * ng)) * kDfRT;
                int cl = 0;
                while ((1 << cl) < f.IT) ++cl;
                for (int r0 = 0; r0 < d.rows; r0 += rows_per_cta) {
                    f.row0 = r0;
                    all_d[cl].push_back(f);
                }
            }
        // the classes of 2 to 64 outputs again in 64-row blocks for k_dthin_mma
        std::vector<ThinDF> all_m[4];
        bool mok[4] = {false, dok, dok, dok};
        for (int lg = 0; lg < 8; ++lg)
            for (auto& d : td[lg]) {
                int cl = 0;
                while ((1 << cl) < std::min(d.SMALL, 8)) ++cl;
                if (cl == 0 || !mok[cl]) continue;
                if (d.SMALL > 64 || d.WIDE % kDmChunk != 0) {
                    mok[cl] = false;
                    continue;
                }
                ThinDF f{};
                f.wide = d.wide;
                f.wide_stride = d.wide_stride;
                f.SMALL = d.SMALL;
                f.WIDE = d.WIDE;
                f.rows = d.rows;
                f.lq_trans = d.lq_trans;
                f.out = d.out;
                f.out_s = d.out_s;
                f.out_i = d.out_i;
                F->dm_smem[cl] = std::max(F->dm_smem[cl], dthin_mma_smem(d.SMALL, d.WIDE));
                for (int r0 = 0; r0 < d.rows; r0 += kDmRows) {
                    f.row0 = r0;
                    all_m[cl].push_back(f);
                }
            }
        int pinned_q = -1, pinned_d = -1, pinned_m = -1, unused = 0;
        tf.get("qf", &pinned_q, &unused);
        tf.get("df", &pinned_d, &unused);
        tf.get("dm", &pinned_m, &unused);  // bit cl: class cl on k_dthin_mma
        if (const char* dm = getenv("BDC_DTHIN")) pinned_m = !strcmp(dm, "mma") ? 14 : 0;  // forces either form
        BDC_CUDA_TRY(cudaMemsetAsync(H->d_st, 0, sizeof(DevState), H->stream));
        if (qok && !all_q.empty()) {
            F->qf_stage = qthin_stage_bytes(all_q);
            BDC_CUDA_TRY(cudaFuncSetAttribute(k_qthin, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              F->qf_stage * kQtStages));
            BDC_CUDA_TRY(cudaMalloc(&F->d_qf, sizeof(ThinQ) * all_q.size()));
            BDC_CUDA_TRY(cudaMemcpy(F->d_qf, all_q.data(), sizeof(ThinQ) * all_q.size(), cudaMemcpyHostToDevice));
            F->n_qf = (int)all_q.size();
            if (pinned_q >= 0) {
                F->use_qf = pinned_q != 0;
            } else {
                const float tc = time_ms(H, [&] { return enqueue_stage(H, ST_QSMALL, -INFINITY); });
                const float tfu = time_ms(H, [&] { return launch_qthin(F->d_qf, F->n_qf, F->qf_stage, H->stream, nullptr); });
                F->use_qf = tfu < tc;
                tf.put("qf", F->use_qf ? 1 : 0, 0);
                if (H->verbose)
                    printf("bdc: tuned q-side term products: %s (one launch %.1f us, per class %.1f us)\n",
                           F->use_qf ? "one launch" : "per class", tfu * 1e3f, tc * 1e3f);
            }
            // the terms of 8..64 small outputs on the FP64 tensor path
            std::vector<ThinQ> q_lo, q_hi;
            bool qmok = ny == 4096;
            for (const ThinQ& x : all_q) {
                if (x.SMALL < 8) {
                    q_lo.push_back(x);
                    continue;
                }
                if (x.SMALL > 64 || x.SMALL * x.WIDE != 4096 || x.WIDE % 64 != 0) qmok = false;
                q_hi.push_back(x);
                F->qm_stage = std::max(F->qm_stage, qmma_stage(x.SMALL, x.WIDE));
            }
            F->qm_stage = (F->qm_stage + 15) & ~15;
            if (F->use_qf && qmok && !q_hi.empty() && 2 * F->qm_stage + 1024 <= 227 * 1024) {
                BDC_CUDA_TRY(cudaFuncSetAttribute(k_qthin_mma, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                  2 * F->qm_stage));
                BDC_CUDA_TRY(cudaMalloc(&F->d_qm, sizeof(ThinQ) * q_hi.size()));
                BDC_CUDA_TRY(cudaMemcpy(F->d_qm, q_hi.data(), sizeof(ThinQ) * q_hi.size(), cudaMemcpyHostToDevice));
                F->n_qm = (int)q_hi.size();
                if (!q_lo.empty()) {
                    F->ql_stage = qthin_stage_bytes(q_lo);
                    BDC_CUDA_TRY(cudaMalloc(&F->d_ql, sizeof(ThinQ) * q_lo.size()));
                    BDC_CUDA_TRY(cudaMemcpy(F->d_ql, q_lo.data(), sizeof(ThinQ) * q_lo.size(), cudaMemcpyHostToDevice));
                    F->n_ql = (int)q_lo.size();
                }
                int pinned_qm = -1;
                tf.get("qm", &pinned_qm, &unused);
                if (const char* qm = getenv("BDC_QTHIN")) pinned_qm = !strcmp(qm, "mma") ? 1 : 0;  // forces either form
                if (pinned_qm >= 0) {
                    F->use_qm = pinned_qm != 0;
                } else {
                    cudaError_t e1 = cudaSuccess, e2 = cudaSuccess;
                    const float t1 = time_ms(H, [&] {
                        return launch_qthin(F->d_qf, F->n_qf, F->qf_stage, H->stream, nullptr);
                    }, &e1);
                    const float t2 = time_ms(H, [&] { return enqueue_qthin_split(H, H->stream, nullptr); }, &e2);
                    BDC_CUDA_TRY(e1);
                    BDC_CUDA_TRY(e2);
                    F->use_qm = t2 < t1;
                    tf.put("qm", F->use_qm ? 1 : 0, 0);
                    if (H->verbose)
                        printf("bdc: tuned q-side terms of 8..64 outputs: %s (with mma.sync %.1f us, CUDA cores %.1f us)\n",
                               F->use_qm ? "mma.sync" : "CUDA cores", t2 * 1e3f, t1 * 1e3f);
                }
            }
        }
        if (dok) {
            const int sm = dthin_smem(k);
            if (sm > 48 * 1024) {
                BDC_CUDA_TRY(cudaFuncSetAttribute(k_dthin<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
                BDC_CUDA_TRY(cudaFuncSetAttribute(k_dthin<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
                BDC_CUDA_TRY(cudaFuncSetAttribute(k_dthin<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
                BDC_CUDA_TRY(cudaFuncSetAttribute(k_dthin<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
            }
            for (int cl = 0; cl < 4; ++cl) {
                if (all_d[cl].empty()) continue;
                BDC_CUDA_TRY(cudaMalloc(&F->d_df[cl], sizeof(ThinDF) * all_d[cl].size()));
                BDC_CUDA_TRY(cudaMemcpy(F->d_df[cl], all_d[cl].data(), sizeof(ThinDF) * all_d[cl].size(),
                                        cudaMemcpyHostToDevice));
                F->n_df[cl] = (int)all_d[cl].size();
            }
            if (pinned_d >= 0) {
                F->use_df = pinned_d != 0;
            } else {
                F->use_df = false;
                const float tc = time_ms(H, [&] { return enqueue_stage(H, ST_DSMALL, -INFINITY); });
                F->use_df = true;
                const float tfu = time_ms(H, [&] { return enqueue_stage(H, ST_DSMALL, -INFINITY); });
                F->use_df = tfu < tc;
                tf.put("df", F->use_df ? 1 : 0, 0);
                if (H->verbose)
                    printf("bdc: tuned D-side term products: %s (fused %.1f us, per class %.1f us)\n",
                           F->use_df ? "fused" : "per class", tfu * 1e3f, tc * 1e3f);
            }
            // classes of the fused launches on the FP64 tensor path
            int dm_bits = 0, dm_max = 0;
            auto dm_ok = [&](int cl) {
                return mok[cl] && !all_m[cl].empty() && F->n_df[cl] > 0 && F->dm_smem[cl] + 1024 <= 227 * 1024;
            };
            for (int cl = 1; cl < 4; ++cl)
                if (dm_ok(cl)) dm_max = std::max(dm_max, F->dm_smem[cl]);
            if (F->use_df && dm_max > 0)
                BDC_CUDA_TRY(cudaFuncSetAttribute(k_dthin_mma, cudaFuncAttributeMaxDynamicSharedMemorySize, dm_max));
            for (int cl = 1; cl < 4 && F->use_df; ++cl) {
                if (!dm_ok(cl)) continue;
                BDC_CUDA_TRY(cudaMalloc(&F->d_dm[cl], sizeof(ThinDF) * all_m[cl].size()));
                BDC_CUDA_TRY(cudaMemcpy(F->d_dm[cl], all_m[cl].data(), sizeof(ThinDF) * all_m[cl].size(),
                                        cudaMemcpyHostToDevice));
                F->n_dm[cl] = (int)all_m[cl].size();
                if (pinned_m >= 0) {
                    F->use_dm[cl] = (pinned_m >> cl) & 1;
                } else {
                    cudaError_t e1 = cudaSuccess, e2 = cudaSuccess;
                    const float tc = time_ms(H, [&] {
                        return launch_dthin(F->d_df[cl], F->n_df[cl], 1 << cl, H->k, F->lnq_full, H->stream, nullptr);
                    }, &e1);
                    const float tm = time_ms(H, [&] {
                        return launch_dthin_mma(F->d_dm[cl], F->n_dm[cl], F->dm_smem[cl], F->lnq_full, H->stream,
                                                nullptr);
                    }, &e2);
                    BDC_CUDA_TRY(e1);
                    BDC_CUDA_TRY(e2);
                    F->use_dm[cl] = tm < tc;
                    if (H->verbose)
                        printf("bdc: tuned D-side terms of class %d (%s outputs): %s (mma.sync %.1f us, CUDA cores %.1f us)\n",
                               cl, cl == 3 ? "8..64" : (cl == 2 ? "4" : "2"), F->use_dm[cl] ? "mma.sync" : "CUDA cores",
                               tm * 1e3f, tc * 1e3f);
                }
                dm_bits |= (int)F->use_dm[cl] << cl;
            }
            if (F->use_df && pinned_m < 0) tf.put("dm", dm_bits, 0);
        }
    }

    // ---- G = LA RB with the BA epilogue; the tile shape is tuned on the
    // zero state (set_p re-initialises everything it touches)
    {
        // (128x128 tiles do not fit the two-CTAs-per-SM register budget of the
        // fused epilogue)
        const int cfgs[3] = {CFG_128x64, CFG_64x128, CFG_64x64};
        int ctas_max = 0;
        for (int c : cfgs) ctas_max = std::max(ctas_max, ((H1 + kCfgBM[c] - 1) / kCfgBM[c]) * ((H2 + kCfgBN[c] - 1) / kCfgBN[c]));
        BDC_CUDA_TRY(al(&F->epart, (size_t)std::max(ctas_max, H->nb_upd) * 8));
        float best = 1e30f;
        int best_cfg = CFG_128x64;
        GemmDesc d = make_desc(op_f64(F->LA, Kp, 0), op_f64(F->RB, H2, 0), nullptr, 0, 0, H1, H2, Kp);
        BaEpilogue ep{};
        ep.n = H->n;
        ep.n2 = H->s.n2;
        ep.hx = F->hx;
        ep.Lt = F->Lt;
        ep.Pw = F->Pw;
        ep.inv_c = H->inv_c;
        ep.part = F->epart;
        ep.eta = 1.0;
        ep.row0 = F->row0;
        // each shape one CTA per tile, or (when the tiles outnumber them) as
        // many CTAs as fit on the SMs at once, each looping over tiles with
        // the next tile's loads in flight during the epilogue
        auto resident = [&](int c) { return H->num_sms * ((kCfgBM[c] * kCfgBN[c] <= 4096) ? 3 : 2); };
        int best_persist = 0;
        const bool pinned = tf.get("g", &best_cfg, &best_persist);
        for (int c : cfgs) {
            if (pinned) break;
            Launch T;
            BDC_CUDA_TRY(make_tile_launch(T, d, c, F->colmax));
            for (int persist = 0; persist < 2; ++persist) {
                if (persist && T.tiles <= resident(c)) break;
                T.grid = persist ? resident(c) : 0;
                const float ms = time_ms(H, [&] { return launch_ba(T, ep, H->stream, H->d_st); });
                if (ms < best) {
                    best = ms;
                    best_cfg = c;
                    best_persist = persist;
                }
            }
            free_launch(T);
        }
        if (!pinned) tf.put("g", best_cfg, best_persist);
        tf.save();
        BDC_CUDA_TRY(make_tile_launch(F->g, d, best_cfg, F->colmax));
        F->g.grid = best_persist ? std::min(F->g.tiles, resident(best_cfg)) : 0;
        F->ctas_g = F->g.grid > 0 ? F->g.grid : F->g.tiles;
        if (H->verbose)
            printf("bdc: tuned G: tile %dx%d, %d of %d tiles hold representatives, %d CTAs, %.1f us%s\n",
                   kCfgBM[best_cfg], kCfgBN[best_cfg], F->g.tiles,
                   ((H1 + kCfgBM[best_cfg] - 1) / kCfgBM[best_cfg]) * ((H2 + kCfgBN[best_cfg] - 1) / kCfgBN[best_cfg]),
                   F->ctas_g, pinned ? 0.f : best * 1e3f, pinned ? " (pinned)" : "");
        BDC_CUDA_TRY(cudaMemsetAsync(F->Pw, 0, sizeof(double) * NX, H->stream));
        BDC_CUDA_TRY(cudaMemsetAsync(F->Lt, 0, sizeof(double) * NX, H->stream));
        BDC_CUDA_TRY(cudaMemsetAsync(H->d_st, 0, sizeof(DevState), H->stream));
        // split slices that the chosen launches never write must read zero
        BDC_CUDA_TRY(cudaMemsetAsync(F->ulpart, 0, sizeof(double) * max_split * H2 * KLa, H->stream));
        BDC_CUDA_TRY(cudaMemsetAsync(F->vrpart, 0, sizeof(double) * max_split * H1 * KRa, H->stream));
    }
    int nq = 0, nd = 0;
    for (int lg = 0; lg < 8; ++lg) {
        nq += F->n_thinq[lg] > 0;
        nd += F->n_thind[lg] > 0;
    }
    if (F->use_qf) nq = (F->use_qm && F->n_ql) ? 2 : 1;
    if (F->use_df) {
        nd = 0;
        for (int cl = 0; cl < 4; ++cl) nd += F->n_df[cl] > 0;
    }
    // G on the int8 tensor cores (bdc_ozaki.cu), with the slicing of its FP64
    // operands, where that times faster than the FP64 product chosen above;
    // BDC_G_KERNEL=dmma or ozaki forces one of the two
    {
        const char* gk = getenv("BDC_G_KERNEL");
        const bool force_fp = gk && !strcmp(gk, "dmma");
        const bool force_oz = gk && !strcmp(gk, "ozaki");
        int pick = -1, unused = 0;
        // a pinned choice (0: FP64, 8 or 16: int8 with that many epilogue
        // warps); a forced int8 G ignores a pinned FP64 one
        const bool has_pick = tf.get("oz", &pick, &unused);
        const bool pinned = has_pick && !(force_oz && pick == 0);
        if (!force_fp && !(pinned && pick == 0)) {
            // an entry of ML (NR) is ln q against a row of B_m (A_j), whose
            // entries add up to C(n2, m) (C(n1, j)); 1 for an identity table
            double cmax = 1.0;
            for (const Term& t : F->terms)
                if (t.left && !t.idB) cmax = std::max(cmax, (double)binom(s.n2, t.m));
                else if (!t.left && !t.idA) cmax = std::max(cmax, (double)binom(s.n1, t.j));
            const OzakiInput in{F->LA, F->RB, Kp, KL, KR, H1, H2, F->colmax.data(), F->lnq_full, H->k, cmax};
            const char* why = nullptr;
            bdc_status rc = ozaki_init(H, in, &F->oz, &why);
            if (rc != BDC_OK) return rc;
            float t_fp = 0.f, t_oz[2] = {0.f, 0.f};
            if (F->oz && pinned) {
                F->oz->epi = pick == 8 ? 8 : 16;
            } else if (F->oz) {
                // both on the zeroed state (the products' cost does not depend
                // on the values); the int8 product with 16 and with 8
                // epilogue warps
                const BaEpilogue ep = make_epilogue(H);
                cudaError_t e = cudaSuccess;
                if (!force_oz) {
                    t_fp = time_ms(H, [&] { return launch_ba(F->g, ep, H->stream, H->d_st); }, &e);
                    BDC_CUDA_TRY(e);
                }
                for (int v = 0; v < 2; ++v) {
                    F->oz->epi = v == 0 ? 16 : 8;
                    t_oz[v] = time_ms(H, [&] {
                        const cudaError_t e1 = ozaki_prepare(F->oz, H->d_st, H->stream);
                        return e1 != cudaSuccess ? e1 : ozaki_product(F->oz, ep, H->d_st, H->stream);
                    }, &e);
                    BDC_CUDA_TRY(e);
                }
                F->oz->epi = t_oz[1] < t_oz[0] ? 8 : 16;
                const bool use = force_oz || std::min(t_oz[0], t_oz[1]) < t_fp;
                tf.put("oz", use ? F->oz->epi : 0, 0);
                tf.save();
                BDC_CUDA_TRY(cudaMemsetAsync(F->Pw, 0, sizeof(double) * NX, H->stream));
                BDC_CUDA_TRY(cudaMemsetAsync(F->Lt, 0, sizeof(double) * NX, H->stream));
                BDC_CUDA_TRY(cudaMemsetAsync(H->d_st, 0, sizeof(DevState), H->stream));
                if (!use) {
                    ozaki_free(F->oz);
                    F->oz = nullptr;
                }
            }
            F->use_oz = F->oz != nullptr;
            if (H->verbose) {
                if (F->use_oz)
                    printf("bdc: G on the int8 tensor cores: %d tiles of %dx%d over %d CTAs, %d epilogue warps, "
                           "%d B shared memory, ring of %d, %d FP64 tile%s%s\n", F->oz->tiles, kOzBM, kOzTN,
                           F->oz->grid, F->oz->epi, F->oz->smem, F->oz->stages, 1 + F->oz->two_tiles,
                           F->oz->two_tiles ? "s" : "", t_oz[0] > 0.f ? "" : " (pinned)");
                else
                    printf("bdc: G stays on the FP64 product: %s\n", why ? why : "timed slower");
                if (t_oz[0] > 0.f)
                    printf("bdc: G timed: FP64 %.1f us, int8 with slicing %.1f us (16 epilogue warps), %.1f us (8)\n",
                           t_fp * 1e3f, t_oz[0] * 1e3f, t_oz[1] * 1e3f);
            }
        }
    }
    // U, V, the split sums; q-side terms; three fold kernels; D-side terms; G
    // (plus the slicing kernel on the int8 path); finalize
    F->launches_per_iter = (F->ul.n > 0) + (F->vr.n > 0) + 1 + nq + 3 + nd + 1 + 1 + (F->use_oz ? 1 : 0);
    BDC_CUDA_TRY(cudaStreamSynchronize(H->stream));
    return BDC_OK;
}

void factored_free(bdc_handle* H) {
    FactoredState* F = H->fac;
    if (!F) return;
    for (double* p : {F->Pw, F->Lt, F->hx, F->LA, F->RB, F->UL, F->VR, F->ulpart, F->vrpart, F->qparts,
                      F->qsum, F->qacc, F->lnq_full, F->epart})
        cudaFree(p);
    cudaFree(F->Bp);
    cudaFree(F->Ddense);
    cudaFree(F->d_rowstart);
    cudaFree(F->rpart);
    cudaFree(F->d_qf);
    cudaFree(F->d_ql);
    cudaFree(F->d_qm);
    for (auto* d : F->d_df) cudaFree(d);
    for (int lg = 0; lg < 8; ++lg) {
        cudaFree(F->d_thinq[lg]);
        cudaFree(F->d_thind[lg]);
        if (F->side[lg]) cudaStreamDestroy(F->side[lg]);
        if (F->ev_join[lg]) cudaEventDestroy(F->ev_join[lg]);
    }
    if (F->ev_fork) cudaEventDestroy(F->ev_fork);
    if (F->graph) cudaGraphExecDestroy(F->graph);
    if (F->cycle) cudaGraphExecDestroy(F->cycle);
    for (auto& m : F->maps)
        if (m.exec) cudaGraphExecDestroy(m.exec);
    cudaFree(F->snap0);
    cudaFree(F->snap1);
    for (Launch* L : {&F->ul, &F->vr, &F->g}) free_launch(*L);
    for (int lg = 0; lg < 8; ++lg) {
        free_launch(F->mq[lg]);
        free_launch(F->md[lg]);
    }
    cudaFree(F->d_fold);
    ozaki_free(F->oz);
    for (auto* d : F->d_dm) cudaFree(d);
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
    ep.Dout = F->dout;
    ep.eta = F->eta;
    ep.row0 = F->row0;
    return ep;
}

// the stages of one iteration (enum Stage), each gated by DevState::done / error

// the fused q side split in two: the terms of fewer than 8 small outputs
// (k_qthin) on a branch beside those of 8 to 64 (k_qthin_mma); neither fills
// the GPU alone
static cudaError_t enqueue_qthin_split(bdc_handle* H, cudaStream_t s, const DevState* st) {
    FactoredState* F = H->fac;
    cudaError_t e;
    if (F->n_ql) {
        if ((e = cudaEventRecord(F->ev_fork, s)) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(F->side[1], F->ev_fork, 0)) != cudaSuccess) return e;
        if ((e = launch_qthin(F->d_ql, F->n_ql, F->ql_stage, F->side[1], st)) != cudaSuccess) return e;
        if ((e = cudaEventRecord(F->ev_join[1], F->side[1])) != cudaSuccess) return e;
    }
    if ((e = launch_qthin_mma(F->d_qm, F->n_qm, F->qm_stage, s, st)) != cudaSuccess) return e;
    return F->n_ql ? cudaStreamWaitEvent(s, F->ev_join[1], 0) : cudaSuccess;
}

static cudaError_t enqueue_stage(bdc_handle* H, int stage, double a) {
    FactoredState* F = H->fac;
    cudaStream_t s = H->stream;
    cudaError_t e = cudaSuccess;
    switch (stage) {
        case ST_QBIG: {
            // U and V are independent: V runs on a branch beside U
            if ((e = cudaEventRecord(F->ev_fork, s)) != cudaSuccess) return e;
            if ((e = cudaStreamWaitEvent(F->side[0], F->ev_fork, 0)) != cudaSuccess) return e;
            if ((e = launch_store(F->vr, F->side[0], H->d_st)) != cudaSuccess) return e;
            if ((e = cudaEventRecord(F->ev_join[0], F->side[0])) != cudaSuccess) return e;
            if ((e = launch_store(F->ul, s, H->d_st)) != cudaSuccess) return e;
            if ((e = cudaStreamWaitEvent(s, F->ev_join[0], 0)) != cudaSuccess) return e;
            const int64_t na = (int64_t)F->KL * F->H2, nb = (int64_t)F->H1h * F->KR;
            k_sum_parts<<<H->num_sms * 4, 256, 0, s>>>(F->ulpart, F->S1, F->KL > 0 ? na : 0, F->UL, F->vrpart,
                                                       F->S2, F->KR > 0 ? nb : 0, F->VR, H->d_st);
            break;
        }
        case ST_QSMALL:
            if (F->use_qf && F->use_qm) return enqueue_qthin_split(H, s, H->d_st);
            if (F->use_qf) return launch_qthin(F->d_qf, F->n_qf, F->qf_stage, s, H->d_st);
            // fork: each size class on its own branch, joined before the fold
            if ((e = cudaEventRecord(F->ev_fork, s)) != cudaSuccess) return e;
            for (int lg = 0; lg < 8; ++lg) {
                if (!F->n_thinq[lg]) continue;
                if ((e = cudaStreamWaitEvent(F->side[lg], F->ev_fork, 0)) != cudaSuccess) return e;
                e = F->use_mq[lg] ? launch_store(F->mq[lg], F->side[lg], H->d_st)
                                  : launch_thin_q(lg, F->d_thinq[lg], F->n_thinq[lg], 1 << H->k, F->side[lg], H->d_st);
                if (e != cudaSuccess) return e;
                if ((e = cudaEventRecord(F->ev_join[lg], F->side[lg])) != cudaSuccess) return e;
                if ((e = cudaStreamWaitEvent(s, F->ev_join[lg], 0)) != cudaSuccess) return e;
            }
            break;
        case ST_FOLD: {
            const int ny = 1 << H->k;
            const int nqs = (F->T * ny + 255) / 256;
            k_qsum<<<nqs < 4096 ? nqs : 4096, 256, 0, s>>>(F->d_fold, F->T, F->qparts, H->k, F->qsum, H->d_st);
            k_fold_acc<<<(ny + 31) / 32, 256, 0, s>>>(F->d_fold, F->T, F->qsum, F->UL, F->KL, F->VR, F->KR,
                                                       F->H1h, F->row0, H->k, F->qacc, H->d_st);
            k_fold_q<<<(ny + 127) / 128, 128, 0, s>>>(F->d_fold, F->T, F->qacc, H->k, H->inv_c, F->lnq_full,
                                                       H->d_lnq, F->RB, F->H2, F->LA, F->Kp, F->KL, F->H1h, F->row0,
                                                       H->d_st);
            break;
        }
        case ST_DSMALL:
            if ((e = cudaEventRecord(F->ev_fork, s)) != cudaSuccess) return e;
            if (F->use_df) {
                // one launch per output-tile width, each on its own branch
                for (int cl = 0; cl < 4; ++cl) {
                    if (!F->n_df[cl]) continue;
                    if ((e = cudaStreamWaitEvent(F->side[cl], F->ev_fork, 0)) != cudaSuccess) return e;
                    e = F->use_dm[cl]
                            ? launch_dthin_mma(F->d_dm[cl], F->n_dm[cl], F->dm_smem[cl], F->lnq_full, F->side[cl], H->d_st)
                            : launch_dthin(F->d_df[cl], F->n_df[cl], 1 << cl, H->k, F->lnq_full, F->side[cl], H->d_st);
                    if (e != cudaSuccess) return e;
                    if ((e = cudaEventRecord(F->ev_join[cl], F->side[cl])) != cudaSuccess) return e;
                    if ((e = cudaStreamWaitEvent(s, F->ev_join[cl], 0)) != cudaSuccess) return e;
                }
                if (F->use_oz) return ozaki_prepare(F->oz, H->d_st, s);
                break;
            }
            for (int lg = 0; lg < 8; ++lg) {
                if (!F->n_thind[lg]) continue;
                if ((e = cudaStreamWaitEvent(F->side[lg], F->ev_fork, 0)) != cudaSuccess) return e;
                e = F->use_md[lg] ? launch_store(F->md[lg], F->side[lg], H->d_st)
                                  : launch_thin_d(lg, F->d_thind[lg], F->n_thind[lg], F->ctas_thind[lg], 1 << H->k,
                                                  F->lnq_full, F->side[lg], H->d_st);
                if (e != cudaSuccess) return e;
                if ((e = cudaEventRecord(F->ev_join[lg], F->side[lg])) != cudaSuccess) return e;
                if ((e = cudaStreamWaitEvent(s, F->ev_join[lg], 0)) != cudaSuccess) return e;
            }
            if (F->use_oz) return ozaki_prepare(F->oz, H->d_st, s);
            break;
        case ST_G:
            if (F->use_oz) return ozaki_product(F->oz, make_epilogue(H), H->d_st, s);
            return launch_ba(F->g, make_epilogue(H), s, H->d_st);
        case ST_FIN:
            k_fac_finalize<<<1, 256, 0, s>>>(F->epart, F->use_oz ? ozaki_partials(F->oz) : F->ctas_g, a, F->eta, H->d_st);
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

cudaError_t factored_enqueue_iteration(bdc_handle* H, double a) { return enqueue_iteration(H, a); }

// the first shift's inputs over every representative (as k_fac_load writes
// them for its own): a shard sets the same p on every rank, so each one
// derives the same shift without an exchange
__global__ void __launch_bounds__(256) k_lnp_all(const double* __restrict__ p, int64_t R, int strict_zero,
                                                 double* __restrict__ part) {
    double mx = -DBL_MAX;
    int zero = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < R; i += (int64_t)gridDim.x * blockDim.x) {
        const double v = p[i];
        if (strict_zero) {
            if (v > 0.0) mx = fmax(mx, log(v));
            continue;
        }
        mx = fmax(mx, (v != 0.0) ? log(v) : 0.0);
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

bdc_status factored_load_p(bdc_handle* H, int strict_zero) {
    FactoredState* F = H->fac;
    const int64_t NX = (int64_t)F->H1h * F->H2;  // the dense rows held
    BDC_CUDA_TRY(cudaMemsetAsync(F->Pw, 0, sizeof(double) * NX, H->stream));
    const int nb = H->nb_upd;
    k_fac_load_rows<<<F->H1h, 256, F->rows_smem, H->stream>>>(F->d_rowstart, H->n, F->row0, H->d_p[0] + F->i0, F->Pw,
                                                              F->Lt, F->rpart, strict_zero);
    if (H->shard_world > 1) {
        // the first shift from every rank's p, not only the held rows
        k_lnp_all<<<nb, 256, 0, H->stream>>>(H->d_p[0], H->R, strict_zero, F->epart);
        k_fac_load_finish<<<1, 32, 0, H->stream>>>(F->epart, nb, H->k, H->d_st);
    } else {
        k_fac_load_finish<<<1, 32, 0, H->stream>>>(F->rpart, F->H1h, H->k, H->d_st);
    }
    BDC_CUDA_TRY(cudaGetLastError());
    return BDC_OK;
}

// ----------------------------------------------- rows over several GPUs
void factored_shard_range(const bdc_handle* H, int* row0, int* rows, int64_t* i0, int64_t* i1) {
    const FactoredState* F = H->fac;
    *row0 = F->row0;
    *rows = F->H1h;
    *i0 = F->i0;
    *i1 = F->i0 + F->Rl;
}

// q side on the held rows: partial sums acc[y] = sum_{held x} |O(x)| e(x) N(x, y)
// of every term (the fold's first two phases), to the host
bdc_status factored_shard_q(bdc_handle* H, double* acc) {
    FactoredState* F = H->fac;
    cudaStream_t s = H->stream;
    BDC_CUDA_TRY(cudaMemsetAsync(&H->d_st->done, 0, sizeof(int), s));
    BDC_CUDA_TRY(enqueue_stage(H, ST_QBIG, -INFINITY));
    BDC_CUDA_TRY(enqueue_stage(H, ST_QSMALL, -INFINITY));
    const int ny = 1 << H->k;
    const int nqs = (F->T * ny + 255) / 256;
    k_qsum<<<nqs < 4096 ? nqs : 4096, 256, 0, s>>>(F->d_fold, F->T, F->qparts, H->k, F->qsum, H->d_st);
    k_fold_acc<<<(ny + 31) / 32, 256, 0, s>>>(F->d_fold, F->T, F->qsum, F->UL, F->KL, F->VR, F->KR, F->H1h, F->row0,
                                               H->k, F->qacc, H->d_st);
    BDC_CUDA_TRY(cudaGetLastError());
    BDC_CUDA_TRY(cudaMemcpyAsync(acc, F->qacc, sizeof(double) * ny, cudaMemcpyDeviceToHost, s));
    BDC_CUDA_TRY(cudaStreamSynchronize(s));
    return BDC_OK;
}

// from the summed acc: ln q, the D side and G with the update on the held
// rows; part5 = this shard's [max D, sum |O| e, max logW, sum |O| p D, zero]
bdc_status factored_shard_d(bdc_handle* H, const double* acc, double* part5) {
    FactoredState* F = H->fac;
    cudaStream_t s = H->stream;
    const int ny = 1 << H->k;
    BDC_CUDA_TRY(cudaMemcpyAsync(F->qacc, acc, sizeof(double) * ny, cudaMemcpyHostToDevice, s));
    k_fold_q<<<(ny + 127) / 128, 128, 0, s>>>(F->d_fold, F->T, F->qacc, H->k, H->inv_c, F->lnq_full, H->d_lnq, F->RB,
                                              F->H2, F->LA, F->Kp, F->KL, F->H1h, F->row0, H->d_st);
    BDC_CUDA_TRY(cudaGetLastError());
    BDC_CUDA_TRY(enqueue_stage(H, ST_DSMALL, -INFINITY));
    BDC_CUDA_TRY(enqueue_stage(H, ST_G, -INFINITY));
    const int nb = F->use_oz ? ozaki_partials(F->oz) : F->ctas_g;
    std::vector<double> part((size_t)nb * 8);
    BDC_CUDA_TRY(cudaMemcpyAsync(part.data(), F->epart, sizeof(double) * part.size(), cudaMemcpyDeviceToHost, s));
    BDC_CUDA_TRY(cudaMemcpyAsync(H->h_st, H->d_st, sizeof(DevState), cudaMemcpyDeviceToHost, s));
    BDC_CUDA_TRY(cudaStreamSynchronize(s));
    if (H->h_st->error) return fail(BDC_ERR_NUMERIC, "sharded iteration: device error %d", H->h_st->error);
    double mD = -DBL_MAX, sE = 0.0, mL = -DBL_MAX, sR = 0.0, zero = 0.0;
    for (int b = 0; b < nb; ++b) {
        mD = std::max(mD, part[(size_t)b * 8 + 0]);
        sE += part[(size_t)b * 8 + 1];
        mL = std::max(mL, part[(size_t)b * 8 + 2]);
        sR += part[(size_t)b * 8 + 3];
        zero = std::max(zero, part[(size_t)b * 8 + 4]);
    }
    part5[0] = mD;
    part5[1] = sE;
    part5[2] = mL;
    part5[3] = sR;
    part5[4] = zero;
    return BDC_OK;
}

// the update's finish from the combined part5 (max, sum, max, sum, max over
// the shards): ln Z, mx, the bound, the stop test and the next shift, the
// same on every shard
bdc_status factored_shard_finish(bdc_handle* H, const double* part5, double a) {
    FactoredState* F = H->fac;
    cudaStream_t s = H->stream;
    double row[8] = {part5[0], part5[1], part5[2], part5[3], part5[4], 0.0, 0.0, 0.0};
    BDC_CUDA_TRY(cudaMemcpyAsync(F->epart, row, sizeof(row), cudaMemcpyHostToDevice, s));
    k_fac_finalize<<<1, 256, 0, s>>>(F->epart, 1, a, 1.0, H->d_st);
    BDC_CUDA_TRY(cudaGetLastError());
    BDC_CUDA_TRY(cudaMemcpyAsync(H->h_st, H->d_st, sizeof(DevState), cudaMemcpyDeviceToHost, s));
    BDC_CUDA_TRY(cudaStreamSynchronize(s));
    if (H->h_st->error)
        return fail(BDC_ERR_NUMERIC, "sharded iteration: exp shift out of range (device error %d)", H->h_st->error);
    return BDC_OK;
}

bdc_status factored_store_p(bdc_handle* H, double* p_out) {
    FactoredState* F = H->fac;
    k_fac_rows<0><<<F->H1h, 256, F->rows_smem, H->stream>>>(F->d_rowstart, H->n, F->row0, F->Pw, p_out + F->i0,
                                                            H->d_st);
    BDC_CUDA_TRY(cudaGetLastError());
    return BDC_OK;
}


static bdc_status rescale(bdc_handle* H, double a);

// One BA map on device vectors: p_in (per representative, sum |O| p = 1; a
// zero entry stays zero) -> p_out.  The bound max_x D(x) and the rate I(p;W)
// of p_in (nats) are left in H->h_st->max_d / rate; with D_out set, D(x) of
// p_in per representative.  Leaves the handle's iterate at p_out.
// the kernels of one map, queued on H->stream: load, iteration, re-scale
// when the iteration flagged an out-of-range shift (the kernels check the
// flag themselves), D gather, store, and the state copied to the host mirror
static cudaError_t enqueue_map(bdc_handle* H, const double* p_in, double* p_out, double* D_out) {
    FactoredState* F = H->fac;
    cudaStream_t s = H->stream;
    cudaError_t e = cudaMemsetAsync(&H->d_st->done, 0, sizeof(int), s);
    if (e != cudaSuccess) return e;
    // (Pw is zero away from the representatives from set-up on: every kernel
    // writes it only there, and the load below rewrites all of them)
    const int nb = H->nb_upd;
    k_fac_load_rows<<<F->H1h, 256, F->rows_smem, s>>>(F->d_rowstart, H->n, F->row0, p_in + F->i0, F->Pw, F->Lt,
                                                      F->rpart, 1);
    k_fac_load_finish<<<1, 32, 0, s>>>(F->rpart, F->H1h, H->k, H->d_st);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    F->dout = D_out ? F->Ddense : nullptr;
    e = enqueue_iteration(H, -INFINITY);
    F->dout = nullptr;
    if (e != cudaSuccess) return e;
    k_fac_rescale<<<nb, 256, 0, s>>>(H->d_reps + F->i0, F->Rl, H->n, F->row0, F->Lt, F->Pw, F->epart, H->d_st, 1);
    k_fac_rescale_finish<<<1, 32, 0, s>>>(F->epart, nb, -INFINITY, H->d_st, 1);
    if (D_out)
        k_fac_rows<1><<<F->H1h, 256, F->rows_smem, s>>>(F->d_rowstart, H->n, F->row0, F->Ddense, D_out + F->i0, H->d_st);
    k_fac_rows<0><<<F->H1h, 256, F->rows_smem, s>>>(F->d_rowstart, H->n, F->row0, F->Pw, p_out + F->i0, H->d_st);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return cudaMemcpyAsync(H->h_st, H->d_st, sizeof(DevState), cudaMemcpyDeviceToHost, s);
}

// One BA map on device vectors: p_in (per representative, sum |O| p = 1; a
// zero entry stays zero) -> p_out.  The bound max_x D(x) and the rate I(p;W)
// of p_in (nats) are left in H->h_st->max_d / rate; with D_out set, D(x) of
// p_in per representative.  The kernels of a map are captured once per
// (p_in, p_out, D_out) into a CUDA graph (the last four are kept), so a map
// costs one graph launch and one synchronisation.
bdc_status factored_map(bdc_handle* H, const double* p_in, double* p_out, double* D_out) {
    FactoredState* F = H->fac;
    const int64_t NX = (int64_t)F->H1h * F->H2;
    if (D_out && !F->Ddense) {
        BDC_CUDA_TRY(cudaMalloc(&F->Ddense, sizeof(double) * NX));
        H->bytes += sizeof(double) * NX;
    }
    cudaGraphExec_t exec = nullptr;
    for (auto& m : F->maps)
        if (m.exec && m.pin == p_in && m.pout == p_out && m.dout == D_out) exec = m.exec;
    if (!exec) {
        // captured on the handle's own stream, launched on the caller's
        cudaStream_t keep = H->stream;
        BDC_CUDA_TRY(cudaStreamSynchronize(keep));
        H->stream = H->own_stream;
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamBeginCapture(H->own_stream, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            e = enqueue_map(H, p_in, p_out, D_out);
            const cudaError_t e2 = cudaStreamEndCapture(H->own_stream, &g);
            if (e == cudaSuccess) e = e2;
        }
        H->stream = keep;
        if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, g, 0);
        if (g) cudaGraphDestroy(g);
        BDC_CUDA_TRY(e);
        auto& slot = F->maps[F->maps_next];
        F->maps_next = (F->maps_next + 1) % 4;
        if (slot.exec) cudaGraphExecDestroy(slot.exec);
        slot.pin = p_in;
        slot.pout = p_out;
        slot.dout = D_out;
        slot.exec = exec;
    }
    BDC_CUDA_TRY(cudaGraphLaunch(exec, H->stream));
    BDC_CUDA_TRY(cudaStreamSynchronize(H->stream));
    if (H->h_st->error) return fail(BDC_ERR_NUMERIC, "factored engine: device error %d", H->h_st->error);
    return BDC_OK;
}

bdc_status factored_recover(bdc_handle* H, double a) {
    if (H->h_st->error != kErrShift) return fail(BDC_ERR_NUMERIC, "factored engine: device error %d", H->h_st->error);
    return rescale(H, a);
}

static bdc_status rescale(bdc_handle* H, double a) {
    FactoredState* F = H->fac;
    k_fac_rescale<<<H->nb_upd, 256, 0, H->stream>>>(H->d_reps + F->i0, F->Rl, H->n, F->row0, F->Lt, F->Pw, F->epart, H->d_st, 0);
    k_fac_rescale_finish<<<1, 32, 0, H->stream>>>(F->epart, H->nb_upd, a, H->d_st, 0);
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
    stats->best_upper_bound = H->h_st->best_ub / ln2;
    stats->best_rate = H->h_st->best_rate / ln2;
    stats->converged = H->h_st->done;
}

// kGraphIters iterations captured once (per threshold a) on the handle's own
// stream and replayed on whatever stream the handle queues on; the device
// done / error flags make iterations past convergence no-ops
constexpr int kGraphIters = 8;

static bdc_status ensure_graph(bdc_handle* H, double a) {
    FactoredState* F = H->fac;
    if (F->graph && F->graph_a == a) return BDC_OK;
    if (F->graph) {
        cudaGraphExecDestroy(F->graph);
        F->graph = nullptr;
    }
    cudaStream_t keep = H->stream;
    H->stream = H->own_stream;
    BDC_CUDA_TRY(cudaStreamSynchronize(keep));
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(H->own_stream, cudaStreamCaptureModeThreadLocal);
    for (int i = 0; i < kGraphIters && e == cudaSuccess; ++i) e = enqueue_iteration(H, a);
    cudaError_t e2 = cudaStreamEndCapture(H->own_stream, &g);
    H->stream = keep;
    if (e == cudaSuccess) e = e2;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&F->graph, g, 0);
    if (g) cudaGraphDestroy(g);
    BDC_CUDA_TRY(e);
    F->graph_a = a;
    return BDC_OK;
}

bdc_status factored_iterate(bdc_handle* H, int64_t max_iters, double a, bdc_stats* stats) {
    FactoredState* F = H->fac;
    BDC_CUDA_TRY(cudaMemsetAsync(&H->d_st->done, 0, sizeof(int), H->stream));
    const long long it0 = H->h_st->iter;
    long long target = it0 + max_iters;
    int64_t chunk = 1;
    for (int guard = 0; guard < 1000000; ++guard) {
        const long long done_iters = H->h_st->iter;
        const int64_t remaining = target - done_iters;
        if (remaining <= 0) break;
        const int64_t c = chunk < remaining ? chunk : remaining;
        // whole graphs for the bulk of the chunk, single iterations for the rest
        const int64_t ng = (c >= kGraphIters) ? c / kGraphIters : 0;
        if (ng > 0) {
            bdc_status rc = ensure_graph(H, a);
            if (rc != BDC_OK) return rc;
        }
        for (int64_t i = 0; i < ng; ++i) BDC_CUDA_TRY(cudaGraphLaunch(F->graph, H->stream));
        for (int64_t i = ng * kGraphIters; i < c; ++i) BDC_CUDA_TRY(enqueue_iteration(H, a));
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
        if (chunk < 256) chunk *= 2;
    }
    fill_stats(H, it0, stats);
    return BDC_OK;
}

// ------------------------------------------------------ accelerated loop
// Nesterov-accelerated exponentiated gradient on the simplex, driven by the
// adjoint of I(p;W): its gradient over the probabilities of the strings is
// dI/dp(x) = D(x) - 1, so the mirror (exponentiated-gradient) step of length
// eta is ln p' = ln y + eta D(y) - ln Z, which for eta = 1 and y = p is the
// BA update.  Per step t (all on the device, kAccSteps steps per graph):
//   y_t     = normalise(exp(x_t + beta_t (x_t - x_{t-1}))),  beta_t = t / (t + 3)
//   D(y_t), I(y_t)                 the fused forward/backward (G epilogue)
//   x_{t+1} = ln y_t + eta D(y_t) - ln Z
// with x the normalised log iterate.  Adaptive restart: when I(y_t) falls
// below I(y_{t-1}), the step is discarded, the momentum is dropped (t = 0)
// and the next point is y = x_t.  Every evaluated y gives a valid bracket
// I(y) <= C <= max_x D(x; y), tracked as best_rate / best_ub; the loop stops
// on the device when best_ub - best_rate < the requested gap.
constexpr int kAccSteps = 8;
constexpr double kAccEta = 1.5;

__device__ __forceinline__ double block_sum256(double v) {
    __shared__ double red[256];
    red[threadIdx.x] = v;
    __syncthreads();
    for (int t = 128; t > 0; t >>= 1) {
        if (threadIdx.x < t) red[threadIdx.x] += red[threadIdx.x + t];
        __syncthreads();
    }
    const double r = red[0];
    __syncthreads();
    return r;
}

__device__ __forceinline__ double block_max256(double v) {
    __shared__ double red[256];
    red[threadIdx.x] = v;
    __syncthreads();
    for (int t = 128; t > 0; t >>= 1) {
        if (threadIdx.x < t) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + t]);
        __syncthreads();
    }
    const double r = red[0];
    __syncthreads();
    return r;
}

__device__ __forceinline__ bool acc_gated(const DevState* st) { return st->error != 0 || st->done; }

// decides what the last evaluation means for the iterate: accept (mode 1),
// restart (mode 2) or nothing yet (mode 0, the fresh start)
__global__ void k_acc_decide(DevState* st) {
    if (acc_gated(st) || threadIdx.x != 0) return;
    if (st->ng_mode < 0) {  // set by the host: nothing evaluated since the start
        st->ng_mode = 0;
        st->ng_t = 0;
        st->ng_prev_rate = -DBL_MAX;
        return;
    }
    if (st->rate >= st->ng_prev_rate) {
        st->ng_mode = 1;
        st->ng_prev_rate = st->rate;
        st->ng_t += 1;
    } else {
        st->ng_mode = 2;
        st->ng_t = 0;
        st->ng_prev_rate = -DBL_MAX;
    }
}

// x_{t-1}, x_t (dense, at representatives) and the extrapolated ln y into Lt;
// block max of ln y
__global__ void __launch_bounds__(256) k_acc_extrap(int64_t nx, int n, int row0, double* __restrict__ xa,
                                                    double* __restrict__ xb, double* __restrict__ Lt,
                                                    double* __restrict__ part, const DevState* st) {
    if (acc_gated(st)) return;
    const int mode = st->ng_mode;
    const double lnz = st->log_z;
    const double beta = (double)st->ng_t / ((double)st->ng_t + 3.0);
    double mx = -DBL_MAX;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nx; i += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t xd = (uint32_t)i;
        if (!is_rep(fac_str(xd, n, row0), n)) continue;
        double y;
        if (mode == 1) {
            const double a_old = xa[xd], a_new = Lt[xd] - lnz;
            xb[xd] = a_old;
            xa[xd] = a_new;
            // an input at exact zero (ln p = -inf) stays there
            y = (a_new == -INFINITY) ? a_new : a_new + beta * (a_new - a_old);
        } else {
            y = xa[xd];
            xb[xd] = y;
        }
        Lt[xd] = y;
        mx = fmax(mx, y);
    }
    mx = block_max256(mx);
    if (threadIdx.x == 0) part[blockIdx.x] = mx;
}

// one warp
__global__ void k_acc_max(const double* __restrict__ part, int nb, DevState* st) {
    if (acc_gated(st)) return;
    const double m = warp_parts<true>(part, nb, 1);
    if (threadIdx.x == 0) st->ng_max = m;
}

// Lt -= max, Pw = |O| exp(Lt); block sums of |O| exp(Lt)
__global__ void __launch_bounds__(256) k_acc_pw(int64_t nx, int n, int row0, double* __restrict__ Lt,
                                                double* __restrict__ Pw, double* __restrict__ part, const DevState* st) {
    if (acc_gated(st)) return;
    const double m = st->ng_max;
    double sum = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nx; i += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t xd = (uint32_t)i, x = fac_str(xd, n, row0);
        if (!is_rep(x, n)) continue;
        const double l = Lt[xd] - m;
        const double o = (double)orbit_size(x, n);
        const double e = exp(l);
        Lt[xd] = l;
        Pw[xd] = o * e;
        sum = fma(o, e, sum);
    }
    sum = block_sum256(sum);
    if (threadIdx.x == 0) part[blockIdx.x] = sum;
}

// ln Z of y and the exp shift of the next update (max ln y + eta * last bound)
// one warp
__global__ void k_acc_setz(const double* __restrict__ part, int nb, double eta, DevState* st) {
    if (acc_gated(st)) return;
    const double s = warp_parts<false>(part, nb, 1);
    if (threadIdx.x != 0) return;
    const double lnz = log(s);
    st->log_z = lnz;
    st->shift = -lnz + eta * st->max_d;
}

// the device-side stop: the bracket of the evaluated points is below the gap
__global__ void k_acc_stop(DevState* st) {
    if (acc_gated(st) || threadIdx.x != 0) return;
    if (st->best_ub - st->best_rate < st->ng_gap) st->done = 1;
}

static cudaError_t enqueue_acc_step(bdc_handle* H, double eta) {
    FactoredState* F = H->fac;
    if (!F->snap0 || !F->snap1) return cudaErrorInvalidValue;  // factored_acc_buffers first
    cudaStream_t s = H->stream;
    const int nb = H->nb_upd;
    k_acc_decide<<<1, 32, 0, s>>>(H->d_st);
    const int64_t nx = (int64_t)F->H1h << H->s.n2;  // the dense positions of the held rows
    k_acc_extrap<<<nb, 256, 0, s>>>(nx, H->n, F->row0, F->snap0, F->snap1, F->Lt, F->epart, H->d_st);
    k_acc_max<<<1, 32, 0, s>>>(F->epart, nb, H->d_st);
    k_acc_pw<<<nb, 256, 0, s>>>(nx, H->n, F->row0, F->Lt, F->Pw, F->epart, H->d_st);
    k_acc_setz<<<1, 32, 0, s>>>(F->epart, nb, eta, H->d_st);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const double keep = F->eta;
    F->eta = eta;
    e = enqueue_iteration(H, -INFINITY);
    F->eta = keep;
    if (e != cudaSuccess) return e;
    k_acc_stop<<<1, 32, 0, s>>>(H->d_st);
    return cudaGetLastError();
}

cudaError_t factored_enqueue_acc_steps(bdc_handle* H, int steps, double eta) {
    for (int i = 0; i < steps; ++i) {
        cudaError_t e = enqueue_acc_step(H, eta);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// the loop's two snapshot vectors (dense, allocated on first use)
bdc_status factored_acc_buffers(bdc_handle* H) {
    FactoredState* F = H->fac;
    if (F->snap0) return BDC_OK;
    const size_t NX = (size_t)F->H1h * F->H2;
    BDC_CUDA_TRY(cudaMalloc(&F->snap0, sizeof(double) * NX));
    BDC_CUDA_TRY(cudaMalloc(&F->snap1, sizeof(double) * NX));
    H->bytes += 2 * sizeof(double) * NX;
    return BDC_OK;
}

// x_t = x_{t-1} = the current normalised log iterate; nothing evaluated yet
__global__ void __launch_bounds__(256) k_acc_init(int64_t nx, int n, int row0, const double* __restrict__ Lt,
                                                  double* __restrict__ xa, double* __restrict__ xb, DevState* st,
                                                  double gap_nats) {
    const double lnz = st->log_z;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nx; i += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t xd = (uint32_t)i;
        if (!is_rep(fac_str(xd, n, row0), n)) continue;
        const double l = Lt[xd] - lnz;
        xa[xd] = l;
        xb[xd] = l;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        st->ng_mode = -1;
        st->ng_gap = gap_nats;
        st->done = 0;
    }
}

bdc_status factored_acc_start(bdc_handle* H, double gap_bits) {
    bdc_status rc = factored_acc_buffers(H);
    if (rc != BDC_OK) return rc;
    FactoredState* F = H->fac;
    k_acc_init<<<H->nb_upd, 256, 0, H->stream>>>((int64_t)F->H1h << H->s.n2, H->n, F->row0, F->Lt, F->snap0, F->snap1, H->d_st,
                                                 gap_bits * 0.69314718055994530942);
    BDC_CUDA_TRY(cudaGetLastError());
    return BDC_OK;
}

double factored_acc_eta() {
    const char* e = getenv("BDC_ACCEL_STEP");
    const double v = (e && *e) ? atof(e) : kAccEta;
    return (v > 0.0 && v <= 4.0) ? v : kAccEta;
}

static bdc_status ensure_cycle_graph(bdc_handle* H, double eta) {
    FactoredState* F = H->fac;
    if (F->cycle && F->cycle_eta == eta) return BDC_OK;
    // the snapshot vectors must exist before the steps are captured
    bdc_status rc = factored_acc_buffers(H);
    if (rc != BDC_OK) return rc;
    if (F->cycle) {
        cudaGraphExecDestroy(F->cycle);
        F->cycle = nullptr;
    }
    cudaStream_t keep = H->stream;
    H->stream = H->own_stream;
    BDC_CUDA_TRY(cudaStreamSynchronize(keep));
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(H->own_stream, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) e = factored_enqueue_acc_steps(H, kAccSteps, eta);
    cudaError_t e2 = cudaStreamEndCapture(H->own_stream, &g);
    H->stream = keep;
    if (e == cudaSuccess) e = e2;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&F->cycle, g, 0);
    if (g) cudaGraphDestroy(g);
    BDC_CUDA_TRY(e);
    F->cycle_eta = eta;
    return BDC_OK;
}

bdc_status factored_accelerate(bdc_handle* H, int64_t max_evals, double gap_bits, bdc_stats* stats) {
    FactoredState* F = H->fac;
    const double ln2 = 0.69314718055994530942;
    const double eta = factored_acc_eta();
    BDC_CUDA_TRY(cudaMemsetAsync(&H->d_st->done, 0, sizeof(int), H->stream));
    BDC_CUDA_TRY(cudaMemcpyAsync(H->h_st, H->d_st, sizeof(DevState), cudaMemcpyDeviceToHost, H->stream));
    BDC_CUDA_TRY(cudaStreamSynchronize(H->stream));
    const long long it0 = H->h_st->iter;
    // a plain step first when the iterate still carries the caller's exact
    // zeros (ln 0 = 0 applies to the first update only)
    if (H->h_st->iter == 0 && max_evals > 0) {
        bdc_status rc = factored_iterate(H, 1, -INFINITY, nullptr);
        if (rc != BDC_OK) return rc;
    }
    bool converged = (H->h_st->best_ub - H->h_st->best_rate) / ln2 < gap_bits;
    if (!converged && H->h_st->iter - it0 < max_evals) {
        bdc_status rc = ensure_cycle_graph(H, eta);
        if (rc != BDC_OK) return rc;
        rc = factored_acc_start(H, gap_bits);
        if (rc != BDC_OK) return rc;
        int64_t chunk = 1;
        for (int guard = 0; guard < 1000000; ++guard) {
            const int64_t remaining = max_evals - (H->h_st->iter - it0);
            // whole graphs while they fit, single steps for the rest
            if (remaining <= 0) break;
            if (remaining >= kAccSteps) {
                const int64_t c = std::min<int64_t>(chunk, remaining / kAccSteps);
                for (int64_t i = 0; i < c; ++i) BDC_CUDA_TRY(cudaGraphLaunch(F->cycle, H->stream));
            } else {
                BDC_CUDA_TRY(factored_enqueue_acc_steps(H, (int)remaining, eta));
            }
            BDC_CUDA_TRY(cudaMemcpyAsync(H->h_st, H->d_st, sizeof(DevState), cudaMemcpyDeviceToHost, H->stream));
            BDC_CUDA_TRY(cudaStreamSynchronize(H->stream));
            if (H->h_st->error == kErrShift) {
                // an exp shift went out of range: finish that evaluation by
                // re-scaling; the next step's decision takes it from there
                rc = rescale(H, -INFINITY);
                if (rc != BDC_OK) return rc;
                BDC_CUDA_TRY(cudaMemcpyAsync(H->h_st, H->d_st, sizeof(DevState), cudaMemcpyDeviceToHost, H->stream));
                BDC_CUDA_TRY(cudaStreamSynchronize(H->stream));
            } else if (H->h_st->error) {
                return fail(BDC_ERR_NUMERIC, "accelerated loop: device error %d", H->h_st->error);
            }
            if (H->h_st->done) break;
            if (chunk < 64) chunk *= 2;
        }
        converged = (H->h_st->best_ub - H->h_st->best_rate) / ln2 < gap_bits;
    }
    BDC_CUDA_TRY(cudaMemsetAsync(&H->d_st->done, 0, sizeof(int), H->stream));
    BDC_CUDA_TRY(cudaStreamSynchronize(H->stream));
    fill_stats(H, it0, stats);
    if (stats) stats->converged = converged;
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
    // algorithmic work of G: one K-long dot product per representative
    out->work_main = 2.0 * (double)H->R * (double)(F->KL + F->KR);
    out->launches = F->launches_per_iter;
    out->iters = iters;
    out->main_kind = F->use_oz ? 2 : 1;
    out->bytes_main = 40.0 * (double)F->Rl;
    return BDC_OK;
}

}  // namespace bdc
