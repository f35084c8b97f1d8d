// bdc_ozaki.cu -- G = [AL | NR] [ML ; BR^T] with the fused BA update on the
// int8 tensor cores of sm_100a (tcgen05.mma kind::i8, TMEM accumulators, TMA
// loads through an mbarrier pipeline).  The splitting of the operands is
// explained in bdc_ozaki.cuh.
//
// Replaces, like the FP64 product it stands beside (k_mma_ba in
// bdc_factored.cu), the D pass and normalised update of the reference
// (backend/BAA.cu:487-530 compute_log_W_gpu, 590-639 baa_iteration): per
// representative D(x) = h(x) - G(x) / C(n,k), logW = ln p + eta D, and the
// block partials of the update.
//
// One persistent CTA per SM loops over the 128 x 32 tiles of G that hold a
// representative.  Warp 0 lane 0 loads by TMA (the static table slices of a
// tile into one of two buffers, the per-weight slices of the FP64 operands
// through a ring), warp 1 lane 0 issues the MMAs into one of two TMEM
// accumulator buffers (8 weights x 32 columns each), and 8 or 16 epilogue
// warps drain the other buffer (a thread per tile row, its TMEM lane) into an
// FP64 tile in shared memory, then run the BA update over the tile in a
// coalesced order (a warp per 256 contiguous bytes of a dense row).  The
// entropy and log iterate of the next tile are loaded before its
// accumulators are drained.  Every wait on an mbarrier is bounded: on
// time-out the CTA records an error in DevState::error, skips the rest, waits
// (bounded) for its loads and frees its TMEM.
#include <cudaTypedefs.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <vector>

#include "bdc_gemm.cuh"
#include "bdc_ozaki.cuh"

namespace bdc {

constexpr int kErrOzakiWait = 3;         // DevState::error: an mbarrier wait ran out
constexpr int kErrOzakiOperand = 4;      // DevState::error: a non-finite FP64 operand
constexpr uint32_t kOzSpin = 1u << 22;   // polls per wait

// ------------------------------------------------------------- PTX helpers
__device__ __forceinline__ uint32_t sm_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// bounded wait for the phase with the given parity to complete
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (uint32_t i = 0; i < kOzSpin; ++i) {
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

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, uint32_t bar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(dst),
        "l"((uint64_t)map), "r"(bar), "r"(x), "r"(y)
        : "memory");
}

// K-major operand in the 128-byte swizzled canonical layout: rows of 128
// bytes, groups of 8 rows 1024 bytes apart (SBO), the start advanced in
// 32-byte steps along the contraction inside a 128-byte atom
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t addr) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);          // start address
    d |= (uint64_t)1 << 16;                          // leading byte offset (unused by swizzled K-major)
    d |= (uint64_t)(1024 >> 4) << 32;                // stride byte offset: 8 rows x 128 B
    d |= (uint64_t)1 << 46;                          // descriptor version (sm_100)
    d |= (uint64_t)2 << 61;                          // 128-byte swizzle
    return d;
}

// instruction descriptor: s8 x s8 -> s32, both K-major, M x N
__host__ __device__ constexpr uint32_t umma_idesc_i8(int M, int N) {
    return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_i8(uint32_t tmem_d, uint64_t ad, uint64_t bd, uint32_t idesc, uint32_t accum) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(ad), "l"(bd), "r"(idesc), "r"(accum)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr));
}

template <int N>
__device__ __forceinline__ void tmem_ld(uint32_t taddr, uint32_t (&v)[N]) {
    if constexpr (N == 16) tmem_ld16(taddr, v);
    else if constexpr (N == 4) {
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
                     : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3])
                     : "r"(taddr));
    } else {
        static_assert(N == 8, "4, 8 or 16 columns");
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                     : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                     : "r"(taddr));
    }
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// --------------------------------------------------------------- the product
struct OzGeomDev {
    int KLp, KRp;
    int aS, bS, aD, bD;  // atom columns
    int M, N;            // rows (H1h) and columns (H2) of G
    int tiles_n;
    int stages;          // ring depth of the per-weight operands (<= kOzStages)
    int two_tiles;       // 1: two FP64 tiles in shared memory (one epilogue barrier per tile), 0: one (two)
};

constexpr int kOzBuf = kOzW * kOzTN;  // TMEM columns of one accumulator buffer
static_assert(2 * kOzBuf <= 512, "two accumulator buffers exceed tensor memory");
static_assert(kOzW % 2 == 0, "the drain reads accumulator pairs");
// threads of the product with EPI epilogue warps (beside one TMA producer
// warp and one MMA warp)
__host__ __device__ constexpr int oz_threads(int EPI) { return 64 + 32 * EPI; }
constexpr int kOzTileLd = kOzTN + 1;                  // row pitch of an FP64 tile in shared memory
constexpr int kOzTileBytes = kOzBM * kOzTileLd * 8;  // one FP64 tile

// named barrier 1 among the EPI epilogue warps only
__device__ __forceinline__ void epi_sync(int EPI) {
    asm volatile("bar.sync 1, %0;" ::"r"(32 * EPI) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// EPI epilogue warps (8 or 16): four per TMEM lane quadrant or two, each
// draining 32 / (EPI / 4) columns of its 32 rows
template <int EPI>
__global__ void __launch_bounds__(oz_threads(EPI), 1)
k_oz_ba(const __grid_constant__ CUtensorMap tmAs, const __grid_constant__ CUtensorMap tmBs,
          const __grid_constant__ CUtensorMap tmAd, const __grid_constant__ CUtensorMap tmBd, OzGeomDev g,
          const int* __restrict__ tiles, int ntiles, const int* __restrict__ d_e, BaEpilogue ep, DevState* st) {
    constexpr int kOzCols = kOzTN / (EPI / 4);  // columns one epilogue warp drains
    extern __shared__ __align__(1024) uint8_t ozp_smem_raw[];
    __shared__ __align__(8) uint64_t sfull[2], sempty[2], full[kOzStages], empty[kOzStages], tfull[2], tempty[2],
        bar_done;
    __shared__ uint32_t tmem_base_sh;
    __shared__ int abort_sh, skip_sh;
    if (threadIdx.x == 0) skip_sh = (st->done || st->error) ? 1 : 0;
    __syncthreads();
    if (skip_sh) return;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int NS = g.stages;
    const int nmine = (ntiles - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x;
    uint8_t* base = (uint8_t*)(((uintptr_t)ozp_smem_raw + 1023) & ~(uintptr_t)1023);
    const uint32_t sA0 = sm_addr(base);
    const uint32_t bytesA = (uint32_t)g.aS * kOzBM * 128, bytesB = (uint32_t)g.bS * kOzTN * 128;
    const uint32_t sB0 = sA0 + 2 * bytesA;
    const uint32_t ring0 = sB0 + 2 * bytesB;
    const uint32_t stageA = (uint32_t)g.aD * kOzBM * 128, stageB = (uint32_t)g.bD * kOzTN * 128;
    const uint32_t stageBytes = stageA + stageB;
    // two FP64 tiles [kOzBM][kOzTileLd] after the ring: the drain of one tile
    // writes one while the pass of the previous tile reads the other
    double* gt = (double*)(base + (ring0 - sA0) + (size_t)NS * stageBytes);

    if (threadIdx.x == 0) {
        for (int i = 0; i < 2; ++i) {
            mbar_init(sm_addr(&sfull[i]), 1);
            mbar_init(sm_addr(&sempty[i]), 1);
            mbar_init(sm_addr(&tfull[i]), 1);
            mbar_init(sm_addr(&tempty[i]), EPI);
        }
        for (int i = 0; i < NS; ++i) {
            mbar_init(sm_addr(&full[i]), 1);
            mbar_init(sm_addr(&empty[i]), 1);
        }
        mbar_init(sm_addr(&bar_done), 1);
        abort_sh = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sm_addr(&tmem_base_sh)),
                     "r"(512u)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base_sh;
    auto aborted = [&]() { return *(volatile int*)&abort_sh != 0; };
    auto give_up = [&]() { atomicExch(&abort_sh, 1); };

    double mD = -DBL_MAX, sE = 0.0, mL = -DBL_MAX, sR = 0.0, zero = 0.0;
    // producer bookkeeping for the bounded drain on an abort
    int last_use[kOzStages], last_static[2];
    for (int i = 0; i < kOzStages; ++i) last_use[i] = -1;
    last_static[0] = last_static[1] = -1;

    if (warp == 0) {
        if (lane == 0) {
            int wc = 0;
            for (int it = 0; it < nmine && !aborted(); ++it) {
                const int t = tiles[blockIdx.x + it * gridDim.x];
                const int m0 = (t / g.tiles_n) * kOzBM, n0 = (t % g.tiles_n) * kOzTN;
                const int sb = it & 1;
                if (it >= 2 && !mbar_wait(sm_addr(&sempty[sb]), ((it >> 1) - 1) & 1)) {
                    give_up();
                    break;
                }
                const uint32_t sfb = sm_addr(&sfull[sb]);
                mbar_expect_tx(sfb, bytesA + bytesB);
                for (int c = 0; c < g.aS; ++c) tma_load_2d(sA0 + sb * bytesA + c * kOzBM * 128, &tmAs, sfb, 128 * c, m0);
                for (int c = 0; c < g.bS; ++c)
                    tma_load_2d(sB0 + sb * bytesB + c * kOzTN * 128, &tmBs, sfb, 128 * c, n0);
                last_static[sb] = it >> 1;
                bool ok = true;
                for (int a = 0; a < kOzW; ++a, ++wc) {
                    const int s = wc % NS, use = wc / NS;
                    if (use > 0 && !mbar_wait(sm_addr(&empty[s]), (use - 1) & 1)) {
                        ok = false;
                        break;
                    }
                    const uint32_t fb = sm_addr(&full[s]);
                    const uint32_t dA = ring0 + s * stageBytes, dB = dA + stageA;
                    mbar_expect_tx(fb, stageBytes);
                    for (int c = 0; c < g.aD; ++c) tma_load_2d(dA + c * kOzBM * 128, &tmAd, fb, a * g.KRp + 128 * c, m0);
                    for (int c = 0; c < g.bD; ++c)
                        tma_load_2d(dB + c * kOzTN * 128, &tmBd, fb, a * g.KLp + 128 * c, n0);
                    last_use[s] = use;
                }
                if (!ok) {
                    give_up();
                    break;
                }
            }
        }
        __syncwarp();
    } else if (warp == 1) {
        if (lane == 0) {
            const uint32_t idesc = umma_idesc_i8(kOzBM, kOzTN);
            int wc = 0;
            for (int it = 0; it < nmine && !aborted(); ++it) {
                const int tb = it & 1, sb = it & 1;
                if (it >= 2 && !mbar_wait(sm_addr(&tempty[tb]), ((it >> 1) - 1) & 1)) {
                    give_up();
                    break;
                }
                if (!mbar_wait(sm_addr(&sfull[sb]), (it >> 1) & 1)) {
                    give_up();
                    break;
                }
                tc_fence_after();
                const uint32_t sA = sA0 + sb * bytesA, sB = sB0 + sb * bytesB;
                bool ok = true;
                for (int a = 0; a < kOzW; ++a, ++wc) {
                    const int s = wc % NS, use = wc / NS;
                    if (!mbar_wait(sm_addr(&full[s]), use & 1) || aborted()) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t dA = ring0 + s * stageBytes, dB = dA + stageA;
                    const uint32_t tacc = tmem + (uint32_t)(tb * kOzBuf + a * kOzTN);
                    uint32_t accum = 0;
                    for (int kb = 0; kb < 2 * g.KLp; kb += 32) {
                        const uint32_t off = (uint32_t)(kb >> 7), in = (uint32_t)(kb & 127);
                        umma_i8(tacc, umma_desc_sw128(sA + off * kOzBM * 128 + in),
                                umma_desc_sw128(dB + off * kOzTN * 128 + in), idesc, accum);
                        accum = 1;
                    }
                    for (int kb = 0; kb < 2 * g.KRp; kb += 32) {
                        const uint32_t off = (uint32_t)(kb >> 7), in = (uint32_t)(kb & 127);
                        umma_i8(tacc, umma_desc_sw128(dA + off * kOzBM * 128 + in),
                                umma_desc_sw128(sB + off * kOzTN * 128 + in), idesc, accum);
                        accum = 1;
                    }
                    umma_commit(sm_addr(&empty[s]));
                }
                if (!ok) {
                    give_up();
                    break;
                }
                umma_commit(sm_addr(&sempty[sb]));
                umma_commit(sm_addr(&tfull[tb]));
            }
            umma_commit(sm_addr(&bar_done));  // every MMA issued above has completed
        }
        __syncwarp();
    } else {
        // ---- epilogue warps.  Drain: TMEM lane quadrant q (warp % 4), the
        // warp's share of the columns, one tile row per thread, into an FP64
        // tile in shared memory.  Pass: element (row, col) = (et / 32 + EPI u,
        // lane), so that a warp reads and writes 256 contiguous bytes of a
        // dense row.  With two tiles in shared memory one barrier per tile:
        // the drain of tile it writes buffer it & 1, which the pass of tile
        // it - 2 was the last to read; with one tile a second barrier before
        // the drain.
        constexpr int PER = kOzBM * kOzTN / (32 * EPI);  // elements per thread in the pass
        const int q = warp & 3;
        const int part = (warp - 2) >> 2;
        const int r = q * 32 + lane;      // the tile row this thread drains
        const int et = threadIdx.x - 64;  // 0 .. 32 EPI - 1 in the pass
        const double shift = st->shift;
        const double lnz = st->log_z;
        const double inv_z = exp(-lnz);
        const int e = *d_e;
        // the entropy, log iterate and weighted iterate of a tile's pass
        // elements, loaded before its accumulators are drained; bit u of reps:
        // element u is a representative
        double hv[PER], lv[PER], pv[PER];
        uint32_t reps = 0;
        auto preload = [&](int it) {
            const int t = tiles[blockIdx.x + it * gridDim.x];
            const int m0 = (t / g.tiles_n) * kOzBM, n = (t % g.tiles_n) * kOzTN + lane;
            reps = 0;
#pragma unroll
            for (int u = 0; u < PER; ++u) {
                const int m = m0 + (et >> 5) + u * EPI;
                const uint32_t xd = ((uint32_t)m << ep.n2) | (uint32_t)n;
                const uint32_t xg = xd + ((uint32_t)ep.row0 << ep.n2);
                const uint32_t x = (xg & ~low_mask(ep.n2)) | reverse_bits(xg & low_mask(ep.n2), ep.n2);
                const bool rep = (m < g.M) && (n < g.N) && is_rep(x, ep.n);
                reps |= (uint32_t)rep << u;
                hv[u] = rep ? __ldg(ep.hx + xd) : 0.0;
                lv[u] = rep ? ep.Lt[xd] : 0.0;
                pv[u] = rep ? ep.Pw[xd] : 0.0;
            }
        };
        if (nmine > 0) preload(0);
        for (int it = 0; it < nmine; ++it) {
            const int tb = it & 1;
            const bool got = mbar_wait(sm_addr(&tfull[tb]), (it >> 1) & 1) && !aborted();
            if (!got) give_up();
            tc_fence_after();
            double* gtb = gt + (g.two_tiles ? tb : 0) * (kOzBM * kOzTileLd);
            if (!g.two_tiles) epi_sync(EPI);  // the previous pass is done with the one tile
            if (got) {
                // four columns at a time, so that few registers are held
                // beside the preloaded values
#pragma unroll 1
                for (int c0 = 0; c0 < kOzCols; c0 += 4) {
                    double gsum[4] = {0.0, 0.0, 0.0, 0.0};
                    const uint32_t trow =
                        tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(tb * kOzBuf + part * kOzCols + c0);
#pragma unroll
                    for (int b = kOzW / 2 - 1; b >= 0; --b) {
                        uint32_t v0[4], v1[4];
                        tmem_ld<4>(trow + (uint32_t)(2 * b * kOzTN), v0);
                        tmem_ld<4>(trow + (uint32_t)((2 * b + 1) * kOzTN), v1);
                        // 2^{e - 7(2b+1)} from its exponent bits (e >= -900, so normal)
                        const double w = __hiloint2double((1023 + e - 7 * (2 * b + 1)) << 20, 0);
                        tmem_wait_ld();
#pragma unroll
                        for (int j = 0; j < 4; ++j)
                            gsum[j] = fma((double)((int32_t)v0[j] * 128 + (int32_t)v1[j]), w, gsum[j]);
                    }
#pragma unroll
                    for (int j = 0; j < 4; ++j) gtb[r * kOzTileLd + part * kOzCols + c0 + j] = gsum[j];
                }
            }
            // this warp's part of the TMEM buffer is free for the tile after next
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(sm_addr(&tempty[tb]));
            epi_sync(EPI);
            if (aborted()) break;  // uniform: read after the barrier
            const int t = tiles[blockIdx.x + it * gridDim.x];
            const int m0 = (t / g.tiles_n) * kOzBM, n = (t % g.tiles_n) * kOzTN + lane;
#pragma unroll
            for (int u = 0; u < PER; ++u) {
                if (!((reps >> u) & 1u)) continue;
                const int row = (et >> 5) + u * EPI;
                const uint32_t xd = ((uint32_t)(m0 + row) << ep.n2) | (uint32_t)n;
                const uint32_t xg = xd + ((uint32_t)ep.row0 << ep.n2);
                const uint32_t x = (xg & ~low_mask(ep.n2)) | reverse_bits(xg & low_mask(ep.n2), ep.n2);
                const double o = (double)orbit_size(x, ep.n);
                const double pw = pv[u];
                const double D = hv[u] - gtb[row * kOzTileLd + lane] * ep.inv_c;
                if (ep.Dout) ep.Dout[xd] = D;
                // exact zeros of the caller's distribution (Lt = NaN) take ln p = 0
                // (backend/BAA.cu:573-580)
                const bool zero_in = (lv[u] != lv[u]);
                const double lnp = zero_in ? 0.0 : lv[u] - lnz;
                const double lw = lnp + ep.eta * D - shift;
                const double ex = exp(lw);
                ep.Lt[xd] = lw;
                ep.Pw[xd] = o * ex;
                mD = fmax(mD, D);
                mL = fmax(mL, lw);
                sE = fma(o, ex, sE);
                sR = fma(pw * inv_z, D, sR);
                if (zero_in) zero = 1.0;
            }
            if (it + 1 < nmine) preload(it + 1);
        }
    }

    // ---- teardown: every MMA done, then the partials, the loads, the TMEM
    const bool mma_done = mbar_wait(sm_addr(&bar_done), 0);
    tc_fence_after();
    if (!mma_done) give_up();
    __syncthreads();
    const bool ran = !aborted();
    if (!ran && threadIdx.x == 0) st->error = kErrOzakiWait;
    __shared__ double red[5][oz_threads(EPI) / 32];
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
        for (int w = 1; w < oz_threads(EPI) / 32; ++w) {
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
    if (!ran && warp == 0 && lane == 0) {
        for (int s = 0; s < NS; ++s)
            if (last_use[s] >= 0) (void)mbar_wait(sm_addr(&full[s]), last_use[s] & 1);
        for (int b = 0; b < 2; ++b)
            if (last_static[b] >= 0) (void)mbar_wait(sm_addr(&sfull[b]), last_static[b] & 1);
    }
    __syncthreads();
    tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512u) : "memory");
}

// ------------------------------------------------------ operand preparation
// The J truncated base-128 digits of v 2^{-e} (|v| < 2^e), sign included:
// with N = trunc(v 2^{7J - e}) (a power-of-two scaling, exact, then a
// truncating conversion, exact since |N| < 2^{7J}), digit s is the sign of v
// times bits [7(J-1-s), 7(J-s)) of |N| -- the digits that repeated
// "multiply by 128, truncate, subtract" would give.  Four values' digit s
// packed into one 32-bit word per call.
__device__ __forceinline__ uint32_t oz_pack4(const long long (&N)[4], int s) {
    uint32_t w = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const unsigned long long a = (unsigned long long)(N[j] < 0 ? -N[j] : N[j]);
        const int d = (int)((a >> (7 * (kOzJ - 1 - s))) & 127u);
        w |= (uint32_t)(uint8_t)(int8_t)(N[j] < 0 ? -d : d) << (8 * j);
    }
    return w;
}

// 4 values -> their J digit slices as 4-byte words dst[s * pitch] (s < J)
__device__ __forceinline__ void oz_slice4(const double (&v)[4], double scale, uint8_t* dst, int pitch) {
    long long N[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) N[j] = __double2ll_rz(v[j] * scale);
#pragma unroll
    for (int s = 0; s < kOzJ; ++s) *(uint32_t*)(dst + (size_t)s * pitch) = oz_pack4(N, s);
}

// The operands' exponent e (max |X| < 2^e, frexp) from the bound |ML|, |NR|
// <= max |ln q| * cmax: each operand entry is ln q summed against a table row
// whose entries add up to at most cmax.  Every block of the slicing launch
// reduces the 2^k values of ln q (from L2) itself; false on a non-finite ln q.
__device__ __forceinline__ bool oz_exponent(const double* __restrict__ lnq, int ny, double cmax, int* e_out) {
    __shared__ double red[8];
    // eight independent maxima, so that eight loads per thread are in flight
    double mu[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    int y = threadIdx.x;
    for (; y + 7 * 256 < ny; y += 8 * 256) {
#pragma unroll
        for (int u = 0; u < 8; ++u) mu[u] = fmax(mu[u], fabs(__ldg(lnq + y + u * 256)));
    }
    for (; y < ny; y += 256) mu[0] = fmax(mu[0], fabs(__ldg(lnq + y)));
    double m = mu[0];
#pragma unroll
    for (int u = 1; u < 8; ++u) m = fmax(m, mu[u]);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) m = fmax(m, __shfl_xor_sync(0xFFFFFFFFu, m, off));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    m = red[0];
    for (int w = 1; w < 8; ++w) m = fmax(m, red[w]);
    // headroom for the rounding of the FP64 operands (sums of at most cmax
    // terms, relative error far below 2^-30), so that |X| < 2^e holds for the
    // computed values too
    m = m * cmax * (1.0 + 0x1p-30);
    if (!isfinite(m)) return false;
    int e = 0;
    if (m > 0.0) frexp(m, &e);  // m = f 2^e, f in [0.5, 1)
    // raising e keeps |X| < 2^e; the weights 2^{e - 7a} stay normal numbers
    *e_out = e < -900 ? -900 : e;
    return true;
}

// NR (LA columns KL + r) -> Ad[m][slot 1 + s][r]; one thread per (row, 4 r),
// over blocks [b0, b0 + nb) of the launch
__device__ __forceinline__ void oz_slice_a(const double* __restrict__ LA, int Kp, int KL, int KR, int rows, int KRp,
                                           uint8_t* __restrict__ Ad, double scale, int b0, int nb) {
    const int chunks = KRp / 4;
    const int64_t total = (int64_t)rows * chunks;
    for (int64_t i = (blockIdx.x - b0) * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)nb * blockDim.x) {
        const int m = (int)(i / chunks), c = (int)(i % chunks);
        double v[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int r = c * 4 + j;
            v[j] = (r < KR) ? LA[(int64_t)m * Kp + KL + r] : 0.0;
        }
        oz_slice4(v, scale, Ad + (int64_t)m * kOzP * KRp + KRp + c * 4, KRp);
    }
}

// ML (RB rows k < KL, column n) -> Bd[n][slot 1 + s][k]: a block covers 32
// columns from n0 and 32 rows from k0; thread (column c, rows k0 + 4 kq ..
// + 3) loads its four values (a warp reads 32 adjacent columns of one row at
// a time) and writes their slices, four bytes per slot
__device__ __forceinline__ void oz_slice_b(const double* __restrict__ RB, int KL, int cols, int KLp,
                                           uint8_t* __restrict__ Bd, double scale, int n0, int k0) {
    const int c = threadIdx.x % 32, kq = threadIdx.x / 32;  // 256 threads: 32 columns x 8 row quads
    if (n0 + c >= cols) return;
    double v[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int k = k0 + 4 * kq + j;
        v[j] = (k < KL) ? RB[(int64_t)k * cols + n0 + c] : 0.0;
    }
    oz_slice4(v, scale, Bd + (int64_t)(n0 + c) * kOzP * KLp + KLp + k0 + 4 * kq, KLp);
}

// the exponent and both slicings in one launch: blocks [0, nb_b) the 32 x 32
// tiles of ML (strip-major), the rest NR; block 0 publishes e for the product
__global__ void __launch_bounds__(256) k_oz_slice(const double* __restrict__ RB, const double* __restrict__ LA, int Kp,
                                                  int KL, int KR, int rows, int cols, int KLp, int KRp,
                                                  uint8_t* __restrict__ Ad, uint8_t* __restrict__ Bd, int nb_b,
                                                  const double* __restrict__ lnq, int ny, double cmax,
                                                  int* __restrict__ d_e, DevState* st) {
    if (st->done || st->error) return;
    int e = 0;
    if (!oz_exponent(lnq, ny, cmax, &e)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) st->error = kErrOzakiOperand;
        return;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *d_e = e;
    const double scale = ldexp(1.0, 7 * kOzJ - e);
    if ((int)blockIdx.x < nb_b) {
        const int strips = (cols + 31) / 32;
        oz_slice_b(RB, KL, cols, KLp, Bd, scale, ((int)blockIdx.x % strips) * 32, ((int)blockIdx.x / strips) * 32);
    } else {
        oz_slice_a(LA, Kp, KL, KR, rows, KRp, Ad, scale, nb_b, (int)gridDim.x - nb_b);
    }
}

// the integer operands, once: As[m] = [lo | hi] of AL[m][k] (LA columns k <
// KL), Bs[n] = [lo | hi] of BR^T[r][n] (RB rows KL + r); flag set when an
// entry does not fit two digits
__global__ void k_oz_static(const double* __restrict__ LA, const double* __restrict__ RB, int Kp, int KL, int KR,
                            int rows, int cols, int KLp, int KRp, uint8_t* __restrict__ As, uint8_t* __restrict__ Bs,
                            int* __restrict__ bad) {
    const int64_t na = (int64_t)rows * KLp, nb = (int64_t)cols * KRp;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < na + nb; i += (int64_t)gridDim.x * blockDim.x) {
        double v;
        uint8_t* lo;
        int len;
        if (i < na) {
            const int m = (int)(i / KLp), k = (int)(i % KLp);
            v = (k < KL) ? LA[(int64_t)m * Kp + k] : 0.0;
            lo = As + (int64_t)m * 2 * KLp + k;
            len = KLp;
        } else {
            const int64_t j = i - na;
            const int n = (int)(j / KRp), r = (int)(j % KRp);
            v = (r < KR) ? RB[(int64_t)(KL + r) * cols + n] : 0.0;
            lo = Bs + (int64_t)n * 2 * KRp + r;
            len = KRp;
        }
        const int iv = (int)v;
        if ((double)iv != v || iv < 0 || iv >= 128 * 127) atomicExch(bad, 1);
        lo[0] = (uint8_t)(iv & 127);
        lo[len] = (uint8_t)((iv >> 7) & 127);
    }
}

// ------------------------------------------------------------------- host
static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    }
    return fn;
}

// a 2-D byte tensor of `rows` rows of `row_bytes` bytes, boxes of 128 bytes x box_rows
static bool make_map(CUtensorMap* map, const void* base, uint64_t row_bytes, uint64_t rows, uint32_t box_rows) {
    auto fn = encode_fn();
    if (!fn) return false;
    const cuuint64_t dims[2] = {row_bytes, rows};
    const cuuint64_t strides[1] = {row_bytes};
    const cuuint32_t box[2] = {128, box_rows};
    const cuuint32_t estr[2] = {1, 1};
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void*>(base), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

void ozaki_free(OzakiG* oz) {
    if (!oz) return;
    cudaFree(oz->As);
    cudaFree(oz->Bs);
    cudaFree(oz->Ad);
    cudaFree(oz->Bd);
    cudaFree(oz->d_e);
    cudaFree(oz->d_tiles);
    delete oz;
}

int ozaki_partials(const OzakiG* oz) { return oz->grid; }

// tile ids (tm * tiles_n + tn) of BM x bn tiles that hold a representative
static std::vector<int> rep_tiles(const OzakiInput& in, int bn, int* tiles_n) {
    const int tiles_m = (in.H1h + kOzBM - 1) / kOzBM;
    *tiles_n = (in.H2 + bn - 1) / bn;
    std::vector<int> ids;
    for (int tm = 0; tm < tiles_m; ++tm)
        for (int tn = 0; tn < *tiles_n; ++tn) {
            int mx = -1;
            for (int c = tn * bn; c < std::min(in.H2, (tn + 1) * bn); ++c) mx = std::max(mx, in.colmax[c]);
            if (mx >= tm * kOzBM) ids.push_back(tm * *tiles_n + tn);
        }
    return ids;
}

bdc_status ozaki_init(bdc_handle* H, const OzakiInput& in, OzakiG** out, const char** why) {
    *out = nullptr;
    *why = nullptr;
    auto round32 = [](int v) { return (v + 31) / 32 * 32; };
    if (in.KL < 1 || in.KR < 1) {
        *why = "a part of the contraction is empty";
        return BDC_OK;
    }
    const int KLp = round32(in.KL), KRp = round32(in.KR);
    if (KLp > 256 || KRp > 256) {
        *why = "contraction longer than 256";
        return BDC_OK;
    }
    if (!encode_fn()) {
        *why = "cuTensorMapEncodeTiled unavailable";
        return BDC_OK;
    }
    OzakiG* oz = new OzakiG();
    oz->in = in;
    oz->KLp = KLp;
    oz->KRp = KRp;
    oz->aS = (2 * KLp + 127) / 128;
    oz->bS = (2 * KRp + 127) / 128;
    oz->aD = (2 * KRp + 127) / 128;
    oz->bD = (2 * KLp + 127) / 128;
    int dev_smem = 0;
    BDC_CUDA_TRY(cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, H->device));
    // the deepest ring (<= kOzStages, >= 2) that fits beside two FP64 tiles,
    // else beside one
    for (oz->two_tiles = 1; oz->two_tiles >= 0; --oz->two_tiles) {
        for (oz->stages = kOzStages; oz->stages >= 2; --oz->stages) {
            oz->smem = 1024 + 2 * (oz->aS * kOzBM + oz->bS * kOzTN) * 128 +
                       oz->stages * (oz->aD * kOzBM + oz->bD * kOzTN) * 128 + (1 + oz->two_tiles) * kOzTileBytes;
            if (oz->smem + 2048 <= dev_smem) break;
        }
        if (oz->stages >= 2) break;
    }
    if (oz->smem + 2048 > dev_smem) {
        ozaki_free(oz);
        *why = "tile operands exceed shared memory";
        return BDC_OK;
    }
    const int rows = in.H1h, cols = in.H2;
    cudaStream_t s = H->stream;
    auto al = [&](uint8_t** p, size_t bytes) -> cudaError_t {
        H->bytes += bytes;
        cudaError_t e = cudaMalloc(p, bytes);
        if (e == cudaSuccess) e = cudaMemsetAsync(*p, 0, bytes, s);
        return e;
    };
    BDC_CUDA_TRY(al(&oz->As, (size_t)rows * 2 * KLp));
    BDC_CUDA_TRY(al(&oz->Bs, (size_t)cols * 2 * KRp));
    BDC_CUDA_TRY(al(&oz->Ad, (size_t)rows * kOzP * KRp));
    BDC_CUDA_TRY(al(&oz->Bd, (size_t)cols * kOzP * KLp));
    BDC_CUDA_TRY(cudaMalloc(&oz->d_e, sizeof(int)));
    BDC_CUDA_TRY(cudaMemsetAsync(oz->d_e, 0, sizeof(int), s));
    {
        int* bad = nullptr;
        BDC_CUDA_TRY(cudaMalloc(&bad, sizeof(int)));
        BDC_CUDA_TRY(cudaMemsetAsync(bad, 0, sizeof(int), s));
        k_oz_static<<<H->num_sms * 4, 256, 0, s>>>(in.LA, in.RB, in.Kp, in.KL, in.KR, rows, cols, KLp, KRp, oz->As,
                                                   oz->Bs, bad);
        BDC_CUDA_TRY(cudaGetLastError());
        int hb = 0;
        BDC_CUDA_TRY(cudaMemcpyAsync(&hb, bad, sizeof(int), cudaMemcpyDeviceToHost, s));
        BDC_CUDA_TRY(cudaStreamSynchronize(s));
        cudaFree(bad);
        if (hb) {
            ozaki_free(oz);
            *why = "a table entry does not fit two base-128 digits";
            return BDC_OK;
        }
    }
    // tiles that hold a representative
    {
        std::vector<int> idsP = rep_tiles(in, kOzTN, &oz->tiles_n);
        oz->tiles = (int)idsP.size();
        oz->grid = std::min(oz->tiles, H->num_sms);
        if (oz->tiles > 0) {
            BDC_CUDA_TRY(cudaMalloc(&oz->d_tiles, sizeof(int) * idsP.size()));
            BDC_CUDA_TRY(cudaMemcpy(oz->d_tiles, idsP.data(), sizeof(int) * idsP.size(), cudaMemcpyHostToDevice));
        }
    }
    const bool ok = make_map(&oz->tmAs, oz->As, 2 * KLp, rows, kOzBM) &&
                    make_map(&oz->tmAd, oz->Ad, (uint64_t)kOzP * KRp, rows, kOzBM) &&
                    make_map(&oz->tmBs, oz->Bs, 2 * KRp, cols, kOzTN) &&
                    make_map(&oz->tmBd, oz->Bd, (uint64_t)kOzP * KLp, cols, kOzTN);
    if (!ok) {
        ozaki_free(oz);
        *why = "tensor map encoding failed";
        return BDC_OK;
    }
    BDC_CUDA_TRY(cudaFuncSetAttribute(k_oz_ba<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, oz->smem));
    BDC_CUDA_TRY(cudaFuncSetAttribute(k_oz_ba<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, oz->smem));
    *out = oz;
    return BDC_OK;
}

cudaError_t ozaki_prepare(OzakiG* oz, DevState* st, cudaStream_t s) {
    const OzakiInput& in = oz->in;
    const int nb_b = ((in.H2 + 31) / 32) * (oz->KLp / 32);
    const int64_t work_a = (int64_t)in.H1h * (oz->KRp / 4);
    const int nb_a = (int)std::max<int64_t>(1, std::min<int64_t>((work_a + 255) / 256, 148 * 8));
    k_oz_slice<<<nb_b + nb_a, 256, 0, s>>>(in.RB, in.LA, in.Kp, in.KL, in.KR, in.H1h, in.H2, oz->KLp, oz->KRp, oz->Ad,
                                          oz->Bd, nb_b, in.lnq, 1 << in.k, in.cmax, oz->d_e, st);
    return cudaGetLastError();
}

cudaError_t ozaki_product(OzakiG* oz, const BaEpilogue& ep, DevState* st, cudaStream_t s) {
    const OzakiInput& in = oz->in;
    if (oz->tiles == 0) return cudaGetLastError();
    const OzGeomDev gp{oz->KLp, oz->KRp, oz->aS, oz->bS, oz->aD, oz->bD, in.H1h, in.H2, oz->tiles_n, oz->stages,
                       oz->two_tiles};
    if (oz->epi == 16)
        k_oz_ba<16><<<oz->grid, oz_threads(16), oz->smem, s>>>(oz->tmAs, oz->tmBs, oz->tmAd, oz->tmBd, gp, oz->d_tiles,
                                                               oz->tiles, oz->d_e, ep, st);
    else
        k_oz_ba<8><<<oz->grid, oz_threads(8), oz->smem, s>>>(oz->tmAs, oz->tmBs, oz->tmAd, oz->tmBd, gp, oz->d_tiles,
                                                             oz->tiles, oz->d_e, ep, st);
    return cudaGetLastError();
}

}  // namespace bdc
