// bdc_gemm.cuh -- FP64 tiled matrix products for the factored engine.
//
// C(m, n) = alpha * sum_k A(m, k) B(k, n) (+ C) on the CUDA cores in FP64
// FMA (the tensor cores have no FP64 path on sm_100).  Operands are logical
// matrices over device memory of three kinds: FP64, uint16 half-table
// entries (exact small integers, widened on load) and the identity.  Element
// (r, c) of an operand lives at ptr[r * ld + c] or, transposed, ptr[c * ld + r].
//
// Kernels:
//   k_gemm_tile<128,128>  8x8 outputs per thread, used for the big products
//   k_gemm_tile<64,64>    4x4 outputs per thread
//   k_gemm_rows           few output rows (<= 8): one output column per
//                         thread, B staged in shared memory
// All launches are "grouped": one launch runs a list of products (GemmDesc)
// and CTA i finds its product through a prefix table of tile counts.
#pragma once

#include "bdc_common.cuh"

namespace bdc {

enum OpKind : int { OP_F64 = 0, OP_U16 = 1, OP_EYE = 2 };

struct Operand {
    const void* ptr = nullptr;
    int64_t ld = 0;
    int kind = OP_F64;
    int trans = 0;  // 0: (r,c) at ptr[r*ld+c]; 1: at ptr[c*ld+r]
};

struct GemmDesc {
    Operand A;        // M x K
    Operand B;        // K x N
    double* C;        // element (m,n) at C[m*ldc_m + n*ldc_n]
    int64_t ldc_m, ldc_n;
    int M, N, K;
    double alpha;
    int accumulate;   // C += alpha AB instead of C = alpha AB
    int tiles_m, tiles_n;  // filled by the planner
    int tile_begin;        // first CTA of this product in its launch
};

// The BA epilogue of the D-side product G = LA * RB (see bdc_factored.cu).
struct BaEpilogue {
    int n;                       // string length; x = m * H2 + col
    int n2;
    const double* __restrict__ hx;  // h(x) at representatives
    double* Lt;                  // log of the unnormalised iterate (in place)
    double* Pw;                  // |O(x)| * exp(Lt - shift) (in place)
    double inv_c;
    double* part;                // per-CTA partials [ctas][4]
    const DevState* st;
    double* Dout;                // optional: D(x) at every representative (dense layout)
    double eta;                  // step of the exponentiated-gradient update: ln p' = ln p + eta D - ln Z
                                 // (1 is the BA update)
    int row0;                    // global x_hi of the product's row 0 (a shard of the rows; 0 on one GPU)
};

}  // namespace bdc
