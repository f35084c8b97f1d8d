// bdc_ozaki.cuh -- the G product of the factored engine on the integer tensor
// cores (tcgen05.mma kind::i8, accumulators in tensor memory), exact up to a
// stated truncation of its FP64 operands.
//
// G = AL * ML + NR * BR^T, where AL and BR^T are half-table entries (exact
// integers < 2^14) and ML, NR are FP64 (ln q contracted with a table).  With
// one power-of-two exponent e for both FP64 operands (|X| < 2^e):
//     X = 2^e * sum_{s<J} x_s 2^{-7(s+1)} + r,   x_s in [-127, 127],  |r| < 2^{e-7J}
//     a = a_lo + 128 a_hi,                         a_lo in [0, 127]
// and the products regroup by power of two into J + 1 integer sums
//     acc_w = sum_k a_lo x_w + a_hi x_{w+1}   (L part, x from ML)
//           + sum_k x_w b_lo + x_{w+1} b_hi   (R part, x from NR),  x_{-1} = x_J = 0
//     G = sum_{w=-1}^{J-1} 2^{e - 7(w+1)} acc_w  (+ the truncation error)
// Each acc_w is one int8 product with the contraction [lo | hi] against
// [x_w | x_{w+1}], exact in int32 (|acc_w| < 2^23 for K <= 256).  The
// truncation leaves |G - G_exact| < (max row sum of AL + max column sum of
// BR^T) * 2^{e - 7J}, which is below 1e-13 nats of D(x) at n = 24.
#pragma once

#include <cuda.h>

#include "bdc_engine.cuh"

namespace bdc {

constexpr int kOzJ = 7;          // int8 slices of each FP64 operand (49 bits)
constexpr int kOzW = kOzJ + 1;   // accumulators (weights 2^{e - 7a}, a = 0..J)
constexpr int kOzP = kOzJ + 2;   // slots per row of a sliced operand: zero, x_0..x_{J-1}, zero
constexpr int kOzBM = 128;       // tile rows (x_hi): one TMEM lane each
constexpr int kOzTN = 32;        // tile columns (dense x_lo): two buffers of kOzW * kOzTN TMEM columns
constexpr int kOzStages = 6;     // deepest ring of the per-weight operands

// what the product reads from the factored engine (bdc_factored.cu)
struct OzakiInput {
    const double* LA;               // [H1h][Kp] = [AL | NR]
    const double* RB;               // [Kp][H2]  = [ML ; BR^T]
    int Kp, KL, KR, H1h, H2;
    const int* colmax;              // [H2] largest row of a representative per dense column, -1 if none
    const double* lnq;              // [2^k] ln q over every output (the operands are ln q contracted with tables)
    int k;
    double cmax;                    // the largest row sum of a table the FP64 operands contract ln q with:
                                    // |ML|, |NR| <= max |ln q| * cmax
};

struct OzakiG {
    OzakiInput in{};
    int KLp = 0, KRp = 0;           // contraction lengths padded to 32
    int aS = 0, bS = 0, aD = 0, bD = 0;  // 128-byte atom columns: static A / B, per-weight A / B
    uint8_t* As = nullptr;          // [H1h][2 KLp]  [a_lo | a_hi] of AL
    uint8_t* Bs = nullptr;          // [H2][2 KRp]   [b_lo | b_hi] of BR^T
    uint8_t* Ad = nullptr;          // [H1h][P KRp]  slots of NR
    uint8_t* Bd = nullptr;          // [H2][P KLp]   slots of ML (transposed)
    int* d_e = nullptr;             // the exponent e of this iteration's FP64 operands
    // persistent product: one CTA per SM over the 128 x 32 tiles that hold
    // representatives, two TMEM accumulator buffers
    int smem = 0, grid = 0, stages = 0, two_tiles = 0;
    int epi = 16;                   // epilogue warps: 16 (8 columns each) or 8 (16 columns each)
    int* d_tiles = nullptr;         // tile ids (tm * tiles_n + tn)
    int tiles = 0, tiles_n = 0;
    CUtensorMap tmAs, tmBs, tmAd, tmBd;
};

// set-up: *out stays null (with the reason in *why) when the shapes or the
// table entries are outside what the kernel covers; the caller then keeps
// the FP64 product
bdc_status ozaki_init(bdc_handle* H, const OzakiInput& in, OzakiG** out, const char** why);
// rows of block partials the product writes (the finalize's count)
int ozaki_partials(const OzakiG* oz);
void ozaki_free(OzakiG* oz);
// the operands of one G product, queued on s once ML and NR are final: the
// exponent of the FP64 operands and their int8 slices
cudaError_t ozaki_prepare(OzakiG* oz, DevState* st, cudaStream_t s);
// the tensor-core product with the fused BA update; block partials as the
// FP64 product writes them (ep.part, one row of 8 per CTA)
cudaError_t ozaki_product(OzakiG* oz, const BaEpilogue& ep, DevState* st, cudaStream_t s);

}  // namespace bdc
