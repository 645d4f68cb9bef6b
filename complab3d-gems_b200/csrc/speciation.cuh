// speciation.cuh -- shared declarations of the speciation solver and its MLP surrogate.
#pragma once

#include <cuda_bf16.h>

#include "clb_internal.cuh"

namespace clb {

constexpr double EQ_MIN_C = 1e-30, EQ_MAX_C = 10.0, EQ_MIN_LOG = -30.0, EQ_MAX_LOG = 1.0;

// Surrogate network: nc log10 totals -> 64 tanh -> 64 tanh -> ns log10 species. Weights are kept
// in FP32 (master copy, Adam state) and BF16 (tensor-core operands). Matrices are [out][in]
// row-major, inputs padded to 16 and outputs to 16 so every layer is whole m16n8k16 tiles.
constexpr int MLP_H = 64;
constexpr int MLP_IN = 16;   // padded input width
constexpr int MLP_OUT = 16;  // padded output width

struct MlpView {
    const __nv_bfloat16* w1b;  // [64][16]
    const __nv_bfloat16* w2b;  // [64][64]
    const __nv_bfloat16* w3b;  // [16][64]
    const __nv_bfloat16* w2t;  // [64][64] W2 transposed (backward operand)
    const __nv_bfloat16* w3t;  // [64][16] W3 transposed (backward operand)
    const float* b1;           // [64]
    const float* b2;           // [64]
    const float* b3;           // [16]
    const float* in_lo;        // [16] mapminmax ranges of the inputs (log10 totals)
    const float* in_hi;
    const float* out_lo;       // [16] and of the outputs (log10 species)
    const float* out_hi;
    int nc, ns;
    float range_margin;        // inputs may exceed the trained range by this fraction
    float resid_tol;           // relative mass-balance residual a kept answer must meet
    int polish;                // FP64 Newton iterations started from the surrogate's answer
};

struct SpecParams {
    int ns, nc, max_it;
    double tol;
    double S[CLB_MAX_EQ_SPECIES * CLB_MAX_COMPONENTS];
    double logK[CLB_MAX_EQ_SPECIES];
    int comp[CLB_MAX_COMPONENTS];
    int eq[CLB_MAX_EQ_SPECIES];
    int ispec[CLB_MAX_EQ_SPECIES];  // internal species index of tableau row i
};

__device__ __forceinline__ bool eq_solve_nr(const SpecParams& P, const double* cin, double* cout, int* iters,
                                            const double* x0, int max_it);
__device__ __forceinline__ void eq_totals(const SpecParams& P, const double* cin, double* T);

MlpView mlp_view(clb_handle* h);

// the handle keeps SpecParams in raw storage (the handle struct is declared before this header)
#define CLB_SP(h) (*reinterpret_cast<clb::SpecParams*>((h)->sp_storage))

// ------------------------------------------------------------------ tensor-core tiles
// mma.sync m16n8k16, BF16 operands, FP32 accumulators. Fragment ownership (PTX ISA): g = lane/4,
// t = lane%4; A regs {a0,a1,a2,a3} hold (row g, cols 2t..2t+1), (g+8, 2t..), (g, 2t+8..),
// (g+8, 2t+8..); B regs {b0,b1} hold (k 2t..2t+1, col g), (k 2t+8.., col g); C/D {c0..c3} hold
// (row g, cols 2t, 2t+1), (row g+8, cols 2t, 2t+1). The D of two adjacent n-tiles is exactly the
// A fragment of the next layer's k-step, so activations never leave registers.
__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&v);
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// B fragment of W (row-major [n][k] BF16, row stride ld) for n-tile nt and k-step kt
__device__ __forceinline__ void load_b(const __nv_bfloat16* W, int ld, int nt, int kt, int lane, uint32_t& b0,
                                       uint32_t& b1) {
    const int g = lane >> 2, t = lane & 3;
    const __nv_bfloat16* p = W + (nt * 8 + g) * ld + kt * 16 + 2 * t;
    b0 = *reinterpret_cast<const uint32_t*>(p);
    b1 = *reinterpret_cast<const uint32_t*>(p + 8);
}

// Forward pass of one 16-row tile held by the whole warp. A0: the input tile's A fragment
// (inputs padded to 16). Outputs the 16x16 output tile as two D fragments (n-tiles 0 and 1);
// optionally keeps the two hidden layers' activations (FP32, D layout) for the backward pass.
__device__ __forceinline__ void mlp_tile_forward(const MlpView& M, const uint32_t (&A0)[4], int lane, float (&y)[2][4],
                                                 float (*h1)[4] = nullptr, float (*h2)[4] = nullptr) {
    const int t = lane & 3;
    float d[8][4];
    // layer 1: 16 x 64 = X (16 x 16) W1^T
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
        d[nt][0] = d[nt][1] = d[nt][2] = d[nt][3] = 0.f;
        uint32_t b0, b1;
        load_b(M.w1b, MLP_IN, nt, 0, lane, b0, b1);
        mma_bf16(d[nt], A0, b0, b1);
    }
    uint32_t A[4][4];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
        const float bb0 = M.b1[nt * 8 + 2 * t], bb1 = M.b1[nt * 8 + 2 * t + 1];
        const float v0 = tanhf(d[nt][0] + bb0), v1 = tanhf(d[nt][1] + bb1);
        const float v2 = tanhf(d[nt][2] + bb0), v3 = tanhf(d[nt][3] + bb1);
        if (h1) { h1[nt][0] = v0; h1[nt][1] = v1; h1[nt][2] = v2; h1[nt][3] = v3; }
        const int kt = nt >> 1, hi = nt & 1;
        A[kt][0 + 2 * hi] = pack_bf16(v0, v1);
        A[kt][1 + 2 * hi] = pack_bf16(v2, v3);
    }
    // layer 2: 16 x 64 = H1 W2^T
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
        d[nt][0] = d[nt][1] = d[nt][2] = d[nt][3] = 0.f;
#pragma unroll
        for (int kt = 0; kt < 4; ++kt) {
            uint32_t b0, b1;
            load_b(M.w2b, MLP_H, nt, kt, lane, b0, b1);
            mma_bf16(d[nt], A[kt], b0, b1);
        }
    }
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
        const float bb0 = M.b2[nt * 8 + 2 * t], bb1 = M.b2[nt * 8 + 2 * t + 1];
        const float v0 = tanhf(d[nt][0] + bb0), v1 = tanhf(d[nt][1] + bb1);
        const float v2 = tanhf(d[nt][2] + bb0), v3 = tanhf(d[nt][3] + bb1);
        if (h2) { h2[nt][0] = v0; h2[nt][1] = v1; h2[nt][2] = v2; h2[nt][3] = v3; }
        const int kt = nt >> 1, hi = nt & 1;
        A[kt][0 + 2 * hi] = pack_bf16(v0, v1);
        A[kt][1 + 2 * hi] = pack_bf16(v2, v3);
    }
    // layer 3: 16 x 16 = H2 W3^T (linear)
#pragma unroll
    for (int nt = 0; nt < 2; ++nt) {
        y[nt][0] = y[nt][1] = y[nt][2] = y[nt][3] = 0.f;
#pragma unroll
        for (int kt = 0; kt < 4; ++kt) {
            uint32_t b0, b1;
            load_b(M.w3b, MLP_H, nt, kt, lane, b0, b1);
            mma_bf16(y[nt], A[kt], b0, b1);
        }
        const float bb0 = M.b3[nt * 8 + 2 * t], bb1 = M.b3[nt * 8 + 2 * t + 1];
        y[nt][0] += bb0; y[nt][1] += bb1; y[nt][2] += bb0; y[nt][3] += bb1;
    }
}

// A fragment of a 16-row tile whose row r (r = 0..15) is given as 16 floats in xs[r*16 ...]
// (shared memory).
__device__ __forceinline__ void load_a_tile(const float* xs, int lane, uint32_t (&A)[4]) {
    const int g = lane >> 2, t = lane & 3;
    A[0] = pack_bf16(xs[g * 16 + 2 * t], xs[g * 16 + 2 * t + 1]);
    A[1] = pack_bf16(xs[(g + 8) * 16 + 2 * t], xs[(g + 8) * 16 + 2 * t + 1]);
    A[2] = pack_bf16(xs[g * 16 + 2 * t + 8], xs[g * 16 + 2 * t + 9]);
    A[3] = pack_bf16(xs[(g + 8) * 16 + 2 * t + 8], xs[(g + 8) * 16 + 2 * t + 9]);
}

// write a 16x16 D tile pair (n-tiles 0, 1) to ys[r*16 + c]
__device__ __forceinline__ void store_d_tile(float* ys, int lane, const float (&y)[2][4]) {
    const int g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int nt = 0; nt < 2; ++nt) {
        ys[g * 16 + nt * 8 + 2 * t] = y[nt][0];
        ys[g * 16 + nt * 8 + 2 * t + 1] = y[nt][1];
        ys[(g + 8) * 16 + nt * 8 + 2 * t] = y[nt][2];
        ys[(g + 8) * 16 + nt * 8 + 2 * t + 1] = y[nt][3];
    }
}

}  // namespace clb
