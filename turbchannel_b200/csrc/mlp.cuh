// mlp.cuh -- the learned eddy-viscosity closure: a 6 -> 64 -> 64 -> 1 MLP (SiLU,
// SiLU, softplus) with BF16 weights and activations on the tensor cores
// (mma.sync m16n8k16, FP32 accumulation).  One warp evaluates a tile of 16 samples.
//
// Arithmetic (the CPU oracle oracle/les_oracle.py restates it, roundings included):
//   xb = bf16(x)                       x: 6 features, padded with zeros to 16
//   z1 = W1^T xb + b1,  h1 = silu(z1),  h1b = bf16(h1)
//   z2 = W2^T h1b + b2, h2 = silu(z2),  h2b = bf16(h2)
//   z3 = w3 . h2b + b3 (FP32),          out = softplus(z3)      (nu_t / nu)
// Backward for the loss L = mean((out - y)^2):
//   gz3 = 2 (out - y) / B * sigmoid(z3)
//   gw3 = sum gz3 h2b, gb3 = sum gz3;   gh2 = gz3 w3b
//   gz2 = gh2 * silu'(z2), gz2b = bf16(gz2)
//   gW2 = sum h1b gz2b^T, gb2 = sum gz2b; gh1 = W2 gz2b
//   gz1 = gh1 * silu'(z1), gz1b = bf16(gz1)
//   gW1 = sum xb gz1b^T,  gb1 = sum gz1b
// Weights live in shared memory in the layouts the B operand wants: W1T[n][k]
// (64 x 16, k >= 6 zero), W2T[n][k] = W2[k][n] (forward), W2R[n][k] = W2[n][k]
// (backward, where the roles of the two indices swap).
#pragma once
#include <cuda_bf16.h>

#include "tc_common.cuh"

namespace tc {

constexpr int MLP_IN = 6, MLP_H = 64, MLP_K1 = 16;
// packed FP32 parameter vector: W1[6][64], b1[64], W2[64][64], b2[64], w3[64], b3
constexpr int MLP_OW1 = 0, MLP_OB1 = MLP_OW1 + MLP_IN * MLP_H, MLP_OW2 = MLP_OB1 + MLP_H,
              MLP_OB2 = MLP_OW2 + MLP_H * MLP_H, MLP_OW3 = MLP_OB2 + MLP_H, MLP_OB3 = MLP_OW3 + MLP_H,
              MLP_NPAR = MLP_OB3 + 1;

// Shared-memory image of the network (bf16 matrices, fp32 vectors).
// row strides padded (24, 72 elements) so that the 8 rows a B-fragment load touches
// fall in different shared-memory banks
constexpr int MLP_LD1 = MLP_K1 + 8, MLP_LD2 = MLP_H + 8;
struct alignas(16) MlpSmem {
    alignas(16) __nv_bfloat16 W1T[MLP_H][MLP_LD1];
    alignas(16) __nv_bfloat16 W2T[MLP_H][MLP_LD2];
    alignas(16) __nv_bfloat16 W2R[MLP_H][MLP_LD2];
    float b1[MLP_H], b2[MLP_H], w3[MLP_H];  // w3 already rounded to bf16
    float b3;
};

// Fill from the packed FP32 parameters (cooperatively by the CTA; caller syncs).
__device__ __forceinline__ void mlp_load_smem(MlpSmem& S, const float* __restrict__ P) {
    for (int e = threadIdx.x; e < MLP_H * MLP_K1; e += blockDim.x) {
        const int n = e / MLP_K1, k = e - n * MLP_K1;
        S.W1T[n][k] = __float2bfloat16_rn(k < MLP_IN ? P[MLP_OW1 + k * MLP_H + n] : 0.f);
    }
    for (int e = threadIdx.x; e < MLP_H * MLP_H; e += blockDim.x) {
        const int n = e / MLP_H, k = e - n * MLP_H;
        S.W2T[n][k] = __float2bfloat16_rn(P[MLP_OW2 + k * MLP_H + n]);
        S.W2R[n][k] = __float2bfloat16_rn(P[MLP_OW2 + n * MLP_H + k]);
    }
    for (int e = threadIdx.x; e < MLP_H; e += blockDim.x) {
        S.b1[e] = P[MLP_OB1 + e];
        S.b2[e] = P[MLP_OB2 + e];
        S.w3[e] = __bfloat162float(__float2bfloat16_rn(P[MLP_OW3 + e]));
    }
    if (threadIdx.x == 0) S.b3 = P[MLP_OB3];
}

__device__ __forceinline__ unsigned pack_bf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);  // .x = lo (low half)
    return *reinterpret_cast<const unsigned*>(&v);
}
__device__ __forceinline__ float bf16r(float v) { return __bfloat162float(__float2bfloat16_rn(v)); }

// D = A(16x16 bf16, row) * B(16x8 bf16, col) + D (fp32)
__device__ __forceinline__ void mma_bf16(float d[4], const unsigned a[4], unsigned b0, unsigned b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// B fragment (16 x 8, col layout) of the k-step kk, n-tile nt, from a [n][k] bf16 array.
template <int LD>
__device__ __forceinline__ void ldb(const __nv_bfloat16 (*M)[LD], int kk, int nt, unsigned& b0, unsigned& b1) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const __nv_bfloat16* row = &M[nt * 8 + g][kk * 16 + 2 * t];
    b0 = *reinterpret_cast<const unsigned*>(row);
    b1 = *reinterpret_cast<const unsigned*>(row + 8);
}

// sigmoid with the fast exponential and division intrinsics (a few float ulps, far
// below the BF16 rounding that follows every activation)
__device__ __forceinline__ float sigm(float z) { return __fdividef(1.f, 1.f + __expf(-z)); }
__device__ __forceinline__ float silu(float z) { return z * sigm(z); }
__device__ __forceinline__ float dsilu(float z) {
    const float s = sigm(z);
    return s * (1.f + z * (1.f - s));
}
__device__ __forceinline__ float softplus(float z) { return z > 20.f ? z : log1pf(expf(z)); }

// The closure's inputs in float (the run's inference path; the training samples use
// les_features in double): same invariants, then rounded to BF16 by the network.
__device__ __forceinline__ void les_features_f(const float G[3][3], float sc, float yplus, float* f) {
    float S[3][3], O[3][3];
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            S[i][j] = 0.5f * (G[i][j] + G[j][i]) * sc;
            O[i][j] = 0.5f * (G[i][j] - G[j][i]) * sc;
        }
    float S2[3][3], O2[3][3];
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            S2[i][j] = S[i][0] * S[0][j] + S[i][1] * S[1][j] + S[i][2] * S[2][j];
            O2[i][j] = O[i][0] * O[0][j] + O[i][1] * O[1][j] + O[i][2] * O[2][j];
        }
    float l1 = 0, l2 = 0, l3 = 0, l4 = 0, l5 = 0;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            l1 += S[i][j] * S[j][i];
            l2 += O[i][j] * O[j][i];
            l3 += S2[i][j] * S[j][i];
            l4 += O2[i][j] * S[j][i];
            l5 += O2[i][j] * S2[j][i];
        }
    f[0] = asinhf(l1);
    f[1] = asinhf(l2);
    f[2] = asinhf(l3);
    f[3] = asinhf(l4);
    f[4] = asinhf(l5);
    f[5] = 0.25f * log1pf(yplus);
}

// Accumulator tile 16 x 64: 8 n-tiles of m16n8, element (row g or g+8, col 8 nt + 2t (+1)).
struct Acc64 {
    float c[8][4];
};

// Rows of a C tile -> A fragments (16 x 64 bf16 = 4 k-steps) of the next product.
__device__ __forceinline__ void c_to_a(const Acc64& C, unsigned A[4][4]) {
#pragma unroll
    for (int kk = 0; kk < 4; kk++) {
        A[kk][0] = pack_bf16(C.c[2 * kk][0], C.c[2 * kk][1]);
        A[kk][1] = pack_bf16(C.c[2 * kk][2], C.c[2 * kk][3]);
        A[kk][2] = pack_bf16(C.c[2 * kk + 1][0], C.c[2 * kk + 1][1]);
        A[kk][3] = pack_bf16(C.c[2 * kk + 1][2], C.c[2 * kk + 1][3]);
    }
}

// Forward pass of one 16-sample tile.  ax: A fragment of the features (16 x 16).
// Returns z1, z2 (pre-activations, for the backward pass), the h1b A fragments and
// z3 for the two rows (g, g+8) this lane holds.
__device__ __forceinline__ void mlp_forward_tile(const MlpSmem& S, const unsigned ax[4], Acc64& z1, Acc64& z2,
                                                 unsigned h1a[4][4], float z3[2]) {
    const int lane = threadIdx.x & 31, t = lane & 3;
#pragma unroll
    for (int nt = 0; nt < 8; nt++) {
        const float b0 = S.b1[8 * nt + 2 * t], b1 = S.b1[8 * nt + 2 * t + 1];
        z1.c[nt][0] = b0;
        z1.c[nt][1] = b1;
        z1.c[nt][2] = b0;
        z1.c[nt][3] = b1;
        unsigned w0, w1;
        ldb<MLP_LD1>(S.W1T, 0, nt, w0, w1);
        mma_bf16(z1.c[nt], ax, w0, w1);
    }
    Acc64 h1;
#pragma unroll
    for (int nt = 0; nt < 8; nt++)
#pragma unroll
        for (int e = 0; e < 4; e++) h1.c[nt][e] = silu(z1.c[nt][e]);
    c_to_a(h1, h1a);
#pragma unroll
    for (int nt = 0; nt < 8; nt++) {
        const float b0 = S.b2[8 * nt + 2 * t], b1 = S.b2[8 * nt + 2 * t + 1];
        z2.c[nt][0] = b0;
        z2.c[nt][1] = b1;
        z2.c[nt][2] = b0;
        z2.c[nt][3] = b1;
#pragma unroll
        for (int kk = 0; kk < 4; kk++) {
            unsigned w0, w1;
            ldb<MLP_LD2>(S.W2T, kk, nt, w0, w1);
            mma_bf16(z2.c[nt], h1a[kk], w0, w1);
        }
    }
    // z3 = w3 . bf16(silu(z2)) + b3: partial over this lane's columns, then the quad
    float p0 = 0.f, p1 = 0.f;
#pragma unroll
    for (int nt = 0; nt < 8; nt++)
#pragma unroll
        for (int e = 0; e < 2; e++) {
            const float w = S.w3[8 * nt + 2 * t + e];
            p0 += w * bf16r(silu(z2.c[nt][e]));
            p1 += w * bf16r(silu(z2.c[nt][2 + e]));
        }
    p0 += __shfl_xor_sync(0xffffffffu, p0, 1);
    p0 += __shfl_xor_sync(0xffffffffu, p0, 2);
    p1 += __shfl_xor_sync(0xffffffffu, p1, 1);
    p1 += __shfl_xor_sync(0xffffffffu, p1, 2);
    z3[0] = p0 + S.b3;
    z3[1] = p1 + S.b3;
}

// A fragment of a 16 x 16 feature tile from 16 rows of 6 floats (row r at X + r*ldx;
// rows >= nrow are zero).
__device__ __forceinline__ void feature_fragment(const float* X, int ldx, int nrow, unsigned ax[4]) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    float v[2][4];
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int r = g + 8 * h;
#pragma unroll
        for (int j = 0; j < 2; j++) {
            const int k = 2 * t + j;
            v[h][j] = (r < nrow && k < MLP_IN) ? X[(size_t)r * ldx + k] : 0.f;
            v[h][2 + j] = 0.f;  // k = 2t+8+j >= 8 > 6
        }
    }
    ax[0] = pack_bf16(v[0][0], v[0][1]);
    ax[1] = pack_bf16(v[1][0], v[1][1]);
    ax[2] = 0u;
    ax[3] = 0u;
}

}  // namespace tc
