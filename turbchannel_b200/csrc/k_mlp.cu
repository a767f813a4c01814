// k_mlp.cu -- training and inference kernels of the learned eddy-viscosity closure
// (network and arithmetic: mlp.cuh).
//
//   k_mlp_grad    one pass over a batch: per 64-sample chunk, each warp runs the
//                 forward and backward pass of 16 samples on the tensor cores and
//                 stores its per-sample factors (h1b, gz2b, xb, gz1b) transposed in
//                 shared memory; the CTA then forms the weight gradients of the chunk
//                 as tensor-core products over the 64 samples (dW2 = H1b^T Gz2b,
//                 dW1 = Xb^T Gz1b) accumulated in registers across chunks.  Each CTA
//                 writes one partial gradient; k_mlp_reduce adds them in CTA order
//                 (deterministic).
//   k_mlp_adam    Adam update of the FP32 master parameters.
//   k_mlp_forward inference of a feature array.
#include "kernels.cuh"
#include "mlp.cuh"

namespace tc {

constexpr int MW = 4;         // warps per CTA
constexpr int MCH = 16 * MW;  // samples per chunk

struct MlpTrainSmem {
    MlpSmem net;
    alignas(16) __nv_bfloat16 H1T[MLP_H][MCH + 8];  // h1b^T  [i][s]   (+8: spreads the rows over the banks)
    alignas(16) __nv_bfloat16 G2T[MLP_H][MCH + 8];  // gz2b^T [j][s]
    alignas(16) __nv_bfloat16 G1T[MLP_H][MCH + 8];  // gz1b^T [j][s]
    alignas(16) __nv_bfloat16 XT[MLP_K1][MCH + 8];  // xb^T   [k][s]
    float red[MW][3 * MLP_H + 2];       // per-warp bias / w3 / loss partials
};

// A fragment (16 x 16, row layout) of rows m0.. of a [m][k] bf16 array, k-step kk.
template <int LD>
__device__ __forceinline__ void lda(const __nv_bfloat16 (*M)[LD], int m0, int kk, unsigned a[4]) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const __nv_bfloat16* r0 = &M[m0 + g][kk * 16 + 2 * t];
    const __nv_bfloat16* r1 = &M[m0 + g + 8][kk * 16 + 2 * t];
    a[0] = *reinterpret_cast<const unsigned*>(r0);
    a[1] = *reinterpret_cast<const unsigned*>(r1);
    a[2] = *reinterpret_cast<const unsigned*>(r0 + 8);
    a[3] = *reinterpret_cast<const unsigned*>(r1 + 8);
}

// X: n x 6 features (row-major), Y: n targets (nu*/nu).  part: gridDim.x x (NPAR + 1).
__global__ void __launch_bounds__(MW * 32) k_mlp_grad(const float* __restrict__ P, const float* __restrict__ X,
                                                      const float* __restrict__ Y, long long n, float* __restrict__ part) {
    extern __shared__ __align__(16) unsigned char smraw[];
    MlpTrainSmem& S = *reinterpret_cast<MlpTrainSmem*>(smraw);
    mlp_load_smem(S.net, P);
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
    const float inv_b = 1.f / (float)n;
    float gw3[8][2] = {};
    float gbias = 0.f;  // lanes 0-15: gb1[16 w + lane], lanes 16-31: gb2[16 w + lane - 16]
    float gb3 = 0.f, loss = 0.f;
    float dW2[8][4] = {};  // rows i = 16 w + g (+8), cols j = 8 nt + 2 t (+1)
    float dW1[2][4] = {};  // rows k = g (+8), cols j = 8 (2 w + q) + 2 t (+1)
    const long long nch = (n + MCH - 1) / MCH;
    for (long long ch = blockIdx.x; ch < nch; ch += gridDim.x) {
        // ---- phase 1: this warp's 16 samples ----
        const long long s0 = ch * MCH + 16 * w;
        const int nrow = (int)max(0LL, min(16LL, n - s0));
        unsigned ax[4];
        feature_fragment(X + (nrow > 0 ? s0 * MLP_IN : 0), MLP_IN, nrow, ax);
        Acc64 z1, z2;
        unsigned h1a[4][4];
        float z3[2];
        mlp_forward_tile(S.net, ax, z1, z2, h1a, z3);
        float gz3[2];
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int r = g + 8 * h;
            if (r < nrow) {
                const float out = softplus(z3[h]), y = Y[s0 + r], d = out - y;
                if (t == 0) loss += d * d;
                gz3[h] = 2.f * d * inv_b * sigm(z3[h]);
            } else {
                gz3[h] = 0.f;
            }
        }
        if (t == 0) gb3 += gz3[0] + gz3[1];
        Acc64 gz2;
#pragma unroll
        for (int nt = 0; nt < 8; nt++)
#pragma unroll
            for (int e = 0; e < 2; e++) {
                const int j = 8 * nt + 2 * t + e;
                const float w3 = S.net.w3[j];
                const float h2a = bf16r(silu(z2.c[nt][e])), h2b = bf16r(silu(z2.c[nt][2 + e]));
                gw3[nt][e] += gz3[0] * h2a + gz3[1] * h2b;
                gz2.c[nt][e] = gz3[0] * w3 * dsilu(z2.c[nt][e]);
                gz2.c[nt][2 + e] = gz3[1] * w3 * dsilu(z2.c[nt][2 + e]);
            }
        unsigned g2a[4][4];
        c_to_a(gz2, g2a);
        Acc64 gz1;
#pragma unroll
        for (int nt = 0; nt < 8; nt++) {
            gz1.c[nt][0] = gz1.c[nt][1] = gz1.c[nt][2] = gz1.c[nt][3] = 0.f;
#pragma unroll
            for (int kk = 0; kk < 4; kk++) {
                unsigned b0, b1;
                ldb<MLP_LD2>(S.net.W2R, kk, nt, b0, b1);
                mma_bf16(gz1.c[nt], g2a[kk], b0, b1);
            }
#pragma unroll
            for (int e = 0; e < 4; e++) gz1.c[nt][e] *= dsilu(z1.c[nt][e]);
        }
        // per-sample factors, transposed, into shared memory
        const int cs = 16 * w;
#pragma unroll
        for (int nt = 0; nt < 8; nt++)
#pragma unroll
            for (int e = 0; e < 2; e++) {
                const int j = 8 * nt + 2 * t + e;
                S.H1T[j][cs + g] = __float2bfloat16_rn(silu(z1.c[nt][e]));
                S.H1T[j][cs + g + 8] = __float2bfloat16_rn(silu(z1.c[nt][2 + e]));
                S.G2T[j][cs + g] = __float2bfloat16_rn(gz2.c[nt][e]);
                S.G2T[j][cs + g + 8] = __float2bfloat16_rn(gz2.c[nt][2 + e]);
                S.G1T[j][cs + g] = __float2bfloat16_rn(gz1.c[nt][e]);
                S.G1T[j][cs + g + 8] = __float2bfloat16_rn(gz1.c[nt][2 + e]);
            }
        for (int e = lane; e < 16 * MLP_K1; e += 32) {
            const int r = e / MLP_K1, k = e - r * MLP_K1;
            S.XT[k][cs + r] = __float2bfloat16_rn((r < nrow && k < MLP_IN) ? X[(s0 + r) * MLP_IN + k] : 0.f);
        }
        __syncthreads();
        // ---- phase 2: weight gradients of the 64-sample chunk ----
        {  // bias gradients: sums of the bf16 factors over the chunk's samples
            const __nv_bfloat16* row = lane < 16 ? &S.G1T[16 * w + lane][0] : &S.G2T[16 * w + lane - 16][0];
#pragma unroll 8
            for (int q = 0; q < MCH; q += 2) {
                const float2 v = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(row + q));
                gbias += v.x + v.y;
            }
        }
#pragma unroll
        for (int kk = 0; kk < MCH / 16; kk++) {
            unsigned a[4];
            lda<MCH + 8>(S.H1T, 16 * w, kk, a);
#pragma unroll
            for (int nt = 0; nt < 8; nt++) {
                unsigned b0, b1;
                ldb<MCH + 8>(S.G2T, kk, nt, b0, b1);
                mma_bf16(dW2[nt], a, b0, b1);
            }
            unsigned ak[4];
            lda<MCH + 8>(S.XT, 0, kk, ak);
#pragma unroll
            for (int q = 0; q < 2; q++) {
                unsigned b0, b1;
                ldb<MCH + 8>(S.G1T, kk, 2 * w + q, b0, b1);
                mma_bf16(dW1[q], ak, b0, b1);
            }
        }
        __syncthreads();
    }
    // ---- reduce the per-lane vectors over the 8 row groups, then over the warps ----
#pragma unroll
    for (int nt = 0; nt < 8; nt++)
#pragma unroll
        for (int e = 0; e < 2; e++)
#pragma unroll
            for (int o = 4; o < 32; o <<= 1) gw3[nt][e] += __shfl_xor_sync(0xffffffffu, gw3[nt][e], o);
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        gb3 += __shfl_xor_sync(0xffffffffu, gb3, o);
        loss += __shfl_xor_sync(0xffffffffu, loss, o);
    }
    if (g == 0) {
#pragma unroll
        for (int nt = 0; nt < 8; nt++)
#pragma unroll
            for (int e = 0; e < 2; e++) {
                const int j = 8 * nt + 2 * t + e;
                S.red[w][2 * MLP_H + j] = gw3[nt][e];
            }
        if (t == 0) {
            S.red[w][3 * MLP_H] = gb3;
            S.red[w][3 * MLP_H + 1] = loss;
        }
    }
    __syncthreads();
    float* out = part + (size_t)blockIdx.x * (MLP_NPAR + 1);
    if (lane < 16) out[MLP_OB1 + 16 * w + lane] = gbias;
    else out[MLP_OB2 + 16 * w + lane - 16] = gbias;
    for (int e = threadIdx.x + 2 * MLP_H; e < 3 * MLP_H + 2; e += blockDim.x) {
        float v = 0.f;
        for (int q = 0; q < MW; q++) v += S.red[q][e];
        if (e < 3 * MLP_H) out[MLP_OW3 + e - 2 * MLP_H] = v;
        else if (e == 3 * MLP_H) out[MLP_OB3] = v;
        else out[MLP_NPAR] = v;
    }
#pragma unroll
    for (int nt = 0; nt < 8; nt++)
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const int i = 16 * w + g + 8 * (e >> 1), j = 8 * nt + 2 * t + (e & 1);
            out[MLP_OW2 + i * MLP_H + j] = dW2[nt][e];
        }
#pragma unroll
    for (int q = 0; q < 2; q++)
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const int k = g + 8 * (e >> 1), j = 8 * (2 * w + q) + 2 * t + (e & 1);
            if (k < MLP_IN) out[MLP_OW1 + k * MLP_H + j] = dW1[q][e];
        }
}

// grad[k] = sum over CTAs (in order) of part[cta][k], k <= NPAR (the last: loss sum)
__global__ void k_mlp_reduce(const float* __restrict__ part, int nblk, float* __restrict__ grad) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k > MLP_NPAR) return;
    float s = 0.f;
    for (int b = 0; b < nblk; b++) s += part[(size_t)b * (MLP_NPAR + 1) + k];
    grad[k] = s;
}

__global__ void k_mlp_adam(float* __restrict__ P, float* __restrict__ M, float* __restrict__ V,
                           const float* __restrict__ grad, float lr, float b1, float b2, float eps, float c1, float c2) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= MLP_NPAR) return;
    const float gk = grad[k];
    const float m = b1 * M[k] + (1.f - b1) * gk, v = b2 * V[k] + (1.f - b2) * gk * gk;
    M[k] = m;
    V[k] = v;
    P[k] -= lr * (m / c1) / (sqrtf(v / c2) + eps);
}

__global__ void __launch_bounds__(MW * 32) k_mlp_forward(const float* __restrict__ P, const float* __restrict__ X,
                                                         long long n, float* __restrict__ out) {
    __shared__ MlpSmem S;
    mlp_load_smem(S, P);
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
    const long long ntile = (n + 15) / 16;
    for (long long tile = (long long)blockIdx.x * MW + w; tile < ntile; tile += (long long)gridDim.x * MW) {
        const long long s0 = tile * 16;
        const int nrow = (int)min(16LL, n - s0);
        unsigned ax[4];
        feature_fragment(X + s0 * MLP_IN, MLP_IN, nrow, ax);
        Acc64 z1, z2;
        unsigned h1a[4][4];
        float z3[2];
        mlp_forward_tile(S, ax, z1, z2, h1a, z3);
        if (t == 0) {
            if (g < nrow) out[s0 + g] = softplus(z3[0]);
            if (g + 8 < nrow) out[s0 + g + 8] = softplus(z3[1]);
        }
    }
}

__global__ void k_mlp_loss_acc(float* acc, const float* grad) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *acc += grad[MLP_NPAR];
}
void launch_mlp_loss_acc(float* acc, const float* grad, cudaStream_t s) { k_mlp_loss_acc<<<1, 32, 0, s>>>(acc, grad); }

int mlp_grad_blocks(long long n) {
    const long long nch = (n + MCH - 1) / MCH;
    return (int)std::max<long long>(1, std::min<long long>(nch, 148 * 4));
}
size_t mlp_train_smem() { return sizeof(MlpTrainSmem); }

void launch_mlp_grad(const float* P, const float* X, const float* Y, long long n, float* part, float* grad,
                     cudaStream_t s) {
    const int nb = mlp_grad_blocks(n);
    const size_t smem = sizeof(MlpTrainSmem);
    cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_mlp_grad<<<nb, MW * 32, smem, s>>>(P, X, Y, n, part);
    k_mlp_reduce<<<(MLP_NPAR + 1 + 255) / 256, 256, 0, s>>>(part, nb, grad);
}

void launch_mlp_adam(float* P, float* M, float* V, const float* grad, float lr, int step, cudaStream_t s) {
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
    k_mlp_adam<<<(MLP_NPAR + 255) / 256, 256, 0, s>>>(P, M, V, grad, lr, b1, b2, 1e-8f, c1, c2);
}

void launch_mlp_forward(const float* P, const float* X, long long n, float* out, cudaStream_t s) {
    const long long ntile = (n + 15) / 16;
    const int nb = (int)std::max<long long>(1, std::min<long long>((ntile + MW - 1) / MW, 148 * 8));
    k_mlp_forward<<<nb, MW * 32, 0, s>>>(P, X, n, out);
}

}  // namespace tc
