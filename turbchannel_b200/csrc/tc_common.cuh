// tc_common.cuh -- types and device building blocks shared by the sm_100a kernels
// of turbchannel_b200 and by the host orchestration.  Internal, not part of the ABI.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/turbch.h"

namespace tc {

// ---------------------------------------------------------------------------
// Plain data passed to kernels by value
// ---------------------------------------------------------------------------
struct Geom {
    int NX, NY, NZ, NXY;
    long long N;  // cells (or nodes)
    int NXH;      // NX/2 + 1 : kx range of the half spectrum
    int scheme, visc_type, turb, stab_type, fd_mode, low_modes;
    double visc, sour_dpdx, inv_ls, hx, hy, inv_hx, inv_hy, area;
    // collocated pressure normalisation: 0 shift sum(p vol) hx hy / area
    // (collocated_AB3/func_global.h:163-170), 1 shift sum(p vol) / area
    // (collocated_SRK/func_global.h:130-137)
    int norm_srk = 0;
};

// Mesh-derived arrays (device pointers into one allocation).  Staggered arrays
// follow struct main_params (staggered/config.h:58-72) in the working type T;
// collocated ones follow collocated_AB3/data_global.h:113-116 (double).  The
// double copies serve the double-precision banded solves of the mixed mode.
// PC: per-plane reciprocals of the staggered stencils, 8 per plane (precomputed on
// the host so the per-cell code has no division): [0] 1/DZ[z], [1] 2/(DZ[z]+DZ[z-1])
// (DZ[-1] = 0), [2] 2/(DZ[z]+DZ[z+1]) (DZ[NZ] = 0), [3] 1/DZ[z-1] (0 at z = 0),
// [4] VV4 convective scale -1/(32 (DZ-DZW/9) hx hy), [5] VV4 w scale -GCZ/(32 hx hy).
constexpr int TC_PC = 8;
// FK (mixed precision): per plane the 24 constants of the flux kernels' interior-plane
// stencils (stencil_vv4_int.cuh), each stored twice (a float2 for the packed arithmetic):
// TC_FK floats per plane.  FK64 (FP64, VV4): the same constants once, TC_FK64 doubles.
constexpr int TC_FK = 48, TC_FK64 = 24;
template <typename T>
struct MeshDev {
    const T *ZZ, *DZ, *DZW, *GC1, *GC2, *GCZ, *KERG, *MAT_A, *cellh, *PC;
    const float* FK = nullptr;
    const double* FK64 = nullptr;
    const double *dZZ, *dDZ, *dDZW, *dKERG, *dMAT_A, *dcellh;
    double MAT_D[6];
    double KERG_norm2;
};

struct ModeTabs {
    const double* cosx;  // cos(2 pi kx / NX),  kx = 0..NX/2
    const double* cosy;  // cos(2 pi ky / NY),  ky = 0..NY-1
    const double* sinx;  // sin(pi kx / NX)
    const double* siny;  // sin(pi ky / NY)
};

constexpr int FFT_MAXF = 24;
struct FftPlan {
    int n, nf;
    int fac[FFT_MAXF];
};

// aligned to its size so that loads and stores are single 8/16-byte accesses
template <typename T>
struct alignas(2 * sizeof(T)) cplx {
    T x, y;
};

// four consecutive elements as one (float) or two (double) 16-byte read-only loads;
// the address must be 16-byte aligned
template <typename T>
struct Acc4 {
    T v[4];
};
template <typename T>
__device__ __forceinline__ Acc4<T> ld4(const T* p) {
    Acc4<T> r;
    if constexpr (sizeof(T) == 4) {
        const float4 q = __ldg(reinterpret_cast<const float4*>(p));
        r.v[0] = q.x; r.v[1] = q.y; r.v[2] = q.z; r.v[3] = q.w;
    } else {
        const double2 q0 = __ldg(reinterpret_cast<const double2*>(p));
        const double2 q1 = __ldg(reinterpret_cast<const double2*>(p) + 1);
        r.v[0] = q0.x; r.v[1] = q0.y; r.v[2] = q1.x; r.v[3] = q1.y;
    }
    return r;
}

template <typename T>
__host__ __device__ __forceinline__ cplx<T> cmul(cplx<T> a, cplx<T> b) {
    return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}

// ---------------------------------------------------------------------------
// Async global->shared copies (LDGSTS).  Sizes 4, 8 or 16 bytes.
// ---------------------------------------------------------------------------
template <int BYTES>
__device__ __forceinline__ void cp_async(void* smem, const void* gmem) {
    unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(sa), "l"(gmem), "n"(BYTES) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// ---------------------------------------------------------------------------
// mbarrier and TMA tiled tensor loads into this CTA's shared memory (no cluster
// multicast; the tensor map covers this GPU's memory only).
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Wait for the phase of `bar` with the given parity; false after `limit` polls (the
// caller records an error instead of waiting for ever).
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity, int limit = 1 << 22) {
    for (int it = 0; it < limit; it++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
// Order this thread's earlier generic-proxy shared-memory accesses before later
// async-proxy (TMA) writes to the same memory.
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
// One box of a 3-D tiled tensor map into shared memory at `dst` (128-byte aligned),
// complete_tx on `bar`.  x * element size must be a multiple of 16 bytes.
__device__ __forceinline__ void tma_load_3d(void* dst, const void* tmap, int x, int y, int z, unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(
            smem_u32(dst)),
        "l"(tmap), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Block-wide sum; result valid in thread 0.  sbuf: >= 32 doubles of shared memory.
__device__ __forceinline__ double block_sum(double v, double* sbuf) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) sbuf[wid] = v;
    __syncthreads();
    double r = 0;
    if (wid == 0) {
        r = lane < nw ? sbuf[lane] : 0.0;
        r = warp_sum(r);
    }
    return r;
}

// Deterministic grid reduction: every block stores its partial, the last block to
// arrive sums all partials in index order and stores the total (then re-arms the
// ticket for the next launch).  Thread 0 of each block passes its partial.
// grid_sum_finish_at: the same over several launches of one stream that share the
// ticket: block `bid` of `nb` in all (the last launch's last block finishes).
__device__ __forceinline__ void grid_sum_finish_at(double partial, double* partials, unsigned* ticket, double* out,
                                                   double* sbuf, unsigned bid, unsigned nb) {
    __shared__ unsigned s_last;
    if (threadIdx.x == 0) {
        partials[bid] = partial;
        __threadfence();
        unsigned t = atomicAdd(ticket, 1u);
        s_last = (t == nb - 1);
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    double s = 0;
    for (unsigned i = threadIdx.x; i < nb; i += blockDim.x) s += ((volatile double*)partials)[i];
    s = block_sum(s, sbuf);
    if (threadIdx.x == 0) {
        *out = s;
        *ticket = 0u;
    }
}
__device__ __forceinline__ void grid_sum_finish(double partial, double* partials, unsigned* ticket, double* out,
                                                double* sbuf) {
    grid_sum_finish_at(partial, partials, ticket, out, sbuf, blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z),
                       gridDim.x * gridDim.y * gridDim.z);
}

__device__ __forceinline__ int wrapi(int i, int n) {
    while (i < 0) i += n;
    while (i >= n) i -= n;
    return i;
}

// ---------------------------------------------------------------------------
// Shared-memory Stockham FFT (radix 4, 2, 3), textbook Cooley-Tukey.
// nl lines of length P.n at stride ls (complex elements) in shared memory;
// tw[k] = exp(-2 pi i k / n), k < n.  sign -1 forward, +1 inverse (unnormalised).
// All threads of the block take part; the result buffer is returned.
// ---------------------------------------------------------------------------
template <typename T, int R>
__device__ __forceinline__ void dft_small(cplx<T>* v, int sign) {
    if (R == 2) {
        cplx<T> a = v[0];
        v[0] = {a.x + v[1].x, a.y + v[1].y};
        v[1] = {a.x - v[1].x, a.y - v[1].y};
    } else if (R == 4) {
        cplx<T> t0 = {v[0].x + v[2].x, v[0].y + v[2].y};
        cplx<T> t1 = {v[0].x - v[2].x, v[0].y - v[2].y};
        cplx<T> t2 = {v[1].x + v[3].x, v[1].y + v[3].y};
        T dr = v[1].x - v[3].x, di = v[1].y - v[3].y;
        cplx<T> t3 = {-sign * di, sign * dr};  // (v1 - v3) * (sign i)
        v[0] = {t0.x + t2.x, t0.y + t2.y};
        v[2] = {t0.x - t2.x, t0.y - t2.y};
        v[1] = {t1.x + t3.x, t1.y + t3.y};
        v[3] = {t1.x - t3.x, t1.y - t3.y};
    } else {  // R == 3
        const T s3 = (T)0.86602540378443864676372317075294;
        cplx<T> t1 = {v[1].x + v[2].x, v[1].y + v[2].y};
        cplx<T> t2 = {v[1].x - v[2].x, v[1].y - v[2].y};
        cplx<T> m = {v[0].x - (T)0.5 * t1.x, v[0].y - (T)0.5 * t1.y};
        cplx<T> e = {-sign * s3 * t2.y, sign * s3 * t2.x};
        v[0] = {v[0].x + t1.x, v[0].y + t1.y};
        v[1] = {m.x + e.x, m.y + e.y};
        v[2] = {m.x - e.x, m.y - e.y};
    }
}

template <typename T, int R>
__device__ __forceinline__ void fft_pass(const cplx<T>* in, cplx<T>* out, int n, int Ns, int nl, int ls,
                                         const cplx<T>* __restrict__ tw, int sign) {
    const int nR = n / R, step = n / (Ns * R), total = nl * nR;
    for (int b = threadIdx.x; b < total; b += blockDim.x) {
        const int l = b / nR, j = b - l * nR;
        const int k = j % Ns;
        const cplx<T>* src = in + l * ls;
        cplx<T>* dst = out + l * ls;
        cplx<T> v[R];
#pragma unroll
        for (int r = 0; r < R; r++) {
            cplx<T> a = src[j + r * nR];
            if (r > 0 && k > 0) {
                cplx<T> w = tw[r * k * step];
                if (sign > 0) w.y = -w.y;
                a = cmul(a, w);
            }
            v[r] = a;
        }
        dft_small<T, R>(v, sign);
        const int d = (j / Ns) * Ns * R + k;
#pragma unroll
        for (int r = 0; r < R; r++) dst[d + r * Ns] = v[r];
    }
}

template <typename T>
__device__ cplx<T>* fft_lines(cplx<T>* A, cplx<T>* B, int nl, int ls, const FftPlan& P, const cplx<T>* tw,
                              int sign) {
    int Ns = 1;
    for (int f = 0; f < P.nf; f++) {
        const int R = P.fac[f];
        __syncthreads();
        if (R == 4) fft_pass<T, 4>(A, B, P.n, Ns, nl, ls, tw, sign);
        else if (R == 2) fft_pass<T, 2>(A, B, P.n, Ns, nl, ls, tw, sign);
        else fft_pass<T, 3>(A, B, P.n, Ns, nl, ls, tw, sign);
        cplx<T>* s = A;
        A = B;
        B = s;
        Ns *= R;
    }
    __syncthreads();
    return A;
}

// ---------------------------------------------------------------------------
// The same transform with the length known at compile time: the radix sequence,
// strides and every index division fold into constants.  fft_lines_any picks
// the compiled length or falls back to the runtime plan.
// ---------------------------------------------------------------------------
template <int N>
struct FftFac {
    static constexpr int count() {
        int m = N, c = 0;
        while (m % 4 == 0) { m /= 4; c++; }
        while (m % 2 == 0) { m /= 2; c++; }
        while (m % 3 == 0) { m /= 3; c++; }
        return c;
    }
    static constexpr int radix(int i) {
        int m = N, c = 0;
        while (m % 4 == 0) { if (c == i) return 4; m /= 4; c++; }
        while (m % 2 == 0) { if (c == i) return 2; m /= 2; c++; }
        while (m % 3 == 0) { if (c == i) return 3; m /= 3; c++; }
        return 1;
    }
    static constexpr int ns(int i) {
        int n = 1;
        for (int k = 0; k < i; k++) n *= radix(k);
        return n;
    }
};

template <typename T, int N, int R, int Ns>
__device__ __forceinline__ void fft_pass_c(const cplx<T>* in, cplx<T>* out, int nl, int ls,
                                           const cplx<T>* __restrict__ tw, int sign) {
    constexpr int nR = N / R, step = N / (Ns * R);
    const int total = nl * nR;
    for (int b = threadIdx.x; b < total; b += blockDim.x) {
        const int l = b / nR, j = b - l * nR;
        const int k = j % Ns;
        const cplx<T>* src = in + l * ls;
        cplx<T>* dst = out + l * ls;
        cplx<T> v[R];
#pragma unroll
        for (int r = 0; r < R; r++) {
            cplx<T> a = src[j + r * nR];
            if (r > 0 && Ns > 1) {
                cplx<T> w = tw[r * k * step];
                if (sign > 0) w.y = -w.y;
                a = cmul(a, w);
            }
            v[r] = a;
        }
        dft_small<T, R>(v, sign);
        const int d = (j / Ns) * Ns * R + k;
#pragma unroll
        for (int r = 0; r < R; r++) dst[d + r * Ns] = v[r];
    }
}

template <typename T, int N, int F>
__device__ __forceinline__ void fft_passes_c(cplx<T>*& A, cplx<T>*& B, int nl, int ls, const cplx<T>* tw, int sign) {
    if constexpr (F < FftFac<N>::count()) {
        constexpr int R = FftFac<N>::radix(F), Ns = FftFac<N>::ns(F);
        __syncthreads();
        fft_pass_c<T, N, R, Ns>(A, B, nl, ls, tw, sign);
        cplx<T>* s = A;
        A = B;
        B = s;
        fft_passes_c<T, N, F + 1>(A, B, nl, ls, tw, sign);
    }
}

template <typename T, int N>
__device__ __forceinline__ cplx<T>* fft_lines_n(cplx<T>* A, cplx<T>* B, int nl, int ls, const cplx<T>* tw, int sign) {
    fft_passes_c<T, N, 0>(A, B, nl, ls, tw, sign);
    __syncthreads();
    return A;
}

template <typename T>
__device__ cplx<T>* fft_lines_any(cplx<T>* A, cplx<T>* B, int nl, int ls, const FftPlan& P, const cplx<T>* tw,
                                  int sign) {
    switch (P.n) {
        case 16: return fft_lines_n<T, 16>(A, B, nl, ls, tw, sign);
        case 24: return fft_lines_n<T, 24>(A, B, nl, ls, tw, sign);
        case 32: return fft_lines_n<T, 32>(A, B, nl, ls, tw, sign);
        case 48: return fft_lines_n<T, 48>(A, B, nl, ls, tw, sign);
        case 64: return fft_lines_n<T, 64>(A, B, nl, ls, tw, sign);
        case 96: return fft_lines_n<T, 96>(A, B, nl, ls, tw, sign);
        case 128: return fft_lines_n<T, 128>(A, B, nl, ls, tw, sign);
        case 192: return fft_lines_n<T, 192>(A, B, nl, ls, tw, sign);
        case 256: return fft_lines_n<T, 256>(A, B, nl, ls, tw, sign);
        case 384: return fft_lines_n<T, 384>(A, B, nl, ls, tw, sign);
        case 512: return fft_lines_n<T, 512>(A, B, nl, ls, tw, sign);
        case 768: return fft_lines_n<T, 768>(A, B, nl, ls, tw, sign);
        case 1024: return fft_lines_n<T, 1024>(A, B, nl, ls, tw, sign);
        default: return fft_lines(A, B, nl, ls, P, tw, sign);
    }
}

}  // namespace tc
