// k_fft_plane.cu -- the pressure solve's 2-D transforms of one z-plane in one kernel.
//
// The separate kernels (k_fft.cu) write the half spectrum after the x-FFT and read it
// back for the y-FFT (and the reverse on the way back): two extra words per cell in each
// direction.  Here a thread-block cluster of PF_CS CTAs owns one plane and keeps its half
// spectrum in distributed shared memory:
//   forward  each CTA x-transforms its NY/PF_CS rows of the real field (two rows per
//            complex line, unpacked as k_xfft_reg does) into its tile[kx][y]; cluster
//            barrier; each CTA then y-transforms the columns kx = rank, rank + PF_CS, ...
//            reading every line's values from the cluster's tiles, and writes
//            spec[z][kx][ky] (the layout of the separate kernels);
//   inverse  each CTA inverse-y-transforms its kx columns straight from spec and stores
//            the values into the tile of the CTA owning each y (remote shared stores);
//            cluster barrier; each CTA inverse-x-transforms its rows (Hermitian-extended
//            half spectrum, two rows per line, as k_ixfft_reg) into p, scaled.
// The line transforms are fft_pass_a / fft_pass_b of fft_reg.cuh with the same twiddle
// tables, so the values are those of the separate kernels.  Compiled for the small planes
// of TC_PLANE_SIZES, where the step is bound by launches and latency: measured at
// 64 x 64 x 64 (HW2), 0.0748 against 0.0770 ms per step in float, 0.0865 against 0.0878 in
// double.  On large planes each CTA's load, transform and exchange phases run in turn with
// two CTAs per SM at most (128 registers, 114 KB of shared memory at 384 x 384), and the
// separate kernels are faster: at 384 x 384 x 256 (VV4, float) forward 0.195 against
// 0.136 ms, inverse 0.163 against 0.132; at 256 x 256 x 192 (collocated) the step 0.500
// against 0.477 ms in float, 0.988 against 0.868 in double.  Other grids keep the
// separate kernels.
#include <cooperative_groups.h>

#include <algorithm>

#include "fft_reg.cuh"
#include "kernels.cuh"

namespace cg = cooperative_groups;

namespace tc {

constexpr int PF_CS = 8;    // CTAs per plane: one portable-size cluster
constexpr int PF_NT = 256;  // threads per CTA

template <typename T, int NX, int NY>
struct PlaneFft {
    using SX = FftSplit<NX>;
    using SY = FftSplit<NY>;
    static constexpr int CS = PF_CS, RY = NY / CS, NXH = NX / 2 + 1;
    static constexpr int TS = RY + 1;  // tile row stride: odd, so column walks spread over the banks
    // rows per x batch: even, divides RY, and one second-pass line segment per thread at most
    static constexpr int br() {
        int b = RY < 32 ? RY : 32;
        b -= b & 1;
        while (b > 0 && (RY % b != 0 || (b / 2) * SX::N1 > PF_NT)) b -= 2;
        return b;
    }
    static constexpr int BR = SX::ok ? br() : 0;
    static constexpr int YLN = SY::ok ? (PF_NT / SY::N2 < 1 ? 1 : PF_NT / SY::N2) : 1;  // lines per y batch
    static constexpr size_t tile_bytes = ((size_t)NXH * TS * sizeof(cplx<T>) + 15) / 16 * 16;
    static constexpr size_t xs = SX::ok ? (size_t)(BR / 2) * SX::YL : 0, ys = SY::ok ? (size_t)YLN * SY::YL : 0;
    static constexpr size_t smem = tile_bytes + (xs > ys ? xs : ys) * sizeof(cplx<T>);
    static constexpr bool ok = SX::ok && SY::ok && NY % (2 * CS) == 0 && BR > 0 && smem <= (size_t)227 * 1024;
};

// One forward plane: rows of the real field src[z][y][x] -> spec[z][kx][ky].
template <typename T, int NX, int NY>
__global__ void __launch_bounds__(PF_NT) k_xyfft_plane(const T* __restrict__ src, cplx<T>* __restrict__ spec,
                                                        const cplx<T>* __restrict__ twx,
                                                        const cplx<T>* __restrict__ twy) {
    using P = PlaneFft<T, NX, NY>;
    constexpr int CS = P::CS, RY = P::RY, NXH = P::NXH, TS = P::TS, BR = P::BR, NL = BR / 2, YLN = P::YLN;
    constexpr int X1 = FftSplit<NX>::N1, X2 = FftSplit<NX>::N2, XYL = FftSplit<NX>::YL, ZS = NX + 1;
    constexpr int Y1 = FftSplit<NY>::N1, Y2 = FftSplit<NY>::N2, YYL = FftSplit<NY>::YL;
    extern __shared__ __align__(16) unsigned char smraw[];
    cplx<T>* tile = reinterpret_cast<cplx<T>*>(smraw);
    cplx<T>* Y = reinterpret_cast<cplx<T>*>(smraw + P::tile_bytes);
    cg::cluster_group cl = cg::this_cluster();
    const int r = (int)cl.block_rank(), z = blockIdx.x / CS, tid = threadIdx.x;

    // x-FFT of rows r*RY .. r*RY+RY-1, BR at a time, into tile[kx][y - r*RY]
    const T* rows = src + ((size_t)z * NY + (size_t)r * RY) * NX;
    for (int b = 0; b < RY; b += BR) {
        for (int it = tid; it < NL * X2; it += PF_NT) {
            const int l = it / X2, n2 = it - l * X2;
            const T* d0 = rows + (size_t)(b + 2 * l) * NX + n2;
            cplx<T> v[X1];
#pragma unroll
            for (int n1 = 0; n1 < X1; n1++) v[n1] = {__ldg(d0 + n1 * X2), __ldg(d0 + NX + n1 * X2)};
            fft_pass_a<T, NX, -1>(v, n2, twx, Y + l * XYL);
        }
        __syncthreads();
        {  // second pass; the transformed lines (stride ZS) overwrite Y once every thread holds its values
            const bool mine = tid < NL * X1;
            const int l = tid / X1, k1 = tid - l * X1;
            cplx<T> v[X2];
            if (mine) fft_pass_b<T, NX, -1>(v, k1, Y + l * XYL);
            __syncthreads();
            if (mine) {
                cplx<T>* zl = Y + l * ZS + k1;
#pragma unroll
                for (int k2 = 0; k2 < X2; k2++) zl[k2 * X1] = v[k2];
            }
        }
        __syncthreads();
        // unpack the two real rows of each line: X_a = (Z_k + conj Z_{N-k}) / 2, X_b = (Z_k - conj Z_{N-k}) / 2i
        for (int e = tid; e < NXH * BR; e += PF_NT) {
            const int kx = e / BR, rr = e - kx * BR, l = rr >> 1;
            const cplx<T> Zk = Y[l * ZS + kx], Zm = Y[l * ZS + (kx == 0 ? 0 : NX - kx)];
            cplx<T> val;
            if ((rr & 1) == 0) val = {T(0.5) * (Zk.x + Zm.x), T(0.5) * (Zk.y - Zm.y)};
            else val = {T(0.5) * (Zk.y + Zm.y), -T(0.5) * (Zk.x - Zm.x)};
            tile[kx * TS + b + rr] = val;
        }
        __syncthreads();  // Y is refilled by the next batch
    }
    cl.sync();  // every tile of the plane is complete

    // y-FFT of the columns kx = r, r + CS, ...: line values y live in tile y / RY of the cluster
    const int ncol = (NXH - r + CS - 1) / CS;
    for (int j0 = 0; j0 < ncol; j0 += YLN) {
        const int nl = min(YLN, ncol - j0);
        for (int it = tid; it < nl * Y2; it += PF_NT) {
            const int l = it / Y2, n2 = it - l * Y2, kx = r + CS * (j0 + l);
            cplx<T> v[Y1];
#pragma unroll
            for (int n1 = 0; n1 < Y1; n1++) {
                const int y = n2 + Y2 * n1, q = y / RY;
                const cplx<T>* t = cl.map_shared_rank(tile, q);
                v[n1] = t[kx * TS + (y - q * RY)];
            }
            fft_pass_a<T, NY, -1>(v, n2, twy, Y + l * YYL);
        }
        __syncthreads();
        for (int it = tid; it < nl * Y1; it += PF_NT) {
            const int l = it / Y1, k1 = it - l * Y1, kx = r + CS * (j0 + l);
            cplx<T> v[Y2];
            fft_pass_b<T, NY, -1>(v, k1, Y + l * YYL);
            cplx<T>* dst = spec + ((size_t)z * NXH + kx) * NY + k1;
#pragma unroll
            for (int k2 = 0; k2 < Y2; k2++) dst[k2 * Y1] = v[k2];
        }
        __syncthreads();
    }
    cl.sync();  // the cluster's reads of this CTA's tile are done before it exits
}

// One inverse plane: spec[z][kx][ky] -> p[z][y][x] * scale.
template <typename T, int NX, int NY>
__global__ void __launch_bounds__(PF_NT) k_ixyfft_plane(const cplx<T>* __restrict__ spec, T* __restrict__ p,
                                                         const cplx<T>* __restrict__ twx,
                                                         const cplx<T>* __restrict__ twy, T scale) {
    using P = PlaneFft<T, NX, NY>;
    constexpr int CS = P::CS, RY = P::RY, NXH = P::NXH, TS = P::TS, BR = P::BR, NL = BR / 2, YLN = P::YLN;
    constexpr int X1 = FftSplit<NX>::N1, X2 = FftSplit<NX>::N2, XYL = FftSplit<NX>::YL, NH = NX / 2;
    constexpr int Y1 = FftSplit<NY>::N1, Y2 = FftSplit<NY>::N2, YYL = FftSplit<NY>::YL;
    extern __shared__ __align__(16) unsigned char smraw[];
    cplx<T>* tile = reinterpret_cast<cplx<T>*>(smraw);
    cplx<T>* Y = reinterpret_cast<cplx<T>*>(smraw + P::tile_bytes);
    cg::cluster_group cl = cg::this_cluster();
    const int r = (int)cl.block_rank(), z = blockIdx.x / CS, tid = threadIdx.x;
    // every CTA of the cluster has started (its shared memory exists) before the first
    // remote store; the arrive is issued now and waited on just before those stores
    asm volatile("barrier.cluster.arrive.relaxed.aligned;\n" ::: "memory");
    bool waited = false;

    // inverse y-FFT of the columns kx = r, r + CS, ...; value y goes to tile y / RY
    const int ncol = (NXH - r + CS - 1) / CS;
    for (int j0 = 0; j0 < ncol; j0 += YLN) {
        const int nl = min(YLN, ncol - j0);
        for (int it = tid; it < nl * Y2; it += PF_NT) {
            const int l = it / Y2, n2 = it - l * Y2, kx = r + CS * (j0 + l);
            const cplx<T>* srcl = spec + ((size_t)z * NXH + kx) * NY + n2;
            cplx<T> v[Y1];
#pragma unroll
            for (int n1 = 0; n1 < Y1; n1++) v[n1] = ldg_c(srcl + n1 * Y2);
            fft_pass_a<T, NY, +1>(v, n2, twy, Y + l * YYL);
        }
        __syncthreads();
        if (!waited) {
            asm volatile("barrier.cluster.wait.aligned;\n" ::: "memory");
            waited = true;
        }
        for (int it = tid; it < nl * Y1; it += PF_NT) {
            const int l = it / Y1, k1 = it - l * Y1, kx = r + CS * (j0 + l);
            cplx<T> v[Y2];
            fft_pass_b<T, NY, +1>(v, k1, Y + l * YYL);
#pragma unroll
            for (int k2 = 0; k2 < Y2; k2++) {
                const int y = k1 + Y1 * k2, q = y / RY;
                cplx<T>* t = cl.map_shared_rank(tile, q);
                t[kx * TS + (y - q * RY)] = v[k2];
            }
        }
        __syncthreads();  // Y is refilled by the next batch
    }
    if (!waited) asm volatile("barrier.cluster.wait.aligned;\n" ::: "memory");
    cl.sync();  // every tile of the plane is complete

    // inverse x-FFT of rows r*RY .. r*RY+RY-1, BR at a time, from the local tile
    T* prow = p + ((size_t)z * NY + (size_t)r * RY) * NX;
    for (int b = 0; b < RY; b += BR) {
        for (int it = tid; it < NL * X2; it += PF_NT) {
            const int l = it / X2, n2 = it - l * X2;
            cplx<T> v[X1];
#pragma unroll
            for (int n1 = 0; n1 < X1; n1++) {  // the Hermitian-extended line of rows b+2l, b+2l+1
                const int k = X2 * n1 + n2;
                const bool up = k > NH;
                const cplx<T>* tp = tile + (up ? NX - k : k) * TS + b + 2 * l;
                cplx<T> av = tp[0], bv = tp[1];
                if (up) {
                    av.y = -av.y;
                    bv.y = -bv.y;
                }
                if (k == 0 || k == NH) {
                    av.y = 0;
                    bv.y = 0;
                }
                v[n1] = {av.x - bv.y, av.y + bv.x};
            }
            fft_pass_a<T, NX, +1>(v, n2, twx, Y + l * XYL);
        }
        __syncthreads();
        for (int it = tid; it < NL * X1; it += PF_NT) {
            const int l = it / X1, k1 = it - l * X1;
            cplx<T> v[X2];
            fft_pass_b<T, NX, +1>(v, k1, Y + l * XYL);
            T* pa = prow + (size_t)(b + 2 * l) * NX + k1;
            T* pb = pa + NX;
#pragma unroll
            for (int k2 = 0; k2 < X2; k2++) {
                pa[k2 * X1] = v[k2].x * scale;
                pb[k2 * X1] = v[k2].y * scale;
            }
        }
        __syncthreads();  // Y is refilled by the next batch
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
static cudaLaunchConfig_t plane_config(cudaLaunchAttribute* at, int nz, size_t smem, cudaStream_t s) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(PF_CS * nz));
    cfg.blockDim = dim3(PF_NT);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    at->id = cudaLaunchAttributeClusterDimension;
    at->val.clusterDim.x = PF_CS;
    at->val.clusterDim.y = 1;
    at->val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cfg;
}

// Whether a cluster of PF_CS CTAs of this kernel, `smem` bytes each, can be resident.
static bool cluster_fits(const void* k, size_t smem) {
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    cudaLaunchAttribute at;
    const cudaLaunchConfig_t cfg = plane_config(&at, 1, smem, 0);
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, k, &cfg) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return n > 0;
}

template <typename T, int NX, int NY>
static bool plane_fits() {
    using P = PlaneFft<T, NX, NY>;
    if constexpr (!P::ok) {
        return false;
    } else {
        // per device (function attributes are per device), resolved at the first call:
        // 0 not resolved, 1 fits, -1 does not
        constexpr int MAXDEV = 64;
        static int state[MAXDEV] = {};
        int dev = 0;
        cudaGetDevice(&dev);
        if (dev < 0 || dev >= MAXDEV) return false;
        if (state[dev] == 0)
            state[dev] = cluster_fits(reinterpret_cast<const void*>(k_xyfft_plane<T, NX, NY>), P::smem) &&
                                 cluster_fits(reinterpret_cast<const void*>(k_ixyfft_plane<T, NX, NY>), P::smem)
                             ? 1
                             : -1;
        return state[dev] == 1;
    }
}

template <typename T, int NX, int NY>
static void plane_fwd(const T* src, cplx<T>* spec, const cplx<T>* twx, const cplx<T>* twy, int nz, cudaStream_t s) {
    using P = PlaneFft<T, NX, NY>;
    if constexpr (P::ok) {
        cudaLaunchAttribute at;
        const cudaLaunchConfig_t cfg = plane_config(&at, nz, P::smem, s);
        cudaLaunchKernelEx(&cfg, k_xyfft_plane<T, NX, NY>, src, spec, twx, twy);
    }
}

template <typename T, int NX, int NY>
static void plane_inv(const cplx<T>* spec, T* p, const cplx<T>* twx, const cplx<T>* twy, T scale, int nz,
                      cudaStream_t s) {
    using P = PlaneFft<T, NX, NY>;
    if constexpr (P::ok) {
        cudaLaunchAttribute at;
        const cudaLaunchConfig_t cfg = plane_config(&at, nz, P::smem, s);
        cudaLaunchKernelEx(&cfg, k_ixyfft_plane<T, NX, NY>, spec, p, twx, twy, scale);
    }
}

// (NX, NY) pairs with plane kernels: planes of up to 64 x 64 (see the top of this file)
#define TC_PLANE_SIZES(X) X(32, 16) X(32, 32) X(64, 32) X(64, 64)

template <typename T>
bool plane_fft_ok(const Geom& g) {
#define TC_CASE(x, y) \
    if (g.NX == x && g.NY == y) return plane_fits<T, x, y>();
    TC_PLANE_SIZES(TC_CASE)
#undef TC_CASE
    return false;
}

// The divergence (vector RHS) and the forward plane transforms: the number of launches,
// 0 when this grid has no plane kernel (nothing launched).
template <typename T>
int launch_div_xyfft_plane(const DivFftArgs<T>& a, const cplx<T>* twy, cudaStream_t s) {
    if (!plane_fft_ok<T>(a.g)) return 0;
    const bool vec = a.src_scalar == nullptr;
    if (vec && !launch_div_quad<T>(a, s)) return 0;
    const T* src = vec ? a.dtmp : a.src_scalar;
#define TC_CASE(x, y)                                              \
    if (a.g.NX == x && a.g.NY == y) {                              \
        plane_fwd<T, x, y>(src, a.spec, a.twx, twy, a.g.NZ, s);   \
        return vec ? 2 : 1;                                        \
    }
    TC_PLANE_SIZES(TC_CASE)
#undef TC_CASE
    return 0;
}

template <typename T>
bool launch_ixyfft_plane(const IxFftArgs<T>& a, const cplx<T>* twy, cudaStream_t s) {
    if (!plane_fft_ok<T>(a.g)) return false;
#define TC_CASE(x, y)                                                        \
    if (a.g.NX == x && a.g.NY == y) {                                        \
        plane_inv<T, x, y>(a.spec, a.p, a.twx, twy, a.scale, a.g.NZ, s);     \
        return true;                                                         \
    }
    TC_PLANE_SIZES(TC_CASE)
#undef TC_CASE
    return false;
}

template bool plane_fft_ok<float>(const Geom&);
template bool plane_fft_ok<double>(const Geom&);
template int launch_div_xyfft_plane<float>(const DivFftArgs<float>&, const cplx<float>*, cudaStream_t);
template int launch_div_xyfft_plane<double>(const DivFftArgs<double>&, const cplx<double>*, cudaStream_t);
template bool launch_ixyfft_plane<float>(const IxFftArgs<float>&, const cplx<float>*, cudaStream_t);
template bool launch_ixyfft_plane<double>(const IxFftArgs<double>&, const cplx<double>*, cudaStream_t);

}  // namespace tc
