// k_fft.cu -- the pressure solve's FFT kernels for the lengths that have a compiled
// two-pass register transform (fft_reg.cuh: 16 ... 1024 = 2^a 3^b); other lengths
// keep the Stockham kernels of k_poisson.cu.  Same data layouts and results:
//   k_div_quad_z   : divergence of the vector RHS (streaming, 16-byte row loads)
//                    into a scratch real field;
//   k_xfft_reg     : forward x-FFT of `rows` y-rows of a real field (the divergence
//                    or the scalar RHS), two rows packed as one complex line,
//                    unpacked to spec[z][kx][y] (kx = 0..NX/2);
//   k_yfft_reg     : complex FFT of contiguous y-lines of spec, in place, straight
//                    from and back to global memory;
//   k_ixfft_reg    : Hermitian-extended half spectrum of two rows packed as one
//                    complex line, inverse x-FFT, scaled real rows into p.
#include <algorithm>

#include "fft_reg.cuh"
#include "kernels.cuh"
#include "stencil_div.cuh"

namespace tc {

// ---------------------------------------------------------------------------
// y-FFT
// ---------------------------------------------------------------------------
constexpr int YFFT_LINE_BUDGET = 128;  // lines x N1 per CTA
// Lines per CTA: few (8 at N = 384: 26 KB of shared memory in float, 51 KB in double),
// so that many CTAs share an SM and hide each other's global-memory latency (measured
// at 384 x 384 x 256: 32 float lines per CTA 0.082 ms, 16 lines 0.074, 8 lines 0.058).
template <typename T, int N>
constexpr int yfft_reg_lines() {
    const int l = YFFT_LINE_BUDGET / FftSplit<N>::N1;
    return l < 1 ? 1 : l;
}

template <typename T, int N, int SIGN>
__global__ void __launch_bounds__(256) k_yfft_reg(cplx<T>* spec, long long nlines, const cplx<T>* __restrict__ tw) {
    constexpr int N1 = FftSplit<N>::N1, N2 = FftSplit<N>::N2, YL = FftSplit<N>::YL;
    constexpr int LINES = yfft_reg_lines<T, N>();
    extern __shared__ __align__(16) unsigned char smraw[];
    cplx<T>* Y = reinterpret_cast<cplx<T>*>(smraw);
    // the forward transform takes the lines in descending z, the reverse of the x-FFT that
    // wrote them (its last planes are still in L2), and leaves the low planes, which the
    // z-solve's forward sweep reads first, written last (384x256x384 float: y-FFT 0.052
    // against 0.059 ms, z-solve 0.144 against 0.152; double 0.097 / 0.283 against 0.101 / 0.292)
    const long long blk = SIGN < 0 ? (long long)gridDim.x - 1 - blockIdx.x : (long long)blockIdx.x;
    const long long L0 = blk * LINES;
    const int nl = (int)min((long long)LINES, nlines - L0);
    cplx<T>* base = spec + L0 * N;
    for (int it = threadIdx.x; it < nl * N2; it += blockDim.x) {
        const int l = it / N2, n2 = it - l * N2;
        const cplx<T>* src = base + (size_t)l * N + n2;
        cplx<T> v[N1];
#pragma unroll
        for (int n1 = 0; n1 < N1; n1++) v[n1] = src[n1 * N2];
        fft_pass_a<T, N, SIGN>(v, n2, tw, Y + l * YL);
    }
    __syncthreads();
    for (int it = threadIdx.x; it < nl * N1; it += blockDim.x) {
        const int l = it / N1, k1 = it - l * N1;
        cplx<T> v[N2];
        fft_pass_b<T, N, SIGN>(v, k1, Y + l * YL);
        cplx<T>* dst = base + (size_t)l * N + k1;
#pragma unroll
        for (int k2 = 0; k2 < N2; k2++) dst[k2 * N1] = v[k2];
    }
}

template <typename T, int N>
static void yfft_reg_launch(const YFftArgs<T>& a, cudaStream_t s) {
    constexpr int LINES = yfft_reg_lines<T, N>();
    const long long total = (long long)a.g.NZ * a.g.NXH;
    const size_t smem = (size_t)LINES * FftSplit<N>::YL * sizeof(cplx<T>);
    auto k = a.sign < 0 ? k_yfft_reg<T, N, -1> : k_yfft_reg<T, N, +1>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k<<<(unsigned)((total + LINES - 1) / LINES), 256, smem, s>>>(a.spec, total, a.twy);
}

// ---------------------------------------------------------------------------
// divergence of the vector RHS (streaming, 4 cells of a row per thread) and the
// forward x-FFT of a real field
// ---------------------------------------------------------------------------
// Same expressions as div_at (stencil_div.cuh), evaluated for x..x+3 from 16-byte row
// loads (NX % 4 == 0: the periodic wrap then moves whole 4-cell chunks), each thread
// marching over ZC consecutive planes of its 4-cell row: the w planes z-1 .. z+2 of the
// stencils stay in registers from one plane to the next (one new w load per plane
// instead of four; measured at 384x384x256, float: 0.188 ms with the x-FFT against 0.223
// ms for one plane per thread).
// Bounded for four CTAs per SM in float (64 registers) and three in double (80 registers;
// 0.351 against 0.359 ms with the x-FFT at 384x256x384; float with one CTA as the bound
// takes 79 registers and 0.193 against 0.184 ms)
template <typename T, int SCHEME, int ZC>
__global__ void __launch_bounds__(256, sizeof(T) == 8 ? 3 : 4) k_div_quad_z(DivFftArgs<T> a, T* __restrict__ out) {
    const Geom& g = a.g;
    const int NX = g.NX, NY = g.NY, NZ = g.NZ, NQ = NX >> 2, NZB = (NZ + ZC - 1) / ZC;
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= (long long)NQ * NY * NZB) return;
    const int row = (int)(q / NQ), x = (int)(q - (long long)row * NQ) * 4;
    // float: plane chunks in descending z, the float flux kernel's last-written planes (high
    // z) being the ones still in L2 (divergence + x-FFT 0.177 against 0.179 ms at
    // 384x256x384); double keeps ascending chunks (the FP64 flux kernel writes in z-chunks,
    // and descending took 0.377 against 0.353 ms)
    const int y = row % NY, z0 = (sizeof(T) == 4 ? NZB - 1 - row / NY : row / NY) * ZC;
    const size_t NXY = (size_t)NX * NY, col = (size_t)y * NX + x;
    const T *u = a.v.c[0], *v = a.v.c[1], *w = a.v.c[2];
    const T ihx = (T)g.inv_hx, ihy = (T)g.inv_hy;
    const int xq = x + 4 == NX ? 0 : x + 4, xm = x == 0 ? NX - 1 : x - 1;
    const int yp = y + 1 == NY ? 0 : y + 1, ym = y == 0 ? NY - 1 : y - 1;
    const int ypp = yp + 1 == NY ? 0 : yp + 1;
    auto ldw = [&](int zz) {
        Acc4<T> r;
        if (zz >= 0 && zz < NZ) r = ld4(w + (size_t)zz * NXY + col);
        else
#pragma unroll
            for (int k = 0; k < 4; k++) r.v[k] = T(0);
        return r;
    };
    Acc4<T> Wz[4];  // w at the planes z-1, z, z+1, z+2
    Wz[0] = ldw(z0 - 1);
    Wz[1] = ldw(z0);
    Wz[2] = ldw(z0 + 1);
    Wz[3] = ldw(z0 + 2);
#pragma unroll
    for (int kz = 0; kz < ZC; kz++) {
        const int z = z0 + kz;
        if (z >= NZ) break;
        if (kz > 0) {
            Wz[0] = Wz[1];
            Wz[1] = Wz[2];
            Wz[2] = Wz[3];
            Wz[3] = ldw(z + 2);
        }
        const size_t pl = (size_t)z * NXY, rb = pl + (size_t)y * NX, id = rb + x;
        T e[9];  // u at x-1 .. x+7
        {
            const Acc4<T> U0 = ld4(u + id), U1 = ld4(u + rb + xq);
            e[0] = __ldg(u + rb + xm);
#pragma unroll
            for (int k = 0; k < 4; k++) {
                e[1 + k] = U0.v[k];
                e[5 + k] = U1.v[k];
            }
        }
        T d[4];
        if constexpr (SCHEME == TC_SCHEME_VV4) {
            const T C27 = T(0.03703703703703703703);
            const T dz = a.m.DZ[z], dzw = a.m.DZW[z];
            const Acc4<T> V0 = ld4(v + id), Vp = ld4(v + pl + (size_t)yp * NX + x),
                          Vpp = ld4(v + pl + (size_t)ypp * NX + x), Vm = ld4(v + pl + (size_t)ym * NX + x);
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const T W0 = Wz[1].v[k];
                const T Wr = z == NZ - 1 ? T(0) : Wz[2].v[k];
                const T Wrr = z == NZ - 1 ? W0 : (z == NZ - 2 ? T(0) : Wz[3].v[k]);
                const T Wll = z == 0 ? Wz[2].v[k] : (z == 1 ? T(0) : Wz[0].v[k]);
                const T dudx = ihx * (dz * (e[k + 2] - e[k + 1]) - C27 * dzw * (e[k + 3] - e[k]));
                const T dvdy = ihy * (dz * (Vp.v[k] - V0.v[k]) - C27 * dzw * (Vpp.v[k] - Vm.v[k]));
                d[k] = dudx + dvdy + (Wr - W0) - C27 * (Wrr - Wll);
            }
        } else if constexpr (SCHEME == TC_SCHEME_HW2) {
            const T hz = a.m.DZ[z];
            const Acc4<T> V0 = ld4(v + id), Vp = ld4(v + pl + (size_t)yp * NX + x);
#pragma unroll
            for (int k = 0; k < 4; k++)
                d[k] = (e[k + 2] - e[k + 1]) * ihx * hz + (Vp.v[k] - V0.v[k]) * ihy * hz +
                       ((z < NZ - 1) ? (Wz[2].v[k] - Wz[1].v[k]) : (-Wz[1].v[k]));
        } else {
            const T hz = a.m.cellh[z], hx = (T)g.hx, hy = (T)g.hy;
            const Acc4<T> Vp = ld4(v + pl + (size_t)yp * NX + x), Vm = ld4(v + pl + (size_t)ym * NX + x);
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const T Wa = z == 0 ? Wz[2].v[k] : (z == NZ - 1 ? Wz[1].v[k] : Wz[2].v[k]);
                const T Wb = z == 0 ? Wz[1].v[k] : Wz[0].v[k];
                T dd = 0;
                dd += T(0.5) * (e[k + 2] - e[k]) * hy * hz;
                dd += T(0.5) * (Vp.v[k] - Vm.v[k]) * hx * hz;
                dd += T(0.5) * (Wa - Wb) * hx * hy;
                d[k] = dd;
            }
        }
        if constexpr (sizeof(T) == 4) {
            *reinterpret_cast<float4*>(out + id) = make_float4(d[0], d[1], d[2], d[3]);
        } else {
            reinterpret_cast<double2*>(out + id)[0] = make_double2(d[0], d[1]);
            reinterpret_cast<double2*>(out + id)[1] = make_double2(d[2], d[3]);
        }
    }
}

// Whether the forward x-FFT of `rows` rows (256 threads) keeps its transformed lines in
// the first pass's buffer: one second-pass line segment per thread at most.
template <int N>
__host__ __device__ constexpr bool xfft_alias(int rows) {
    return (rows / 2) * FftSplit<N>::N1 <= 256;
}

// Three CTAs per SM in float (79 registers at N = 384, no spill), two in double.
template <typename T, int N>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 3 : 2) k_xfft_reg(DivFftArgs<T> a, const T* __restrict__ src, int rows, int lrows) {
    constexpr int N1 = FftSplit<N>::N1, N2 = FftSplit<N>::N2, YL = FftSplit<N>::YL, ZS = N + 1;
    extern __shared__ __align__(16) unsigned char smraw[];
    const Geom& g = a.g;
    const int NY = g.NY, NXH = N / 2 + 1, nl = rows >> 1;
    cplx<T>* Y = reinterpret_cast<cplx<T>*>(smraw);
    // transformed lines, stride N+1: over Y itself when every thread holds at most one
    // line segment of the second pass (read all, barrier, write), else after Y
    const bool alias = xfft_alias<N>(rows);
    cplx<T>* Zs = alias ? Y : Y + nl * YL;
    const int z = blockIdx.y, y0 = blockIdx.x * rows;
    const T* plane = src + ((size_t)z * NY + y0) * N;
    for (int it = threadIdx.x; it < nl * N2; it += blockDim.x) {
        const int l = it / N2, n2 = it - l * N2;
        const T* d0 = plane + (size_t)(2 * l) * N + n2;
        cplx<T> v[N1];
#pragma unroll
        for (int n1 = 0; n1 < N1; n1++) v[n1] = {__ldg(d0 + n1 * N2), __ldg(d0 + N + n1 * N2)};
        fft_pass_a<T, N, -1>(v, n2, a.twx, Y + l * YL);
    }
    __syncthreads();
    if (alias) {
        const bool mine = (int)threadIdx.x < nl * N1;
        const int l = threadIdx.x / N1, k1 = threadIdx.x - l * N1;
        cplx<T> v[N2];
        if (mine) fft_pass_b<T, N, -1>(v, k1, Y + l * YL);
        __syncthreads();
        if (mine) {
            cplx<T>* zl = Zs + l * ZS + k1;
#pragma unroll
            for (int k2 = 0; k2 < N2; k2++) zl[k2 * N1] = v[k2];
        }
    } else {
        for (int it = threadIdx.x; it < nl * N1; it += blockDim.x) {
            const int l = it / N1, k1 = it - l * N1;
            cplx<T> v[N2];
            fft_pass_b<T, N, -1>(v, k1, Y + l * YL);
            cplx<T>* zl = Zs + l * ZS + k1;
#pragma unroll
            for (int k2 = 0; k2 < N2; k2++) zl[k2 * N1] = v[k2];
        }
    }
    __syncthreads();
    // unpack the two real rows of each line: X_a = (Z_k + conj Z_{N-k}) / 2, X_b = (Z_k - conj Z_{N-k}) / 2i
    for (int e = threadIdx.x; e < NXH * rows; e += blockDim.x) {
        const int kx = e >> lrows, r = e & (rows - 1), l = r >> 1;
        const cplx<T> Zk = Zs[l * ZS + kx], Zm = Zs[l * ZS + (kx == 0 ? 0 : N - kx)];
        cplx<T> val;
        if ((r & 1) == 0) val = {T(0.5) * (Zk.x + Zm.x), T(0.5) * (Zk.y - Zm.y)};
        else val = {T(0.5) * (Zk.y + Zm.y), -T(0.5) * (Zk.x - Zm.x)};
        a.spec[((size_t)z * NXH + kx) * NY + y0 + r] = val;
    }
}

template <typename T, int N>
static size_t div_xfft_reg_smem(int rows) {
    return (size_t)(rows / 2) * (FftSplit<N>::YL + (xfft_alias<N>(rows) ? 0 : N + 1)) * sizeof(cplx<T>);
}

template <typename T, int N>
static void xfft_reg_launch(const DivFftArgs<T>& a, const T* src, int rows, cudaStream_t s) {
    const size_t smem = div_xfft_reg_smem<T, N>(rows);
    int lr = 0;
    while ((1 << lr) < rows) lr++;
    auto k = k_xfft_reg<T, N>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k<<<dim3(a.g.NY / rows, a.g.NZ), 256, smem, s>>>(a, src, rows, lr);
}

// ---------------------------------------------------------------------------
// inverse x-FFT, persistent and double-buffered (float)
// ---------------------------------------------------------------------------
constexpr int XP_NT = 256;
// As k_ixfft_reg (the Hermitian-extended
// half spectrum of two rows per complex line, inverse transform, scaled rows into p), with
// each CTA walking tiles of RB (16) y-values of one plane and copying the next tile's half
// spectrum (NX/2+1 rows of RB contiguous values) into its second buffer while it
// transforms the current one.
template <typename T, int N>
struct IPipe {
    static constexpr int RB = sizeof(T) == 4 ? 16 : 8, NL = RB / 2, TS = RB + 2, NXH = N / 2 + 1;
    static constexpr int PC = 16 / sizeof(cplx<T>), CPK = RB / PC;  // 16-byte chunks per kx row
    static constexpr size_t buf = ((size_t)NXH * TS * sizeof(cplx<T>) + 15) / 16 * 16;
    static constexpr size_t smem = 2 * buf + (size_t)NL * FftSplit<N>::YL * sizeof(cplx<T>);
};

template <typename T, int N>
__global__ void __launch_bounds__(XP_NT) k_ixfft_pipe(IxFftArgs<T> a) {
    using P = IPipe<T, N>;
    constexpr int RB = P::RB, NL = P::NL, TS = P::TS, NXH = P::NXH, PC = P::PC, CPK = P::CPK;
    constexpr int N1 = FftSplit<N>::N1, N2 = FftSplit<N>::N2, YL = FftSplit<N>::YL, NH = N / 2;
    extern __shared__ __align__(16) unsigned char smraw[];
    cplx<T>* Y = reinterpret_cast<cplx<T>*>(smraw + 2 * P::buf);
    const Geom& g = a.g;
    const int NY = g.NY, YB = NY / RB;
    const long long ntile = (long long)YB * g.NZ;
    // tiles in ascending z: the correction that reads p next walks the planes downwards,
    // so that the next step's flux kernel, which starts at z = 0, finds the low planes of
    // the new velocity in L2 (at 384x256x384 the flux kernel gains more, 7 us, than this
    // kernel loses against descending tiles, 1.5 us)
    auto fetch = [&](long long t, int b) {
        const int z = (int)(t / YB), y0 = (int)(t - (long long)z * YB) * RB;
        cplx<T>* tile = reinterpret_cast<cplx<T>*>(smraw + b * P::buf);
        for (int e = threadIdx.x; e < NXH * CPK; e += XP_NT) {
            const int kx = e / CPK, c = e - kx * CPK;
            cp_async<16>(tile + kx * TS + c * PC, a.spec + ((size_t)z * NXH + kx) * NY + y0 + c * PC);
        }
    };
    long long t = blockIdx.x;
    if (t < ntile) fetch(t, 0);
    cp_async_commit();
    const T sc = a.scale;
    for (int b = 0; t < ntile; t += gridDim.x, b ^= 1) {
        if (t + gridDim.x < ntile) fetch(t + gridDim.x, b ^ 1);
        cp_async_commit();
        cp_async_wait<1>();
        __syncthreads();  // tile t is in buffer b
        const int z = (int)(t / YB), y0 = (int)(t - (long long)z * YB) * RB;
        const cplx<T>* tile = reinterpret_cast<const cplx<T>*>(smraw + b * P::buf);
        for (int it = threadIdx.x; it < NL * N2; it += XP_NT) {
            const int l = it / N2, n2 = it - l * N2;
            cplx<T> v[N1];
#pragma unroll
            for (int n1 = 0; n1 < N1; n1++) {  // the Hermitian-extended line of rows 2l, 2l+1
                const int k = N2 * n1 + n2;
                const bool up = k > NH;
                const cplx<T>* tp = tile + (up ? N - k : k) * TS + 2 * l;
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
            fft_pass_a<T, N, +1>(v, n2, a.twx, Y + l * YL);
        }
        __syncthreads();
        for (int it = threadIdx.x; it < NL * N1; it += XP_NT) {
            const int l = it / N1, k1 = it - l * N1;
            cplx<T> v[N2];
            fft_pass_b<T, N, +1>(v, k1, Y + l * YL);
            T* pa = a.p + ((size_t)z * NY + y0 + 2 * l) * N + k1;
            T* pb = pa + N;
#pragma unroll
            for (int k2 = 0; k2 < N2; k2++) {
                pa[k2 * N1] = v[k2].x * sc;
                pb[k2 * N1] = v[k2].y * sc;
            }
        }
        __syncthreads();  // buffer b and Y are refilled by the next iterations
    }
}

template <typename T, int N>
static bool ixfft_pipe_launch(const IxFftArgs<T>& a, cudaStream_t s) {
    // float only: in double the tiles halve and the k_ixfft_reg form measured faster
    if constexpr (sizeof(T) != 4) {
        return false;
    } else {
        using P = IPipe<T, N>;
        if (a.g.NY % P::RB != 0) return false;
        auto k = k_ixfft_pipe<T, N>;
        // per size and device (function attributes are per device), resolved at the first launch
        constexpr int MAXDEV = 64;
        static int sms_of[MAXDEV] = {}, occ_of[MAXDEV] = {};  // occ 0: not resolved yet, -1: does not fit
        int dev = 0;
        cudaGetDevice(&dev);
        if (dev < 0 || dev >= MAXDEV) return false;
        if (occ_of[dev] == 0) {
            int optin = 0, o = 0, n = 0;
            cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
            cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
            if (P::smem <= (size_t)optin) {
                cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)P::smem);
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, k, XP_NT, P::smem);
            }
            sms_of[dev] = n;
            occ_of[dev] = o > 0 ? o : -1;
        }
        const int occ = occ_of[dev], sms = sms_of[dev];
        if (occ < 1) return false;
        const long long ntile = (long long)(a.g.NY / P::RB) * a.g.NZ;
        const int grid = (int)std::min<long long>(ntile, (long long)sms * occ);
        k<<<grid, XP_NT, P::smem, s>>>(a);
        return true;
    }
}

constexpr int DIV_ZC = 4;  // planes per thread of k_div_quad_z
template <typename T>
static void div_quad_launch(const DivFftArgs<T>& a, T* out, cudaStream_t s) {
    const long long nq = (long long)(a.g.NX / 4) * a.g.NY * ((a.g.NZ + DIV_ZC - 1) / DIV_ZC);
    const unsigned nb = (unsigned)((nq + 255) / 256);
    if (a.g.scheme == TC_SCHEME_VV4) k_div_quad_z<T, TC_SCHEME_VV4, DIV_ZC><<<nb, 256, 0, s>>>(a, out);
    else if (a.g.scheme == TC_SCHEME_HW2) k_div_quad_z<T, TC_SCHEME_HW2, DIV_ZC><<<nb, 256, 0, s>>>(a, out);
    else k_div_quad_z<T, TC_SCHEME_COLLOC, DIV_ZC><<<nb, 256, 0, s>>>(a, out);
}

// ---------------------------------------------------------------------------
// inverse x-FFT
// ---------------------------------------------------------------------------
template <typename T, int N>
__global__ void __launch_bounds__(512) k_ixfft_reg(IxFftArgs<T> a, int rows, int lrows, int alias) {
    constexpr int N1 = FftSplit<N>::N1, N2 = FftSplit<N>::N2, YL = FftSplit<N>::YL, NH = N / 2, NXH = NH + 1;
    constexpr int PC = 16 / sizeof(cplx<T>);  // complex values per 16-byte chunk
    extern __shared__ __align__(16) unsigned char smraw[];
    const Geom& g = a.g;
    const int NY = g.NY, nl = rows >> 1, TS = rows + 2;
    cplx<T>* tile = reinterpret_cast<cplx<T>*>(smraw);  // tile[kx * TS + r]
    // alias: the first pass's output over the tile itself, every thread holding at most
    // one line segment (gather all, barrier, transform and write); else after the tile
    cplx<T>* Y = alias ? tile : tile + NXH * TS;
    // planes in descending z, the reverse of the inverse y-FFT that wrote them
    const int z = gridDim.y - 1 - blockIdx.y, y0 = blockIdx.x * rows;
    {
        const int cpr = rows / PC, lc = lrows - (PC == 2 ? 1 : 0);
        for (int e = threadIdx.x; e < NXH * cpr; e += blockDim.x) {
            const int kx = e >> lc, c = e & (cpr - 1);
            cp_async<16>(tile + kx * TS + c * PC, a.spec + ((size_t)z * NXH + kx) * NY + y0 + c * PC);
        }
        cp_async_commit();
        cp_async_wait<0>();
    }
    __syncthreads();
    // the Hermitian-extended line of two packed rows at the first pass's positions
    auto gather = [&](int l, int n2, cplx<T>(&v)[N1]) {
#pragma unroll
        for (int n1 = 0; n1 < N1; n1++) {
            const int k = N2 * n1 + n2;
            const bool up = k > NH;
            const cplx<T>* t = tile + (up ? N - k : k) * TS + 2 * l;
            cplx<T> av = t[0], bv = t[1];
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
    };
    if (alias) {
        const bool mine = (int)threadIdx.x < nl * N2;
        const int l = threadIdx.x / N2, n2 = threadIdx.x - l * N2;
        cplx<T> v[N1];
        if (mine) gather(l, n2, v);
        __syncthreads();
        if (mine) fft_pass_a<T, N, +1>(v, n2, a.twx, Y + l * YL);
    } else {
        for (int it = threadIdx.x; it < nl * N2; it += blockDim.x) {
            const int l = it / N2, n2 = it - l * N2;
            cplx<T> v[N1];
            gather(l, n2, v);
            fft_pass_a<T, N, +1>(v, n2, a.twx, Y + l * YL);
        }
    }
    __syncthreads();
    const T sc = a.scale;
    for (int it = threadIdx.x; it < nl * N1; it += blockDim.x) {
        const int l = it / N1, k1 = it - l * N1;
        cplx<T> v[N2];
        fft_pass_b<T, N, +1>(v, k1, Y + l * YL);
        T* pa = a.p + ((size_t)z * NY + y0 + 2 * l) * N + k1;
        T* pb = pa + N;
#pragma unroll
        for (int k2 = 0; k2 < N2; k2++) {
            pa[k2 * N1] = v[k2].x * sc;
            pb[k2 * N1] = v[k2].y * sc;
        }
    }
}

// Double: one thread per first-pass line segment when that takes at most 512 threads, and
// the tile and the first pass's output share their buffer, which doubles the rows that
// fit the shared-memory budget (measured at 384x384x256: 0.139 ms against 0.164 ms).
// Float keeps 256 threads and separate buffers (0.083 ms against 0.087 ms aliased).
template <typename T, int N>
static bool ixfft_alias(int rows) {
    return sizeof(T) == 8 && (rows / 2) * FftSplit<N>::N2 <= 512;
}
template <typename T, int N>
static int ixfft_threads(int rows) {
    const int items = (rows / 2) * FftSplit<N>::N2;
    return ixfft_alias<T, N>(rows) ? std::max(256, (items + 31) / 32 * 32) : 256;
}

template <typename T, int N>
static size_t ixfft_reg_smem(int rows) {
    const size_t tile = (size_t)(N / 2 + 1) * (rows + 2), y = (size_t)(rows / 2) * FftSplit<N>::YL;
    return (ixfft_alias<T, N>(rows) ? std::max(tile, y) : tile + y) * sizeof(cplx<T>);
}

template <typename T, int N>
static void ixfft_reg_launch(const IxFftArgs<T>& a, int rows, cudaStream_t s) {
    const size_t smem = ixfft_reg_smem<T, N>(rows);
    int lr = 0;
    while ((1 << lr) < rows) lr++;
    auto k = k_ixfft_reg<T, N>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k<<<dim3(a.g.NY / rows, a.g.NZ), ixfft_threads<T, N>(rows), smem, s>>>(a, rows, lr,
                                                                           ixfft_alias<T, N>(rows) ? 1 : 0);
}

// ---------------------------------------------------------------------------
// dispatch on the transform length
// ---------------------------------------------------------------------------
// Rows per CTA of the x-FFT kernels: the largest of 32, 16, 8 that divides NY and
// whose shared memory stays within XFFT_SMEM_PREF (four CTAs per SM: measured faster
// than two), else within 110 KB (two CTAs per SM); 0 if none.
constexpr size_t XFFT_SMEM_PREF = 56 * 1024;
template <typename T, int N>
static int xfft_reg_rows(int NY, bool inverse) {
    for (size_t cap : {XFFT_SMEM_PREF, (size_t)110 * 1024})
        for (int r : {32, 16, 8}) {
            if (NY % r) continue;
            const size_t sm = inverse ? ixfft_reg_smem<T, N>(r) : div_xfft_reg_smem<T, N>(r);
            if (sm <= cap) return r;
        }
    return 0;
}

#define TC_FFT_SIZES(X) X(16) X(24) X(32) X(48) X(64) X(96) X(128) X(192) X(256) X(384) X(512) X(768) X(1024)

template <typename T>
bool launch_yfft_reg(const YFftArgs<T>& a, cudaStream_t s) {
    switch (a.g.NY) {
#define TC_CASE(n)                  \
    case n:                         \
        yfft_reg_launch<T, n>(a, s); \
        return true;
        TC_FFT_SIZES(TC_CASE)
#undef TC_CASE
        default: return false;
    }
}

// The vector RHS first goes through k_div_quad_z into a.dtmp (needs NX % 4 == 0 and a
// scratch buffer), then the real field is transformed.
template <typename T>
int launch_div_xfft_reg(const DivFftArgs<T>& a, cudaStream_t s) {
    const bool vec = a.src_scalar == nullptr;
    if (vec && (a.dtmp == nullptr || a.g.NX % 4 != 0)) return 0;
    switch (a.g.NX) {
#define TC_CASE(n)                                           \
    case n: {                                                \
        const int rows = xfft_reg_rows<T, n>(a.g.NY, false); \
        if (!rows) return 0;                                 \
        if (vec) div_quad_launch<T>(a, a.dtmp, s);           \
        xfft_reg_launch<T, n>(a, vec ? a.dtmp : a.src_scalar, rows, s); \
        return vec ? 2 : 1;                                  \
    }
        TC_FFT_SIZES(TC_CASE)
#undef TC_CASE
        default: return 0;
    }
}

template <typename T>
bool launch_ixfft_reg(const IxFftArgs<T>& a, cudaStream_t s) {
    switch (a.g.NX) {
#define TC_CASE(n)                                          \
    case n: {                                               \
        const int rows = xfft_reg_rows<T, n>(a.g.NY, true); \
        if (!rows) return false;                            \
        if (!ixfft_pipe_launch<T, n>(a, s)) ixfft_reg_launch<T, n>(a, rows, s); \
        return true;                                        \
    }
        TC_FFT_SIZES(TC_CASE)
#undef TC_CASE
        default: return false;
    }
}

// The divergence pass alone (for the plane transforms of k_fft_plane.cu): false when the
// vector RHS has no scratch or NX % 4 != 0.
template <typename T>
bool launch_div_quad(const DivFftArgs<T>& a, cudaStream_t s) {
    if (a.dtmp == nullptr || a.g.NX % 4 != 0) return false;
    div_quad_launch<T>(a, a.dtmp, s);
    return true;
}

template bool launch_div_quad<double>(const DivFftArgs<double>&, cudaStream_t);
template bool launch_div_quad<float>(const DivFftArgs<float>&, cudaStream_t);
template bool launch_yfft_reg<double>(const YFftArgs<double>&, cudaStream_t);
template bool launch_yfft_reg<float>(const YFftArgs<float>&, cudaStream_t);
template int launch_div_xfft_reg<double>(const DivFftArgs<double>&, cudaStream_t);
template int launch_div_xfft_reg<float>(const DivFftArgs<float>&, cudaStream_t);
template bool launch_ixfft_reg<double>(const IxFftArgs<double>&, cudaStream_t);
template bool launch_ixfft_reg<float>(const IxFftArgs<float>&, cudaStream_t);

}  // namespace tc
