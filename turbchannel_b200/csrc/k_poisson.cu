// k_poisson.cu -- pressure Poisson solve of the SBDF3 step on sm_100a.
//
// The reference solves L p = div(RHS) with a 2-D FFT over each z-plane (cuFFT
// D2Z / FFTW), one banded solve per (kx, ky) mode along z, the inverse FFT, a 1/NXY
// scale and a separate normalisation pass (staggered/func_global.h:214-248,
// 71-189, 657-675).  Here the same algorithm runs as four kernels over a half
// spectrum laid out spec[z][kx][ky] (ky fastest, kx = 0..NX/2):
//   k_div_xfft : divergence of the RHS (HW2 :306-312, VV4 :325-333, collocated
//                collocated_AB3/func_global.h:310-325) computed straight into shared
//                memory, two rows packed as one complex FFT along x, unpacked to the
//                half spectrum;
//   k_yfft     : complex FFT along y of contiguous lines (forward and inverse);
//   k_zsolve   : banded elimination per mode (tridiagonal for HW2 and collocated,
//                7-diagonal for VV4) with the pin of the mean mode; the pressure
//                normalisation only touches mode (0,0), so it is applied there in
//                spectral space instead of as a separate pass;
//   k_ixfft    : inverse real FFT along x (two rows per complex FFT) and the 1/NXY
//                scale, writing p.
// In the mixed mode the modes with small |k| (including (0,0)) are solved in
// double from the float spectrum; all others in float.
#include <algorithm>

#include "kernels.cuh"
#include "stencil_div.cuh"

namespace tc {

// ---------------------------------------------------------------------------
// divergence + forward x-FFT
// ---------------------------------------------------------------------------
template <typename T, int SCHEME, bool SCALAR, int ROWS>
__global__ void __launch_bounds__(256) k_div_xfft(DivFftArgs<T> a) {
    constexpr int rows = ROWS;
    extern __shared__ __align__(16) unsigned char smraw[];
    const Geom& g = a.g;
    const int NX = g.NX, NY = g.NY, NXH = g.NXH;
    const int nl = rows >> 1;
    cplx<T>* A = reinterpret_cast<cplx<T>*>(smraw);
    cplx<T>* B = A + nl * NX;
    const int z = blockIdx.y, y0 = blockIdx.x * rows;
    T* Ar = reinterpret_cast<T*>(A);
    for (int e = threadIdx.x; e < rows * NX; e += blockDim.x) {
        const int r = e / NX, x = e - r * NX;
        Ar[2 * ((r >> 1) * NX + x) + (r & 1)] = div_at<T, SCHEME, SCALAR>(g, a.m, a.v, a.src_scalar, x, y0 + r, z);
    }
    const cplx<T>* R = fft_lines_any(A, B, nl, NX, a.px, a.twx, -1);
    for (int e = threadIdx.x; e < NXH * rows; e += blockDim.x) {
        const int kx = e / rows, r = e - kx * rows, l = r >> 1;
        const cplx<T> Zk = R[l * NX + kx], Zm = R[l * NX + (kx == 0 ? 0 : NX - kx)];
        cplx<T> val;
        if ((r & 1) == 0) val = {T(0.5) * (Zk.x + Zm.x), T(0.5) * (Zk.y - Zm.y)};
        else val = {T(0.5) * (Zk.y + Zm.y), -T(0.5) * (Zk.x - Zm.x)};
        a.spec[((size_t)z * NXH + kx) * NY + y0 + r] = val;
    }
}

static int pick_rows(int NX, int NY, size_t cbytes) {
    for (int r : {8, 4, 2})
        if (NY % r == 0 && (size_t)r * NX * cbytes <= 100 * 1024) return r;
    return 2;
}

template <typename T>
int launch_div_xfft(const DivFftArgs<T>& a, cudaStream_t s) {
    if (const int n = launch_div_xfft_reg<T>(a, s)) return n;
    const int rows = pick_rows(a.g.NX, a.g.NY, sizeof(cplx<T>));
    const size_t smem = (size_t)rows * a.g.NX * sizeof(cplx<T>);
    dim3 grid(a.g.NY / rows, a.g.NZ);
#define TC_LDX(SCH, SC)                                                                                 \
    {                                                                                                   \
        auto k = rows == 8 ? k_div_xfft<T, SCH, SC, 8> : rows == 4 ? k_div_xfft<T, SCH, SC, 4> : k_div_xfft<T, SCH, SC, 2>; \
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);               \
        k<<<grid, 256, smem, s>>>(a);                                                                   \
    }
    if (a.src_scalar) TC_LDX(TC_SCHEME_HW2, true)
    else if (a.g.scheme == TC_SCHEME_HW2) TC_LDX(TC_SCHEME_HW2, false)
    else if (a.g.scheme == TC_SCHEME_VV4) TC_LDX(TC_SCHEME_VV4, false)
    else TC_LDX(TC_SCHEME_COLLOC, false)
#undef TC_LDX
    return 1;
}

// ---------------------------------------------------------------------------
// y-FFT on contiguous lines
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_yfft(YFftArgs<T> a, int lines) {
    extern __shared__ __align__(16) unsigned char smraw[];
    const int NY = a.g.NY;
    const long long total = (long long)a.g.NZ * a.g.NXH;
    const long long L0 = (long long)blockIdx.x * lines;
    const int nl = (int)min((long long)lines, total - L0);
    cplx<T>* A = reinterpret_cast<cplx<T>*>(smraw);
    cplx<T>* B = A + lines * NY;
    cplx<T>* src = a.spec + L0 * NY;
    // nl*NY complex values, contiguous and 16-byte aligned (NY even)
    constexpr int PC = 16 / sizeof(cplx<T>);  // complex values per 16-byte chunk
    const int nch = nl * NY / PC;
    for (int e = threadIdx.x; e < nch; e += blockDim.x) cp_async<16>(A + e * PC, src + e * PC);
    cp_async_commit();
    cp_async_wait<0>();
    const cplx<T>* R = fft_lines_any(A, B, nl, NY, a.py, a.twy, a.sign);
    const int4* r4 = reinterpret_cast<const int4*>(R);
    int4* d4 = reinterpret_cast<int4*>(src);
    for (int e = threadIdx.x; e < nch; e += blockDim.x) d4[e] = r4[e];
}

template <typename T>
void launch_yfft(const YFftArgs<T>& a, cudaStream_t s) {
    if (launch_yfft_reg<T>(a, s)) return;
    int lines = std::max(1, std::min(16, 4096 / a.g.NY));
    while (lines > 1 && (size_t)2 * lines * a.g.NY * sizeof(cplx<T>) > 96 * 1024) lines >>= 1;
    const size_t smem = (size_t)2 * lines * a.g.NY * sizeof(cplx<T>);
    const long long total = (long long)a.g.NZ * a.g.NXH;
    auto k = k_yfft<T>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k<<<(unsigned)((total + lines - 1) / lines), 256, smem, s>>>(a, lines);
}

// ---------------------------------------------------------------------------
// Banded z-solve per mode
// ---------------------------------------------------------------------------
template <typename C, typename T>
__device__ __forceinline__ const C* pickm(const T* t, const double* d) {
    if constexpr (sizeof(C) == sizeof(double)) return reinterpret_cast<const C*>(d);
    else return reinterpret_cast<const C*>(t);
}

template <typename C, typename T>
__device__ __forceinline__ cplx<C> ldc(const cplx<T>* p) {
    const cplx<T> v = *p;
    return {(C)v.x, (C)v.y};
}
template <typename C, typename T>
__device__ __forceinline__ void stc(cplx<T>* p, cplx<C> v) {
    *p = {(T)v.x, (T)v.y};
}

// Mean-mode normalisation in spectral space (equivalent to NormalizePressure
// applied after the inverse FFT): x_iz -= NXY * p_shift * profile_iz.
template <typename T>
__device__ void normalize_mean_mode(const ZSolveArgs<T>& a) {
    const Geom& g = a.g;
    const size_t zs = (size_t)g.NXH * g.NY;
    cplx<T>* x = a.spec;
    double psum = 0;
    if (g.scheme == TC_SCHEME_VV4) {
        for (int i = 0; i < g.NZ; i++) psum += (double)x[i * zs].x * a.m.dKERG[i] * a.m.dDZ[i];
        const double c = psum / a.m.KERG_norm2;
        for (int i = 0; i < g.NZ; i++) x[i * zs].x = (T)((double)x[i * zs].x - c * a.m.dKERG[i]);
    } else if (g.scheme == TC_SCHEME_HW2) {
        for (int i = 0; i < g.NZ; i++) psum += (double)x[i * zs].x * a.m.dDZ[i];
        const double c = psum / (a.m.dZZ[g.NZ] - a.m.dZZ[0]);
        for (int i = 0; i < g.NZ; i++) x[i * zs].x = (T)((double)x[i * zs].x - c);
    } else {
        // collocated_AB3/func_global.h:163-170 (shift = sum(p vol) hx hy / area) or, for
        // the SRK step, collocated_SRK/func_global.h:130-137 (shift = sum(p vol) / area)
        for (int i = 0; i < g.NZ; i++) psum += (double)x[i * zs].x * (a.m.dcellh[i] * g.hx * g.hy);
        const double c = (double)g.NXY * (g.norm_srk ? psum / g.area : psum * g.hx * g.hy / g.area);
        for (int i = 0; i < g.NZ; i++) x[i * zs].x = (T)((double)x[i * zs].x - c);
    }
}

// x: the mode's column (stride zs between z), sc: its elimination coefficients
// (stride M between rows); MA, DZ, DZW: the banded-matrix mesh arrays (global or
// shared memory).  Rows are fetched ZR at a time ahead of the recurrence so their
// load latency overlaps it.
constexpr int ZR = 4;

template <typename C, typename T, int SCHEME>
__device__ void zsolve_mode_at(const ZSolveArgs<T>& a, int kx, int ky, C* sc, cplx<T>* x, size_t zs, size_t M,
                               const C* MA, const C* DZ, const C* DZW) {
    const Geom& g = a.g;
    const int NZ = g.NZ;
    const bool pin = (kx == 0 && ky == 0);
    if (SCHEME == TC_SCHEME_HW2 || SCHEME == TC_SCHEME_COLLOC) {
        C MM;
        if (SCHEME == TC_SCHEME_HW2) {
            MM = 2 * ((1 - (C)a.tabs.cosx[kx]) * (C)g.inv_hx * (C)g.inv_hx + (1 - (C)a.tabs.cosy[ky]) * (C)g.inv_hy * (C)g.inv_hy);
        } else {
            MM = (1 - (C)a.tabs.cosx[kx]) * (C)g.hy / (C)g.hx + (1 - (C)a.tabs.cosy[ky]) * (C)g.hx / (C)g.hy;
        }
        C b0;
        if (SCHEME == TC_SCHEME_HW2) b0 = -DZ[0] * MM - MA[1];
        else {
            b0 = -MA[1];
            if (!g.fd_mode) b0 += DZ[0] * MM;
        }
        if (pin) b0 *= 2;
        const C ib0 = 1 / b0;
        cplx<C> prev = ldc<C>(x);
        prev.x *= ib0;
        prev.y *= ib0;
        stc(x, prev);
        C pp = MA[1] * ib0;
        sc[0] = pp;
        for (int i0 = 1; i0 <= NZ - 1; i0 += ZR) {
            cplx<C> xv[ZR];
#pragma unroll
            for (int k = 0; k < ZR; k++)
                if (i0 + k <= NZ - 1) xv[k] = ldc<C>(x + (size_t)(i0 + k) * zs);
#pragma unroll
            for (int k = 0; k < ZR; k++) {
                const int i = i0 + k;
                if (i > NZ - 1) break;
                C d;
                if (SCHEME == TC_SCHEME_HW2) {
                    d = -MA[i] - DZ[i] * MM;
                    if (i != NZ - 1) d -= MA[i + 1];
                } else {
                    const C mm = (g.fd_mode && (i == NZ - 1)) ? C(0) : MM;
                    d = 0;
                    d -= MA[i] + DZ[i - 1] * mm;
                    if (i != NZ - 1) d -= MA[i + 1] + DZ[i] * mm;
                }
                d -= MA[i] * pp;
                d = 1 / d;
                if (i != NZ - 1) {
                    pp = MA[i + 1] * d;
                    sc[(size_t)i * M] = pp;
                }
                cplx<C> xi = xv[k];
                xi.x = (xi.x - MA[i] * prev.x) * d;
                xi.y = (xi.y - MA[i] * prev.y) * d;
                stc(x + (size_t)i * zs, xi);
                prev = xi;
            }
        }
        for (int i0 = NZ - 2; i0 >= 0; i0 -= ZR) {
            cplx<C> xv[ZR];
            C pv[ZR];
#pragma unroll
            for (int k = 0; k < ZR; k++)
                if (i0 - k >= 0) {
                    xv[k] = ldc<C>(x + (size_t)(i0 - k) * zs);
                    pv[k] = sc[(size_t)(i0 - k) * M];
                }
#pragma unroll
            for (int k = 0; k < ZR; k++) {
                const int i = i0 - k;
                if (i < 0) break;
                cplx<C> xi = xv[k];
                xi.x -= prev.x * pv[k];
                xi.y -= prev.y * pv[k];
                stc(x + (size_t)i * zs, xi);
                prev = xi;
            }
        }
    } else {  // VV4, staggered/func_global.h:110-189
        const C C27 = C(0.03703703703703703703), C9 = C(0.11111111111111111111);
        const C sx = (C)a.tabs.sinx[kx], sy = (C)a.tabs.siny[ky];
        const C s3x = 3 * sx - 4 * sx * sx * sx, s3y = 3 * sy - 4 * sy * sy * sy;
        const C ihx = (C)g.inv_hx, ihy = (C)g.inv_hy;
        const C tiny = C(1e-30);
        C b[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};  // b[j][k]: row i-3+j, coefficient of x_{row+k+1}
        cplx<C> xr[3] = {{0, 0}, {0, 0}, {0, 0}};       // eliminated rhs of rows i-3, i-2, i-1
        for (int i0 = 0; i0 < NZ; i0 += ZR) {
            cplx<C> xv[ZR];
#pragma unroll
            for (int k = 0; k < ZR; k++)
                if (i0 + k < NZ) xv[k] = ldc<C>(x + (size_t)(i0 + k) * zs);
#pragma unroll
            for (int kk = 0; kk < ZR; kk++) {
                const int i = i0 + kk;
                if (i >= NZ) break;
                C row[7] = {0, 0, 0, 0, 0, 0, 0};
                C sum = 0;
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    if (i + k - 3 < 0 || i + k - 3 >= NZ) continue;
                    row[k] = MA[i * 3 + k];
                    sum += MA[i * 3 + k];
                }
#pragma unroll
                for (int k = 1; k <= 3; k++) {
                    if (i + k >= NZ) continue;
                    row[3 + k] = MA[(i + k) * 3 + 3 - k];
                    sum += MA[(i + k) * 3 + 3 - k];
                }
                if (i <= 2) row[3] = (C)a.m.MAT_D[i];
                else if (i >= NZ - 3) row[3] = (C)a.m.MAT_D[i - (NZ - 3) + 3];
                else row[3] = -sum;
                if (pin && i == 0) row[3] *= 2;
                {
                    C ci = DZ[i] * sx - C27 * DZW[i] * s3x;
                    row[3] -= 4 * ihx * ihx * ci * ci / (DZ[i] - C9 * DZW[i]);
                    ci = DZ[i] * sy - C27 * DZW[i] * s3y;
                    row[3] -= 4 * ihy * ihy * ci * ci / (DZ[i] - C9 * DZW[i]);
                }
                cplx<C> xi = xv[kk];
#pragma unroll
                for (int j = -3; j < 0; j++) {
                    if (i + j < 0) continue;
                    const C mult = -row[3 + j];
#pragma unroll
                    for (int k = 1; k <= 3; k++) {
                        if (i + j + k >= NZ) continue;
                        row[3 + j + k] += mult * b[3 + j][k - 1];
                    }
                    xi.x += mult * xr[3 + j].x;
                    xi.y += mult * xr[3 + j].y;
                }
                if (fabs((double)row[3]) < (double)tiny) {
                    if (a.err_flag) atomicExch(a.err_flag, 1);
                    cplx<T> bad = {(T)(sizeof(T) == 8 ? -1e50 : -1e30), (T)0};
                    x[0] = bad;
                    return;
                }
                const C mult = C(1) / row[3];
                C nb[3];
#pragma unroll
                for (int k = 1; k <= 3; k++) nb[k - 1] = (i + k >= NZ) ? C(0) : row[3 + k] * mult;
                xi.x *= mult;
                xi.y *= mult;
                stc(x + (size_t)i * zs, xi);
#pragma unroll
                for (int k = 0; k < 3; k++) sc[((size_t)i * 3 + k) * M] = nb[k];
#pragma unroll
                for (int j = 0; j < 2; j++) {
                    xr[j] = xr[j + 1];
#pragma unroll
                    for (int k = 0; k < 3; k++) b[j][k] = b[j + 1][k];
                }
                xr[2] = xi;
#pragma unroll
                for (int k = 0; k < 3; k++) b[2][k] = nb[k];
            }
        }
        cplx<C> xs[3] = {{0, 0}, {0, 0}, {0, 0}};  // x_{i+1}, x_{i+2}, x_{i+3}
        for (int i0 = NZ - 1; i0 >= 0; i0 -= ZR) {
            cplx<C> xv[ZR];
            C bv[ZR][3];
#pragma unroll
            for (int k = 0; k < ZR; k++)
                if (i0 - k >= 0) {
                    xv[k] = ldc<C>(x + (size_t)(i0 - k) * zs);
#pragma unroll
                    for (int j = 0; j < 3; j++) bv[k][j] = sc[((size_t)(i0 - k) * 3 + j) * M];
                }
#pragma unroll
            for (int kk = 0; kk < ZR; kk++) {
                const int i = i0 - kk;
                if (i < 0) break;
                cplx<C> xi = xv[kk];
#pragma unroll
                for (int j = 1; j <= 3; j++) {
                    if (i + j >= NZ) continue;
                    xi.x -= bv[kk][j - 1] * xs[j - 1].x;
                    xi.y -= bv[kk][j - 1] * xs[j - 1].y;
                }
                stc(x + (size_t)i * zs, xi);
                xs[2] = xs[1];
                xs[1] = xs[0];
                xs[0] = xi;
            }
        }
    }
}

// All modes (FP64) or, in the mixed mode, all modes outside the low set (float).
template <typename C, typename T, int SCHEME>
__global__ void __launch_bounds__(64) k_zsolve_all(ZSolveArgs<T> a, int skip_low) {
    const Geom& g = a.g;
    const size_t M = (size_t)g.NXH * g.NY;
    const size_t m = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M) return;
    const int kx = (int)(m / g.NY), ky = (int)(m - (size_t)kx * g.NY);
    const int LM = g.low_modes;
    if (skip_low && kx < LM && (ky < LM || ky > g.NY - LM)) return;
    zsolve_mode_at<C, T, SCHEME>(a, kx, ky, reinterpret_cast<C*>(a.scratch) + m, a.spec + m, M, M,
                                 pickm<C>(a.m.MAT_A, a.m.dMAT_A), pickm<C>(a.m.DZ, a.m.dDZ),
                                 pickm<C>(a.m.DZW, a.m.dDZW));
    if (!skip_low && m == 0) normalize_mean_mode(a);
}

// The low-|k| modes (kx < LM, |ky| < LM) in double; mode (0,0) also normalised.
// One CTA per mode: the column is staged into shared memory by all threads (so
// the sequential elimination by one thread runs at shared-memory latency), the
// elimination coefficients stay in shared memory, the result is written back by
// all threads.
template <typename T, int SCHEME>
__global__ void __launch_bounds__(128) k_zsolve_low(ZSolveArgs<T> a) {
    extern __shared__ __align__(16) unsigned char smraw[];
    const Geom& g = a.g;
    const int LM = g.low_modes, nky = 2 * LM - 1;
    const int idx = blockIdx.x;
    const int kx = idx / nky, j = idx - kx * nky;
    const int ky = j < LM ? j : g.NY - (j - LM + 1);
    if (kx >= g.NXH || ky < 0 || ky >= g.NY) return;
    const int NZ = g.NZ;
    const size_t M = (size_t)g.NXH * g.NY;
    const size_t m = (size_t)kx * g.NY + ky;
    const int nc = SCHEME == TC_SCHEME_VV4 ? 3 : 1;
    const int nma = SCHEME == TC_SCHEME_VV4 ? 3 * NZ : NZ;
    cplx<double>* xs = reinterpret_cast<cplx<double>*>(smraw);
    double* sc = reinterpret_cast<double*>(xs + NZ);
    double* sMA = sc + (size_t)nc * NZ;
    double* sDZ = sMA + nma;
    double* sDZW = sDZ + NZ;
    for (int i = threadIdx.x; i < NZ; i += blockDim.x) {
        const cplx<T> v = a.spec[(size_t)i * M + m];
        xs[i] = {(double)v.x, (double)v.y};
        sDZ[i] = a.m.dDZ[i];
        sDZW[i] = a.m.dDZW[i];
    }
    for (int i = threadIdx.x; i < nma; i += blockDim.x) sMA[i] = a.m.dMAT_A[i];
    __syncthreads();
    if (threadIdx.x == 0) {
        ZSolveArgs<double> b;
        b.g = g;
        b.g.NXH = 1;
        b.g.NY = 1;  // a single column: stride 1 between z, mode index 0
        b.m.MAT_A = a.m.dMAT_A; b.m.DZ = a.m.dDZ; b.m.DZW = a.m.dDZW; b.m.KERG = a.m.dKERG; b.m.cellh = a.m.dcellh;
        b.m.ZZ = a.m.dZZ; b.m.GC1 = b.m.GC2 = b.m.GCZ = nullptr;
        b.m.dMAT_A = a.m.dMAT_A; b.m.dDZ = a.m.dDZ; b.m.dDZW = a.m.dDZW; b.m.dKERG = a.m.dKERG;
        b.m.dcellh = a.m.dcellh; b.m.dZZ = a.m.dZZ;
        for (int k = 0; k < 6; k++) b.m.MAT_D[k] = a.m.MAT_D[k];
        b.m.KERG_norm2 = a.m.KERG_norm2;
        b.tabs = a.tabs;
        b.spec = xs;
        b.scratch = sc;
        b.err_flag = a.err_flag;
        zsolve_mode_at<double, double, SCHEME>(b, kx, ky, sc, xs, 1, 1, sMA, sDZ, sDZW);
        if (m == 0) {
            b.g.NXH = 1;
            b.g.NY = 1;
            normalize_mean_mode(b);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < NZ; i += blockDim.x) {
        const cplx<double> v = xs[i];
        a.spec[(size_t)i * M + m] = {(T)v.x, (T)v.y};
    }
}

size_t zsolve_scratch_bytes(const Geom& g, int elem_bytes) {
    (void)elem_bytes;
    const int nc = g.scheme == TC_SCHEME_VV4 ? 3 : 1;
    return (size_t)g.NXH * g.NY * g.NZ * nc * sizeof(double);
}

template <typename T, int SCHEME>
static void zsolve_scheme(const ZSolveArgs<T>& a, cudaStream_t s, cudaStream_t side, cudaEvent_t fork, cudaEvent_t join) {
    const size_t M = (size_t)a.g.NXH * a.g.NY;
    if (sizeof(T) == sizeof(double)) {
        k_zsolve_all<double, T, SCHEME><<<(unsigned)((M + 63) / 64), 64, 0, s>>>(a, 0);
    } else {
        // Modes outside the low set in float first, then the low set in double.  Both
        // launches share the scratch buffer, which is sized for double entries; the
        // float kernel indexes it as float (so the low-set double entries are disjoint
        // only in time: the launches are stream-ordered).
        // the low modes (double, few and sequential) run on a side stream next to the
        // float modes; the two sets are disjoint
        cudaEventRecord(fork, s);
        cudaStreamWaitEvent(side, fork, 0);
        const int nlow = a.g.low_modes * (2 * a.g.low_modes - 1);
        const int nc = SCHEME == TC_SCHEME_VV4 ? 3 : 1;
        const int nma = SCHEME == TC_SCHEME_VV4 ? 3 * a.g.NZ : a.g.NZ;
        const size_t smem = (size_t)a.g.NZ * (sizeof(cplx<double>) + nc * sizeof(double)) + (size_t)(nma + 2 * a.g.NZ) * sizeof(double);
        auto k = k_zsolve_low<T, SCHEME>;
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k<<<nlow, 128, smem, side>>>(a);
        cudaEventRecord(join, side);
        k_zsolve_all<float, T, SCHEME><<<(unsigned)((M + 63) / 64), 64, 0, s>>>(a, 1);
        cudaStreamWaitEvent(s, join, 0);
    }
}

template <typename T>
void launch_zsolve(const ZSolveArgs<T>& a, cudaStream_t s, cudaStream_t side, cudaEvent_t fork, cudaEvent_t join) {
    if (a.g.scheme == TC_SCHEME_VV4) zsolve_scheme<T, TC_SCHEME_VV4>(a, s, side, fork, join);
    else if (a.g.scheme == TC_SCHEME_HW2) zsolve_scheme<T, TC_SCHEME_HW2>(a, s, side, fork, join);
    else zsolve_scheme<T, TC_SCHEME_COLLOC>(a, s, side, fork, join);
}

// ---------------------------------------------------------------------------
// Factored z-solve.  The z-matrix of a mode depends on the mesh and the mode only,
// not on the time step, so its elimination (the same row order, pivots and
// multipliers as zsolve_mode_at) is done once, in double, at solver creation and
// stored in the working precision T as
//   forward   z_i = F0_i r_i - F1_i z_{i-1} - F2_i z_{i-2} - F3_i z_{i-3}
//   backward  x_i = z_i - B0_i x_{i+1} - B1_i x_{i+2} - B2_i x_{i+3}
// (tridiagonal schemes: F0, F1, B0).  The matrix of mode (kx, ky) depends on ky only
// through cos(2 pi ky/NY) or sin^2(pi ky/NY), so ky and NY-ky share their factors:
// they are stored for kh = 0..NY/2 (mode index mh = kx*(NY/2+1) + kh).  Layout: VV4
// F[i][mh] = {F0,F1,F2,F3} then B[i][mh] = {B0,B1,B2,0}; tridiagonal F[i][mh] =
// {F0,F1} then B[i][mh] = B0.  The per-step solve streams r, F, B with no divide and
// a one-FMA recurrence chain, one thread per pair (ky, NY-ky) reading the factors once.
// ---------------------------------------------------------------------------

size_t zfactor_low_bytes(const Geom& g) {
    const size_t per = g.scheme == TC_SCHEME_VV4 ? 8 : 3;
    return (size_t)g.low_modes * g.low_modes * g.NZ * per * sizeof(double);
}

size_t zfactor_bytes(const Geom& g, int elem_bytes) {
    const size_t per = g.scheme == TC_SCHEME_VV4 ? 8 : 3;
    return (size_t)g.NXH * (g.NY / 2 + 1) * g.NZ * per * elem_bytes;
}

template <typename T, int SCHEME>
__global__ void __launch_bounds__(128) k_zfactor(ZSolveArgs<T> a) {
    const Geom& g = a.g;
    const int NYH1 = g.NY / 2 + 1;
    const size_t M = (size_t)g.NXH * NYH1;  // factor modes (kx, ky <= NY/2)
    const size_t m = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M) return;
    const int kx = (int)(m / NYH1), ky = (int)(m - (size_t)kx * NYH1);
    const int NZ = g.NZ;
    const bool pin = (kx == 0 && ky == 0);
    // low modes (kx, ky < LM): a double copy, mode-major [jl][row], for k_zsolve_low
    const int LM = g.low_modes;
    const bool low = a.fac_low != nullptr && kx < LM && ky < LM;
    const size_t jl = (size_t)kx * LM + ky;
    const double* MA = a.m.dMAT_A;
    const double* DZ = a.m.dDZ;
    const double* DZW = a.m.dDZW;
    if (SCHEME == TC_SCHEME_HW2 || SCHEME == TC_SCHEME_COLLOC) {
        Q2<T>* F = reinterpret_cast<Q2<T>*>(a.fac);
        T* B = reinterpret_cast<T*>(F + (size_t)NZ * M);
        double MM;
        if (SCHEME == TC_SCHEME_HW2)
            MM = 2 * ((1 - a.tabs.cosx[kx]) * g.inv_hx * g.inv_hx + (1 - a.tabs.cosy[ky]) * g.inv_hy * g.inv_hy);
        else
            MM = (1 - a.tabs.cosx[kx]) * g.hy / g.hx + (1 - a.tabs.cosy[ky]) * g.hx / g.hy;
        double b0;
        if (SCHEME == TC_SCHEME_HW2) b0 = -DZ[0] * MM - MA[1];
        else {
            b0 = -MA[1];
            if (!g.fd_mode) b0 += DZ[0] * MM;
        }
        if (pin) b0 *= 2;
        const double ib0 = 1 / b0;
        double pp = MA[1] * ib0;
        F[m] = {(T)ib0, (T)0};
        B[m] = (T)pp;
        Q2<double>* FL = reinterpret_cast<Q2<double>*>(a.fac_low) + jl * NZ;
        double* BL = reinterpret_cast<double*>(reinterpret_cast<Q2<double>*>(a.fac_low) + (size_t)LM * LM * NZ) + jl * NZ;
        if (low) {
            FL[0] = {ib0, 0.0};
            BL[0] = pp;
        }
        for (int i = 1; i <= NZ - 1; i++) {
            double d;
            if (SCHEME == TC_SCHEME_HW2) {
                d = -MA[i] - DZ[i] * MM;
                if (i != NZ - 1) d -= MA[i + 1];
            } else {
                const double mm = (g.fd_mode && (i == NZ - 1)) ? 0.0 : MM;
                d = 0;
                d -= MA[i] + DZ[i - 1] * mm;
                if (i != NZ - 1) d -= MA[i + 1] + DZ[i] * mm;
            }
            d -= MA[i] * pp;
            d = 1 / d;
            pp = i != NZ - 1 ? MA[i + 1] * d : 0.0;
            F[(size_t)i * M + m] = {(T)d, (T)(MA[i] * d)};
            B[(size_t)i * M + m] = (T)pp;
            if (low) {
                FL[i] = {d, MA[i] * d};
                BL[i] = pp;
            }
        }
    } else {
        Q4<T>* F = reinterpret_cast<Q4<T>*>(a.fac);
        Q4<T>* B = F + (size_t)NZ * M;
        Q4<double>* FL = reinterpret_cast<Q4<double>*>(a.fac_low) + jl * NZ;
        Q4<double>* BL = reinterpret_cast<Q4<double>*>(a.fac_low) + (size_t)LM * LM * NZ + jl * NZ;
        const double C27 = 0.03703703703703703703, C9 = 0.11111111111111111111;
        const double sx = a.tabs.sinx[kx], sy = a.tabs.siny[ky];
        const double s3x = 3 * sx - 4 * sx * sx * sx, s3y = 3 * sy - 4 * sy * sy * sy;
        const double ihx = g.inv_hx, ihy = g.inv_hy;
        double b[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        for (int i = 0; i < NZ; i++) {
            double row[7] = {0, 0, 0, 0, 0, 0, 0};
            double sum = 0;
            for (int k = 0; k < 3; k++) {
                if (i + k - 3 < 0 || i + k - 3 >= NZ) continue;
                row[k] = MA[i * 3 + k];
                sum += MA[i * 3 + k];
            }
            for (int k = 1; k <= 3; k++) {
                if (i + k >= NZ) continue;
                row[3 + k] = MA[(i + k) * 3 + 3 - k];
                sum += MA[(i + k) * 3 + 3 - k];
            }
            if (i <= 2) row[3] = a.m.MAT_D[i];
            else if (i >= NZ - 3) row[3] = a.m.MAT_D[i - (NZ - 3) + 3];
            else row[3] = -sum;
            if (pin && i == 0) row[3] *= 2;
            {
                double ci = DZ[i] * sx - C27 * DZW[i] * s3x;
                row[3] -= 4 * ihx * ihx * ci * ci / (DZ[i] - C9 * DZW[i]);
                ci = DZ[i] * sy - C27 * DZW[i] * s3y;
                row[3] -= 4 * ihy * ihy * ci * ci / (DZ[i] - C9 * DZW[i]);
            }
            double used[3] = {0, 0, 0};  // row entry eliminated against z_{i-3}, z_{i-2}, z_{i-1}
            for (int j = -3; j < 0; j++) {
                if (i + j < 0) continue;
                used[3 + j] = row[3 + j];
                const double mult = -row[3 + j];
                for (int k = 1; k <= 3; k++) {
                    if (i + j + k >= NZ) continue;
                    row[3 + j + k] += mult * b[3 + j][k - 1];
                }
            }
            if (fabs(row[3]) < 1e-30) {
                if (a.err_flag) atomicExch(a.err_flag, 1);
                return;
            }
            const double inv = 1.0 / row[3];
            double nb[3];
            for (int k = 1; k <= 3; k++) nb[k - 1] = (i + k >= NZ) ? 0.0 : row[3 + k] * inv;
            F[(size_t)i * M + m] = {(T)inv, (T)(used[2] * inv), (T)(used[1] * inv), (T)(used[0] * inv)};
            B[(size_t)i * M + m] = {(T)nb[0], (T)nb[1], (T)nb[2], (T)0};
            if (low) {
                FL[i] = {inv, used[2] * inv, used[1] * inv, used[0] * inv};
                BL[i] = {nb[0], nb[1], nb[2], 0.0};
            }
            for (int j = 0; j < 2; j++)
                for (int k = 0; k < 3; k++) b[j][k] = b[j + 1][k];
            for (int k = 0; k < 3; k++) b[2][k] = nb[k];
        }
    }
}

template <typename T>
void launch_zfactor(const ZSolveArgs<T>& a, cudaStream_t s) {
    const size_t M = (size_t)a.g.NXH * (a.g.NY / 2 + 1);
    const unsigned nb = (unsigned)((M + 127) / 128);
    if (a.g.scheme == TC_SCHEME_VV4) k_zfactor<T, TC_SCHEME_VV4><<<nb, 128, 0, s>>>(a);
    else if (a.g.scheme == TC_SCHEME_HW2) k_zfactor<T, TC_SCHEME_HW2><<<nb, 128, 0, s>>>(a);
    else k_zfactor<T, TC_SCHEME_COLLOC><<<nb, 128, 0, s>>>(a);
}

// One thread per mode outside the low set.  Adjacent lanes take the two modes
// (kx, kh), (kx, NY-kh) that share their factors, so a warp's factor loads fetch each
// factor row once (two lanes, one address).  Rows are moved R at a time through two
// register batches: the loads of batch b+1 are issued before batch b is consumed.
template <typename T, int SCHEME>
__global__ void __launch_bounds__(128) k_zsolve_fac(ZSolveArgs<T> a) {
    constexpr bool VV = SCHEME == TC_SCHEME_VV4;
    // rows per register batch: as deep as keeps the kernel at 4 (float, 120 registers) or 5
    // (double, 96) CTAs of 128 threads per SM, so that the ~74 k mode threads of a
    // 384 x 384 plane run as one wave (measured at 384x256x384: float 8 rows, 152 registers,
    // 1.3 waves: 0.176 ms; 6 rows 0.152; 5 rows 0.158; double 4 rows 0.318, 3 rows 0.296,
    // 2 rows 0.292)
    constexpr int R = sizeof(T) == 4 ? 6 : 2;
    using FQ = typename std::conditional<VV, Q4<T>, Q2<T>>::type;
    using BQ = typename std::conditional<VV, Q4<T>, T>::type;
    const Geom& g = a.g;
    const int NY = g.NY, NYH1 = NY / 2 + 1;
    const size_t M = (size_t)g.NXH * NY, MH = (size_t)g.NXH * NYH1;
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t mh = t >> 1;
    if (mh >= MH) return;
    const int kx = (int)(mh / NYH1), kh = (int)(mh - (size_t)kx * NYH1);
    if ((t & 1) && (kh == 0 || 2 * kh == NY)) return;  // no partner mode
    const int LM = g.low_modes;
    if (kx < LM && kh < LM) return;
    const int ky = (t & 1) ? NY - kh : kh;
    const int NZ = g.NZ;
    const FQ* F = reinterpret_cast<const FQ*>(a.fac) + mh;
    const BQ* B = reinterpret_cast<const BQ*>(reinterpret_cast<const FQ*>(a.fac) + (size_t)NZ * MH) + mh;
    cplx<T>* x = a.spec + (size_t)kx * NY + ky;

    // forward
    {
        cplx<T> z1 = {0, 0}, z2 = {0, 0}, z3 = {0, 0};
        cplx<T> ra[R], rb[R];
        FQ fa[R], fb[R];
        auto load = [&](int i0, cplx<T>(&r)[R], FQ(&f)[R]) {
#pragma unroll
            for (int k = 0; k < R; k++)
                if (i0 + k < NZ) {
                    r[k] = x[(size_t)(i0 + k) * M];
                    f[k] = F[(size_t)(i0 + k) * MH];
                }
        };
        auto run = [&](int i0, const cplx<T>(&r)[R], const FQ(&f)[R]) {
#pragma unroll
            for (int k = 0; k < R; k++) {
                if (i0 + k >= NZ) break;
                cplx<T> z;
                if constexpr (VV) {
                    z.x = r[k].x * f[k].x - f[k].w * z3.x - f[k].z * z2.x;
                    z.y = r[k].y * f[k].x - f[k].w * z3.y - f[k].z * z2.y;
                } else {
                    z.x = r[k].x * f[k].x;
                    z.y = r[k].y * f[k].x;
                }
                z.x -= f[k].y * z1.x;
                z.y -= f[k].y * z1.y;
                x[(size_t)(i0 + k) * M] = z;
                z3 = z2;
                z2 = z1;
                z1 = z;
            }
        };
        load(0, ra, fa);
        for (int i0 = 0; i0 < NZ; i0 += 2 * R) {
            load(i0 + R, rb, fb);
            run(i0, ra, fa);
            load(i0 + 2 * R, ra, fa);
            run(i0 + R, rb, fb);
        }
    }
    // backward (row NZ-1 first)
    {
        cplx<T> x1 = {0, 0}, x2 = {0, 0}, x3 = {0, 0};
        cplx<T> za[R], zb[R];
        BQ ba[R], bb[R];
        auto load = [&](int i0, cplx<T>(&zz)[R], BQ(&bq)[R]) {
#pragma unroll
            for (int k = 0; k < R; k++)
                if (i0 - k >= 0) {
                    zz[k] = x[(size_t)(i0 - k) * M];
                    bq[k] = B[(size_t)(i0 - k) * MH];
                }
        };
        auto run = [&](int i0, const cplx<T>(&zz)[R], const BQ(&bq)[R]) {
#pragma unroll
            for (int k = 0; k < R; k++) {
                if (i0 - k < 0) break;
                cplx<T> v;
                if constexpr (VV) {
                    v.x = zz[k].x - bq[k].z * x3.x - bq[k].y * x2.x;
                    v.y = zz[k].y - bq[k].z * x3.y - bq[k].y * x2.y;
                    v.x -= bq[k].x * x1.x;
                    v.y -= bq[k].x * x1.y;
                } else {
                    v.x = zz[k].x - bq[k] * x1.x;
                    v.y = zz[k].y - bq[k] * x1.y;
                }
                x[(size_t)(i0 - k) * M] = v;
                x3 = x2;
                x2 = x1;
                x1 = v;
            }
        };
        load(NZ - 1, za, ba);
        for (int i0 = NZ - 1; i0 >= 0; i0 -= 2 * R) {
            load(i0 - R, zb, bb);
            run(i0, za, ba);
            load(i0 - 2 * R, za, ba);
            run(i0 - R, zb, bb);
        }
    }
}

// The low-|k| modes (kx < LM, |ky| < LM) in double from their double factors; mode
// (0,0) also normalised.  One CTA per mode: the column and its factors are staged into
// shared memory by all threads, one thread runs the two sweeps there, LOWB rows at a
// time (the batch's shared loads issued before its recurrence, so only the one-FMA
// chain per row is serial), all threads normalise the mean mode and write the column
// back.
constexpr int LOWB = 8;

// Mean-mode normalisation of a column held in shared memory (stride 1), every thread
// of the CTA taking part: the same shift as normalize_mean_mode, the weighted sum
// reduced over the CTA instead of one thread.
template <typename MD>
__device__ void normalize_mean_column(const Geom& g, const MD& m, cplx<double>* xs, double* red) {
    const int NZ = g.NZ;
    double part = 0;
    for (int i = threadIdx.x; i < NZ; i += blockDim.x) {
        double wgt;
        if (g.scheme == TC_SCHEME_VV4) wgt = m.dKERG[i] * m.dDZ[i];
        else if (g.scheme == TC_SCHEME_HW2) wgt = m.dDZ[i];
        else wgt = m.dcellh[i] * g.hx * g.hy;
        part += xs[i].x * wgt;
    }
    part = warp_sum(part);
    const int nw = (int)(blockDim.x >> 5);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = part;
    __syncthreads();
    double psum = 0;
    for (int w = 0; w < nw; w++) psum += red[w];
    double c;
    if (g.scheme == TC_SCHEME_VV4) c = psum / m.KERG_norm2;
    else if (g.scheme == TC_SCHEME_HW2) c = psum / (m.dZZ[NZ] - m.dZZ[0]);
    else c = (double)g.NXY * (g.norm_srk ? psum / g.area : psum * g.hx * g.hy / g.area);
    for (int i = threadIdx.x; i < NZ; i += blockDim.x)
        xs[i].x -= g.scheme == TC_SCHEME_VV4 ? c * m.dKERG[i] : c;
    __syncthreads();
}

template <typename T, int SCHEME>
__global__ void __launch_bounds__(128) k_zsolve_low_fac(ZSolveArgs<T> a) {
    constexpr bool VV = SCHEME == TC_SCHEME_VV4;
    using FQ = typename std::conditional<VV, Q4<double>, Q2<double>>::type;
    using BQ = typename std::conditional<VV, Q4<double>, double>::type;
    extern __shared__ __align__(32) unsigned char smraw[];
    __shared__ double red[4];
    const Geom& g = a.g;
    const int LM = g.low_modes, nky = 2 * LM - 1;
    const int idx = blockIdx.x;
    const int kx = idx / nky, j = idx - kx * nky;
    const int ky = j < LM ? j : g.NY - (j - LM + 1);
    if (kx >= g.NXH || ky < 0 || ky >= g.NY) return;
    const int kh = j < LM ? j : j - LM + 1;  // min(ky, NY - ky)
    const int NZ = g.NZ;
    const size_t M = (size_t)g.NXH * g.NY;
    const size_t m = (size_t)kx * g.NY + ky;
    const size_t jl = (size_t)kx * LM + kh;
    // shared layout: F rows, B rows, then the column at a 32-byte boundary
    FQ* sF = reinterpret_cast<FQ*>(smraw);
    BQ* sB = reinterpret_cast<BQ*>(sF + NZ);
    const size_t xo = ((size_t)NZ * (sizeof(FQ) + sizeof(BQ)) + 31) & ~(size_t)31;
    cplx<double>* xs = reinterpret_cast<cplx<double>*>(smraw + xo);
    const FQ* F = reinterpret_cast<const FQ*>(a.fac_low) + jl * NZ;
    const BQ* B = reinterpret_cast<const BQ*>(reinterpret_cast<const FQ*>(a.fac_low) + (size_t)LM * LM * NZ) + jl * NZ;
    for (int i = threadIdx.x; i < NZ; i += blockDim.x) {
        const cplx<T> v = a.spec[(size_t)i * M + m];
        xs[i] = {(double)v.x, (double)v.y};
        sF[i] = F[i];
        sB[i] = B[i];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        cplx<double> z1 = {0, 0}, z2 = {0, 0}, z3 = {0, 0};
        for (int i0 = 0; i0 < NZ; i0 += LOWB) {
            FQ f[LOWB];
            cplx<double> r[LOWB];
#pragma unroll
            for (int k = 0; k < LOWB; k++)
                if (i0 + k < NZ) {
                    f[k] = sF[i0 + k];
                    r[k] = xs[i0 + k];
                }
#pragma unroll
            for (int k = 0; k < LOWB; k++) {
                if (i0 + k >= NZ) break;
                cplx<double> z;
                if constexpr (VV) {
                    z.x = r[k].x * f[k].x - f[k].w * z3.x - f[k].z * z2.x;
                    z.y = r[k].y * f[k].x - f[k].w * z3.y - f[k].z * z2.y;
                } else {
                    z.x = r[k].x * f[k].x;
                    z.y = r[k].y * f[k].x;
                }
                z.x -= f[k].y * z1.x;
                z.y -= f[k].y * z1.y;
                xs[i0 + k] = z;
                z3 = z2;
                z2 = z1;
                z1 = z;
            }
        }
        cplx<double> x1 = {0, 0}, x2 = {0, 0}, x3 = {0, 0};
        for (int i0 = NZ - 1; i0 >= 0; i0 -= LOWB) {
            BQ bq[LOWB];
            cplx<double> zz[LOWB];
#pragma unroll
            for (int k = 0; k < LOWB; k++)
                if (i0 - k >= 0) {
                    bq[k] = sB[i0 - k];
                    zz[k] = xs[i0 - k];
                }
#pragma unroll
            for (int k = 0; k < LOWB; k++) {
                if (i0 - k < 0) break;
                cplx<double> v;
                if constexpr (VV) {
                    v.x = zz[k].x - bq[k].z * x3.x - bq[k].y * x2.x;
                    v.y = zz[k].y - bq[k].z * x3.y - bq[k].y * x2.y;
                    v.x -= bq[k].x * x1.x;
                    v.y -= bq[k].x * x1.y;
                } else {
                    v.x = zz[k].x - bq[k] * x1.x;
                    v.y = zz[k].y - bq[k] * x1.y;
                }
                xs[i0 - k] = v;
                x3 = x2;
                x2 = x1;
                x1 = v;
            }
        }
    }
    __syncthreads();
    if (m == 0) normalize_mean_column(g, a.m, xs, red);
    for (int i = threadIdx.x; i < NZ; i += blockDim.x) {
        const cplx<double> v = xs[i];
        a.spec[(size_t)i * M + m] = {(T)v.x, (T)v.y};
    }
}

template <typename T, int SCHEME>
static void zsolve_low_scheme(const ZSolveArgs<T>& a, cudaStream_t s) {
    const int nlow = a.g.low_modes * (2 * a.g.low_modes - 1);
    const size_t smem = (((size_t)a.g.NZ * (SCHEME == TC_SCHEME_VV4 ? 64 : 24) + 31) & ~(size_t)31) +
                        (size_t)a.g.NZ * sizeof(cplx<double>);
    auto k = k_zsolve_low_fac<T, SCHEME>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k<<<nlow, 128, smem, s>>>(a);
}

template <typename T, int SCHEME>
static void zsolve_fac_scheme(const ZSolveArgs<T>& a, cudaStream_t s, cudaStream_t side, cudaEvent_t fork,
                              cudaEvent_t join) {
        // the low modes (exact elimination in double, mode (0,0) normalised) on a side
    // stream next to the factored solve of all other modes; the two sets are disjoint
    cudaEventRecord(fork, s);
    cudaStreamWaitEvent(side, fork, 0);
    zsolve_low_scheme<T, SCHEME>(a, side);
    cudaEventRecord(join, side);
    const size_t MH = (size_t)a.g.NXH * (a.g.NY / 2 + 1);
    k_zsolve_fac<T, SCHEME><<<(unsigned)((2 * MH + 127) / 128), 128, 0, s>>>(a);
    cudaStreamWaitEvent(s, join, 0);
}

template <typename T>
void launch_zsolve_fac(const ZSolveArgs<T>& a, cudaStream_t s, cudaStream_t side, cudaEvent_t fork, cudaEvent_t join) {
    if (a.g.scheme == TC_SCHEME_VV4) zsolve_fac_scheme<T, TC_SCHEME_VV4>(a, s, side, fork, join);
    else if (a.g.scheme == TC_SCHEME_HW2) zsolve_fac_scheme<T, TC_SCHEME_HW2>(a, s, side, fork, join);
    else zsolve_fac_scheme<T, TC_SCHEME_COLLOC>(a, s, side, fork, join);
}

// ---------------------------------------------------------------------------
// inverse x-FFT (complex-to-real, two rows per complex FFT) and scaling
// ---------------------------------------------------------------------------
template <typename T, int ROWS>
__global__ void __launch_bounds__(256) k_ixfft(IxFftArgs<T> a) {
    constexpr int rows = ROWS;
    extern __shared__ __align__(16) unsigned char smraw[];
    const Geom& g = a.g;
    const int NX = g.NX, NY = g.NY, NXH = g.NXH;
    const int nl = rows >> 1;
    cplx<T>* A = reinterpret_cast<cplx<T>*>(smraw);
    cplx<T>* B = A + nl * NX;  // also holds the loaded tile (rows x NXH)
    cplx<T>* tile = B;
    const int z = blockIdx.y, y0 = blockIdx.x * rows;
    for (int e = threadIdx.x; e < NXH * rows; e += blockDim.x) {
        const int kx = e / rows, r = e - kx * rows;
        tile[r * NXH + kx] = a.spec[((size_t)z * NXH + kx) * NY + y0 + r];
    }
    __syncthreads();  // (row-major tile: rows x NXH)
    const int nh = NX / 2;
    for (int e = threadIdx.x; e < nl * NX; e += blockDim.x) {
        const int l = e / NX, k = e - l * NX;
        const int ra = 2 * l, rb = 2 * l + 1;
        cplx<T> av, bv;
        if (k <= nh) {
            av = tile[ra * NXH + k];
            bv = tile[rb * NXH + k];
        } else {
            av = tile[ra * NXH + NX - k];
            bv = tile[rb * NXH + NX - k];
            av.y = -av.y;
            bv.y = -bv.y;
        }
        if (k == 0 || k == nh) {
            av.y = 0;
            bv.y = 0;
        }
        A[l * NX + k] = {av.x - bv.y, av.y + bv.x};
    }
    const cplx<T>* R = fft_lines_any(A, B, nl, NX, a.px, a.twx, +1);
    const T sc = a.scale;
    for (int e = threadIdx.x; e < rows * NX; e += blockDim.x) {
        const int r = e / NX, x = e - r * NX;
        const cplx<T> zv = R[(r >> 1) * NX + x];
        a.p[((size_t)z * NY + y0 + r) * NX + x] = ((r & 1) ? zv.y : zv.x) * sc;
    }
}

template <typename T>
void launch_ixfft(const IxFftArgs<T>& a, cudaStream_t s) {
    if (launch_ixfft_reg<T>(a, s)) return;
    const int rows = pick_rows(a.g.NX, a.g.NY, sizeof(cplx<T>));
    const size_t nl = rows / 2;
    const size_t smem = (nl * a.g.NX + std::max(nl * a.g.NX, (size_t)rows * a.g.NXH)) * sizeof(cplx<T>);
    auto k = rows == 8 ? k_ixfft<T, 8> : rows == 4 ? k_ixfft<T, 4> : k_ixfft<T, 2>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k<<<dim3(a.g.NY / rows, a.g.NZ), 256, smem, s>>>(a);
}

template int launch_div_xfft<double>(const DivFftArgs<double>&, cudaStream_t);
template int launch_div_xfft<float>(const DivFftArgs<float>&, cudaStream_t);
template void launch_yfft<double>(const YFftArgs<double>&, cudaStream_t);
template void launch_yfft<float>(const YFftArgs<float>&, cudaStream_t);
template void launch_zsolve<double>(const ZSolveArgs<double>&, cudaStream_t, cudaStream_t, cudaEvent_t, cudaEvent_t);
template void launch_zsolve<float>(const ZSolveArgs<float>&, cudaStream_t, cudaStream_t, cudaEvent_t, cudaEvent_t);
template void launch_zsolve_fac<double>(const ZSolveArgs<double>&, cudaStream_t, cudaStream_t, cudaEvent_t, cudaEvent_t);
template void launch_zsolve_fac<float>(const ZSolveArgs<float>&, cudaStream_t, cudaStream_t, cudaEvent_t, cudaEvent_t);
template void launch_zfactor<double>(const ZSolveArgs<double>&, cudaStream_t);
template void launch_zfactor<float>(const ZSolveArgs<float>&, cudaStream_t);
template void launch_ixfft<double>(const IxFftArgs<double>&, cudaStream_t);
template void launch_ixfft<float>(const IxFftArgs<float>&, cudaStream_t);

}  // namespace tc
