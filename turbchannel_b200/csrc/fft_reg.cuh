// fft_reg.cuh -- line FFTs of compile-time length N done mostly in registers.
//
// N = N1 * N2 (Cooley-Tukey, n = N2*n1 + n2, k = k1 + N1*k2):
//   pass A  one item per (line, n2): the thread holds x[N2*n1 + n2], n1 < N1, does a
//           length-N1 DFT in registers, multiplies by W_N^(n2*k1) and writes
//           Y[k1][n2] to shared memory (row stride N2+1, which keeps the column reads
//           of pass B free of bank conflicts);
//   pass B  one item per (line, k1): the thread reads Y[k1][0..N2), does a length-N2
//           DFT in registers and holds X[k1 + N1*k2], k2 < N2.
// The register DFTs are mixed radix-4/2/3 with every inner twiddle a compile-time
// constant.  Against a Stockham transform through shared memory this is one shared
// round trip instead of one per radix pass, and no run-time index arithmetic inside
// the butterflies.
#pragma once
#include <utility>

#include "tc_common.cuh"

namespace tc {

// ---- compile-time cos/sin(2 pi k / n) -------------------------------------------
// The angle is reduced on the integers to an octant, so the Taylor series (summed
// to well below double rounding) only sees arguments in [0, pi/4].
constexpr double kc_sin_series(double x) {
    double t = x, s = x;
    for (int i = 1; i < 14; i++) {
        t *= -x * x / ((2.0 * i) * (2.0 * i + 1));
        s += t;
    }
    return s;
}
constexpr double kc_cos_series(double x) {
    double t = 1, s = 1;
    for (int i = 1; i < 14; i++) {
        t *= -x * x / ((2.0 * i - 1) * (2.0 * i));
        s += t;
    }
    return s;
}
struct KCS {
    double c, s;
};
constexpr KCS kcs(long long k, long long n) {
    const double PI = 3.14159265358979323846264338327950288;
    k %= n;
    if (k < 0) k += n;
    const long long q = (4 * k) / n, r = 4 * k - q * n;  // k/n = (q + r/n) / 4, r in [0, n)
    double c = 0, s = 0;
    if (2 * r <= n) {  // phi = pi r / (2n) in [0, pi/4]
        const double phi = PI * (double)r / (2.0 * (double)n);
        c = kc_cos_series(phi);
        s = kc_sin_series(phi);
    } else {  // phi in (pi/4, pi/2): use the complement
        const double psi = PI * (double)(n - r) / (2.0 * (double)n);
        c = kc_sin_series(psi);
        s = kc_cos_series(psi);
    }
    switch (q) {
        case 0: return {c, s};
        case 1: return {-s, c};
        case 2: return {-c, -s};
        default: return {s, -c};
    }
}

// ---- register DFTs ---------------------------------------------------------------
template <typename T, int N, int SIGN>
__device__ __forceinline__ void rdft(cplx<T> (&v)[N]);

// multiply t[r][k] by W_N^(SIGN * r * k) (I = r * M + k); quarter turns without a multiply
template <typename T, int N, int SIGN, int R, int M, int I>
__device__ __forceinline__ void rdft_tw1(cplx<T> (&t)[R][M]) {
    constexpr int r = I / M, k = I % M;
    constexpr long long e = ((long long)r * k) % N;
    if constexpr (e != 0) {
        cplx<T>& a = t[r][k];
        if constexpr (4 * e == N) {
            a = {-SIGN * a.y, SIGN * a.x};
        } else if constexpr (2 * e == N) {
            a = {-a.x, -a.y};
        } else if constexpr (4 * e == 3 * N) {
            a = {SIGN * a.y, -SIGN * a.x};
        } else {
            constexpr KCS w = kcs(e, N);
            constexpr double wc = w.c, ws = SIGN * w.s;
            a = cmul(a, cplx<T>{(T)wc, (T)ws});
        }
    }
}
template <typename T, int N, int SIGN, int R, int M, int... I>
__device__ __forceinline__ void rdft_tw(cplx<T> (&t)[R][M], std::integer_sequence<int, I...>) {
    (rdft_tw1<T, N, SIGN, R, M, I>(t), ...);
}

template <typename T, int N, int SIGN>
__device__ __forceinline__ void rdft(cplx<T> (&v)[N]) {
    if constexpr (N == 1) {
    } else if constexpr (N == 2 || N == 3 || N == 4) {
        dft_small<T, N>(v, SIGN);
    } else {
        constexpr int R = N % 4 == 0 ? 4 : (N % 2 == 0 ? 2 : 3);
        constexpr int M = N / R;
        cplx<T> t[R][M];
#pragma unroll
        for (int r = 0; r < R; r++)
#pragma unroll
            for (int m = 0; m < M; m++) t[r][m] = v[m * R + r];
#pragma unroll
        for (int r = 0; r < R; r++) rdft<T, M, SIGN>(t[r]);
        rdft_tw<T, N, SIGN, R, M>(t, std::make_integer_sequence<int, R * M>{});
#pragma unroll
        for (int k = 0; k < M; k++) {
            cplx<T> u[R];
#pragma unroll
            for (int r = 0; r < R; r++) u[r] = t[r][k];
            dft_small<T, R>(u, SIGN);
#pragma unroll
            for (int q = 0; q < R; q++) v[k + M * q] = u[q];
        }
    }
}

// ---- two-pass line transform -----------------------------------------------------
template <int N>
struct FftSplit {
    static constexpr bool ok = false;
};
#define TC_FFT_SPLIT(n, a, b)                     \
    template <>                                   \
    struct FftSplit<n> {                          \
        static constexpr bool ok = true;          \
        static constexpr int N1 = a, N2 = b;      \
        static constexpr int YL = a * (b + 1);    \
    };
TC_FFT_SPLIT(16, 4, 4)
TC_FFT_SPLIT(24, 4, 6)
TC_FFT_SPLIT(32, 4, 8)
TC_FFT_SPLIT(48, 6, 8)
TC_FFT_SPLIT(64, 8, 8)
TC_FFT_SPLIT(96, 8, 12)
TC_FFT_SPLIT(128, 8, 16)
TC_FFT_SPLIT(192, 12, 16)
TC_FFT_SPLIT(256, 16, 16)
TC_FFT_SPLIT(384, 16, 24)
TC_FFT_SPLIT(512, 16, 32)
TC_FFT_SPLIT(768, 24, 32)
TC_FFT_SPLIT(1024, 32, 32)
#undef TC_FFT_SPLIT

template <typename T>
__device__ __forceinline__ cplx<T> ldg_c(const cplx<T>* p) {
    if constexpr (sizeof(T) == 4) {
        const float2 q = __ldg(reinterpret_cast<const float2*>(p));
        return {q.x, q.y};
    } else {
        const double2 q = __ldg(reinterpret_cast<const double2*>(p));
        return {q.x, q.y};
    }
}

// Pass A of one item; Yl is the line's block of YL complex values.  tw[k] = exp(-2 pi i k / N).
template <typename T, int N, int SIGN>
__device__ __forceinline__ void fft_pass_a(cplx<T> (&v)[FftSplit<N>::N1], int n2, const cplx<T>* __restrict__ tw,
                                           cplx<T>* Yl) {
    constexpr int N1 = FftSplit<N>::N1, N2 = FftSplit<N>::N2;
    rdft<T, N1, SIGN>(v);
    Yl[n2] = v[0];
#pragma unroll
    for (int k1 = 1; k1 < N1; k1++) {
        cplx<T> w = ldg_c(tw + n2 * k1);
        if (SIGN > 0) w.y = -w.y;
        Yl[k1 * (N2 + 1) + n2] = cmul(v[k1], w);
    }
}

// Pass B of one item: v[k2] = X[k1 + N1 * k2].
template <typename T, int N, int SIGN>
__device__ __forceinline__ void fft_pass_b(cplx<T> (&v)[FftSplit<N>::N2], int k1, const cplx<T>* Yl) {
    constexpr int N2 = FftSplit<N>::N2;
    const cplx<T>* row = Yl + k1 * (N2 + 1);
#pragma unroll
    for (int n2 = 0; n2 < N2; n2++) v[n2] = row[n2];
    rdft<T, N2, SIGN>(v);
}

}  // namespace tc
