/*
 * orc_fft.h -- mixed-radix (4, 2, 3) Stockham complex FFT (textbook Cooley-Tukey),
 * shared by the oracle (tc_oracle.c) and the FFTW-API stand-in used to build the
 * reference's CPU path (ref/fftw_shim.c).  TEST INFRASTRUCTURE ONLY.
 */
#ifndef ORC_FFT_H
#define ORC_FFT_H
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* Mixed-radix (4, 2, 3) Stockham complex FFT, textbook Cooley-Tukey.        */
/* Stands in for FFTW's complex DFT used by the reference CPU path           */
/* (staggered/func_global.h:250-258): forward sign -1, backward +1, no scale. */
/* ------------------------------------------------------------------------ */
typedef struct {
    int n, nf, fac[64];
    double* tw; /* tw[2k], tw[2k+1] = cos, sin of (-2 pi k / n) */
} fftplan;

static inline int fft_plan_init(fftplan* P, int n) {
    int m = n;
    P->n = n;
    P->nf = 0;
    P->tw = NULL;
    if (n <= 0) return -1;
    while (m % 4 == 0) { P->fac[P->nf++] = 4; m /= 4; }
    while (m % 2 == 0) { P->fac[P->nf++] = 2; m /= 2; }
    while (m % 3 == 0) { P->fac[P->nf++] = 3; m /= 3; }
    if (m != 1) return -1;
    P->tw = (double*)malloc(sizeof(double) * 2 * (size_t)n);
    for (int k = 0; k < n; k++) {
        long double a = -2.0L * 3.14159265358979323846264338327950288L * (long double)k / (long double)n;
        P->tw[2 * k] = (double)cosl(a);
        P->tw[2 * k + 1] = (double)sinl(a);
    }
    return 0;
}

static inline void fft_plan_free(fftplan* P) { free(P->tw); P->tw = NULL; }

/* a: n complex (interleaved), tmp: scratch of the same size. */
static inline void fft_exec(const fftplan* P, int sign, double* a, double* tmp) {
    const int n = P->n;
    double* in = a;
    double* out = tmp;
    int Ns = 1;
    const double s3 = 0.86602540378443864676372317075294;
    for (int f = 0; f < P->nf; f++) {
        const int R = P->fac[f], nR = n / R, step = n / (Ns * R);
        for (int j = 0; j < nR; j++) {
            const int k = j % Ns;
            double vr[4], vi[4];
            for (int r = 0; r < R; r++) {
                const int idx = j + r * nR, t = r * k * step;
                const double xr = in[2 * idx], xi = in[2 * idx + 1];
                const double c = P->tw[2 * t], s = sign < 0 ? P->tw[2 * t + 1] : -P->tw[2 * t + 1];
                vr[r] = xr * c - xi * s;
                vi[r] = xr * s + xi * c;
            }
            if (R == 2) {
                double ar = vr[0], ai = vi[0];
                vr[0] = ar + vr[1]; vi[0] = ai + vi[1];
                vr[1] = ar - vr[1]; vi[1] = ai - vi[1];
            } else if (R == 4) {
                double t0r = vr[0] + vr[2], t0i = vi[0] + vi[2];
                double t1r = vr[0] - vr[2], t1i = vi[0] - vi[2];
                double t2r = vr[1] + vr[3], t2i = vi[1] + vi[3];
                double dr = vr[1] - vr[3], di = vi[1] - vi[3];
                /* (dr + i di) * (sign * i) */
                double t3r = -sign * di, t3i = sign * dr;
                vr[0] = t0r + t2r; vi[0] = t0i + t2i;
                vr[2] = t0r - t2r; vi[2] = t0i - t2i;
                vr[1] = t1r + t3r; vi[1] = t1i + t3i;
                vr[3] = t1r - t3r; vi[3] = t1i - t3i;
            } else { /* R == 3 */
                double t1r = vr[1] + vr[2], t1i = vi[1] + vi[2];
                double t2r = vr[1] - vr[2], t2i = vi[1] - vi[2];
                double mr = vr[0] - 0.5 * t1r, mi = vi[0] - 0.5 * t1i;
                /* sign * i * s3 * t2 */
                double er = -sign * s3 * t2i, ei = sign * s3 * t2r;
                vr[0] += t1r; vi[0] += t1i;
                vr[1] = mr + er; vi[1] = mi + ei;
                vr[2] = mr - er; vi[2] = mi - ei;
            }
            const int d = (j / Ns) * Ns * R + k;
            for (int r = 0; r < R; r++) {
                out[2 * (d + r * Ns)] = vr[r];
                out[2 * (d + r * Ns) + 1] = vi[r];
            }
        }
        Ns *= R;
        double* sw = in; in = out; out = sw;
    }
    if (in != a) memcpy(a, in, sizeof(double) * 2 * (size_t)n);
}

#endif
