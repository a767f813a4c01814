/* fftw_shim.c -- implementation of the FFTW-API stand-in (see fftw3.h).
   TEST INFRASTRUCTURE ONLY. */
#include "fftw3.h"
#include "../orc_fft.h"

struct tcref_fftw_plan_s {
    int rank, n[2], howmany, istride, idist, ostride, odist, sign;
    double *in, *out;
    fftplan p[2];
};

fftw_plan fftw_plan_many_dft(int rank, const int* n, int howmany, fftw_complex* in, const int* inembed, int istride,
                             int idist, fftw_complex* out, const int* onembed, int ostride, int odist, int sign,
                             unsigned flags) {
    (void)inembed; (void)onembed; (void)flags;
    if (rank < 1 || rank > 2) return 0;
    struct tcref_fftw_plan_s* P = (struct tcref_fftw_plan_s*)calloc(1, sizeof(*P));
    P->rank = rank;
    for (int r = 0; r < rank; r++) {
        P->n[r] = n[r];
        if (fft_plan_init(&P->p[r], n[r])) { free(P); return 0; }
    }
    P->howmany = howmany; P->istride = istride; P->idist = idist; P->ostride = ostride; P->odist = odist;
    P->sign = sign; P->in = (double*)in; P->out = (double*)out;
    return P;
}

void fftw_execute(const fftw_plan P) {
    const int n0 = P->n[0], n1 = P->rank == 2 ? P->n[1] : 1, tot = n0 * n1;
    const int mx = n0 > n1 ? n0 : n1;
#pragma omp parallel
    {
        double* a = (double*)malloc(sizeof(double) * 2 * (size_t)tot);
        double* tmp = (double*)malloc(sizeof(double) * 2 * (size_t)mx);
        double* col = (double*)malloc(sizeof(double) * 2 * (size_t)mx);
#pragma omp for schedule(static)
        for (int b = 0; b < P->howmany; b++) {
            const double* src = P->in + 2 * (size_t)b * P->idist;
            for (int i = 0; i < tot; i++) { a[2 * i] = src[2 * (size_t)i * P->istride]; a[2 * i + 1] = src[2 * (size_t)i * P->istride + 1]; }
            if (P->rank == 1) fft_exec(&P->p[0], P->sign, a, tmp);
            else {
                /* row-major n0 x n1: transform the contiguous rows (length n1), then the columns */
                for (int r = 0; r < n0; r++) fft_exec(&P->p[1], P->sign, a + 2 * (size_t)r * n1, tmp);
                for (int c = 0; c < n1; c++) {
                    for (int r = 0; r < n0; r++) { col[2 * r] = a[2 * ((size_t)r * n1 + c)]; col[2 * r + 1] = a[2 * ((size_t)r * n1 + c) + 1]; }
                    fft_exec(&P->p[0], P->sign, col, tmp);
                    for (int r = 0; r < n0; r++) { a[2 * ((size_t)r * n1 + c)] = col[2 * r]; a[2 * ((size_t)r * n1 + c) + 1] = col[2 * r + 1]; }
                }
            }
            double* dst = P->out + 2 * (size_t)b * P->odist;
            for (int i = 0; i < tot; i++) { dst[2 * (size_t)i * P->ostride] = a[2 * i]; dst[2 * (size_t)i * P->ostride + 1] = a[2 * i + 1]; }
        }
        free(a); free(tmp); free(col);
    }
}

void fftw_destroy_plan(fftw_plan P) {
    if (!P) return;
    for (int r = 0; r < P->rank; r++) fft_plan_free(&P->p[r]);
    free(P);
}
