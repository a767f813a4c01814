/*
 * fftw3.h -- stand-in for the subset of FFTW's API that the reference's CPU
 * path calls (staggered/func_global.h:250-258, collocated_AB3/func_global.h:117-125):
 * fftw_plan_many_dft (rank 1 or 2, contiguous rows) and fftw_execute.  FFTW is not
 * installed in this image; the transform behind this header is the textbook
 * mixed-radix FFT of ../orc_fft.h.  TEST INFRASTRUCTURE ONLY: used solely to build
 * the reference sources into oracle/_ref/.
 */
#ifndef TCREF_FFTW3_SHIM_H
#define TCREF_FFTW3_SHIM_H
typedef double fftw_complex[2];
typedef struct tcref_fftw_plan_s* fftw_plan;
#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)
#ifdef __cplusplus
extern "C" {
#endif
fftw_plan fftw_plan_many_dft(int rank, const int* n, int howmany, fftw_complex* in, const int* inembed, int istride,
                             int idist, fftw_complex* out, const int* onembed, int ostride, int odist, int sign,
                             unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
#ifdef __cplusplus
}
#endif
#endif
