/*
 * tc_oracle.c -- CPU restatement of TurbChannel's per-time-step path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker).  Only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline / reference legs load this library.  See
 * tc_oracle.h for the API.  Every function cites the reference file:line whose
 * arithmetic it restates.  Sizes are runtime values; periodic wrap is done by
 * explicit index arithmetic (the reference uses power-of-two bit masks,
 * staggered/data_global_inc.h:4-9).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "tc_oracle.h"

#ifndef ORC_REAL
#define ORC_REAL double
#endif
typedef ORC_REAL real;

#define RL(x) ((real)(x))
/* Constants of staggered/func_global.h:12-26, converted to the working type. */
#define C1_36 RL(0.02777777777777777777)
#define C1_27 RL(0.03703703703703703703)
#define C1_18 RL(0.05555555555555555555)
#define C1_9 RL(0.11111111111111111111)
#define C1_6 RL(0.16666666666666666666)
#define C1_3 RL(0.33333333333333333333)
#define PI_R RL(3.14159265358979323846)

#include "orc_fft.h"

int orc_fft(int n, int sign, double* data) {
    fftplan P;
    if (fft_plan_init(&P, n)) return -1;
    double* tmp = (double*)malloc(sizeof(double) * 2 * (size_t)n);
    fft_exec(&P, sign, data, tmp);
    free(tmp);
    fft_plan_free(&P);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Solver state                                                             */
/* ------------------------------------------------------------------------ */
struct orc {
    int scheme, visc_type, turb, stab_type, fd_mode;
    int NX, NY, NZ, NXY, N3D;
    real visc, sour_dpdx, inv_length_scale, xmin, ymin, hx, hy, inv_hx, inv_hy, area;
    /* staggered mesh data, 'real' like main_params (staggered/config.h:47-73) */
    real *ZZ, *DZ, *DZW, *GC1, *GC2, *GCZ, *MAT_A, MAT_D[6], *KERG, KERG_norm2;
    /* collocated mesh data, double like collocated_AB3/data_global.h:113-116 */
    double *cZZ, *cDZ, *cMAT_A;
    double *cosx, *cosy;
    real *vel[4], *flux[4], *pres[4], *divv, *nu_t;
    double* spec; /* NX*NY*NZ complex */
    fftplan px, py;
};

static int g_threads = 0;
void orc_set_threads(int n) {
    g_threads = n;
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#endif
}
int orc_get_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
int orc_real_size(void) { return (int)sizeof(real); }

/* Wrapped neighbour index helper: cell (ix,iy,iz) displaced by (dx,dy,dz). */
typedef struct { int xi[7], yi[7], ix, iy, iz, in; } nbh;
static inline void nbh_set(const orc* o, nbh* b, int in) {
    b->in = in;
    b->ix = in % o->NX;
    b->iy = (in / o->NX) % o->NY;
    b->iz = in / o->NXY;
    for (int k = 0; k < 7; k++) {
        b->xi[k] = ((b->ix + k - 3) % o->NX + o->NX) % o->NX;
        b->yi[k] = (((b->iy + k - 3) % o->NY + o->NY) % o->NY) * o->NX;
    }
}
#define NB(dx, dy, dz) (b.xi[(dx) + 3] + b.yi[(dy) + 3] + o->NXY * (b.iz + (dz)))

/* ------------------------------------------------------------------------ */
/* Mesh-derived data: staggered/main.cpp:12-48 (FillMatrix), :74-109        */
/* (solve_banded), :112-156 (InitDerivativeMeshData)                         */
/* ------------------------------------------------------------------------ */
static int banded_solve(int N, int NB_, double* M, double* x, double tiny) {
    /* Gauss elimination without pivoting on an N x NB_ band (staggered/main.cpp:74-109). */
    const int w = NB_ / 2;
    if (!(NB_ & 1)) return 1;
    for (int i = 0; i < N; i++) {
        for (int j = -w; j < 0; j++) {
            if (i + j < 0) continue;
            double mult = -M[i * NB_ + w + j];
            for (int k = 0; k <= w; k++) {
                if (i + j + k >= N) continue;
                M[i * NB_ + (w + j) + k] += mult * M[(i + j) * NB_ + w + k];
            }
            x[i] += mult * x[i + j];
        }
        if (fabs(M[i * NB_ + w]) < tiny) return 2;
        double mult = 1.0 / M[i * NB_ + w];
        for (int k = 0; k <= w; k++) {
            if (i + k >= N) continue;
            M[i * NB_ + w + k] *= mult;
        }
        x[i] *= mult;
    }
    for (int i = N - 1; i >= 0; i--)
        for (int j = 1; j <= w; j++) {
            if (i + j >= N) continue;
            x[i] -= M[i * NB_ + w + j] * x[i + j];
        }
    return 0;
}

/* The same elimination in the working precision (solve_banded<real>, used for KERG). */
static int banded_solve_r(int N, int NB_, real* M, real* x, real tiny) {
    const int w = NB_ / 2;
    for (int i = 0; i < N; i++) {
        for (int j = -w; j < 0; j++) {
            if (i + j < 0) continue;
            real mult = -M[i * NB_ + w + j];
            for (int k = 0; k <= w; k++) {
                if (i + j + k >= N) continue;
                M[i * NB_ + (w + j) + k] += mult * M[(i + j) * NB_ + w + k];
            }
            x[i] += mult * x[i + j];
        }
        if (fabs((double)M[i * NB_ + w]) < tiny) return 2;
        real mult = RL(1) / M[i * NB_ + w];
        for (int k = 0; k <= w; k++) {
            if (i + k >= N) continue;
            M[i * NB_ + w + k] *= mult;
        }
        x[i] *= mult;
    }
    for (int i = N - 1; i >= 0; i--)
        for (int j = 1; j <= w; j++) {
            if (i + j >= N) continue;
            x[i] -= M[i * NB_ + w + j] * x[i + j];
        }
    return 0;
}

/* 7-diagonal VV4 z-Laplacian of the xy-constant mode (staggered/main.cpp:12-48). */
static void fill_matrix_vv4(const orc* o, real* M) {
    const int NZ = o->NZ, w = 3, NBd = 7;
    const real gc[4] = {RL(1. / 27.), RL(-1.), RL(1.), RL(-1. / 27.)};
    for (int j = 0; j < NZ; j++) {
        for (int pos = 0; pos < NBd; pos++) M[j * NBd + pos] = 0;
        for (int ll = -1; ll <= 2; ll++) {
            real c1 = gc[ll + 1];
            int l = j + ll; /* z-face carrying the gradient */
            if (l == 0 || l == NZ) continue; /* no mass flux through the walls */
            if (l < 0) l = -l;
            if (l > NZ) l = 2 * NZ - l;
            for (int mm = -2; mm <= 1; mm++) {
                real c2 = gc[mm + 2];
                int m = l + mm;
                if (m < 0) { m = -m - 1; c2 = -c2; }
                if (m >= NZ) { m = 2 * NZ - m - 1; c2 = -c2; }
                int pos = m - j + w;
                if (pos < 0 || pos >= NBd) continue;
                M[j * NBd + pos] += c1 * c2 * o->GCZ[l];
            }
        }
    }
}

static int init_mesh(orc* o, const double* zz) {
    const int NZ = o->NZ;
    if (o->scheme == ORC_COLLOC) {
        for (int i = 0; i < NZ; i++) o->cZZ[i] = zz[i];
        for (int i = 0; i < NZ - 1; i++) o->cDZ[i] = o->cZZ[i + 1] - o->cZZ[i];
        /* collocated_AB3/main.cpp:295-300 */
        o->cMAT_A[0] = 0.;
        for (int j = 1; j < NZ; j++) o->cMAT_A[j] = (real)(o->hx * o->hy) / o->cDZ[j - 1];
        if (o->fd_mode) { o->cMAT_A[1] *= 0.5; o->cMAT_A[NZ - 1] *= 0.5; }
        return 0;
    }
    for (int i = 0; i <= NZ; i++) o->ZZ[i] = (real)zz[i];
    for (int i = 0; i < NZ; i++) o->DZ[i] = o->ZZ[i + 1] - o->ZZ[i];
    if (o->scheme == ORC_HW2) {
        o->MAT_A[0] = 0;
        for (int j = 1; j <= NZ - 1; j++) o->MAT_A[j] = (real)(2. / (o->DZ[j - 1] + o->DZ[j]));
        return 0;
    }
    /* VV4 (staggered/main.cpp:122-155) */
    for (int iz = 0; iz < NZ; iz++) {
        /* double-precision literals as in the reference (the result is rounded to real) */
        o->DZW[iz] = (real)((o->DZ[iz] + o->DZ[iz == 0 ? iz : iz - 1] + o->DZ[iz == NZ - 1 ? iz : iz + 1]) / 3.);
        o->GC1[iz] = (real)(o->DZ[iz] / (o->DZ[iz] - o->DZW[iz] / 9.));
        o->GC2[iz] = (real)(-(1. / 27.) * o->DZW[iz] / (o->DZ[iz] - o->DZW[iz] / 9.));
        if (iz == 0) { o->GCZ[iz] = 0; continue; } /* never used: no w-DOF on the bottom wall */
        o->GCZ[iz] = (real)(1 / (0.5 * (o->DZ[iz] + o->DZ[iz - 1]) -
                                 (1. / 27.) * (o->DZ[iz] + o->DZ[iz - 1] +
                                               0.5 * (o->DZ[iz == NZ - 1 ? iz : iz + 1] + o->DZ[iz == 1 ? 0 : iz - 2]))));
    }
    real* MAT = (real*)calloc((size_t)7 * NZ, sizeof(real));
    fill_matrix_vv4(o, MAT);
    for (int iz = 0; iz < NZ; iz++)
        for (int i = 0; i < 3; i++) o->MAT_A[iz * 3 + i] = (iz + i - 3 >= 0) ? MAT[iz * 7 + i] : RL(0);
    o->MAT_D[0] = MAT[3]; o->MAT_D[1] = MAT[7 + 3]; o->MAT_D[2] = MAT[7 * 2 + 3];
    o->MAT_D[3] = MAT[(NZ - 3) * 7 + 3]; o->MAT_D[4] = MAT[(NZ - 2) * 7 + 3]; o->MAT_D[5] = MAT[(NZ - 1) * 7 + 3];
    free(MAT);
    /* Null vector of the VV4 z-gradient: tridiagonal system with RHS 1 (main.cpp:140-148). */
    real* T = (real*)calloc((size_t)3 * NZ, sizeof(real));
    real* K = (real*)malloc(sizeof(real) * NZ);
    const real eps = RL(1. / 27.);
    T[1] = -1; T[2] = eps;
    for (int iz = 1; iz < NZ - 1; iz++) { T[iz * 3 + 0] = T[iz * 3 + 2] = eps; T[iz * 3 + 1] = -1 + eps; }
    T[(NZ - 1) * 3] = eps; T[(NZ - 1) * 3 + 1] = -1;
    for (int iz = 0; iz < NZ; iz++) K[iz] = 1;
    int err = banded_solve_r(NZ, 3, T, K, RL(1e-10));
    o->KERG_norm2 = 0;
    for (int iz = 0; iz < NZ; iz++) {
        o->KERG[iz] = (real)K[iz];
        o->KERG_norm2 += o->KERG[iz] * o->KERG[iz] * o->DZ[iz];
    }
    free(T); free(K);
    return err;
}

int orc_get_mesh(const orc* o, const char* name, double* out) {
    const int NZ = o->NZ;
#define CP(arr, n) do { for (int i = 0; i < (n); i++) out[i] = (double)(arr)[i]; return (n); } while (0)
    if (!strcmp(name, "ZZ")) { if (o->scheme == ORC_COLLOC) CP(o->cZZ, NZ); CP(o->ZZ, NZ + 1); }
    if (!strcmp(name, "DZ")) { if (o->scheme == ORC_COLLOC) CP(o->cDZ, NZ - 1); CP(o->DZ, NZ); }
    if (o->scheme == ORC_COLLOC) {
        if (!strcmp(name, "cMAT_A")) CP(o->cMAT_A, NZ);
        return 0;
    }
    if (!strcmp(name, "MAT_A")) { if (o->scheme == ORC_HW2) CP(o->MAT_A, NZ); CP(o->MAT_A, 3 * NZ); }
    if (o->scheme != ORC_VV4) return 0;
    if (!strcmp(name, "DZW")) CP(o->DZW, NZ);
    if (!strcmp(name, "GC1")) CP(o->GC1, NZ);
    if (!strcmp(name, "GC2")) CP(o->GC2, NZ);
    if (!strcmp(name, "GCZ")) CP(o->GCZ, NZ);
    if (!strcmp(name, "MAT_D")) CP(o->MAT_D, 6);
    if (!strcmp(name, "KERG")) CP(o->KERG, NZ);
    if (!strcmp(name, "KERG_norm2")) { out[0] = o->KERG_norm2; return 1; }
#undef CP
    return 0;
}

orc* orc_create(const orc_params* p, const double* zz, int* err) {
    orc* o = (orc*)calloc(1, sizeof(orc));
    o->scheme = p->scheme; o->visc_type = p->visc_type; o->turb = p->turb;
    o->stab_type = p->stab_type; o->fd_mode = p->fd_mode;
    o->NX = p->NX; o->NY = p->NY; o->NZ = p->NZ;
    o->NXY = p->NX * p->NY; o->N3D = o->NXY * p->NZ;
    o->visc = (real)p->visc; o->sour_dpdx = (real)p->sour_dpdx; o->inv_length_scale = (real)p->inv_length_scale;
    o->xmin = (real)p->xmin; o->ymin = (real)p->ymin; o->hx = (real)p->hx; o->hy = (real)p->hy;
    o->inv_hx = (real)(1. / o->hx); o->inv_hy = (real)(1. / o->hy); o->area = (real)p->area;
    const int NZ = o->NZ;
    o->ZZ = (real*)calloc(NZ + 1, sizeof(real));
    o->DZ = (real*)calloc(NZ + 1, sizeof(real));
    o->DZW = (real*)calloc(NZ, sizeof(real));
    o->GC1 = (real*)calloc(NZ, sizeof(real));
    o->GC2 = (real*)calloc(NZ, sizeof(real));
    o->GCZ = (real*)calloc(NZ, sizeof(real));
    o->MAT_A = (real*)calloc(3 * NZ + 1, sizeof(real));
    o->KERG = (real*)calloc(NZ, sizeof(real));
    o->cZZ = (double*)calloc(NZ + 1, sizeof(double));
    o->cDZ = (double*)calloc(NZ + 1, sizeof(double));
    o->cMAT_A = (double*)calloc(NZ + 1, sizeof(double));
    o->cosx = (double*)malloc(sizeof(double) * o->NX);
    o->cosy = (double*)malloc(sizeof(double) * o->NY);
    for (int i = 0; i < o->NX; i++) o->cosx[i] = cos(2. * 3.14159265358979323846 * i / o->NX);
    for (int i = 0; i < o->NY; i++) o->cosy[i] = cos(2. * 3.14159265358979323846 * i / o->NY);
    size_t N = (size_t)o->N3D;
    for (int l = 0; l < 4; l++) {
        o->vel[l] = (real*)calloc(3 * N, sizeof(real));
        o->flux[l] = (real*)calloc(3 * N, sizeof(real));
        o->pres[l] = (real*)calloc(N, sizeof(real));
    }
    o->divv = (real*)calloc(N, sizeof(real));
    o->nu_t = p->turb ? (real*)calloc(N, sizeof(real)) : NULL;
    o->spec = (double*)malloc(sizeof(double) * 2 * N);
    int e = 0;
    if (fft_plan_init(&o->px, o->NX) || fft_plan_init(&o->py, o->NY)) e = 3;
    if (!e) e = init_mesh(o, zz);
    if (err) *err = e;
    return o;
}

void orc_destroy(orc* o) {
    if (!o) return;
    free(o->ZZ); free(o->DZ); free(o->DZW); free(o->GC1); free(o->GC2); free(o->GCZ);
    free(o->MAT_A); free(o->KERG); free(o->cZZ); free(o->cDZ); free(o->cMAT_A);
    free(o->cosx); free(o->cosy);
    for (int l = 0; l < 4; l++) { free(o->vel[l]); free(o->flux[l]); free(o->pres[l]); }
    free(o->divv); free(o->nu_t); free(o->spec);
    fft_plan_free(&o->px); fft_plan_free(&o->py);
    free(o);
}

/* host <-> working-type copies */
static void to_real(real* dst, const double* src, size_t n) {
    for (size_t i = 0; i < n; i++) dst[i] = (real)src[i];
}
static void to_double(double* dst, const real* src, size_t n) {
    for (size_t i = 0; i < n; i++) dst[i] = (double)src[i];
}
void orc_set_level(orc* o, int l, const double* vel, const double* p) {
    if (vel) to_real(o->vel[l], vel, 3 * (size_t)o->N3D);
    if (p) to_real(o->pres[l], p, (size_t)o->N3D);
}
void orc_get_level(const orc* o, int l, double* vel, double* p) {
    if (vel) to_double(vel, o->vel[l], 3 * (size_t)o->N3D);
    if (p) to_double(p, o->pres[l], (size_t)o->N3D);
}
void orc_get_flux(const orc* o, int l, double* f) { to_double(f, o->flux[l], 3 * (size_t)o->N3D); }
void orc_set_nu_t(orc* o, const double* nt) { if (o->nu_t) to_real(o->nu_t, nt, (size_t)o->N3D); }
void orc_get_nu_t(const orc* o, double* nt) {
    if (o->nu_t) to_double(nt, o->nu_t, (size_t)o->N3D);
    else memset(nt, 0, sizeof(double) * (size_t)o->N3D);
}

/* ======================================================================== */
/* Staggered scheme                                                         */
/* ======================================================================== */
#define U(dx, dy, dz) vel[3 * NB(dx, dy, dz) + 0]
#define V(dx, dy, dz) vel[3 * NB(dx, dy, dz) + 1]
#define W(dx, dy, dz) vel[3 * NB(dx, dy, dz) + 2]

/* HW2 convection, staggered/func_global.h:345-370 */
static void conv_hw2(const orc* o, int in, const real* vel, real s[3]) {
    nbh b; nbh_set(o, &b, in);
    const int iz = b.iz, NZ = o->NZ;
    const real* DZ = o->DZ;
    real inv_hz = RL(1) / DZ[iz];
    real inv_hz_alt = RL(2) / (DZ[iz] + (iz == 0 ? RL(0) : DZ[iz - 1]));
    real U0 = U(0, 0, 0), V0 = V(0, 0, 0), W0 = W(0, 0, 0);
    s[0] = s[1] = s[2] = 0;
    real a = U0 + U(1, 0, 0), c = U0 + U(-1, 0, 0);
    s[0] -= (a * a - c * c) * o->inv_hx;
    s[0] -= ((U0 + U(0, 1, 0)) * (V(0, 1, 0) + V(-1, 1, 0)) - (U0 + U(0, -1, 0)) * (V0 + V(-1, 0, 0))) * o->inv_hy;
    if (iz != NZ - 1) s[0] -= (U0 + U(0, 0, 1)) * (W(0, 0, 1) + W(-1, 0, 1)) * inv_hz;
    if (iz != 0) s[0] += (U0 + U(0, 0, -1)) * (W0 + W(-1, 0, 0)) * inv_hz;

    s[1] -= ((V0 + V(1, 0, 0)) * (U(1, 0, 0) + U(1, -1, 0)) - (V0 + V(-1, 0, 0)) * (U0 + U(0, -1, 0))) * o->inv_hx;
    a = V0 + V(0, 1, 0); c = V0 + V(0, -1, 0);
    s[1] -= (a * a - c * c) * o->inv_hy;
    if (iz != NZ - 1) s[1] -= (V0 + V(0, 0, 1)) * (W(0, 0, 1) + W(0, -1, 1)) * inv_hz;
    if (iz != 0) s[1] += (V0 + V(0, 0, -1)) * (W0 + W(0, -1, 0)) * inv_hz;

    if (iz != 0) {
        s[2] -= ((W0 + W(1, 0, 0)) * (U(1, 0, 0) * DZ[iz] + U(1, 0, -1) * DZ[iz - 1]) -
                 (W0 + W(-1, 0, 0)) * (U0 * DZ[iz] + U(0, 0, -1) * DZ[iz - 1])) * o->inv_hx * inv_hz_alt;
        s[2] -= ((W0 + W(0, 1, 0)) * (V(0, 1, 0) * DZ[iz] + V(0, 1, -1) * DZ[iz - 1]) -
                 (W0 + W(0, -1, 0)) * (V0 * DZ[iz] + V(0, 0, -1) * DZ[iz - 1])) * o->inv_hy * inv_hz_alt;
        a = W0 + (iz == NZ - 1 ? RL(0) : W(0, 0, 1));
        s[2] -= a * a * inv_hz_alt;
        a = W0 + W(0, 0, -1);
        s[2] += a * a * inv_hz_alt;
    }
    s[0] *= RL(0.25); s[1] *= RL(0.25); s[2] *= RL(0.25);
}

/* VV4 convection, staggered/func_global.h:374-529.  'bar' quantities carry a
   factor 16, 'barbar' 16/9, exactly as in the reference. */
static void conv_vv4(const orc* o, int in, const real* vel, real s[3]) {
    nbh b; nbh_set(o, &b, in);
    const int iz = b.iz, NZ = o->NZ;
    const real *DZ = o->DZ, *DZW = o->DZW, hx = o->hx, hy = o->hy;
    const real dz = DZ[iz], dzw = DZW[iz], hxhy = hx * hy;
    const real U0 = U(0, 0, 0), V0 = V(0, 0, 0), W0 = W(0, 0, 0);
    s[0] = s[1] = s[2] = 0;
    { /* u: x-faces */
        real br = dz * hy * (9 * (U0 + U(1, 0, 0)) - (U(-1, 0, 0) + U(2, 0, 0)));
        real bl = dz * hy * (9 * (U(-1, 0, 0) + U0) - (U(-2, 0, 0) + U(1, 0, 0)));
        real bbr = dzw * hy * (9 * (U(1, 0, 0) + U(2, 0, 0)) - (U0 + U(3, 0, 0)));
        real bbl = dzw * hy * (9 * (U(-2, 0, 0) + U(-1, 0, 0)) - (U(-3, 0, 0) + U0));
        s[0] += br * (U0 + U(1, 0, 0)) - C1_27 * bbr * (U0 + U(3, 0, 0)) - bl * (U(-1, 0, 0) + U0) + C1_27 * bbl * (U(-3, 0, 0) + U0);
    }
    { /* u: y-faces */
        real br = dz * hx * (9 * (V(0, 1, 0) + V(-1, 1, 0)) - (V(-2, 1, 0) + V(1, 1, 0)));
        real bl = dz * hx * (9 * (V0 + V(-1, 0, 0)) - (V(-2, 0, 0) + V(1, 0, 0)));
        real bbr = dzw * hx * (9 * (V(0, 2, 0) + V(-1, 2, 0)) - (V(-2, 2, 0) + V(1, 2, 0)));
        real bbl = dzw * hx * (9 * (V(0, -1, 0) + V(-1, -1, 0)) - (V(-2, -1, 0) + V(1, -1, 0)));
        s[0] += br * (U0 + U(0, 1, 0)) - C1_27 * bbr * (U0 + U(0, 3, 0)) - bl * (U(0, -1, 0) + U0) + C1_27 * bbl * (U(0, -3, 0) + U0);
    }
    { /* u: z-faces */
        real wzl, wzr, wbzl, wbzr;
        if (iz == 0) wzl = 0;
        else wzl = hxhy * (9 * (W0 + W(-1, 0, 0)) - (W(-2, 0, 0) + W(1, 0, 0)));
        if (iz == NZ - 1) wzr = 0;
        else wzr = hxhy * (9 * (W(0, 0, 1) + W(-1, 0, 1)) - (W(-2, 0, 1) + W(1, 0, 1)));
        if (iz == 1) wbzl = 0;
        else if (iz == 0) wbzl = wzr;
        else wbzl = hxhy * (9 * (W(0, 0, -1) + W(-1, 0, -1)) - (W(-2, 0, -1) + W(1, 0, -1)));
        if (iz == NZ - 2) wbzr = 0;
        else if (iz == NZ - 1) wbzr = wzl;
        else wbzr = hxhy * (9 * (W(0, 0, 2) + W(-1, 0, 2)) - (W(-2, 0, 2) + W(1, 0, 2)));
        real uzr = iz == NZ - 1 ? RL(0) : U0 + U(0, 0, 1);
        real uzrr = U0 + (iz == NZ - 3 ? -U(0, 0, 2) : iz == NZ - 2 ? RL(0) : iz == NZ - 1 ? U(0, 0, -2) : U(0, 0, 3));
        real uzl = iz == 0 ? RL(0) : U(0, 0, -1) + U0;
        real uzll = U0 + (iz == 2 ? -U(0, 0, -2) : iz == 1 ? RL(0) : iz == 0 ? U(0, 0, 2) : U(0, 0, -3));
        s[0] += wzr * uzr - C1_27 * wbzr * uzrr - wzl * uzl + C1_27 * wbzl * uzll;
    }
    { /* v: x-faces */
        real br = dz * hy * (9 * (U(1, 0, 0) + U(1, -1, 0)) - (U(1, -2, 0) + U(1, 1, 0)));
        real bl = dz * hy * (9 * (U0 + U(0, -1, 0)) - (U(0, -2, 0) + U(0, 1, 0)));
        real bbr = dzw * hy * (9 * (U(2, 0, 0) + U(2, -1, 0)) - (U(2, -2, 0) + U(2, 1, 0)));
        real bbl = dzw * hy * (9 * (U(-1, 0, 0) + U(-1, -1, 0)) - (U(-1, -2, 0) + U(-1, 1, 0)));
        s[1] += br * (V0 + V(1, 0, 0)) - C1_27 * bbr * (V0 + V(3, 0, 0)) - bl * (V(-1, 0, 0) + V0) + C1_27 * bbl * (V(-3, 0, 0) + V0);
    }
    { /* v: y-faces */
        real br = dz * hx * (9 * (V0 + V(0, 1, 0)) - (V(0, -1, 0) + V(0, 2, 0)));
        real bl = dz * hx * (9 * (V(0, -1, 0) + V0) - (V(0, -2, 0) + V(0, 1, 0)));
        real bbr = dzw * hx * (9 * (V(0, 1, 0) + V(0, 2, 0)) - (V0 + V(0, 3, 0)));
        real bbl = dzw * hx * (9 * (V(0, -2, 0) + V(0, -1, 0)) - (V(0, -3, 0) + V0));
        s[1] += br * (V0 + V(0, 1, 0)) - C1_27 * bbr * (V0 + V(0, 3, 0)) - bl * (V(0, -1, 0) + V0) + C1_27 * bbl * (V(0, -3, 0) + V0);
    }
    { /* v: z-faces */
        real wzl, wzr, wbzl, wbzr;
        if (iz == 0) wzl = 0;
        else wzl = hxhy * (9 * (W0 + W(0, -1, 0)) - (W(0, -2, 0) + W(0, 1, 0)));
        if (iz == NZ - 1) wzr = 0;
        else wzr = hxhy * (9 * (W(0, 0, 1) + W(0, -1, 1)) - (W(0, -2, 1) + W(0, 1, 1)));
        if (iz == 1) wbzl = 0;
        else if (iz == 0) wbzl = wzr;
        else wbzl = hxhy * (9 * (W(0, 0, -1) + W(0, -1, -1)) - (W(0, -2, -1) + W(0, 1, -1)));
        if (iz == NZ - 2) wbzr = 0;
        else if (iz == NZ - 1) wbzr = wzl;
        else wbzr = hxhy * (9 * (W(0, 0, 2) + W(0, -1, 2)) - (W(0, -2, 2) + W(0, 1, 2)));
        real vzr = iz == NZ - 1 ? RL(0) : V0 + V(0, 0, 1);
        real vzrr = V0 + (iz == NZ - 3 ? -V(0, 0, 2) : iz == NZ - 2 ? RL(0) : iz == NZ - 1 ? V(0, 0, -2) : V(0, 0, 3));
        real vzl = iz == 0 ? RL(0) : V(0, 0, -1) + V0;
        real vzll = V0 + (iz == 2 ? -V(0, 0, -2) : iz == 1 ? RL(0) : iz == 0 ? V(0, 0, 2) : V(0, 0, -3));
        s[1] += wzr * vzr - C1_27 * wbzr * vzrr - wzl * vzl + C1_27 * wbzl * vzll;
    }
    if (iz != 0) {
        { /* w: x-faces (mass flux averaged to the w-face in z) */
            real br, bl, bbr, bbl;
#define WFACE_X(dst, ox, D)                                                                   \
    dst = 9 * (U(ox, 0, 0) * D[iz] + U(ox, 0, -1) * D[iz - 1]);                                  \
    dst -= (iz == 1) ? -U(ox, 0, -1) * D[0] : U(ox, 0, -2) * D[iz - 2];                          \
    dst -= (iz == NZ - 1) ? -U(ox, 0, 0) * D[NZ - 1] : U(ox, 0, 1) * D[iz + 1];                  \
    dst *= hy;
            WFACE_X(br, 1, DZ) WFACE_X(bl, 0, DZ) WFACE_X(bbr, 2, DZW) WFACE_X(bbl, -1, DZW)
#undef WFACE_X
            s[2] += br * (W0 + W(1, 0, 0)) - C1_27 * bbr * (W0 + W(3, 0, 0)) - bl * (W(-1, 0, 0) + W0) + C1_27 * bbl * (W(-3, 0, 0) + W0);
        }
        { /* w: y-faces.  The reference scales these by hy as well (func_global.h:475-487). */
            real br, bl, bbr, bbl;
#define WFACE_Y(dst, oy, D)                                                                   \
    dst = 9 * (V(0, oy, 0) * D[iz] + V(0, oy, -1) * D[iz - 1]);                                  \
    dst -= (iz == 1) ? -V(0, oy, -1) * D[0] : V(0, oy, -2) * D[iz - 2];                          \
    dst -= (iz == NZ - 1) ? -V(0, oy, 0) * D[NZ - 1] : V(0, oy, 1) * D[iz + 1];                  \
    dst *= hy;
            WFACE_Y(br, 1, DZ) WFACE_Y(bl, 0, DZ) WFACE_Y(bbr, 2, DZW) WFACE_Y(bbl, -1, DZW)
#undef WFACE_Y
            s[2] += br * (W0 + W(0, 1, 0)) - C1_27 * bbr * (W0 + W(0, 3, 0)) - bl * (W(0, -1, 0) + W0) + C1_27 * bbl * (W(0, -3, 0) + W0);
        }
        { /* w: z-faces */
            real wzl = W(0, 0, -1);
            real wzr = iz == NZ - 1 ? RL(0) : W(0, 0, 1);
            real wzll = iz == 1 ? W0 : W(0, 0, -2);
            real wzrr = iz == NZ - 2 ? RL(0) : iz == NZ - 1 ? W0 : W(0, 0, 2);
            real wzlll = iz == 1 ? W(0, 0, 1) : iz == 2 ? W(0, 0, -1) : W(0, 0, -3);
            real wzrrr = iz == NZ - 3 ? RL(0) : iz == NZ - 2 ? W(0, 0, 1) : iz == NZ - 1 ? W(0, 0, -1) : W(0, 0, 3);
            real bl = hxhy * (9 * (wzl + W0) - (wzll + wzr));
            real br = hxhy * (9 * (W0 + wzr) - (wzl + wzrr));
            real bbl = hxhy * (9 * (wzll + wzl) - (wzlll + W0));
            real bbr = hxhy * (9 * (wzr + wzrr) - (W0 + wzrrr));
            s[2] += br * (W0 + wzr) - bl * (wzl + W0);
            if (iz < NZ - 2) s[2] -= C1_27 * bbr * (W0 + wzrrr);
            else if (iz == NZ - 2) s[2] -= C1_27 * bbr * (-W(0, 0, 1) + W0);
            else s[2] -= C1_27 * bbr * (W(0, 0, -1) + W0);
            if (iz > 2) s[2] += C1_27 * bbl * (wzlll + W0);
            else if (iz == 2) s[2] += C1_27 * bbl * (-W(0, 0, -1) + W0);
            else s[2] += C1_27 * bbl * (W(0, 0, 1) + W0);
        }
    }
    real miv = RL(-1) / (32 * (dz - C1_9 * dzw) * hx * hy);
    s[0] *= miv;
    s[1] *= miv;
    s[2] *= (-RL(1. / 32.) * o->inv_hx * o->inv_hy * o->GCZ[iz]);
}

/* CROSS viscous term, staggered/func_global.h:533-562 */
static void visc_cross(const orc* o, int in, const real* vel, real s[3]) {
    nbh b; nbh_set(o, &b, in);
    const int iz = b.iz, NZ = o->NZ;
    const real* DZ = o->DZ;
    real inv_hz = RL(1) / DZ[iz];
    real inv_hz_alt = RL(2) / (DZ[iz] + (iz == 0 ? RL(0) : DZ[iz - 1]));
    for (int c = 0; c < 3; c++) {
        const real v0 = vel[3 * in + c];
        s[c] = o->inv_hx * o->inv_hx * (vel[3 * NB(1, 0, 0) + c] + vel[3 * NB(-1, 0, 0) + c] - RL(2.) * v0);
        s[c] += o->inv_hy * o->inv_hy * (vel[3 * NB(0, 1, 0) + c] + vel[3 * NB(0, -1, 0) + c] - RL(2.) * v0);
    }
    const real U0 = U(0, 0, 0), V0 = V(0, 0, 0), W0 = W(0, 0, 0);
    if (iz != NZ - 1) {
        real up = RL(2) / (DZ[iz] + DZ[iz + 1]);
        s[0] += (U(0, 0, 1) - U0) * up * inv_hz;
        s[1] += (V(0, 0, 1) - V0) * up * inv_hz;
        s[2] += (W(0, 0, 1) - W0) * inv_hz * inv_hz_alt;
    } else {
        real up = RL(2) / (DZ[iz]);
        s[0] += (-U0) * up * inv_hz;
        s[1] += (-V0) * up * inv_hz;
        s[2] += (-W0) * inv_hz * inv_hz_alt;
    }
    if (iz != 0) {
        s[0] += (U(0, 0, -1) - U0) * inv_hz_alt * inv_hz;
        s[1] += (V(0, 0, -1) - V0) * inv_hz_alt * inv_hz;
        s[2] += (W(0, 0, -1) - W0) * (RL(1) / DZ[iz - 1]) * inv_hz_alt;
    } else {
        s[0] += (-U0) * inv_hz_alt * inv_hz;
        s[1] += (-V0) * inv_hz_alt * inv_hz;
    }
    s[0] *= o->visc; s[1] *= o->visc; s[2] *= o->visc;
}

/* NAIVE (stress-divergence) viscous term with mu = visc + nu_t,
   staggered/func_global.h:564-625 (including its mu(XR(YR)) weight in sxy_190). */
static void visc_naive(const orc* o, int in, const real* vel, real s[3]) {
    nbh b; nbh_set(o, &b, in);
    const int iz = b.iz, NZ = o->NZ;
    const real *DZ = o->DZ, ihx = o->inv_hx, ihy = o->inv_hy, visc = o->visc;
    const real* nt = o->nu_t;
#define MU(dx, dy, dz) (nt ? visc + nt[NB(dx, dy, dz)] : visc)
    real inv_hz = RL(1) / DZ[iz];
    real up = 2 / (DZ[iz] + (iz == NZ - 1 ? RL(0) : DZ[iz + 1]));
    real dn = 2 / (DZ[iz] + (iz == 0 ? RL(0) : DZ[iz - 1]));
    const real U0 = U(0, 0, 0), V0 = V(0, 0, 0), W0 = W(0, 0, 0);
    const real q = RL(0.25);
    s[0] = s[1] = s[2] = 0;
    real sxx000 = 2 * (U(1, 0, 0) - U0) * ihx * MU(0, 0, 0);
    real sxx800 = 2 * (U0 - U(-1, 0, 0)) * ihx * MU(-1, 0, 0);
    s[0] += (sxx000 - sxx800) * ihx;
    real sxy910 = ((U(0, 1, 0) - U0) * ihy + (V(0, 1, 0) - V(-1, 1, 0)) * ihx) * q * (MU(0, 0, 0) + MU(-1, 0, 0) + MU(0, 1, 0) + MU(-1, 1, 0));
    real sxy990 = ((U0 - U(0, -1, 0)) * ihy + (V0 - V(-1, 0, 0)) * ihx) * q * (MU(0, -1, 0) + MU(-1, -1, 0) + MU(0, 0, 0) + MU(-1, 0, 0));
    s[0] += (sxy910 - sxy990) * ihy;
    real sxz901 = (iz == NZ - 1) ? (-2 * U0 * inv_hz * visc)
                                 : ((U(0, 0, 1) - U0) * up + (W(0, 0, 1) - W(-1, 0, 1)) * ihx) * q * (MU(0, 0, 0) + MU(-1, 0, 0) + MU(0, 0, 1) + MU(-1, 0, 1));
    real sxz909 = (iz == 0) ? (2 * U0 * inv_hz * visc)
                            : ((U0 - U(0, 0, -1)) * dn + (W0 - W(-1, 0, 0)) * ihx) * q * (MU(0, 0, -1) + MU(-1, 0, -1) + MU(0, 0, 0) + MU(-1, 0, 0));
    s[0] += (sxz901 - sxz909) * inv_hz;

    real sxy190 = ((U(1, 0, 0) - U(1, -1, 0)) * ihy + (V(1, 0, 0) - V0) * ihx) * q * (MU(0, 0, 0) + MU(1, 0, 0) + MU(0, -1, 0) + MU(1, 1, 0));
    s[1] += (sxy190 - sxy990) * ihx;
    real syy000 = 2 * (V(0, 1, 0) - V0) * ihy * MU(0, 0, 0);
    real syy080 = 2 * (V0 - V(0, -1, 0)) * ihy * MU(0, -1, 0);
    s[1] += (syy000 - syy080) * ihy;
    real syz091 = (iz == NZ - 1) ? (-2 * V0 * inv_hz * visc)
                                 : ((V(0, 0, 1) - V0) * up + (W(0, 0, 1) - W(0, -1, 1)) * ihy) * q * (MU(0, 0, 0) + MU(0, -1, 0) + MU(0, 0, 1) + MU(0, -1, 1));
    real syz099 = (iz == 0) ? (2 * V0 * inv_hz * visc)
                            : ((V0 - V(0, 0, -1)) * dn + (W0 - W(0, -1, 0)) * ihy) * q * (MU(0, 0, -1) + MU(0, -1, -1) + MU(0, 0, 0) + MU(0, -1, 0));
    s[1] += (syz091 - syz099) * inv_hz;

    if (iz == 0) return;
    real sxz109 = ((U(1, 0, 0) - U(1, 0, -1)) * dn + (W(1, 0, 0) - W0) * ihx) * q * (MU(0, 0, -1) + MU(1, 0, -1) + MU(0, 0, 0) + MU(1, 0, 0));
    s[2] += (sxz109 - sxz909) * ihx;
    real syz019 = ((V(0, 1, 0) - V(0, 1, -1)) * dn + (W(0, 1, 0) - W0) * ihy) * q * (MU(0, 0, -1) + MU(0, 1, -1) + MU(0, 0, 0) + MU(0, 1, 0));
    s[2] += (syz019 - syz099) * ihy;
    real szz000 = 2 * ((iz == NZ - 1 ? RL(0) : W(0, 0, 1)) - W0) * inv_hz * MU(0, 0, 0);
    real szz008 = 2 * (W0 - W(0, 0, -1)) * MU(0, 0, -1) / DZ[iz - 1];
    s[2] += (szz000 - szz008) * dn;
#undef MU
}

static void stag_flux_cell(const orc* o, int in, const real* vel, int do_conv, int do_visc, int add_src, real f[3]) {
    real c[3] = {0, 0, 0}, v[3] = {0, 0, 0};
    f[0] = add_src ? o->sour_dpdx : 0;
    f[1] = f[2] = 0;
    if (do_conv) {
        if (o->scheme == ORC_VV4) conv_vv4(o, in, vel, c);
        else conv_hw2(o, in, vel, c);
        f[0] += c[0]; f[1] += c[1]; f[2] += c[2];
    }
    if (do_visc) {
        if (o->visc_type == ORC_VISC_CROSS) visc_cross(o, in, vel, v);
        else visc_naive(o, in, vel, v);
        f[0] += v[0]; f[1] += v[1]; f[2] += v[2];
    }
    if (in < o->NXY) f[2] = 0;
}

/* Strain-rate magnitude at the cell centre, staggered/func_global.h:823-870 */
static real calc_abs_s(const orc* o, int in, const real* vel) {
    nbh b; nbh_set(o, &b, in);
    const int iz = b.iz, NZ = o->NZ;
    const real *DZ = o->DZ, ihx = o->inv_hx, ihy = o->inv_hy;
    real inv_hz = RL(1) / DZ[iz];
    real up = 2 / (DZ[iz] + (iz == NZ - 1 ? RL(0) : DZ[iz + 1]));
    real dn = 2 / (DZ[iz] + (iz == 0 ? RL(0) : DZ[iz - 1]));
    const real U0 = U(0, 0, 0), V0 = V(0, 0, 0), W0 = W(0, 0, 0);
    real sxx = (U(1, 0, 0) - U0) * ihx;
    real syy = (V(0, 1, 0) - V0) * ihy;
    real szz = ((iz == NZ - 1 ? RL(0) : W(0, 0, 1)) - W0) * inv_hz;
    real A = sxx * sxx + syy * syy + szz * szz;
    {
        real a = (U(0, 1, 0) - U0) * ihy + (V(0, 1, 0) - V(-1, 1, 0)) * ihx;
        real c = (U0 - U(0, -1, 0)) * ihy + (V0 - V(-1, 0, 0)) * ihx;
        real d = (U(1, 1, 0) - U(1, 0, 0)) * ihy + (V(1, 1, 0) - V(0, 1, 0)) * ihx;
        real e = (U(1, 0, 0) - U(1, -1, 0)) * ihy + (V(1, 0, 0) - V0) * ihx;
        A += RL(0.125) * (a * a + c * c + d * d + e * e);
    }
    {
        real a = (iz == NZ - 1) ? (-2 * U0 * inv_hz) : (U(0, 0, 1) - U0) * up + (W(0, 0, 1) - W(-1, 0, 1)) * ihx;
        real c = (iz == 0) ? (2 * U0 * inv_hz) : (U0 - U(0, 0, -1)) * dn + (W0 - W(-1, 0, 0)) * ihx;
        real d = (iz == NZ - 1) ? (-2 * U(1, 0, 0) * inv_hz) : (U(1, 0, 1) - U(1, 0, 0)) * up + (W(1, 0, 1) - W(0, 0, 1)) * ihx;
        real e = (iz == 0) ? (2 * U(1, 0, 0) * inv_hz) : (U(1, 0, 0) - U(1, 0, -1)) * dn + (W(1, 0, 0) - W0) * ihx;
        A += RL(0.125) * (a * a + c * c + d * d + e * e);
    }
    {
        real a = (iz == NZ - 1) ? (-2 * V0 * inv_hz) : (V(0, 0, 1) - V0) * up + (W(0, 0, 1) - W(0, -1, 1)) * ihy;
        real c = (iz == 0) ? (2 * V0 * inv_hz) : (V0 - V(0, 0, -1)) * dn + (W0 - W(0, -1, 0)) * ihy;
        real d = (iz == NZ - 1) ? (-2 * V(0, 1, 0) * inv_hz) : (V(0, 1, 1) - V(0, 1, 0)) * up + (W(0, 1, 1) - W(0, 0, 1)) * ihy;
        real e = (iz == 0) ? (2 * V(0, 1, 0) * inv_hz) : (V(0, 1, 0) - V(0, 1, -1)) * dn + (W(0, 1, 0) - W0) * ihy;
        A += RL(0.125) * (a * a + c * c + d * d + e * e);
    }
    return (real)sqrt(2 * A);
}

/* Smagorinsky-van Driest, staggered/func_global.h:875-890 */
static void stag_turb_visc(orc* o, const real* vel) {
    if (!o->nu_t) return;
    const int NXY = o->NXY, NZ = o->NZ;
#pragma omp parallel for schedule(static)
    for (int in = 0; in < o->N3D; in++) {
        int iz = in / NXY;
        const real H = RL(0.5) * (o->ZZ[NZ] - o->ZZ[0]);
        const real Z = RL(0.5) * (o->ZZ[iz] + o->ZZ[iz + 1]) - o->ZZ[0];
        const real d = (Z < H) ? Z : 2 * H - Z;
        const real yp = d * o->inv_length_scale;
        const real C_SMAG = RL(0.1), C_exp = RL(0.04 * 0.04 * 0.04);
        const real S = calc_abs_s(o, in, vel);
        const real fvd = 1 - (real)exp(-C_exp * yp * yp * yp);
        const real Vol = o->hx * o->hy * o->DZ[iz];
        real Dl = C_SMAG * (real)pow(Vol, C1_3);
        if (Dl > RL(0.41) * d) Dl = RL(0.41) * d;
        o->nu_t[in] = fvd * Dl * Dl * S;
    }
}

/* Gradient of a cell-centred scalar onto the faces: HW2 func_global.h:297-303,
   VV4 :316-322. */
static void stag_gradient(const orc* o, const real* a, real* ga) {
    const int NZ = o->NZ;
#pragma omp parallel for schedule(static)
    for (int in = 0; in < o->N3D; in++) {
        nbh b; nbh_set(o, &b, in);
        const int iz = b.iz;
        const real a0 = a[in];
        if (o->scheme == ORC_HW2) {
            ga[3 * in + 0] = o->inv_hx * (a0 - a[NB(-1, 0, 0)]);
            ga[3 * in + 1] = o->inv_hy * (a0 - a[NB(0, -1, 0)]);
            ga[3 * in + 2] = iz == 0 ? RL(0) : (a0 - a[NB(0, 0, -1)]) * (2 / (o->DZ[iz] + o->DZ[iz - 1]));
        } else {
            ga[3 * in + 0] = o->inv_hx * (o->GC1[iz] * (a0 - a[NB(-1, 0, 0)]) + o->GC2[iz] * (a[NB(1, 0, 0)] - a[NB(-2, 0, 0)]));
            ga[3 * in + 1] = o->inv_hy * (o->GC1[iz] * (a0 - a[NB(0, -1, 0)]) + o->GC2[iz] * (a[NB(0, 1, 0)] - a[NB(0, -2, 0)]));
            if (iz == 0) ga[3 * in + 2] = 0;
            else {
                real ar = iz == NZ - 1 ? -a0 : a[NB(0, 0, 1)];
                real all = iz == 1 ? -a[NB(0, 0, -1)] : a[NB(0, 0, -2)];
                ga[3 * in + 2] = ((a0 - a[NB(0, 0, -1)]) - C1_27 * (ar - all)) * o->GCZ[iz];
            }
        }
    }
}

/* Divergence times cell height: HW2 func_global.h:306-312, VV4 :325-333. */
static void stag_divergence(const orc* o, const real* v, real* dv) {
    const int NZ = o->NZ;
#pragma omp parallel for schedule(static)
    for (int in = 0; in < o->N3D; in++) {
        nbh b; nbh_set(o, &b, in);
        const int iz = b.iz;
        if (o->scheme == ORC_HW2) {
            real hz = o->DZ[iz];
            dv[in] = (v[3 * NB(1, 0, 0)] - v[3 * in]) * o->inv_hx * hz +
                     (v[3 * NB(0, 1, 0) + 1] - v[3 * in + 1]) * o->inv_hy * hz +
                     ((iz < NZ - 1) ? (v[3 * NB(0, 0, 1) + 2] - v[3 * in + 2]) : (-v[3 * in + 2]));
        } else {
            real dudx = o->inv_hx * (o->DZ[iz] * (v[3 * NB(1, 0, 0)] - v[3 * in]) - C1_27 * o->DZW[iz] * (v[3 * NB(2, 0, 0)] - v[3 * NB(-1, 0, 0)]));
            real dvdy = o->inv_hy * (o->DZ[iz] * (v[3 * NB(0, 1, 0) + 1] - v[3 * in + 1]) - C1_27 * o->DZW[iz] * (v[3 * NB(0, 2, 0) + 1] - v[3 * NB(0, -1, 0) + 1]));
            real wr = (iz == NZ - 1) ? RL(0) : v[3 * NB(0, 0, 1) + 2];
            real wrr = (iz == NZ - 1) ? v[3 * in + 2] : (iz == NZ - 2) ? RL(0) : v[3 * NB(0, 0, 2) + 2];
            real wll = (iz == 0) ? v[3 * NB(0, 0, 1) + 2] : (iz == 1) ? RL(0) : v[3 * NB(0, 0, -1) + 2];
            dv[in] = dudx + dvdy + (wr - v[3 * in + 2]) - C1_27 * (wrr - wll);
        }
    }
}

/* ======================================================================== */
/* Collocated scheme (collocated_AB3/func_global.h, func_fluxes.h)          */
/* ======================================================================== */
static inline int c_is_wall(const orc* o, int iz) { return iz == 0 || iz == o->NZ - 1; }
static inline real c_cell_height(const orc* o, int iz) {
    /* collocated_AB3/func_global.h:150-155 */
    if (iz == 0) return (real)(0.5 * o->cDZ[0]);
    if (iz == o->NZ - 1) return (real)(0.5 * o->cDZ[o->NZ - 2]);
    return (real)(0.5 * (o->cDZ[iz - 1] + o->cDZ[iz]));
}

static void coll_gradient(const orc* o, const real* a, real* R) {
#pragma omp parallel for schedule(static)
    for (int in = 0; in < o->N3D; in++) {
        nbh b; nbh_set(o, &b, in);
        if (c_is_wall(o, b.iz)) { R[3 * in] = R[3 * in + 1] = R[3 * in + 2] = 0; continue; }
        R[3 * in + 0] = RL(0.5) * o->inv_hx * (a[NB(1, 0, 0)] - a[NB(-1, 0, 0)]);
        R[3 * in + 1] = RL(0.5) * o->inv_hy * (a[NB(0, 1, 0)] - a[NB(0, -1, 0)]);
        R[3 * in + 2] = RL(0.5) * (a[NB(0, 0, 1)] - a[NB(0, 0, -1)]) / c_cell_height(o, b.iz);
    }
}

static void coll_divergence(const orc* o, const real* v, real* dv) {
    const int NZ = o->NZ;
#pragma omp parallel for schedule(static)
    for (int in = 0; in < o->N3D; in++) {
        nbh b; nbh_set(o, &b, in);
        const int iz = b.iz;
        real hz = c_cell_height(o, iz), d = 0;
        d += RL(0.5) * (v[3 * NB(1, 0, 0)] - v[3 * NB(-1, 0, 0)]) * o->hy * hz;
        d += RL(0.5) * (v[3 * NB(0, 1, 0) + 1] - v[3 * NB(0, -1, 0) + 1]) * o->hx * hz;
        if (iz == 0) d += RL(0.5) * (v[3 * NB(0, 0, 1) + 2] - v[3 * in + 2]) * o->hx * o->hy;
        else if (iz == NZ - 1) d += RL(0.5) * (v[3 * in + 2] - v[3 * NB(0, 0, -1) + 2]) * o->hx * o->hy;
        else d += RL(0.5) * (v[3 * NB(0, 0, 1) + 2] - v[3 * NB(0, 0, -1) + 2]) * o->hx * o->hy;
        dv[in] = d;
    }
}

/* Galerkin 27-point viscous term, collocated_AB3/func_fluxes.h:21-85 */
static void coll_visc_galerkin(const orc* o, int in, const real* u, real s[3]) {
    nbh b; nbh_set(o, &b, in);
    const int iz = b.iz;
    s[0] = s[1] = s[2] = 0;
    for (int oz = 0; oz <= 1; oz++) {
        const int sz = oz ? 1 : -1;
        real hz = (real)(oz == 0 ? o->cDZ[iz == 0 ? 0 : iz - 1] : o->cDZ[iz]);
        real inv_hz = (real)(1. / hz);
        for (int oy = 0; oy <= 1; oy++) {
            const int sy = oy ? 1 : -1;
            for (int ox = 0; ox <= 1; ox++) {
                const int sx = ox ? 1 : -1;
                const real* q0 = u + 3 * in;
                const real* qx = u + 3 * NB(sx, 0, 0);
                const real* qy = u + 3 * NB(0, sy, 0);
                const real* qz = u + 3 * NB(0, 0, sz);
                const real* qxy = u + 3 * NB(sx, sy, 0);
                const real* qxz = u + 3 * NB(sx, 0, sz);
                const real* qyz = u + 3 * NB(0, sy, sz);
                const real* qxyz = u + 3 * NB(sx, sy, sz);
                real mx = o->inv_hx * o->hy * hz, my = o->inv_hy * o->hx * hz, mz = inv_hz * o->hx * o->hy;
                real g[3];
                for (int c = 0; c < 3; c++)
                    g[c] = (C1_9 * (qx[c] - q0[c]) + C1_18 * (qxy[c] - qy[c]) + C1_18 * (qxz[c] - qz[c]) + C1_36 * (qxyz[c] - qyz[c])) * mx +
                           (C1_9 * (qy[c] - q0[c]) + C1_18 * (qxy[c] - qx[c]) + C1_18 * (qyz[c] - qz[c]) + C1_36 * (qxyz[c] - qxz[c])) * my +
                           (C1_9 * (qz[c] - q0[c]) + C1_18 * (qxz[c] - qx[c]) + C1_18 * (qyz[c] - qy[c]) + C1_36 * (qxyz[c] - qxy[c])) * mz;
                real gxx = C1_9 * (qx[0] - q0[0]) + C1_18 * (qxy[0] - qy[0]) + C1_18 * (qxz[0] - qz[0]) + C1_36 * (qxyz[0] - qyz[0]);
                real gxy = RL(0.25) * (C1_3 * (qx[1] - q0[1] + qxy[1] - qy[1]) + C1_6 * (qxz[1] - qz[1] + qxyz[1] - qyz[1]));
                real gxz = RL(0.25) * (C1_3 * (qx[2] - q0[2] + qxz[2] - qz[2]) + C1_6 * (qxy[2] - qy[2] + qxyz[2] - qyz[2]));
                real gyy = C1_9 * (qy[1] - q0[1]) + C1_18 * (qxy[1] - qx[1]) + C1_18 * (qyz[1] - qz[1]) + C1_36 * (qxyz[1] - qxz[1]);
                real gyx = RL(0.25) * (C1_3 * (qy[0] - q0[0] + qxy[0] - qx[0]) + C1_6 * (qyz[0] - qz[0] + qxyz[0] - qxz[0]));
                real gyz = RL(0.25) * (C1_3 * (qy[2] - q0[2] + qyz[2] - qz[2]) + C1_6 * (qxy[2] - qx[2] + qxyz[2] - qxz[2]));
                real gzz = C1_9 * (qz[2] - q0[2]) + C1_18 * (qyz[2] - qy[2]) + C1_18 * (qxz[2] - qx[2]) + C1_36 * (qxyz[2] - qxy[2]);
                real gzx = RL(0.25) * (C1_3 * (qz[0] - q0[0] + qxz[0] - qx[0]) + C1_6 * (qyz[0] - qy[0] + qxyz[0] - qxy[0]));
                real gzy = RL(0.25) * (C1_3 * (qz[1] - q0[1] + qyz[1] - qy[1]) + C1_6 * (qxz[1] - qx[1] + qxyz[1] - qxy[1]));
                const real sxy = (ox ^ oy) ? RL(-1) : RL(1), sxz = (ox ^ oz) ? RL(-1) : RL(1), syz = (oy ^ oz) ? RL(-1) : RL(1);
                gxx *= mx; gxy *= hz * sxy; gxz *= o->hy * sxz;
                gyy *= my; gyx *= hz * sxy; gyz *= o->hx * syz;
                gzz *= mz; gzx *= o->hy * sxz; gzy *= o->hx * syz;
                g[0] += gxx + gxy + gxz;
                g[1] += gyy + gyx + gyz;
                g[2] += gzz + gzx + gzy;
                real vc = o->visc;
                if (o->nu_t) vc += o->nu_t[NB(ox ? 0 : -1, oy ? 0 : -1, oz ? 0 : -1)];
                s[0] += g[0] * vc; s[1] += g[1] * vc; s[2] += g[2] * vc;
            }
        }
    }
}

/* Collocated flux, collocated_AB3/func_fluxes.h:87-120 */
static void coll_flux_cell(const orc* o, int in, const real* u, int do_conv, int do_visc, real f[3]) {
    nbh b; nbh_set(o, &b, in);
    const int iz = b.iz;
    f[0] = f[1] = f[2] = 0;
    if (c_is_wall(o, iz)) return;
    real inv_hz = (real)(2. / (o->cDZ[iz - 1] + o->cDZ[iz]));
    if (do_conv) {
        const double invh[3] = {(double)o->inv_hx, (double)o->inv_hy, (double)inv_hz};
        for (int d = 0; d < 3; d++) {
            int jn = d == 0 ? NB(-1, 0, 0) : d == 1 ? NB(0, -1, 0) : NB(0, 0, -1);
            int kn = d == 0 ? NB(1, 0, 0) : d == 1 ? NB(0, 1, 0) : NB(0, 0, 1);
            for (int c = 0; c < 3; c++) {
                real cd = RL(0.5) * (u[3 * kn + c] * u[3 * kn + d] - u[3 * jn + c] * u[3 * jn + d]);
                real ca = u[3 * in + d] * (RL(0.5) * (u[3 * kn + c] - u[3 * jn + c]));
                f[c] -= (real)(RL(0.5) * (cd + ca) * invh[d]);
            }
        }
    }
    if (do_visc) {
        if (o->visc_type == ORC_VISC_GALERKIN) {
            real g[3];
            coll_visc_galerkin(o, in, u, g);
            for (int c = 0; c < 3; c++) f[c] += g[c] * o->inv_hx * o->inv_hy * inv_hz;
        } else {
            for (int c = 0; c < 3; c++) {
                f[c] += o->visc * o->inv_hx * o->inv_hx * (u[3 * NB(1, 0, 0) + c] + u[3 * NB(-1, 0, 0) + c] - RL(2.) * u[3 * in + c]);
                f[c] += o->visc * o->inv_hy * o->inv_hy * (u[3 * NB(0, 1, 0) + c] + u[3 * NB(0, -1, 0) + c] - RL(2.) * u[3 * in + c]);
                f[c] += o->visc * (real)(((double)u[3 * NB(0, 0, 1) + c] - u[3 * in + c]) / o->cDZ[iz] -
                                         ((double)u[3 * in + c] - u[3 * NB(0, 0, -1) + c]) / o->cDZ[iz - 1]) * inv_hz;
            }
        }
    }
    f[0] += o->sour_dpdx;
}

/* Smagorinsky on elements, collocated_AB3/func_global.h:342-384 */
static void coll_turb_visc(orc* o, const real* u) {
    if (!o->nu_t) return;
    const int NZ = o->NZ;
#pragma omp parallel for schedule(static)
    for (int ie = 0; ie < o->N3D; ie++) {
        nbh b; nbh_set(o, &b, ie);
        const int iz = b.iz;
        if (iz >= NZ - 1) continue;
        const real hz = (real)o->cDZ[iz];
        const real *q = u + 3 * ie, *qx = u + 3 * NB(1, 0, 0), *qy = u + 3 * NB(0, 1, 0), *qxy = u + 3 * NB(1, 1, 0);
        const real *qz = u + 3 * NB(0, 0, 1), *qxz = u + 3 * NB(1, 0, 1), *qyz = u + 3 * NB(0, 1, 1), *qxyz = u + 3 * NB(1, 1, 1);
        real g[3][3];
        for (int c = 0; c < 3; c++) {
            g[0][c] = ((qx[c] + qxy[c] + qxz[c] + qxyz[c]) - (q[c] + qy[c] + qz[c] + qyz[c])) * (RL(0.25) * o->inv_hx);
            g[1][c] = ((qy[c] + qxy[c] + qyz[c] + qxyz[c]) - (q[c] + qx[c] + qz[c] + qxz[c])) * (RL(0.25) * o->inv_hy);
            g[2][c] = ((qz[c] + qxz[c] + qyz[c] + qxyz[c]) - (q[c] + qx[c] + qy[c] + qxy[c])) / (4 * hz);
        }
        g[0][1] = RL(0.5) * (g[0][1] + g[1][0]);
        g[0][2] = RL(0.5) * (g[0][2] + g[2][0]);
        g[1][2] = RL(0.5) * (g[1][2] + g[2][1]);
        real A = g[0][0] * g[0][0] + g[1][1] * g[1][1] + g[2][2] * g[2][2] + 2 * (g[0][1] * g[0][1] + g[0][2] * g[0][2] + g[1][2] * g[1][2]);
        A = (real)sqrt(2 * A);
        const real H = (real)(0.5 * (o->cZZ[NZ - 1] - o->cZZ[0]));
        const real Z = (real)(0.5 * (o->cZZ[iz] + o->cZZ[iz + 1]));
        const real d = (Z < H) ? Z : 2 * H - Z;
        const real yp = d * o->inv_length_scale;
        const real C_SMAG = RL(0.1), C_exp = RL(0.04 * 0.04 * 0.04);
        const real fvd = 1 - (real)exp(-C_exp * yp * yp * yp);
        const real Vol = o->hx * o->hy * hz;
        real Dl = C_SMAG * (real)pow(Vol, C1_3);
        if (Dl > RL(0.41) * d) Dl = RL(0.41) * d;
        o->nu_t[ie] = fvd * Dl * Dl * A;
    }
}

/* ======================================================================== */
/* Pressure solve: 2-D FFT per z-plane, banded solve per mode, inverse FFT  */
/* (staggered/func_global.h:71-189, 250-281; collocated_AB3/func_global.h:8-61, */
/* 117-147)                                                                  */
/* ======================================================================== */
static void fft2_planes(orc* o, int sign) {
    const int NX = o->NX, NY = o->NY, NZ = o->NZ, NXY = o->NXY;
    const int mx = NX > NY ? NX : NY;
#pragma omp parallel
    {
        double* tmp = (double*)malloc(sizeof(double) * 2 * mx);
        double* col = (double*)malloc(sizeof(double) * 2 * mx);
#pragma omp for schedule(static)
        for (int r = 0; r < NY * NZ; r++) fft_exec(&o->px, sign, o->spec + 2 * (size_t)r * NX, tmp);
#pragma omp for schedule(static)
        for (int c = 0; c < NX * NZ; c++) {
            const int iz = c / NX, ix = c % NX;
            double* base = o->spec + 2 * ((size_t)iz * NXY + ix);
            for (int iy = 0; iy < NY; iy++) { col[2 * iy] = base[2 * (size_t)iy * NX]; col[2 * iy + 1] = base[2 * (size_t)iy * NX + 1]; }
            fft_exec(&o->py, sign, col, tmp);
            for (int iy = 0; iy < NY; iy++) { base[2 * (size_t)iy * NX] = col[2 * iy]; base[2 * (size_t)iy * NX + 1] = col[2 * iy + 1]; }
        }
        free(tmp); free(col);
    }
}

/* HW2 tridiagonal solve for mode ixy, staggered/func_global.h:71-106 */
static void thomas_hw2(const orc* o, int ixy, double* p) {
    const int NX = o->NX, NZ = o->NZ, stride = o->NXY;
    const int ix = ixy % NX, iy = ixy / NX;
    const real *MA = o->MAT_A, *DZ = o->DZ;
    real MM = 2 * ((real)(1 - o->cosx[ix]) * o->inv_hx * o->inv_hx + (real)(1 - o->cosy[iy]) * o->inv_hy * o->inv_hy);
    double* x = o->spec + 2 * (size_t)ixy;
    real b0 = -DZ[0] * MM - MA[1];
    if (ixy == 0) b0 *= 2;
    real ib0 = 1 / b0;
    x[0] *= ib0; x[1] *= ib0;
    p[0] = MA[1] * ib0;
    for (int i = 1; i <= NZ - 1; i++) {
        real d = -MA[i] - DZ[i] * MM;
        if (i != NZ - 1) d -= MA[i + 1];
        d -= MA[i] * (real)p[i - 1];
        d = 1 / d;
        if (i != NZ - 1) p[i] = MA[i + 1] * d;
        double* xi = x + 2 * (size_t)i * stride;
        const double* xm = x + 2 * (size_t)(i - 1) * stride;
        xi[0] = (xi[0] - MA[i] * xm[0]) * d;
        xi[1] = (xi[1] - MA[i] * xm[1]) * d;
    }
    for (int i = NZ - 2; i >= 0; i--) {
        double* xi = x + 2 * (size_t)i * stride;
        const double* xp = x + 2 * (size_t)(i + 1) * stride;
        xi[0] -= xp[0] * p[i];
        xi[1] -= xp[1] * p[i];
    }
}

/* VV4 7-diagonal Gauss elimination for mode ixy, staggered/func_global.h:110-189 */
static void thomas_vv4(const orc* o, int ixy, double* buf) {
    const int NX = o->NX, NY = o->NY, N = o->NZ, stride = o->NXY, w = 3;
    const real tiny = RL(1e-30);
    const int ix = ixy % NX, iy = ixy / NX;
    double* x = o->spec + 2 * (size_t)ixy;
    const real sx = (real)sin(PI_R * ix / NX), sy = (real)sin(PI_R * iy / NY);
    const real s3x = 3 * sx - 4 * sx * sx * sx, s3y = 3 * sy - 4 * sy * sy * sy;
    for (int i = 0; i < N; i++) {
        real row[7] = {0, 0, 0, 0, 0, 0, 0};
        real sum = 0;
        for (int k = 0; k < w; k++) {
            if (i + k - w < 0 || i + k - w >= N) continue;
            row[k] = o->MAT_A[i * w + k];
            sum += o->MAT_A[i * w + k];
        }
        for (int k = 1; k <= w; k++) {
            if (i + k >= N) continue;
            row[w + k] = o->MAT_A[(i + k) * w + w - k];
            sum += o->MAT_A[(i + k) * w + w - k];
        }
        if (i <= 2) row[w] = o->MAT_D[i];
        else if (i >= N - 3) row[w] = o->MAT_D[i - (N - 3) + 3];
        else row[w] = -sum;
        if (ixy == 0 && i == 0) row[w] *= 2; /* pin of the singular mean mode */
        {
            real ci = o->DZ[i] * sx - C1_27 * o->DZW[i] * s3x;
            row[w] -= 4 * o->inv_hx * o->inv_hx * ci * ci / (o->DZ[i] - C1_9 * o->DZW[i]);
            ci = o->DZ[i] * sy - C1_27 * o->DZW[i] * s3y;
            row[w] -= 4 * o->inv_hy * o->inv_hy * ci * ci / (o->DZ[i] - C1_9 * o->DZW[i]);
        }
        double* xi = x + 2 * (size_t)i * stride;
        for (int j = -w; j < 0; j++) {
            if (i + j < 0) continue;
            real mult = -row[w + j];
            for (int k = 1; k <= w; k++) {
                if (i + j + k >= N) continue;
                row[w + j + k] += mult * (real)buf[(i + j) * w + k - 1];
            }
            const double* xj = x + 2 * (size_t)(i + j) * stride;
            xi[0] += mult * xj[0];
            xi[1] += mult * xj[1];
        }
        if (fabs((double)row[w]) < tiny) { x[0] = -1e50; return; }
        real mult = RL(1) / row[w];
        for (int k = 1; k <= w; k++) {
            if (i + k >= N) continue;
            buf[i * w + k - 1] = row[w + k] * mult;
        }
        xi[0] *= mult;
        xi[1] *= mult;
    }
    for (int i = N - 1; i >= 0; i--) {
        double* xi = x + 2 * (size_t)i * stride;
        for (int j = 1; j <= w; j++) {
            if (i + j >= N) continue;
            const double* xj = x + 2 * (size_t)(i + j) * stride;
            xi[0] -= buf[i * w + j - 1] * xj[0];
            xi[1] -= buf[i * w + j - 1] * xj[1];
        }
    }
}

/* Collocated tridiagonal solve, collocated_AB3/func_global.h:8-61 */
static void thomas_coll(const orc* o, int ixy, double* p) {
    const int NX = o->NX, NZ = o->NZ, stride = o->NXY;
    const int ix = ixy % NX, iy = ixy / NX;
    const double* MA = o->cMAT_A;
    real MM = (real)(1 - o->cosx[ix]) * o->hy / o->hx + (real)(1 - o->cosy[iy]) * o->hx / o->hy;
    double* x = o->spec + 2 * (size_t)ixy;
    real b0 = (real)(-MA[1]);
    if (!o->fd_mode) b0 += (real)(o->cDZ[0] * MM);
    if (ixy == 0) b0 *= 2;
    real ib0 = 1 / b0;
    x[0] *= ib0; x[1] *= ib0;
    p[0] = (real)(MA[1] * ib0);
    for (int i = 1; i <= NZ - 1; i++) {
        const real mm = (o->fd_mode && (i == 0 || i == NZ - 1)) ? RL(0) : MM;
        real d = 0;
        if (i != 0) d -= (real)(MA[i] + o->cDZ[i - 1] * mm);
        if (i != NZ - 1) d -= (real)(MA[i + 1] + o->cDZ[i] * mm);
        d -= (real)(MA[i] * (real)p[i - 1]);
        d = 1 / d;
        if (i != NZ - 1) p[i] = (real)(MA[i + 1] * d);
        double* xi = x + 2 * (size_t)i * stride;
        const double* xm = x + 2 * (size_t)(i - 1) * stride;
        xi[0] = (xi[0] - MA[i] * xm[0]) * d;
        xi[1] = (xi[1] - MA[i] * xm[1]) * d;
    }
    for (int i = NZ - 2; i >= 0; i--) {
        double* xi = x + 2 * (size_t)i * stride;
        const double* xp = x + 2 * (size_t)(i + 1) * stride;
        xi[0] -= xp[0] * p[i];
        xi[1] -= xp[1] * p[i];
    }
}

static void normalize_pressure_r(const orc* o, real* f) {
    const int NXY = o->NXY;
    double psum = 0;
    if (o->scheme == ORC_COLLOC) {
        /* collocated_AB3/func_global.h:163-170, including its extra hx*hy factor */
#pragma omp parallel for reduction(+ : psum) schedule(static)
        for (int i = 0; i < o->N3D; i++) psum += (double)f[i] * (double)(c_cell_height(o, i / NXY) * o->hx * o->hy);
        real shift = (real)(psum * o->hx * o->hy / o->area);
#pragma omp parallel for schedule(static)
        for (int i = 0; i < o->N3D; i++) f[i] -= shift;
    } else if (o->scheme == ORC_HW2) {
        /* staggered/func_global.h:660-666 */
#pragma omp parallel for reduction(+ : psum) schedule(static)
        for (int i = 0; i < o->N3D; i++) psum += (double)f[i] * (double)o->DZ[i / NXY];
        real shift = (real)(psum / ((double)(o->ZZ[o->NZ] - o->ZZ[0]) * NXY));
#pragma omp parallel for schedule(static)
        for (int i = 0; i < o->N3D; i++) f[i] -= shift;
    } else {
        /* staggered/func_global.h:667-673: remove the KERG component */
#pragma omp parallel for reduction(+ : psum) schedule(static)
        for (int i = 0; i < o->N3D; i++) psum += (double)f[i] * (double)o->KERG[i / NXY] * (double)o->DZ[i / NXY];
        real shift = (real)(psum / ((double)o->KERG_norm2 * NXY));
#pragma omp parallel for schedule(static)
        for (int i = 0; i < o->N3D; i++) f[i] -= shift * o->KERG[i / NXY];
    }
}

static void lin_solve_fft(orc* o, real* XX, const real* f) {
    const size_t N = (size_t)o->N3D;
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < N; i++) { o->spec[2 * i] = f[i]; o->spec[2 * i + 1] = 0; }
    fft2_planes(o, -1);
#pragma omp parallel
    {
        double* buf = (double*)malloc(sizeof(double) * 3 * (o->NZ + 1));
#pragma omp for schedule(static)
        for (int m = 0; m < o->NXY; m++) {
            if (o->scheme == ORC_HW2) thomas_hw2(o, m, buf);
            else if (o->scheme == ORC_VV4) thomas_vv4(o, m, buf);
            else thomas_coll(o, m, buf);
        }
        free(buf);
    }
    fft2_planes(o, +1);
    const double inv = 1. / o->NXY;
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < N; i++) XX[i] = (real)(o->spec[2 * i] * inv);
    normalize_pressure_r(o, XX);
}

static void gradient_r(const orc* o, const real* a, real* g) {
    if (o->scheme == ORC_COLLOC) coll_gradient(o, a, g);
    else stag_gradient(o, a, g);
}
static void divergence_r(const orc* o, const real* v, real* dv) {
    if (o->scheme == ORC_COLLOC) coll_divergence(o, v, dv);
    else stag_divergence(o, v, dv);
}
static void unapply_gradient_r(orc* o, const real* v, real* p) {
    divergence_r(o, v, o->divv);
    lin_solve_fft(o, p, o->divv);
}
static void explicit_term_r(orc* o, const real* v, real* f) {
#pragma omp parallel for schedule(static)
    for (int in = 0; in < o->N3D; in++) {
        real r[3];
        if (o->scheme == ORC_COLLOC) coll_flux_cell(o, in, v, 1, 1, r);
        else stag_flux_cell(o, in, v, 1, 1, 1, r);
        f[3 * in] = r[0]; f[3 * in + 1] = r[1]; f[3 * in + 2] = r[2];
    }
}
static void turb_visc_r(orc* o, const real* v) {
    if (o->scheme == ORC_COLLOC) coll_turb_visc(o, v);
    else stag_turb_visc(o, v);
}

/* ------------------------------------------------------------------------ */
/* Public operator wrappers on double host buffers                           */
/* ------------------------------------------------------------------------ */
void orc_apply_gradient(orc* o, const double* p, double* gp) {
    size_t N = (size_t)o->N3D;
    real *a = (real*)malloc(sizeof(real) * N), *g = (real*)malloc(sizeof(real) * 3 * N);
    to_real(a, p, N);
    gradient_r(o, a, g);
    to_double(gp, g, 3 * N);
    free(a); free(g);
}
void orc_apply_divergence(orc* o, const double* v, double* dv) {
    size_t N = (size_t)o->N3D;
    real *a = (real*)malloc(sizeof(real) * 3 * N), *d = (real*)malloc(sizeof(real) * N);
    to_real(a, v, 3 * N);
    divergence_r(o, a, d);
    to_double(dv, d, N);
    free(a); free(d);
}
void orc_unapply_gradient(orc* o, const double* v, double* p) {
    size_t N = (size_t)o->N3D;
    real *a = (real*)malloc(sizeof(real) * 3 * N), *q = (real*)malloc(sizeof(real) * N);
    to_real(a, v, 3 * N);
    unapply_gradient_r(o, a, q);
    to_double(p, q, N);
    free(a); free(q);
}
void orc_pressure_solve(orc* o, const double* rhs, double* p) {
    size_t N = (size_t)o->N3D;
    real *a = (real*)malloc(sizeof(real) * N), *q = (real*)malloc(sizeof(real) * N);
    to_real(a, rhs, N);
    lin_solve_fft(o, q, a);
    to_double(p, q, N);
    free(a); free(q);
}
void orc_normalize_pressure(orc* o, double* p) {
    size_t N = (size_t)o->N3D;
    real* a = (real*)malloc(sizeof(real) * N);
    to_real(a, p, N);
    normalize_pressure_r(o, a);
    to_double(p, a, N);
    free(a);
}
void orc_explicit_term(orc* o, const double* v, double* f) {
    size_t N = (size_t)o->N3D;
    real *a = (real*)malloc(sizeof(real) * 3 * N), *r = (real*)malloc(sizeof(real) * 3 * N);
    to_real(a, v, 3 * N);
    explicit_term_r(o, a, r);
    to_double(f, r, 3 * N);
    free(a); free(r);
}
void orc_flux_fd(orc* o, const double* v, int do_conv, int do_visc, double* f) {
    size_t N = (size_t)o->N3D;
    real *a = (real*)malloc(sizeof(real) * 3 * N), *r = (real*)malloc(sizeof(real) * 3 * N);
    to_real(a, v, 3 * N);
#pragma omp parallel for schedule(static)
    for (int in = 0; in < o->N3D; in++) {
        real q[3];
        if (o->scheme == ORC_COLLOC) coll_flux_cell(o, in, a, do_conv, do_visc, q);
        else stag_flux_cell(o, in, a, do_conv, do_visc, 0, q);
        r[3 * in] = q[0]; r[3 * in + 1] = q[1]; r[3 * in + 2] = q[2];
    }
    to_double(f, r, 3 * N);
    free(a); free(r);
}
void orc_recalc_turb_visc(orc* o, const double* v) {
    size_t N = (size_t)o->N3D;
    real* a = (real*)malloc(sizeof(real) * 3 * N);
    to_real(a, v, 3 * N);
    turb_visc_r(o, a);
    free(a);
}

/* ------------------------------------------------------------------------ */
/* Diagnostics: staggered/func_global.h:678-808, collocated_AB3/func_global.h:173-289 */
/* ------------------------------------------------------------------------ */
static double cell_weight_u(const orc* o, int iz) {
    return o->scheme == ORC_COLLOC ? (double)c_cell_height(o, iz) : (double)o->DZ[iz];
}
static double cell_weight_w(const orc* o, int iz) {
    if (o->scheme == ORC_COLLOC) return (double)c_cell_height(o, iz);
    return iz == 0 ? 0. : (double)(RL(0.5) * (o->DZ[iz] + o->DZ[iz - 1]));
}

void orc_integral(const orc* o, int level, double out[3]) {
    const real* u = o->vel[level];
    double s0 = 0, s1 = 0, s2 = 0;
#pragma omp parallel for reduction(+ : s0, s1, s2) schedule(static)
    for (int i = 0; i < o->N3D; i++) {
        int iz = i / o->NXY;
        double wu = cell_weight_u(o, iz), ww = cell_weight_w(o, iz);
        s0 += u[3 * i] * wu;
        s1 += u[3 * i + 1] * wu;
        s2 += u[3 * i + 2] * ww;
    }
    double hxy = (double)o->hx * o->hy;
    out[0] = s0 * hxy; out[1] = s1 * hxy; out[2] = s2 * hxy;
}

double orc_kinetic_energy(const orc* o, int level) {
    const real* u = o->vel[level];
    double s = 0;
#pragma omp parallel for reduction(+ : s) schedule(static)
    for (int i = 0; i < o->N3D; i++) {
        int iz = i / o->NXY;
        double wu = cell_weight_u(o, iz), ww = cell_weight_w(o, iz);
        s += ((double)u[3 * i] * u[3 * i] + (double)u[3 * i + 1] * u[3 * i + 1]) * wu + (double)u[3 * i + 2] * u[3 * i + 2] * ww;
    }
    return 0.5 * s * o->hx * o->hy;
}

static double coll_nut_node(const orc* o, int in) {
    nbh b; nbh_set(o, &b, in);
    if (!o->nu_t || c_is_wall(o, b.iz)) return 0.;
    const real* n = o->nu_t;
    return 0.125 * ((double)n[in] + n[NB(-1, 0, 0)] + n[NB(0, -1, 0)] + n[NB(-1, -1, 0)] + n[NB(0, 0, -1)] + n[NB(-1, 0, -1)] +
                    n[NB(0, -1, -1)] + n[NB(-1, -1, -1)]);
}

double orc_cfl(const orc* o, int level, double tau, int mode) {
    const real* u = o->vel[level];
    double m = 0;
#pragma omp parallel for reduction(max : m) schedule(static)
    for (int i = 0; i < o->N3D; i++) {
        int iz = i / o->NXY;
        double ihz = o->scheme == ORC_COLLOC ? 1. / c_cell_height(o, iz) : 1. / o->DZ[iz];
        double c = 0;
        if (mode & 1) c += tau * (fabs((double)u[3 * i]) * o->inv_hx + fabs((double)u[3 * i + 1]) * o->inv_hy + fabs((double)u[3 * i + 2]) * ihz);
        if (mode & 2) {
            double nt = 0, k;
            if (o->scheme == ORC_COLLOC) { nt = coll_nut_node(o, i); k = o->visc_type == ORC_VISC_GALERKIN ? 2 : 1; }
            else { nt = o->nu_t ? (double)o->nu_t[i] : 0.; k = o->visc_type != ORC_VISC_CROSS ? 2 : 1; }
            c += 4 * k * tau * ((double)o->visc + nt) * ((double)o->inv_hx * o->inv_hx + (double)o->inv_hy * o->inv_hy + ihz * ihz);
        }
        if (c > m) m = c;
    }
    return m;
}

void orc_profiles(const orc* o, int level, double* out) {
    const real *u = o->vel[level], *p = o->pres[level];
    const int NXY = o->NXY, NZ = o->NZ;
#pragma omp parallel for schedule(static)
    for (int iz = 0; iz < NZ; iz++) {
        double s[12] = {0};
        for (int in = iz * NXY; in < (iz + 1) * NXY; in++) {
            double a = u[3 * in], b = u[3 * in + 1], c;
            if (o->scheme == ORC_COLLOC) c = u[3 * in + 2];
            else c = 0.5 * (u[3 * in + 2] + (iz == NZ - 1 ? 0. : (double)u[3 * (in + NXY) + 2]));
            s[0] += a; s[1] += b; s[2] += c;
            s[3] += a * a; s[4] += b * b; s[5] += c * c; s[6] += a * b; s[7] += a * c; s[8] += b * c;
            if (o->nu_t) s[9] += o->nu_t[in];
            s[10] += p[in]; s[11] += (double)p[in] * p[in];
        }
        for (int k = 0; k < 12; k++) out[iz * 12 + k] = s[k] / NXY;
    }
}

/* ------------------------------------------------------------------------ */
/* Step: staggered/func_global.h:897-942, collocated_AB3/func_global.h:387-450 */
/* ------------------------------------------------------------------------ */
int orc_step(orc* o, double t, double tau, int cur, int order, int cfr_on, double cfr_target, double* dpdx_out) {
    (void)t;
    if (order < 1 || order > 3) return -1;
    const int nxt = (cur + 1) % 4, prv = (cur + 3) % 4, pr2 = (cur + 2) % 4;
    const real inv_tau = (real)(1. / tau);
    const real bd0 = order == 3 ? RL(1.5 + C1_3) : order == 2 ? RL(1.5) : RL(1.0);
    const real tob = (real)(tau / bd0);
    const size_t N = (size_t)o->N3D;
    if (o->turb) turb_visc_r(o, o->vel[cur]);
    explicit_term_r(o, o->vel[cur], o->flux[cur]);
    real *Fn = o->flux[nxt], *Fc = o->flux[cur], *Fp = o->flux[prv], *Fq = o->flux[pr2];
    real *Vc = o->vel[cur], *Vp = o->vel[prv], *Vq = o->vel[pr2];
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < 3 * N; i++) {
        if (order == 1) Fn[i] = Fc[i] + inv_tau * Vc[i];
        else if (order == 2) Fn[i] = RL(2.) * Fc[i] - Fp[i] + inv_tau * (2 * Vc[i] - RL(0.5) * Vp[i]);
        else Fn[i] = 3 * Fc[i] - 3 * Fp[i] + Fq[i] + inv_tau * (3 * Vc[i] - RL(1.5) * Vp[i] + C1_3 * Vq[i]);
    }
    real* Vn = o->vel[nxt];
    if (o->scheme == ORC_COLLOC && o->stab_type == 1) {
        gradient_r(o, o->pres[cur], Vn);
#pragma omp parallel for schedule(static)
        for (size_t i = 0; i < 3 * N; i++) Fn[i] -= Vn[i];
        unapply_gradient_r(o, Fn, o->pres[nxt]);
        gradient_r(o, o->pres[nxt], Vn);
#pragma omp parallel for schedule(static)
        for (size_t i = 0; i < N; i++) o->pres[nxt][i] += o->pres[cur][i];
    } else {
        unapply_gradient_r(o, Fn, o->pres[nxt]);
        gradient_r(o, o->pres[nxt], Vn);
    }
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < 3 * N; i++) Vn[i] = (Fn[i] - Vn[i]) * tob;
    double dpdx = (double)o->sour_dpdx;
    if (cfr_on) {
        /* Constant flow rate: shift u uniformly (fluid nodes only) so that the bulk
           velocity equals the target; report the equivalent mean pressure gradient. */
        double I[3];
        orc_integral(o, nxt, I);
        double ub = I[0] / o->area;
        double vf = o->area;
        if (o->scheme == ORC_COLLOC) {
            vf = 0;
            for (int iz = 1; iz < o->NZ - 1; iz++) vf += (double)c_cell_height(o, iz);
            vf *= (double)o->hx * o->hy * o->NXY;
        }
        double du = (cfr_target - ub) * o->area / vf;
        const real dur = (real)du;
#pragma omp parallel for schedule(static)
        for (size_t i = 0; i < N; i++) {
            int iz = (int)(i / o->NXY);
            if (o->scheme == ORC_COLLOC && c_is_wall(o, iz)) continue;
            Vn[3 * i] += dur;
        }
        dpdx += du * bd0 / tau;
    }
    if (dpdx_out) *dpdx_out = dpdx;
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Seeded initial field and mesh                                             */
/* ------------------------------------------------------------------------ */
/* MT19937-64 (Matsumoto & Nishimura 2004), the generator of std::mt19937_64. */
typedef struct { uint64_t mt[312]; int mti; } mt64;
static void mt64_seed(mt64* g, uint64_t s) {
    g->mt[0] = s;
    for (int i = 1; i < 312; i++) g->mt[i] = 6364136223846793005ULL * (g->mt[i - 1] ^ (g->mt[i - 1] >> 62)) + (uint64_t)i;
    g->mti = 312;
}
static uint64_t mt64_next(mt64* g) {
    static const uint64_t MAG[2] = {0ULL, 0xB5026F5AA96619E9ULL};
    const uint64_t UM = 0xFFFFFFFF80000000ULL, LM = 0x7FFFFFFFULL;
    if (g->mti >= 312) {
        int i;
        uint64_t x;
        for (i = 0; i < 312 - 156; i++) {
            x = (g->mt[i] & UM) | (g->mt[i + 1] & LM);
            g->mt[i] = g->mt[i + 156] ^ (x >> 1) ^ MAG[x & 1ULL];
        }
        for (; i < 311; i++) {
            x = (g->mt[i] & UM) | (g->mt[i + 1] & LM);
            g->mt[i] = g->mt[i + (156 - 312)] ^ (x >> 1) ^ MAG[x & 1ULL];
        }
        x = (g->mt[311] & UM) | (g->mt[0] & LM);
        g->mt[311] = g->mt[155] ^ (x >> 1) ^ MAG[x & 1ULL];
        g->mti = 0;
    }
    uint64_t x = g->mt[g->mti++];
    x ^= (x >> 29) & 0x5555555555555555ULL;
    x ^= (x << 17) & 0x71D67FFFEDA60000ULL;
    x ^= (x << 37) & 0xFFF7EEE000000000ULL;
    x ^= (x >> 43);
    return x;
}
void orc_mt64_fill(unsigned long long seed, int n, unsigned long long* out) {
    mt64 g;
    mt64_seed(&g, seed);
    for (int i = 0; i < n; i++) out[i] = mt64_next(&g);
}

void orc_mesh_tanh(int n, double gamma, double H, double* z) {
    for (int j = 0; j <= n; j++) z[j] = H * (1. + tanh(gamma * (2. * j / n - 1.)) / tanh(gamma));
}

void orc_init_channel(orc* o, int level, unsigned long long seed, double amp, int project) {
    const size_t N = (size_t)o->N3D;
    real* v = o->vel[level];
    mt64 g;
    mt64_seed(&g, seed);
    const double H = o->scheme == ORC_COLLOC ? 0.5 * (o->cZZ[o->NZ - 1] - o->cZZ[0]) : 0.5 * (double)(o->ZZ[o->NZ] - o->ZZ[0]);
    const double z0 = o->scheme == ORC_COLLOC ? o->cZZ[0] : (double)o->ZZ[0];
    for (size_t in = 0; in < N; in++) {
        const int iz = (int)(in / o->NXY);
        double r[3];
        for (int c = 0; c < 3; c++) r[c] = amp * (2. * (double)(mt64_next(&g) >> 11) * (1.0 / 9007199254740992.0) - 1.);
        double zc = o->scheme == ORC_COLLOC ? o->cZZ[iz] : 0.5 * ((double)o->ZZ[iz] + o->ZZ[iz + 1]);
        double y = (zc - z0) / H - 1.;
        v[3 * in + 0] = (real)(1.5 * (1. - y * y) + r[0]);
        v[3 * in + 1] = (real)r[1];
        v[3 * in + 2] = (real)r[2];
        if (o->scheme == ORC_COLLOC) {
            if (c_is_wall(o, iz)) v[3 * in] = v[3 * in + 1] = v[3 * in + 2] = 0;
        } else if (iz == 0) v[3 * in + 2] = 0;
    }
    memset(o->pres[level], 0, sizeof(real) * N);
    if (project) {
        /* divergence-free projection as in staggered/selftest.cpp:224-227 */
        real *p = (real*)malloc(sizeof(real) * N), *gp = (real*)malloc(sizeof(real) * 3 * N);
        unapply_gradient_r(o, v, p);
        gradient_r(o, p, gp);
        for (size_t i = 0; i < 3 * N; i++) v[i] -= gp[i];
        free(p); free(gp);
    }
}

/* ------------------------------------------------------------------------ */
/* Self-tests restated from staggered/selftest.cpp                           */
/* ------------------------------------------------------------------------ */
double orc_check_gradient_kernel(orc* o) { /* selftest.cpp:79-87 */
    size_t N = (size_t)o->N3D;
    real *p = (real*)malloc(sizeof(real) * N), *g = (real*)malloc(sizeof(real) * 3 * N);
    for (size_t in = 0; in < N; in++) p[in] = o->KERG[in / o->NXY];
    gradient_r(o, p, g);
    double e = 0;
    for (size_t in = 0; in < N; in++) {
        double a = sqrt((double)g[3 * in] * g[3 * in] + (double)g[3 * in + 1] * g[3 * in + 1] + (double)g[3 * in + 2] * g[3 * in + 2]);
        if (a > e) e = a;
    }
    free(p); free(g);
    return e;
}
double orc_check_normalization_projection(orc* o) { /* selftest.cpp:89-95 */
    size_t N = (size_t)o->N3D;
    real *p = (real*)malloc(sizeof(real) * N), *q = (real*)malloc(sizeof(real) * N);
    for (size_t in = 0; in < N; in++) p[in] = (real)sin((double)in * in);
    normalize_pressure_r(o, p);
    memcpy(q, p, sizeof(real) * N);
    normalize_pressure_r(o, p);
    double e = 0;
    for (size_t in = 0; in < N; in++) { double a = fabs((double)p[in] - q[in]); if (a > e) e = a; }
    free(p); free(q);
    return e;
}
double orc_check_matrix_symmetry(orc* o) { /* selftest.cpp:100-114 */
    real* M = (real*)calloc((size_t)7 * o->NZ, sizeof(real));
    fill_matrix_vv4(o, M);
    double e = 0;
    for (int i = 0; i < o->NZ; i++)
        for (int j = -3; j <= 3; j++) {
            if (i + j < 0 || i + j >= o->NZ) continue;
            double a = fabs((double)M[i * 7 + 3 + j] - M[(i + j) * 7 + 3 - j]);
            if (a > e) e = a;
        }
    free(M);
    return e;
}
double orc_check_pressure_matrix(orc* o) { /* selftest.cpp:116-141 */
    size_t N = (size_t)o->N3D;
    const int NZ = o->NZ, NXY = o->NXY;
    real* M = (real*)calloc((size_t)7 * NZ, sizeof(real));
    fill_matrix_vv4(o, M);
    real *p = (real*)malloc(sizeof(real) * N), *g = (real*)malloc(sizeof(real) * 3 * N), *d = (real*)malloc(sizeof(real) * N);
    for (int iz = 0; iz < NZ; iz++)
        for (int ixy = 0; ixy < NXY; ixy++) p[iz * NXY + ixy] = (real)sin((double)(iz * iz) + 51.);
    gradient_r(o, p, g);
    divergence_r(o, g, d);
    double e = 0;
    for (int i = 0; i < NZ; i++) {
        double s = 0;
        for (int j = -3; j <= 3; j++) {
            if (i + j < 0 || i + j >= NZ) continue;
            s += (double)M[7 * i + j + 3] * p[(i + j) * NXY];
        }
        for (int ixy = 0; ixy < NXY; ixy++) { double a = fabs(s - d[i * NXY + ixy]); if (a > e) e = a; }
    }
    free(M); free(p); free(g); free(d);
    return e;
}
double orc_check_pressure_solver(orc* o, int itest) { /* selftest.cpp:144-181 */
    size_t N = (size_t)o->N3D;
    real *p = (real*)malloc(sizeof(real) * N), *g = (real*)malloc(sizeof(real) * 3 * N), *d = (real*)malloc(sizeof(real) * N);
    real* pn = (real*)malloc(sizeof(real) * N);
    for (size_t in = 0; in < N; in++) {
        int iz = (int)(in / o->NXY);
        p[in] = itest == 0 ? (real)sin((double)(o->scheme == ORC_COLLOC ? o->cZZ[iz] : o->ZZ[iz])) : (real)sin((double)in * in);
    }
    normalize_pressure_r(o, p);
    gradient_r(o, p, g);
    divergence_r(o, g, d);
    lin_solve_fft(o, pn, d);
    normalize_pressure_r(o, pn);
    double e = 0;
    for (size_t in = 0; in < N; in++) { double a = fabs((double)p[in] - pn[in]); if (a > e) e = a; }
    free(p); free(g); free(d); free(pn);
    return e;
}
double orc_check_conservation(orc* o, int itest, double out_K[3]) { /* selftest.cpp:186-254 (3-D case) */
    (void)itest;
    size_t N = (size_t)o->N3D;
    const int NXY = o->NXY;
    real *v = (real*)malloc(sizeof(real) * 3 * N), *g = (real*)malloc(sizeof(real) * 3 * N), *p = (real*)malloc(sizeof(real) * N);
    real* f = (real*)malloc(sizeof(real) * 3 * N);
    for (size_t in = 0; in < N; in++) {
        for (int c = 0; c < 3; c++) v[3 * in + c] = (real)sin((double)in * in + cos(10. * c));
        if (in < (size_t)NXY) v[3 * in + 2] = 0;
    }
    unapply_gradient_r(o, v, p);
    gradient_r(o, p, g);
    for (size_t i = 0; i < 3 * N; i++) v[i] -= g[i];
    unapply_gradient_r(o, v, p);
    double ediv = 0;
    for (size_t in = 0; in < N; in++) if (fabs((double)p[in]) > ediv) ediv = fabs((double)p[in]);
#pragma omp parallel for schedule(static)
    for (int in = 0; in < o->N3D; in++) {
        real q[3];
        stag_flux_cell(o, in, v, 1, 0, 0, q);
        f[3 * in] = q[0]; f[3 * in + 1] = q[1]; f[3 * in + 2] = q[2];
    }
    double K[3] = {0, 0, 0};
    for (size_t in = 0; in < N; in++) {
        int iz = (int)(in / NXY);
        double hz = 1.125 * o->DZ[iz] - 0.125 * o->DZW[iz];
        double hzw = iz > 0 ? 1. / o->GCZ[iz] : 0.;
        K[0] += (double)f[3 * in] * v[3 * in] * hz;
        K[1] += (double)f[3 * in + 1] * v[3 * in + 1] * hz;
        if (iz > 0) K[2] += (double)f[3 * in + 2] * v[3 * in + 2] * hzw;
    }
    if (out_K) { out_K[0] = K[0]; out_K[1] = K[1]; out_K[2] = K[2]; }
    free(v); free(g); free(p); free(f);
    return ediv;
}
