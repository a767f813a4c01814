/*
 * ref_stag_driver.cu -- C entry points over the reference's own CPU solver object
 * (data_cpu::D of staggered/func_cpu.cpp) so that tests can run the unmodified
 * staggered numerics on seeded inputs.  Setup follows staggered/main.cpp:209-262
 * with the mesh supplied by the caller.  TEST INFRASTRUCTURE ONLY (oracle/_ref/).
 */
#include <omp.h>
#include <cstring>
#include <vector>
#include "data_global.h"

using data_cpu::D;

static void put3(real3* dst, const double* src) {
    for (int i = 0; i < D.N3D; i++) for (int c = 0; c < 3; c++) dst[i][c] = (real)src[3 * i + c];
}
static void get3(double* dst, const real3* src) {
    for (int i = 0; i < D.N3D; i++) for (int c = 0; c < 3; c++) dst[3 * i + c] = (double)src[i][c];
}
static void put1(real* dst, const double* src) { for (int i = 0; i < D.N3D; i++) dst[i] = (real)src[i]; }
static void get1(double* dst, const real* src) { for (int i = 0; i < D.N3D; i++) dst[i] = (double)src[i]; }

extern "C" {
int ref_kind(void) { return 0; }
int ref_nx(void) { return NX; }
int ref_ny(void) { return NY; }
int ref_nzmax(void) { return NZ_MAX; }
int ref_conv(void) { return CONV_APPR_TYPE; }
int ref_turb(void) { return ENABLE_TURB_VISC; }
int ref_visc_naive(void) { return VISC_APPR_TYPE == tViscApproximation::NAIVE; }
int ref_real_size(void) { return (int)sizeof(real); }
void ref_set_threads(int n) { if (n > 0) omp_set_num_threads(n); }

int ref_setup(int nz, const double* zz, double visc, double sour_dpdx, double inv_ls, double hx, double hy, double area) {
    if (nz > NZ_MAX || nz < 6) return 1;
    D.NZ = nz;
    D.N3D = NX * NY * nz;
    D.visc = visc;
    D.sour_dpdx = sour_dpdx;
    D.inv_length_scale = inv_ls;
    D.hx = hx;
    D.hy = hy;
    D.inv_hx = 1. / D.hx;
    D.inv_hy = 1. / D.hy;
    D.area = area;
    D.xmin = 0.;
    D.ymin = 0.;
    for (int i = 0; i <= nz; i++) D.ZZ[i] = zz[i];
    D.InitDerivativeMeshData();
    D.alloc_all();
    D.InitFourier();
    for (int l = 0; l < 4; l++) {
        memset((void*)D.vel[l], 0, sizeof(real3) * D.N3D);
        memset((void*)D.flux[l], 0, sizeof(real3) * D.N3D);
        memset((void*)D.pres[l], 0, sizeof(real) * D.N3D);
    }
    memset((void*)D.divv, 0, sizeof(real) * D.N3D);
    if (D.nu_t) memset((void*)D.nu_t, 0, sizeof(real) * D.N3D);
    return 0;
}

int ref_get_mesh(const char* name, double* out) {
    const int NZ = D.NZ;
    auto cp = [&](const real* a, int n) { for (int i = 0; i < n; i++) out[i] = a[i]; return n; };
    if (!strcmp(name, "ZZ")) return cp(D.ZZ, NZ + 1);
    if (!strcmp(name, "DZ")) return cp(D.DZ, NZ);
#if (CONV_APPR_TYPE == CONV_HW)
    if (!strcmp(name, "MAT_A")) return cp(D.MAT_A, NZ);
#else
    if (!strcmp(name, "MAT_A")) return cp(D.MAT_A, 3 * NZ);
    if (!strcmp(name, "DZW")) return cp(D.DZW, NZ);
    if (!strcmp(name, "GC1")) return cp(D.GC1, NZ);
    if (!strcmp(name, "GC2")) return cp(D.GC2, NZ);
    if (!strcmp(name, "GCZ")) return cp(D.GCZ, NZ);
    if (!strcmp(name, "MAT_D")) return cp(D.MAT_D, 6);
    if (!strcmp(name, "KERG")) return cp(D.KERG, NZ);
    if (!strcmp(name, "KERG_norm2")) { out[0] = D.KERG_norm2; return 1; }
#endif
    return 0;
}

void ref_set_level(int l, const double* vel, const double* p) { if (vel) put3(D.vel[l], vel); if (p) put1(D.pres[l], p); }
void ref_get_level(int l, double* vel, double* p) { if (vel) get3(vel, D.vel[l]); if (p) get1(p, D.pres[l]); }
void ref_get_flux(int l, double* f) { get3(f, D.flux[l]); }
void ref_set_nu_t(const double* nt) { if (D.nu_t) put1(D.nu_t, nt); }
void ref_get_nu_t(double* nt) { if (D.nu_t) get1(nt, D.nu_t); else memset(nt, 0, sizeof(double) * D.N3D); }

void ref_step(double t, double tau, int cur, int order) { D.Step(t, tau, cur, order); }

void ref_explicit_term(const double* v, double* f) {
    std::vector<real3> a(D.N3D), r(D.N3D);
    put3(a.data(), v);
    D.ExplicitTerm(a.data(), r.data());
    get3(f, r.data());
}
void ref_flux_fd(const double* v, int dc, int dv, double* f) {
    std::vector<real3> a(D.N3D), r(D.N3D);
    put3(a.data(), v);
    D.CalcFluxTerm_FD(a.data(), dc, dv, r.data());
    get3(f, r.data());
}
void ref_recalc_turb_visc(const double* v) {
    std::vector<real3> a(D.N3D);
    put3(a.data(), v);
    D.RecalcTurbVisc(a.data());
}
void ref_apply_gradient(const double* p, double* g) {
    std::vector<real> a(D.N3D);
    std::vector<real3> r(D.N3D);
    put1(a.data(), p);
    D.ApplyGradient(a.data(), r.data());
    get3(g, r.data());
}
void ref_apply_divergence(const double* v, double* dv) {
    std::vector<real3> a(D.N3D);
    std::vector<real> r(D.N3D);
    put3(a.data(), v);
    for (int i = 0; i < D.N3D; i++) D.ApplyDivergence(i, a.data(), r.data());
    get1(dv, r.data());
}
void ref_unapply_gradient(const double* v, double* p) {
    std::vector<real3> a(D.N3D);
    std::vector<real> r(D.N3D);
    put3(a.data(), v);
    D.UnapplyGradient(a.data(), r.data());
    get1(p, r.data());
}
void ref_pressure_solve(const double* rhs, double* p) {
    std::vector<real> a(D.N3D), r(D.N3D);
    put1(a.data(), rhs);
    D.LinearSystemSolveFFT(r.data(), a.data());
    get1(p, r.data());
}
void ref_normalize_pressure(double* p) {
    std::vector<real> a(D.N3D);
    put1(a.data(), p);
    D.NormalizePressure(a.data());
    get1(p, a.data());
}
void ref_integral(int l, double* out) { real3 r = D.CalcIntegral(D.vel[l]); for (int c = 0; c < 3; c++) out[c] = r[c]; }
double ref_kinetic_energy(int l) { return D.CalcKineticEnergy(D.vel[l]); }
double ref_cfl(int l, double tau, int mode) { return D.CalcCFL(D.vel[l], tau, mode); }
void ref_profiles(int l, double* out) {
    D.CalcProfiles(D.vel[l], D.pres[l]);
    for (int iz = 0; iz < D.NZ; iz++) {
        const real9<real>& a = D.av_u[iz];
        double* o = out + 12 * iz;
        for (int c = 0; c < 3; c++) o[c] = a.u[c];
        for (int c = 0; c < 6; c++) o[3 + c] = a.uu[c];
        o[9] = a.nu_t; o[10] = a.p; o[11] = a.pp;
    }
}
}
