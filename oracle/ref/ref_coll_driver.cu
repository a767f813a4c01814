/*
 * ref_coll_driver.cu -- C entry points over the reference's collocated_AB3 CPU
 * solver object.  The reference keeps main() and both solver namespaces in one
 * translation unit, so this file compiles that unit in place (its main renamed)
 * and adds the entry points after it.  Setup follows collocated_AB3/main.cpp:
 * 236-300 with the node coordinates supplied by the caller.
 * TEST INFRASTRUCTURE ONLY (oracle/_ref/).
 */
#define main tcref_collocated_reference_main
#include "main.cpp"
#undef main
#include <cstring>

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
int ref_kind(void) { return 2; }
int ref_nx(void) { return NX; }
int ref_ny(void) { return NY; }
int ref_nzmax(void) { return NZ_MAX; }
int ref_conv(void) { return 2; }
int ref_turb(void) { return D.EnableTurbVisc; }
int ref_visc_naive(void) { return VISC_TERM_GALERKIN; }
int ref_real_size(void) { return (int)sizeof(real); }
void ref_set_threads(int n) { if (n > 0) omp_set_num_threads(n); }

int ref_setup_colloc(int nz, const double* zz, double visc, double sour_dpdx, double inv_ls, double hx, double hy,
                     double area, int turb, int stab_type, int fd_mode) {
    if (nz > NZ_MAX || nz < 4) return 1;
    for (int i = 0; i < nz; i++) data_cpu::ZZ[i] = zz[i];
    for (int i = 0; i < nz - 1; i++) data_cpu::DZ[i] = data_cpu::ZZ[i + 1] - data_cpu::ZZ[i];
    main_params& MD = D;
    MD.StabType = stab_type;
    MD.visc = visc;
    MD.sour_dpdx = sour_dpdx;
    MD.inv_length_scale = inv_ls;
    MD.EnableTurbVisc = turb;
    MD.NZ = nz;
    MD.N3D = NX * NY * nz;
    MD.hx = hx;
    MD.hy = hy;
    MD.inv_hx = 1. / MD.hx;
    MD.inv_hy = 1. / MD.hy;
    MD.area = area;
    MD.xmin = 0.;
    MD.ymin = 0.;
    MD.FDmode = fd_mode;
    D.alloc_all();
    D.InitFourier();
    double* A = data_cpu::MAT_A;
    A[0] = 0.;
    for (int j = 1; j < nz; j++) A[j] = D.hx * D.hy / data_cpu::DZ[j - 1];
    if (D.FDmode) { A[1] *= 0.5; A[nz - 1] *= 0.5; }
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
    if (!strcmp(name, "ZZ")) { for (int i = 0; i < NZ; i++) out[i] = data_cpu::ZZ[i]; return NZ; }
    if (!strcmp(name, "DZ")) { for (int i = 0; i < NZ - 1; i++) out[i] = data_cpu::DZ[i]; return NZ - 1; }
    if (!strcmp(name, "cMAT_A")) { for (int i = 0; i < NZ; i++) out[i] = data_cpu::MAT_A[i]; return NZ; }
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
    std::vector<real> p(D.N3D);
    put3(a.data(), v);
    D.ExplicitTerm(0., a.data(), p.data(), r.data());
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
    D.CalcVelocityProfile(D.vel[l]);
    for (int iz = 0; iz < D.NZ; iz++) {
        const real9& a = D.av_u[iz];
        double* o = out + 12 * iz;
        for (int c = 0; c < 3; c++) o[c] = a.u[c];
        for (int c = 0; c < 6; c++) o[3 + c] = a.uu[c];
        o[9] = a.nu_t; o[10] = 0.; o[11] = 0.;
    }
}
}
