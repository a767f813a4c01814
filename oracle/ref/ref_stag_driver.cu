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

/* ---------------------------------------------------------------------------
 * The reference's own GPU solver, data_cuda::data of staggered/func_cuda.cpp
 * (lambda Forall kernels, cuFFT D2Z/Z2D, Thrust reductions), set up as
 * staggered/main.cpp:209-262 does (the CPU object holds the parameters and mesh
 * data; the GPU object gets a copy of them, its own buffers and the constant-memory
 * image), and stepped as its time loop does (main.cpp:306-340).  Used to time the
 * reference's GPU path on the same device as the product.  The GPU object holds
 * device buffers only; the CPU object's field buffers are not allocated here.
 * ------------------------------------------------------------------------- */
extern "C++" void CopyDataToDevice(const data_cuda::data&);  // staggered/func_cuda.cpp
static data_cuda::data G;
static int g_gpu_ready = 0;

__global__ void refgpu_subtract(real3* v, const real3* g, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] -= g[i];
}

int refgpu_setup(int nz, const double* zz, double visc, double sour_dpdx, double inv_ls, double hx, double hy,
                 double area, int device) {
    if (nz > NZ_MAX || nz < 6 || g_gpu_ready) return 1;
    if (cudaSetDevice(device) != cudaSuccess) return 2;
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
    *(static_cast<main_params*>(&G)) = *(static_cast<main_params*>(&D));
    G.alloc_all();
    CopyDataToDevice(G);
    G.InitFourier();
    for (int l = 0; l < 4; l++) {
        cudaMemset((void*)G.vel[l], 0, sizeof(real3) * D.N3D);
        cudaMemset((void*)G.flux[l], 0, sizeof(real3) * D.N3D);
        cudaMemset((void*)G.pres[l], 0, sizeof(real) * D.N3D);
    }
    cudaMemset((void*)G.divv, 0, sizeof(real) * D.N3D);
    if (G.nu_t) cudaMemset((void*)G.nu_t, 0, sizeof(real) * D.N3D);
    g_gpu_ready = cudaDeviceSynchronize() == cudaSuccess;
    return g_gpu_ready ? 0 : 3;
}

/* Host AoS double <-> the GPU object's level `l` (real3 / real in `real`). */
int refgpu_set_level(int l, const double* vel, const double* p) {
    if (!g_gpu_ready) return 1;
    std::vector<real3> a(vel ? D.N3D : 0);
    std::vector<real> b(p ? D.N3D : 0);
    if (vel) { put3(a.data(), vel); cudaMemcpy(G.vel[l], a.data(), sizeof(real3) * D.N3D, cudaMemcpyHostToDevice); }
    if (p) { put1(b.data(), p); cudaMemcpy(G.pres[l], b.data(), sizeof(real) * D.N3D, cudaMemcpyHostToDevice); }
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 2;
}
int refgpu_get_level(int l, double* vel, double* p) {
    if (!g_gpu_ready) return 1;
    std::vector<real3> a(vel ? D.N3D : 0);
    std::vector<real> b(p ? D.N3D : 0);
    if (vel) { cudaMemcpy(a.data(), G.vel[l], sizeof(real3) * D.N3D, cudaMemcpyDeviceToHost); get3(vel, a.data()); }
    if (p) { cudaMemcpy(b.data(), G.pres[l], sizeof(real) * D.N3D, cudaMemcpyDeviceToHost); get1(p, b.data()); }
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 2;
}

/* Project level `l` divergence-free with the GPU object's own operators, as
 * staggered/selftest.cpp:224-226 does: v -= grad(L^-1 div v) (flux[(l+1)%4] is the
 * scratch gradient). */
int refgpu_project(int l) {
    if (!g_gpu_ready) return 1;
    real3* g = G.flux[(l + 1) % 4];
    G.UnapplyGradient(G.vel[l], G.pres[l]);
    G.ApplyGradient(G.pres[l], g);
    refgpu_subtract<<<(D.N3D + 255) / 256, 256>>>(G.vel[l], g, D.N3D);
    cudaMemset((void*)G.pres[l], 0, sizeof(real) * D.N3D);
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 2;
}

/* `nsteps` steps of the reference's time loop from ring level *cur (order ramped
 * from *it as main.cpp:308 does), timed with CUDA events on the default stream that
 * the reference launches on.  with_diag != 0 adds the loop's per-step diagnostics
 * (CalcIntegral, CalcProfiles + the av_u device->host copy, CalcCFL:
 * main.cpp:313-338).  Returns the elapsed milliseconds, or a negative value on a
 * CUDA error. */
double refgpu_run(int nsteps, double tau, int with_diag, int* cur, int* it) {
    if (!g_gpu_ready) return -1.0;
    std::vector<real9<real>> prof(D.NZ);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaDeviceSynchronize();
    cudaEventRecord(e0, 0);
    for (int s = 0; s < nsteps; s++) {
        const int order = *it + 1 < 3 ? *it + 1 : 3;
        G.Step(*it * tau, tau, *cur, order);
        *cur = (*cur + 1) % 4;
        *it += 1;
        if (with_diag) {
            volatile real3 fr = G.CalcIntegral(G.vel[*cur]);
            (void)fr;
            G.CalcProfiles(G.vel[*cur], G.pres[*cur]);
            cudaMemcpy(prof.data(), G.av_u, sizeof(real9<real>) * D.NZ, cudaMemcpyDeviceToHost);
            volatile real cfl = G.CalcCFL(G.vel[*cur], (real)tau, 3);
            (void)cfl;
        }
    }
    cudaEventRecord(e1, 0);
    cudaEventSynchronize(e1);
    float ms = -1.f;
    const cudaError_t err = cudaGetLastError();
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return err == cudaSuccess ? (double)ms : -1.0;
}

int refgpu_integral(int l, double* out) {
    if (!g_gpu_ready) return 1;
    real3 r = G.CalcIntegral(G.vel[l]);
    for (int c = 0; c < 3; c++) out[c] = r[c];
    return 0;
}

void refgpu_free(void) {
    if (!g_gpu_ready) return;
    G.dealloc_all();
    g_gpu_ready = 0;
}

/* Project level `l` of the CPU object divergence-free with the reference's own
 * operators (staggered/selftest.cpp:224-226; flux[(l+1)%4] is the scratch gradient). */
void ref_project(int l) {
    real3* g = D.flux[(l + 1) % 4];
    D.UnapplyGradient(D.vel[l], D.pres[l]);
    D.ApplyGradient(D.pres[l], g);
    real3* v = D.vel[l];
#pragma omp parallel for schedule(static)
    for (int i = 0; i < D.N3D; i++) v[i] -= g[i];
    memset((void*)D.pres[l], 0, sizeof(real) * D.N3D);
    memset((void*)g, 0, sizeof(real3) * D.N3D);
}

/* Constant flow rate for the reference's CPU object, as the oracle's driver applies
 * it after each step (shift u uniformly so that the bulk velocity is `target`;
 * the reference itself forces with a constant sour_dpdx). */
void ref_cfr_shift(int l, double target) {
    const real3 I = D.CalcIntegral(D.vel[l]);
    const real du = (real)((target - I[0] / D.area));
    real3* v = D.vel[l];
#pragma omp parallel for schedule(static)
    for (int i = 0; i < D.N3D; i++) v[i][0] += du;
}
}
