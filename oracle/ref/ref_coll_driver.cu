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

/* ---------------------------------------------------------------------------
 * The reference's own GPU solver (data_cuda::data of collocated_AB3/main.cpp:114-178:
 * lambda Forall kernels, the shared-memory flux kernel, cuFFT, Thrust), set up as
 * collocated_AB3/main.cpp:264-300 does and stepped as its time loop does
 * (main.cpp:405-440).  Used to time the reference's GPU path on the same device as
 * the product; the CPU object's field buffers are not allocated here.
 * ------------------------------------------------------------------------- */
static data_cuda::data G;
static int g_gpu_ready = 0;

__global__ void refgpu_subtract(real3* v, const real3* g, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] -= g[i];
}

int refgpu_setup_colloc(int nz, const double* zz, double visc, double sour_dpdx, double inv_ls, double hx, double hy,
                        double area, int turb, int stab_type, int fd_mode, int device) {
    if (nz > NZ_MAX || nz < 4 || g_gpu_ready) return 1;
    if (cudaSetDevice(device) != cudaSuccess) return 2;
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
    *(static_cast<main_params*>(&G)) = *(static_cast<main_params*>(&D));
    G.alloc_all();
    cudaMemcpyToSymbol(data_cuda::D, &G, sizeof(data_cuda::data));
    G.InitFourier();
    cudaMemcpyToSymbol(data_cuda::D, &G, sizeof(data_cuda::data));
    cudaMemcpyToSymbol(data_cuda::DZ, data_cpu::DZ, sizeof(double) * nz);
    cudaMemcpyToSymbol(data_cuda::ZZ, data_cpu::ZZ, sizeof(double) * nz);
    double* A = data_cpu::MAT_A;
    A[0] = 0.;
    for (int j = 1; j < nz; j++) A[j] = D.hx * D.hy / data_cpu::DZ[j - 1];
    if (D.FDmode) { A[1] *= 0.5; A[nz - 1] *= 0.5; }
    cudaMemcpyToSymbol(data_cuda::MAT_A, data_cpu::MAT_A, sizeof(double) * nz);
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

/* v -= grad(L^-1 div v) with the GPU object's own operators (flux[(l+1)%4] is the
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

/* `nsteps` steps of the reference's time loop (order ramped as main.cpp:409 does),
 * timed with CUDA events on the default stream; with_diag adds the loop's per-step
 * CalcIntegral, CalcVelocityProfile (+ the av_u copy) and CalcCFL (main.cpp:414-439). */
double refgpu_run(int nsteps, double tau, int with_diag, int* cur, int* it) {
    if (!g_gpu_ready) return -1.0;
    std::vector<real9> prof(D.NZ);
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
            volatile double fr = G.CalcIntegral(G.vel[*cur])[0];
            (void)fr;
            G.CalcVelocityProfile(G.vel[*cur]);
            cudaMemcpy(prof.data(), G.av_u, sizeof(real9) * D.NZ, cudaMemcpyDeviceToHost);
            volatile double cfl = G.CalcCFL(G.vel[*cur], (real)tau, 3);
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
}
