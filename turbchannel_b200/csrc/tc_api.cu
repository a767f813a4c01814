// tc_api.cu -- host orchestration and the C ABI (include/turbch.h).
//
// A tc_handle owns everything the reference's `struct data` owns
// (staggered/data_global_inc.h:11-76): the 4-level rings vel/flux/pres, nu_t, the
// spectrum buffer and the mesh-derived arrays, here on one CUDA device and one
// stream.  Fields are stored structure-of-arrays in the working precision; the
// boundary converts from/to the reference's AoS double layout.  One step is
// seven launches (eight with a Smagorinsky model):
//   flux+combine -> div+xFFT -> yFFT -> zsolve -> inverse yFFT -> inverse xFFT -> correction
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <random>
#include <string>
#include <initializer_list>
#include <utility>
#include <vector>

#include "../../include/turbch_les.h"
#include "kernels.cuh"
#include "mlp.cuh"

using namespace tc;

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
static thread_local std::string g_err;
static int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}
#define TC_CUDA(call)                                                                         \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) return fail(TC_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

extern "C" const char* tc_last_error(void) { return g_err.c_str(); }
extern "C" const char* tc_version(void) { return "turbchannel_b200 0.1 (sm_100a)"; }

// ---------------------------------------------------------------------------
// Mesh-derived data on the host (double).  Staggered: staggered/main.cpp:112-156
// (InitDerivativeMeshData) with FillMatrix (:12-48) and the banded elimination of
// :74-109 for the null vector of the VV4 gradient.  Collocated:
// collocated_AB3/main.cpp:238-300.
// ---------------------------------------------------------------------------
struct HostMesh {
    std::vector<double> ZZ, DZ, DZW, GC1, GC2, GCZ, KERG, MAT_A, cellh;
    double MAT_D[6] = {0, 0, 0, 0, 0, 0};
    double KERG_norm2 = 0;
};

static int banded_solve(int N, int NB, std::vector<double>& M, std::vector<double>& x, double tiny) {
    const int w = NB / 2;
    for (int i = 0; i < N; i++) {
        for (int j = -w; j < 0; j++) {
            if (i + j < 0) continue;
            const double mult = -M[i * NB + w + j];
            for (int k = 0; k <= w; k++) {
                if (i + j + k >= N) continue;
                M[i * NB + (w + j) + k] += mult * M[(i + j) * NB + w + k];
            }
            x[i] += mult * x[i + j];
        }
        if (std::fabs(M[i * NB + w]) < tiny) return 2;
        const double mult = 1.0 / M[i * NB + w];
        for (int k = 0; k <= w; k++)
            if (i + k < N) M[i * NB + w + k] *= mult;
        x[i] *= mult;
    }
    for (int i = N - 1; i >= 0; i--)
        for (int j = 1; j <= w; j++)
            if (i + j < N) x[i] -= M[i * NB + w + j] * x[i + j];
    return 0;
}

// 7-diagonal VV4 z-Laplacian of the xy-constant mode (div o grad with the 4-point
// stencils; symmetric reflections at the walls).
static void vv4_matrix(const HostMesh& hm, int NZ, std::vector<double>& M) {
    const double gc[4] = {1. / 27., -1., 1., -1. / 27.};
    M.assign((size_t)7 * NZ, 0.0);
    for (int j = 0; j < NZ; j++)
        for (int ll = -1; ll <= 2; ll++) {
            const double c1 = gc[ll + 1];
            int l = j + ll;
            if (l == 0 || l == NZ) continue;
            if (l < 0) l = -l;
            if (l > NZ) l = 2 * NZ - l;
            for (int mm = -2; mm <= 1; mm++) {
                double c2 = gc[mm + 2];
                int m = l + mm;
                if (m < 0) { m = -m - 1; c2 = -c2; }
                if (m >= NZ) { m = 2 * NZ - m - 1; c2 = -c2; }
                const int pos = m - j + 3;
                if (pos < 0 || pos >= 7) continue;
                M[j * 7 + pos] += c1 * c2 * hm.GCZ[l];
            }
        }
}

static int build_mesh(const tc_params& p, const double* zz, HostMesh& hm) {
    const int NZ = p.NZ;
    if (p.scheme == TC_SCHEME_COLLOC) {
        hm.ZZ.assign(zz, zz + NZ);
        hm.DZ.assign(NZ, 0.0);
        for (int i = 0; i < NZ - 1; i++) hm.DZ[i] = hm.ZZ[i + 1] - hm.ZZ[i];
        hm.MAT_A.assign(NZ, 0.0);
        for (int j = 1; j < NZ; j++) hm.MAT_A[j] = p.hx * p.hy / hm.DZ[j - 1];
        if (p.fd_mode) {
            hm.MAT_A[1] *= 0.5;
            hm.MAT_A[NZ - 1] *= 0.5;
        }
        hm.cellh.assign(NZ, 0.0);
        for (int iz = 0; iz < NZ; iz++)
            hm.cellh[iz] = iz == 0 ? 0.5 * hm.DZ[0] : iz == NZ - 1 ? 0.5 * hm.DZ[NZ - 2] : 0.5 * (hm.DZ[iz - 1] + hm.DZ[iz]);
        hm.DZW = hm.GC1 = hm.GC2 = hm.GCZ = hm.KERG = std::vector<double>(NZ, 0.0);
        return 0;
    }
    hm.ZZ.assign(zz, zz + NZ + 1);
    hm.DZ.assign(NZ, 0.0);
    for (int i = 0; i < NZ; i++) hm.DZ[i] = hm.ZZ[i + 1] - hm.ZZ[i];
    hm.cellh = hm.DZ;
    hm.DZW = hm.GC1 = hm.GC2 = hm.GCZ = hm.KERG = std::vector<double>(NZ, 0.0);
    if (p.scheme == TC_SCHEME_HW2) {
        hm.MAT_A.assign(NZ, 0.0);
        for (int j = 1; j <= NZ - 1; j++) hm.MAT_A[j] = 2. / (hm.DZ[j - 1] + hm.DZ[j]);
        return 0;
    }
    const std::vector<double>& DZ = hm.DZ;
    for (int iz = 0; iz < NZ; iz++) {
        hm.DZW[iz] = (DZ[iz] + DZ[iz == 0 ? iz : iz - 1] + DZ[iz == NZ - 1 ? iz : iz + 1]) / 3.;
        hm.GC1[iz] = DZ[iz] / (DZ[iz] - hm.DZW[iz] / 9.);
        hm.GC2[iz] = -(1. / 27.) * hm.DZW[iz] / (DZ[iz] - hm.DZW[iz] / 9.);
        hm.GCZ[iz] = iz == 0 ? 0.0  // no w-DOF on the bottom wall: never used
                             : 1 / (0.5 * (DZ[iz] + DZ[iz - 1]) -
                                    (1. / 27.) * (DZ[iz] + DZ[iz - 1] + 0.5 * (DZ[iz == NZ - 1 ? iz : iz + 1] + DZ[iz == 1 ? 0 : iz - 2])));
    }
    std::vector<double> M;
    vv4_matrix(hm, NZ, M);
    hm.MAT_A.assign((size_t)3 * NZ, 0.0);
    for (int iz = 0; iz < NZ; iz++)
        for (int i = 0; i < 3; i++) hm.MAT_A[iz * 3 + i] = (iz + i - 3 >= 0) ? M[iz * 7 + i] : 0.0;
    hm.MAT_D[0] = M[3];
    hm.MAT_D[1] = M[7 + 3];
    hm.MAT_D[2] = M[14 + 3];
    hm.MAT_D[3] = M[(NZ - 3) * 7 + 3];
    hm.MAT_D[4] = M[(NZ - 2) * 7 + 3];
    hm.MAT_D[5] = M[(NZ - 1) * 7 + 3];
    std::vector<double> T3((size_t)3 * NZ, 0.0), K(NZ, 1.0);
    const double eps = 1. / 27.;
    T3[1] = -1;
    T3[2] = eps;
    for (int iz = 1; iz < NZ - 1; iz++) {
        T3[iz * 3 + 0] = T3[iz * 3 + 2] = eps;
        T3[iz * 3 + 1] = -1 + eps;
    }
    T3[(NZ - 1) * 3] = eps;
    T3[(NZ - 1) * 3 + 1] = -1;
    if (banded_solve(NZ, 3, T3, K, 1e-10)) return 1;
    hm.KERG = K;
    hm.KERG_norm2 = 0;
    for (int iz = 0; iz < NZ; iz++) hm.KERG_norm2 += K[iz] * K[iz] * DZ[iz];
    return 0;
}

// ---------------------------------------------------------------------------
// The handle
// ---------------------------------------------------------------------------
static int plan_fft(int n, FftPlan& P) {
    P.n = n;
    P.nf = 0;
    int m = n;
    while (m % 4 == 0 && P.nf < FFT_MAXF) { P.fac[P.nf++] = 4; m /= 4; }
    while (m % 2 == 0 && P.nf < FFT_MAXF) { P.fac[P.nf++] = 2; m /= 2; }
    while (m % 3 == 0 && P.nf < FFT_MAXF) { P.fac[P.nf++] = 3; m /= 3; }
    return m == 1 ? 0 : 1;
}

struct tc_handle {
    tc_params prm;
    Geom g;
    HostMesh hm;
    cudaStream_t st = nullptr;
    cudaStream_t side = nullptr;  // low-wavenumber double solves of the mixed mode
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    bool fp64 = true;
    size_t esz = 8;
    void* vel[4] = {};
    void* flux[4] = {};
    // The flux ring's level l holds A_l = F_l + hist_it[l] v_l / 2 (sbdf_rhs in kernels.cuh):
    // hist_it[l] is the 1/tau (in the working precision) of the step that wrote it; 0 =
    // plain F (a new handle, a checkpoint of the first format).
    double hist_it[4] = {0.0, 0.0, 0.0, 0.0};
    bool hist_a = true;  // false: the step's flux kernel keeps plain F (k_flux_pair), hist_it stays 0
    void* pres[4] = {};
    void* nu_t = nullptr;
    void* ptmp = nullptr;
    void* spec = nullptr;
    void* zfac = nullptr;  // time-independent factors of the z-matrices (k_zfactor)
    void* zfac_low = nullptr;  // double factors of the low modes
    void* mesh_t = nullptr;     // mesh arrays in T
    void* fk = nullptr;         // flux kernels' interior-plane constants (float pairs mixed, doubles FP64 VV4)
    double* mesh_d = nullptr;   // mesh arrays in double
    double* tabs = nullptr;     // cos/sin tables
    void* tw = nullptr;         // twiddles (x then y), T complex
    FftPlan px{}, py{};
    double* red = nullptr;      // [0] ub_sum, [1] du, [2..] partials
    unsigned* ticket = nullptr;
    int* err_flag = nullptr;
    double* planes = nullptr;
    double* stats = nullptr;     // time-averaged profile sums (NZ x 12) and the total weight
    // tc_run_graph: the instantiated loop and the parameters it was captured for
    cudaGraph_t run_graph = nullptr;
    cudaGraphExec_t run_exec = nullptr;
    RunCtl* run_ctl = nullptr;
    double run_tau = 0.0;
    int run_cur = -1, run_every = 0, run_mode = 0;
    double* diag_part = nullptr;  // per-chunk partial sums of the diagnostics
    double* planes_h = nullptr;  // pinned
    double* stage = nullptr;     // AoS double staging (3N), lazily
    void* opv = nullptr;         // operator scratch (lazily): vector T
    void* opf = nullptr;
    void* ops = nullptr;         // scalar T
    int nblocks_flux = 0;
    int forcing_mode = 0;
    double forcing_value = 0;
    double last_tau = 0, last_bd0 = 1;
    int turb_kind = TC_TURB_NONE;
    float* mlp_params = nullptr;  // learned closure (TC_TURB_MLP): packed FP32 parameters
    // diagnostics fused into the step's correction (tc_set_diag_fusion)
    int diag_fuse = 0;             // 0 off (default), 1 always, 2 when the caller reads every step's diagnostics
    int mlp_fuse = 0;              // TC_TURB_MLP: 1 = closure evaluated inside the flux kernel (k_flux_mlp)
    int fft_plane = 1;             // 1 = x- and y-FFTs of a plane in one cluster kernel where the grid has one
    int flux_staging = 0;          // float pair flux kernel: 0 cp.async ring fill, 1 TMA tensor boxes
    bool diag_follow = false;      // mode 2: the last step's output level was read
    bool fused_valid = false, fused_used = false;
    int fused_level = -1, last_out = -1;
    double fused_tau = 0.0;
    double* fdiag_part = nullptr;  // NZ x correct_diag_chunks x TC_DIAG_STRIDE
    float* les_buf = nullptr;     // box-filter / feature scratch (tc_les_*), grown on demand
    size_t les_bytes = 0;
    // segregated IMEX Runge-Kutta step of the collocated scheme (tc_srk_init/tc_srk_step)
    struct Srk {
        int S = 0, type = 0, stab = 1;
        double BE[TC_SRK_MAX_STAGES * (TC_SRK_MAX_STAGES + 1)] = {}, BI[TC_SRK_MAX_STAGES * (TC_SRK_MAX_STAGES + 1)] = {};
        double d[TC_SRK_MAX_STAGES] = {}, alpha_tau = 0;
        void* buf = nullptr;  // one allocation: kuhat[S], bufv, nu1 (vectors); mujt[S], qj[S], bufs, pjhat, pj
    } srk;
    // instrumentation
    unsigned long long launches = 0;
    bool timing = false;
    std::vector<cudaEvent_t> ev;  // pool
    size_t ev_used = 0;
    int timed_steps = 0;
    double phase_ms[TC_NPHASE] = {};
};

// Phase markers of one step: slot k marks the end of phase k-1.
static void mark(tc_handle* h, int slot, size_t base) {
    if (!h->timing) return;
    const size_t idx = base + (size_t)slot;
    while (h->ev.size() <= idx) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        h->ev.push_back(e);
    }
    cudaEventRecord(h->ev[idx], h->st);
}

template <typename T>
static V3<T> vec(void* base, long long N) {
    T* b = (T*)base;
    return V3<T>{{b, b + N, b + 2 * N}};
}
template <typename T>
static CV3<T> cvec(void* base, long long N) {
    const T* b = (const T*)base;
    return CV3<T>{{b, b + N, b + 2 * N}};
}

template <typename T>
static MeshDev<T> mesh_dev(const tc_handle* h) {
    const int NZ = h->g.NZ, L = NZ + 2;
    const T* t = (const T*)h->mesh_t;
    const double* d = h->mesh_d;
    MeshDev<T> m;
    m.ZZ = t + 0 * L; m.DZ = t + 1 * L; m.DZW = t + 2 * L; m.GC1 = t + 3 * L; m.GC2 = t + 4 * L;
    m.GCZ = t + 5 * L; m.KERG = t + 6 * L; m.cellh = t + 7 * L; m.MAT_A = t + 8 * L; m.PC = t + 11 * L;
    m.FK = h->fp64 ? nullptr : (const float*)h->fk;
    m.FK64 = h->fp64 ? (const double*)h->fk : nullptr;
    m.dZZ = d + 0 * L; m.dDZ = d + 1 * L; m.dDZW = d + 2 * L; m.dKERG = d + 6 * L; m.dcellh = d + 7 * L;
    m.dMAT_A = d + 8 * L;
    for (int i = 0; i < 6; i++) m.MAT_D[i] = h->hm.MAT_D[i];
    m.KERG_norm2 = h->hm.KERG_norm2;
    return m;
}

static ModeTabs mode_tabs(const tc_handle* h) {
    ModeTabs t;
    const int NXH = h->g.NXH, NY = h->g.NY;
    t.cosx = h->tabs;
    t.cosy = h->tabs + NXH;
    t.sinx = h->tabs + NXH + NY;
    t.siny = h->tabs + 2 * NXH + NY;
    return t;
}

template <typename T>
static const cplx<T>* twx(const tc_handle* h) { return (const cplx<T>*)h->tw; }
template <typename T>
static const cplx<T>* twy(const tc_handle* h) { return (const cplx<T>*)h->tw + h->g.NX; }

static void free_all(tc_handle* h) {
    void* ptrs[] = {h->nu_t, h->ptmp, h->spec, h->zfac, h->zfac_low, h->mesh_t, h->fk, h->stats, h->mesh_d, h->tabs, h->tw, h->red, h->ticket,
                    h->err_flag, h->planes, h->diag_part, h->stage, h->opv, h->opf, h->ops, h->mlp_params, h->les_buf, h->fdiag_part,
                    h->srk.buf};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    for (int l = 0; l < 4; l++) {
        if (h->vel[l]) cudaFree(h->vel[l]);
        if (h->flux[l]) cudaFree(h->flux[l]);
        if (h->pres[l]) cudaFree(h->pres[l]);
    }
    if (h->planes_h) cudaFreeHost(h->planes_h);
    for (cudaEvent_t e : h->ev) cudaEventDestroy(e);
    h->ev.clear();
    if (h->ev_fork) cudaEventDestroy(h->ev_fork);
    if (h->ev_join) cudaEventDestroy(h->ev_join);
    if (h->side) cudaStreamDestroy(h->side);
    if (h->st) cudaStreamDestroy(h->st);
}

static bool is_23(int n) {
    if (n < 2) return false;
    while (n % 2 == 0) n /= 2;
    while (n % 3 == 0) n /= 3;
    return n == 1;
}

#define TC_ALLOC(ptr, bytes)                                                                        \
    do {                                                                                            \
        if (cudaMalloc((void**)&(ptr), (bytes)) != cudaSuccess) {                                   \
            cudaGetLastError();                                                                     \
            free_all(h);                                                                            \
            delete h;                                                                               \
            return fail(TC_E_NOMEM, "device allocation of " + std::to_string((size_t)(bytes)) + " bytes failed"); \
        }                                                                                           \
    } while (0)

// Per-plane reciprocals of the staggered stencils (layout in MeshDev::PC), computed in
// the working type T from the T-valued mesh (t: the mesh slots as uploaded).
template <typename T>
static void fill_plane_consts(const Geom& g, const HostMesh& hm, const T* t, T* pc) {
    const int NZ = g.NZ, L = NZ + 2;
    const T* DZ = t + 1 * L;
    const T* DZW = t + 2 * L;
    const T* GCZ = t + 5 * L;
    const T hx = (T)g.hx, hy = (T)g.hy, ihx = (T)g.inv_hx, ihy = (T)g.inv_hy;
    const T C9 = T(0.11111111111111111111);
    (void)hm;
    for (int z = 0; z < NZ; z++) {
        T* c = pc + (size_t)TC_PC * z;
        c[0] = T(1) / DZ[z];
        c[1] = T(2) / (DZ[z] + (z == 0 ? T(0) : DZ[z - 1]));
        c[2] = T(2) / (DZ[z] + (z == NZ - 1 ? T(0) : DZ[z + 1]));
        c[3] = z == 0 ? T(0) : T(1) / DZ[z - 1];
        c[4] = T(-1) / (32 * (DZ[z] - C9 * DZW[z]) * hx * hy);
        c[5] = -T(1. / 32.) * ihx * ihy * GCZ[z];
        c[6] = c[7] = T(0);
    }
}

// Constants of the flux kernels' interior VV4 planes (stencil_vv4_int.cuh: the float
// pair kernel stores each twice as a float2, the FP64 kernel once), from the double mesh:
// per plane z, with miv and w5 the VV4 momentum and w scales of PC[4], PC[5] and
// C27 = 1/27,
//   [0..5]   miv dz hy, -miv C27 dzw hy, miv dz hx, -miv C27 dzw hx, miv hx hy, -miv C27 hx hy
//   [6..9]   w5 hy, -w5 C27 hy, w5 hx hy, -w5 C27 hx hy
//   [10..13] -9 DZ[z], -9 DZ[z-1], DZ[z-2], DZ[z+1]; [14..17] the same of DZW
//   [18..21] visc (2/(DZ[z]+DZ[z+1])) / DZ[z], visc (2/(DZ[z]+DZ[z-1])) / DZ[z],
//            visc (2/(DZ[z]+DZ[z-1])) / DZ[z], visc (2/(DZ[z]+DZ[z-1])) / DZ[z-1]
//   [22..23] visc / hx^2, visc / hy^2
// (0 where an index leaves the mesh; those planes use the generic stencils).
static void fill_flux_plane_consts(const Geom& g, const HostMesh& hm, std::vector<double>& fk) {
    const int NZ = g.NZ;
    fk.assign((size_t)TC_FK64 * NZ, 0.0);
    const double hx = g.hx, hy = g.hy, nu = g.visc, C27 = 1.0 / 27.0;
    const std::vector<double>&DZ = hm.DZ, &DZW = hm.DZW, &GCZ = hm.GCZ;
    for (int z = 0; z < NZ; z++) {
        double k[24] = {0};
        const double miv = -1.0 / (32.0 * (DZ[z] - DZW[z] / 9.0) * hx * hy);
        const double w5 = -(1.0 / 32.0) * GCZ[z] / (hx * hy);
        k[0] = miv * DZ[z] * hy; k[1] = -miv * C27 * DZW[z] * hy;
        k[2] = miv * DZ[z] * hx; k[3] = -miv * C27 * DZW[z] * hx;
        k[4] = miv * hx * hy; k[5] = -miv * C27 * hx * hy;
        k[6] = w5 * hy; k[7] = -w5 * C27 * hy; k[8] = w5 * hx * hy; k[9] = -w5 * C27 * hx * hy;
        if (z >= 2 && z + 1 < NZ) {
            k[10] = -9.0 * DZ[z]; k[11] = -9.0 * DZ[z - 1]; k[12] = DZ[z - 2]; k[13] = DZ[z + 1];
            k[14] = -9.0 * DZW[z]; k[15] = -9.0 * DZW[z - 1]; k[16] = DZW[z - 2]; k[17] = DZW[z + 1];
        }
        if (z >= 1 && z + 1 < NZ) {
            const double up = 2.0 / (DZ[z] + DZ[z + 1]), dn = 2.0 / (DZ[z] + DZ[z - 1]);
            k[18] = nu * up / DZ[z]; k[19] = nu * dn / DZ[z];
            k[20] = nu * dn / DZ[z]; k[21] = nu * dn / DZ[z - 1];
        }
        k[22] = nu / (hx * hx); k[23] = nu / (hy * hy);
        for (int i = 0; i < TC_FK64; i++) fk[(size_t)TC_FK64 * z + i] = k[i];
    }
}

static int static_zscr(void** out);

extern "C" int tc_create(const tc_params* prm, const double* zz, tc_handle** out) {
    if (!prm || !zz || !out) return fail(TC_E_ARG, "tc_create: null argument");
    *out = nullptr;
    const tc_params& p = *prm;
    if (p.scheme < 0 || p.scheme > 2) return fail(TC_E_ARG, "tc_create: unknown scheme");
    if (p.precision != TC_FP64 && p.precision != TC_MIXED) return fail(TC_E_ARG, "tc_create: unknown precision");
    if (!is_23(p.NX) || !is_23(p.NY) || (p.NX & 1) || (p.NY & 1))
        return fail(TC_E_ARG, "tc_create: NX and NY must be even products of powers of 2 and 3");
    if (p.NX < 8 || p.NY < 8) return fail(TC_E_ARG, "tc_create: NX, NY must be >= 8");
    if (p.NZ < 6) return fail(TC_E_ARG, "tc_create: NZ must be >= 6");
    if (p.scheme != TC_SCHEME_COLLOC && p.visc_type == TC_VISC_GALERKIN)
        return fail(TC_E_ARG, "tc_create: Galerkin viscosity is collocated-only");
    if (p.scheme == TC_SCHEME_COLLOC && p.visc_type == TC_VISC_NAIVE)
        return fail(TC_E_ARG, "tc_create: NAIVE viscosity is staggered-only");
    if (p.turb_model != TC_TURB_NONE && p.visc_type == TC_VISC_CROSS)
        return fail(TC_E_ARG, "tc_create: a turbulence model needs NAIVE (staggered) or GALERKIN (collocated) viscosity");
    if (!(p.hx > 0) || !(p.hy > 0) || !(p.visc > 0) || !(p.area > 0)) return fail(TC_E_ARG, "tc_create: bad mesh steps");
    const int nzz = p.scheme == TC_SCHEME_COLLOC ? p.NZ : p.NZ + 1;
    for (int i = 0; i + 1 < nzz; i++)
        if (!(zz[i + 1] > zz[i])) return fail(TC_E_ARG, "tc_create: z coordinates must increase");
    int ndev = 0;
    TC_CUDA(cudaGetDeviceCount(&ndev));
    if (p.device < 0 || p.device >= ndev) return fail(TC_E_ARG, "tc_create: device id out of range");
    TC_CUDA(cudaSetDevice(p.device));

    tc_handle* h = new tc_handle();
    h->prm = p;
    if (build_mesh(p, zz, h->hm)) {
        delete h;
        return fail(TC_E_NUMERIC, "tc_create: singular system for the VV4 gradient null vector");
    }
    Geom& g = h->g;
    g.NX = p.NX; g.NY = p.NY; g.NZ = p.NZ; g.NXY = p.NX * p.NY;
    g.N = (long long)g.NXY * p.NZ;
    g.NXH = p.NX / 2 + 1;
    g.scheme = p.scheme; g.visc_type = p.visc_type; g.turb = p.turb_model; g.stab_type = p.stab_type; g.fd_mode = p.fd_mode;
    int lm = p.low_modes > 0 ? p.low_modes : 4;
    lm = std::min(lm, std::min(g.NXH, (p.NY + 1) / 2));
    g.low_modes = lm;
    g.visc = p.visc; g.sour_dpdx = p.sour_dpdx; g.inv_ls = p.inv_length_scale; g.hx = p.hx; g.hy = p.hy;
    g.inv_hx = 1. / p.hx; g.inv_hy = 1. / p.hy; g.area = p.area;
    h->fp64 = p.precision == TC_FP64;
    h->esz = h->fp64 ? 8 : 4;
    h->hist_a = h->fp64 || !flux_pair_covers(g);
    h->turb_kind = p.turb_model;
    if (plan_fft(p.NX, h->px) || plan_fft(p.NY, h->py)) {
        delete h;
        return fail(TC_E_ARG, "tc_create: FFT length not supported");
    }
    if (cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&h->side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming) != cudaSuccess) {
        free_all(h);
        delete h;
        return fail(TC_E_CUDA, "tc_create: stream creation failed");
    }
    {
        // loads the module holding tc_op_pressure_solve_static's scratch array on this
        // device now, so that array's memory is reserved before the caller's own pools
        void* scr = nullptr;
        if (static_zscr(&scr)) {
            const std::string msg = "tc_create: " + g_err;
            free_all(h);
            delete h;
            return fail(TC_E_CUDA, msg);
        }
    }
    if ((long long)3 * g.N >= 4294967296LL) {
        free_all(h);
        delete h;
        return fail(TC_E_ARG, "tc_create: grid too large (3 N must stay below 2^32)");
    }
    const size_t N = (size_t)g.N, E = h->esz;
    for (int l = 0; l < 4; l++) {
        TC_ALLOC(h->vel[l], 3 * N * E);
        TC_ALLOC(h->flux[l], 3 * N * E);
        TC_ALLOC(h->pres[l], N * E);
    }
    if (p.turb_model != TC_TURB_NONE) TC_ALLOC(h->nu_t, N * E);
    TC_ALLOC(h->ptmp, N * E);
    TC_ALLOC(h->spec, (size_t)g.NXH * g.NY * g.NZ * 2 * E);
    TC_ALLOC(h->zfac, zfactor_bytes(g, (int)E));
    TC_ALLOC(h->zfac_low, zfactor_low_bytes(g));
    // mesh arrays, 9 slots of NZ+2 (the last one holds MAT_A, up to 3 NZ entries), then
    // the per-plane reciprocals (TC_PC per plane)
    const int L = g.NZ + 2;
    const size_t mlen = (size_t)8 * L + 3 * (size_t)L + (size_t)TC_PC * L;
    TC_ALLOC(h->mesh_t, mlen * E);
    TC_ALLOC(h->mesh_d, mlen * sizeof(double));
    {
        std::vector<double> md(mlen, 0.0);
        const HostMesh& hm = h->hm;
        auto put = [&](int slot, const std::vector<double>& v) {
            for (size_t i = 0; i < v.size() && i < (size_t)(slot == 8 ? 3 * L : L); i++) md[(size_t)slot * L + i] = v[i];
        };
        put(0, hm.ZZ); put(1, hm.DZ); put(2, hm.DZW); put(3, hm.GC1); put(4, hm.GC2); put(5, hm.GCZ);
        put(6, hm.KERG); put(7, hm.cellh); put(8, hm.MAT_A);
        const size_t pc0 = (size_t)11 * L;
        fill_plane_consts<double>(g, hm, md.data(), md.data() + pc0);
        if (cudaMemcpy(h->mesh_d, md.data(), mlen * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
            free_all(h); delete h;
            return fail(TC_E_CUDA, "tc_create: mesh upload failed");
        }
        if (h->fp64) {
            cudaMemcpy(h->mesh_t, md.data(), mlen * sizeof(double), cudaMemcpyHostToDevice);
        } else {
            std::vector<float> mf(mlen);
            for (size_t i = 0; i < mlen; i++) mf[i] = (float)md[i];
            fill_plane_consts<float>(g, hm, mf.data(), mf.data() + pc0);
            cudaMemcpy(h->mesh_t, mf.data(), mlen * sizeof(float), cudaMemcpyHostToDevice);
            if (p.scheme != TC_SCHEME_COLLOC) {  // each constant twice: a float2 for the packed arithmetic
                std::vector<double> k;
                fill_flux_plane_consts(g, hm, k);
                std::vector<float> fk((size_t)TC_FK * g.NZ);
                for (size_t i = 0; i < k.size(); i++) fk[2 * i] = fk[2 * i + 1] = (float)k[i];
                TC_ALLOC(h->fk, fk.size() * sizeof(float));
                cudaMemcpy(h->fk, fk.data(), fk.size() * sizeof(float), cudaMemcpyHostToDevice);
            }
        }
        if (h->fp64 && p.scheme == TC_SCHEME_VV4) {
            std::vector<double> k;
            fill_flux_plane_consts(g, hm, k);
            TC_ALLOC(h->fk, k.size() * sizeof(double));
            cudaMemcpy(h->fk, k.data(), k.size() * sizeof(double), cudaMemcpyHostToDevice);
        }
    }
    // mode tables (staggered/func_global.h:208-211 cos tables; VV4 sin(pi k / N))
    {
        const double PI = 3.14159265358979323846;
        std::vector<double> tb(2 * g.NXH + 2 * g.NY);
        for (int i = 0; i < g.NXH; i++) tb[i] = std::cos(2. * PI * i / g.NX);
        for (int i = 0; i < g.NY; i++) tb[g.NXH + i] = std::cos(2. * PI * i / g.NY);
        for (int i = 0; i < g.NXH; i++) tb[g.NXH + g.NY + i] = std::sin(PI * i / g.NX);
        for (int i = 0; i < g.NY; i++) tb[2 * g.NXH + g.NY + i] = std::sin(PI * i / g.NY);
        TC_ALLOC(h->tabs, tb.size() * sizeof(double));
        cudaMemcpy(h->tabs, tb.data(), tb.size() * sizeof(double), cudaMemcpyHostToDevice);
    }
    // twiddles exp(-2 pi i k / n) for n = NX then NY
    {
        const size_t nt = (size_t)g.NX + g.NY;
        std::vector<double> tw(2 * nt);
        auto fill = [&](int n, size_t off) {
            for (int k = 0; k < n; k++) {
                long double a = -2.0L * 3.14159265358979323846264338327950288L * (long double)k / (long double)n;
                tw[2 * (off + k)] = (double)cosl(a);
                tw[2 * (off + k) + 1] = (double)sinl(a);
            }
        };
        fill(g.NX, 0);
        fill(g.NY, g.NX);
        TC_ALLOC(h->tw, 2 * nt * E);
        if (h->fp64) cudaMemcpy(h->tw, tw.data(), 2 * nt * 8, cudaMemcpyHostToDevice);
        else {
            std::vector<float> tf(2 * nt);
            for (size_t i = 0; i < 2 * nt; i++) tf[i] = (float)tw[i];
            cudaMemcpy(h->tw, tf.data(), 2 * nt * 4, cudaMemcpyHostToDevice);
        }
    }
    h->nblocks_flux = flux_grid_blocks(g);
    TC_ALLOC(h->red, (size_t)(2 + h->nblocks_flux) * sizeof(double));
    TC_ALLOC(h->ticket, sizeof(unsigned));
    TC_ALLOC(h->err_flag, sizeof(int));
    TC_ALLOC(h->planes, (size_t)g.NZ * TC_DIAG_STRIDE * sizeof(double));
    TC_ALLOC(h->stats, ((size_t)g.NZ * 12 + 1) * sizeof(double));
    cudaMemset(h->stats, 0, ((size_t)g.NZ * 12 + 1) * sizeof(double));
    TC_ALLOC(h->diag_part, (size_t)g.NZ * diag_chunks(g) * TC_DIAG_STRIDE * sizeof(double));
    if (cudaMallocHost((void**)&h->planes_h, (size_t)g.NZ * TC_DIAG_STRIDE * sizeof(double)) != cudaSuccess) {
        free_all(h); delete h;
        return fail(TC_E_NOMEM, "tc_create: pinned host allocation failed");
    }
    cudaMemsetAsync(h->ticket, 0, sizeof(unsigned), h->st);
    cudaMemsetAsync(h->err_flag, 0, sizeof(int), h->st);
    cudaMemsetAsync(h->red, 0, (size_t)(2 + h->nblocks_flux) * sizeof(double), h->st);
    for (int l = 0; l < 4; l++) {
        cudaMemsetAsync(h->vel[l], 0, 3 * N * E, h->st);
        cudaMemsetAsync(h->flux[l], 0, 3 * N * E, h->st);
        cudaMemsetAsync(h->pres[l], 0, N * E, h->st);
    }
    if (h->nu_t) cudaMemsetAsync(h->nu_t, 0, N * E, h->st);
    cudaMemsetAsync(h->zfac, 0, zfactor_bytes(g, (int)E), h->st);
    cudaMemsetAsync(h->zfac_low, 0, zfactor_low_bytes(g), h->st);
    if (h->fp64) {
        ZSolveArgs<double> za{g, mesh_dev<double>(h), mode_tabs(h), (cplx<double>*)h->spec, nullptr, h->err_flag, h->zfac,
                              h->zfac_low};
        launch_zfactor<double>(za, h->st);
    } else {
        ZSolveArgs<float> za{g, mesh_dev<float>(h), mode_tabs(h), (cplx<float>*)h->spec, nullptr, h->err_flag, h->zfac,
                             h->zfac_low};
        launch_zfactor<float>(za, h->st);
    }
    cudaError_t e = cudaStreamSynchronize(h->st);
    if (e != cudaSuccess) {
        free_all(h); delete h;
        return fail(TC_E_CUDA, std::string("tc_create: ") + cudaGetErrorString(e));
    }
    *out = h;
    return TC_OK;
}

extern "C" int tc_destroy(tc_handle* h) {
    if (!h) return TC_OK;
    cudaSetDevice(h->prm.device);
    cudaStreamSynchronize(h->st);
    if (h->run_exec) cudaGraphExecDestroy(h->run_exec);
    if (h->run_graph) cudaGraphDestroy(h->run_graph);
    if (h->run_ctl) cudaFree(h->run_ctl);
    free_all(h);
    delete h;
    return TC_OK;
}

static int check_launch(const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(TC_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return TC_OK;
}

static int ensure_stage(tc_handle* h) {
    if (!h->stage && cudaMalloc((void**)&h->stage, 3 * (size_t)h->g.N * sizeof(double)) != cudaSuccess) {
        cudaGetLastError();
        return fail(TC_E_NOMEM, "staging allocation failed");
    }
    return TC_OK;
}
static int ensure_ops(tc_handle* h) {
    const size_t N = (size_t)h->g.N, E = h->esz;
    if (!h->opv && cudaMalloc(&h->opv, 3 * N * E) != cudaSuccess) return fail(TC_E_NOMEM, "operator scratch");
    if (!h->opf && cudaMalloc(&h->opf, 3 * N * E) != cudaSuccess) return fail(TC_E_NOMEM, "operator scratch");
    if (!h->ops && cudaMalloc(&h->ops, N * E) != cudaSuccess) return fail(TC_E_NOMEM, "operator scratch");
    return TC_OK;
}

// ---- host <-> device transfers of AoS double data ----
template <typename T>
static int up_vec(tc_handle* h, const double* src, void* dst) {
    int rc = ensure_stage(h);
    if (rc) return rc;
    const long long N = h->g.N;
    TC_CUDA(cudaMemcpyAsync(h->stage, src, 3 * (size_t)N * sizeof(double), cudaMemcpyHostToDevice, h->st));
    launch_aos_to_soa<T>(h->stage, vec<T>(dst, N), N, h->st);
    return check_launch("aos_to_soa");
}
template <typename T>
static int up_scal(tc_handle* h, const double* src, void* dst) {
    int rc = ensure_stage(h);
    if (rc) return rc;
    const long long N = h->g.N;
    TC_CUDA(cudaMemcpyAsync(h->stage, src, (size_t)N * sizeof(double), cudaMemcpyHostToDevice, h->st));
    launch_d2t<T>(h->stage, (T*)dst, N, h->st);
    return check_launch("d2t");
}
template <typename T>
static int down_vec(tc_handle* h, const void* src, double* dst) {
    int rc = ensure_stage(h);
    if (rc) return rc;
    const long long N = h->g.N;
    launch_soa_to_aos<T>(cvec<T>((void*)src, N), h->stage, N, h->st);
    TC_CUDA(cudaMemcpyAsync(dst, h->stage, 3 * (size_t)N * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    TC_CUDA(cudaStreamSynchronize(h->st));
    return TC_OK;
}
template <typename T>
static int down_scal(tc_handle* h, const void* src, double* dst) {
    int rc = ensure_stage(h);
    if (rc) return rc;
    const long long N = h->g.N;
    launch_t2d<T>((const T*)src, h->stage, N, h->st);
    TC_CUDA(cudaMemcpyAsync(dst, h->stage, (size_t)N * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    TC_CUDA(cudaStreamSynchronize(h->st));
    return TC_OK;
}

#define TC_DISPATCH(h, fn, ...) ((h)->fp64 ? fn<double>(__VA_ARGS__) : fn<float>(__VA_ARGS__))

// Brings flux level l to A_l = F_l + it v_l / 2 (one pass, only when the step's 1/tau
// differs from the one the level was written with: the reference restarts the BDF
// order after a change of tau, so a continuing order meets this only after a checkpoint
// of the first format or a caller that changes tau without restarting).
template <typename T>
static void rebase_hist(tc_handle* h, int l, double it) {
    if (!h->hist_a) it = 0.0;
    if (h->hist_it[l] == it) return;
    LinComb<T> lc{};
    lc.out = (T*)h->flux[l];
    lc.x[0] = (const T*)h->flux[l];
    lc.c[0] = 1.0;
    lc.x[1] = (const T*)h->vel[l];
    lc.c[1] = 0.5 * (it - h->hist_it[l]);
    lc.post = 1.0;
    lc.nt = 2;
    lc.n = 3 * h->g.N;
    launch_lincomb<T>(lc, h->st);
    h->launches += 1;
    h->hist_it[l] = it;
}

// Before a caller may change v_l (upload, zero-copy pointers, a new initial field), flux
// level l goes back to plain F_l, so the history means what the reference's would.
static void hist_plain(tc_handle* h, int l) {
    if (h->hist_it[l] == 0.0) return;
    if (h->fp64) rebase_hist<double>(h, l, 0.0);
    else rebase_hist<float>(h, l, 0.0);
}

extern "C" int tc_upload_level(tc_handle* h, int level, const double* vel, const double* p) {
    if (!h || level < 0 || level > 3) return fail(TC_E_ARG, "tc_upload_level: bad handle or level");
    if (h) h->fused_valid = false;
    cudaSetDevice(h->prm.device);
    int rc = TC_OK;
    if (vel) hist_plain(h, level);
    if (vel) rc = TC_DISPATCH(h, up_vec, h, vel, h->vel[level]);
    if (!rc && p) rc = TC_DISPATCH(h, up_scal, h, p, h->pres[level]);
    if (!rc) TC_CUDA(cudaStreamSynchronize(h->st));
    return rc;
}
extern "C" int tc_download_level(tc_handle* h, int level, double* vel, double* p) {
    if (!h || level < 0 || level > 3) return fail(TC_E_ARG, "tc_download_level: bad handle or level");
    cudaSetDevice(h->prm.device);
    int rc = TC_OK;
    if (vel) rc = TC_DISPATCH(h, down_vec, h, h->vel[level], vel);
    if (!rc && p) rc = TC_DISPATCH(h, down_scal, h, h->pres[level], p);
    return rc;
}
extern "C" int tc_download_flux(tc_handle* h, int level, double* f) {
    if (!h || level < 0 || level > 3 || !f) return fail(TC_E_ARG, "tc_download_flux: bad argument");
    cudaSetDevice(h->prm.device);
    int rc = TC_DISPATCH(h, down_vec, h, h->flux[level], f);
    if (rc || h->hist_it[level] == 0.0) return rc;
    // the reference's F_l = A_l - v_l / (2 tau)
    const size_t n = 3 * (size_t)h->g.N;
    std::vector<double> v(n);
    rc = TC_DISPATCH(h, down_vec, h, h->vel[level], v.data());
    if (rc) return rc;
    const double c = 0.5 * h->hist_it[level];
    for (size_t i = 0; i < n; i++) f[i] -= c * v[i];
    return TC_OK;
}
extern "C" int tc_device_level(tc_handle* h, int level, void** vel, void** p) {
    if (h) h->fused_valid = false;  // the caller may write the level
    if (!h || level < 0 || level > 3) return fail(TC_E_ARG, "tc_device_level: bad handle or level");
    if (vel) {
        cudaSetDevice(h->prm.device);
        hist_plain(h, level);
    }
    if (vel) *vel = h->vel[level];
    if (p) *p = h->pres[level];
    return TC_OK;
}
extern "C" int tc_get_stream(tc_handle* h, void** s) {
    if (!h || !s) return fail(TC_E_ARG, "tc_get_stream: null argument");
    *s = (void*)h->st;
    return TC_OK;
}
extern "C" int tc_sync(tc_handle* h) {
    if (!h) return fail(TC_E_ARG, "tc_sync: null handle");
    cudaSetDevice(h->prm.device);
    TC_CUDA(cudaStreamSynchronize(h->st));
    int flag = 0;
    TC_CUDA(cudaMemcpy(&flag, h->err_flag, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag) {
        cudaMemset(h->err_flag, 0, sizeof(int));
        if (flag == 2) return fail(TC_E_CUDA, "flux kernel: a TMA tile load did not complete (bounded wait gave up)");
        return fail(TC_E_NUMERIC, "banded pressure solve met a vanishing pivot");
    }
    return TC_OK;
}
extern "C" int tc_set_nu_t(tc_handle* h, const double* nt) {
    if (h) h->fused_valid = false;
    if (!h || !nt) return fail(TC_E_ARG, "tc_set_nu_t: null argument");
    if (!h->nu_t) return fail(TC_E_STATE, "tc_set_nu_t: no turbulence model configured");
    cudaSetDevice(h->prm.device);
    int rc = TC_DISPATCH(h, up_scal, h, nt, h->nu_t);
    if (!rc) TC_CUDA(cudaStreamSynchronize(h->st));
    return rc;
}
extern "C" int tc_get_nu_t(tc_handle* h, double* nt) {
    if (!h || !nt) return fail(TC_E_ARG, "tc_get_nu_t: null argument");
    if (!h->nu_t) {
        memset(nt, 0, sizeof(double) * (size_t)h->g.N);
        return TC_OK;
    }
    cudaSetDevice(h->prm.device);
    return TC_DISPATCH(h, down_scal, h, h->nu_t, nt);
}

// ---------------------------------------------------------------------------
// Pressure solve pipeline: RHS (vector, divergence taken) or scalar -> p
// ---------------------------------------------------------------------------
template <typename T>
static void poisson(tc_handle* h, const void* rhs_vec, const void* rhs_scalar, void* p_out, size_t eb = (size_t)-1) {
    const bool mk = eb != (size_t)-1;
    const Geom& g = h->g;
    DivFftArgs<T> da;
    da.g = g;
    da.m = mesh_dev<T>(h);
    da.v = rhs_vec ? cvec<T>((void*)rhs_vec, g.N) : CV3<T>{{nullptr, nullptr, nullptr}};
    da.src_scalar = (const T*)rhs_scalar;
    da.spec = (cplx<T>*)h->spec;
    da.px = h->px;
    da.twx = twx<T>(h);
    da.dtmp = (T*)p_out;
    // plane kernels (x- and y-FFT of a plane in one launch) where the grid has them: the
    // forward pair is timed as the x-FFT phase, the inverse pair as the inverse x-FFT phase
    const bool plane = h->fft_plane && plane_fft_ok<T>(g);
    int ndx = plane ? launch_div_xyfft_plane<T>(da, twy<T>(h), h->st) : 0;
    const bool pf = ndx > 0;
    if (!pf) ndx = launch_div_xfft<T>(da, h->st);
    if (mk) mark(h, 3, eb);
    YFftArgs<T> ya{g, (cplx<T>*)h->spec, h->py, twy<T>(h), -1};
    if (!pf) launch_yfft<T>(ya, h->st);
    if (mk) mark(h, 4, eb);
    ZSolveArgs<T> za{g, mesh_dev<T>(h), mode_tabs(h), (cplx<T>*)h->spec, nullptr, h->err_flag, h->zfac, h->zfac_low};
    launch_zsolve_fac<T>(za, h->st, h->side, h->ev_fork, h->ev_join);
    if (mk) mark(h, 5, eb);
    ya.sign = +1;
    if (!plane) launch_yfft<T>(ya, h->st);
    if (mk) mark(h, 6, eb);
    IxFftArgs<T> ia{g, (const cplx<T>*)h->spec, (T*)p_out, h->px, twx<T>(h), (T)(1.0 / ((double)g.NX * g.NY))};
    if (!(plane && launch_ixyfft_plane<T>(ia, twy<T>(h), h->st))) launch_ixfft<T>(ia, h->st);
    if (mk) mark(h, 7, eb);
    h->launches += ndx + (pf ? 0 : 1) + 2 + (plane ? 1 : 2);
}

template <typename T>
static void turb_visc(tc_handle* h, const void* v) {
    TurbArgs<T> ta{h->g, mesh_dev<T>(h), cvec<T>((void*)v, h->g.N), (T*)h->nu_t};
    if (h->turb_kind == TC_TURB_MLP) launch_turb_mlp<T>(ta, h->mlp_params, h->st);
    else launch_turb<T>(ta, h->st);
}

template <typename T>
static int step_impl(tc_handle* h, double tau, int cur, int order) {
    const Geom& g = h->g;
    const long long N = g.N;
    const int nxt = (cur + 1) % 4, prv = (cur + 3) % 4, pr2 = (cur + 2) % 4;
    const T inv_tau = (T)(1. / tau);
    const T bd0 = order == 3 ? (T)(1.5 + 0.33333333333333333333) : order == 2 ? (T)1.5 : (T)1.0;
    const T tob = (T)(tau / bd0);
    const bool coll = g.scheme == TC_SCHEME_COLLOC;
    const bool stab1 = coll && g.stab_type == 1;
    const bool les = h->nu_t && (h->turb_kind == TC_TURB_SMAGORINSKY || h->turb_kind == TC_TURB_MLP);
    const bool mlp_in_flux = les && h->turb_kind == TC_TURB_MLP && h->mlp_fuse && !coll;
    const size_t eb = h->ev_used;
    mark(h, 0, eb);
    if (les && !mlp_in_flux) {
        turb_visc<T>(h, h->vel[cur]);
        h->launches += 1;
    }
    mark(h, 1, eb);
    FluxArgs<T> fa;
    fa.g = g;
    fa.m = mesh_dev<T>(h);
    fa.vel = cvec<T>(h->vel[cur], N);
    fa.velp = cvec<T>(h->vel[prv], N);
    fa.velq = cvec<T>(h->vel[pr2], N);
    fa.fp = cvec<T>(h->flux[prv], N);
    fa.fq = cvec<T>(h->flux[pr2], N);
    fa.fout = vec<T>(h->flux[cur], N);
    fa.rhs = vec<T>(h->flux[nxt], N);
    fa.nu_t = (h->nu_t && h->turb_kind != TC_TURB_NONE) ? (const T*)h->nu_t : nullptr;
    fa.pcur = stab1 ? (const T*)h->pres[cur] : nullptr;
    fa.inv_tau = inv_tau;
    fa.order = order;
    const bool cfr = h->forcing_mode == 1;
    fa.ub_partial = h->red + 2;
    fa.ticket = h->ticket;
    fa.ub_out = cfr ? h->red : nullptr;
    fa.err_flag = h->err_flag;
    fa.staging = h->flux_staging;
    const double itd = (double)inv_tau;
    if (order >= 2) rebase_hist<T>(h, prv, itd);
    if (order == 3) rebase_hist<T>(h, pr2, itd);
    if (coll) launch_flux_coll<T>(fa, h->st);
    else if (mlp_in_flux) launch_flux_mlp<T>(fa, h->mlp_params, (T*)h->nu_t, h->st);
    else launch_flux_stag<T>(fa, h->st);
    h->hist_it[cur] = h->hist_a ? itd : 0.0;
    h->hist_it[nxt] = 0.0;  // that level now holds the right-hand side (the reference's flux[next]), not an A
    h->launches += 1;
    mark(h, 2, eb);
    void* pdest = stab1 ? h->ptmp : h->pres[nxt];
    poisson<T>(h, h->flux[nxt], nullptr, pdest, eb);
    CorrArgs<T> ca;
    ca.g = g;
    ca.m = mesh_dev<T>(h);
    ca.rhs = cvec<T>(h->flux[nxt], N);
    ca.p = (const T*)pdest;
    ca.vout = vec<T>(h->vel[nxt], N);
    ca.pcur = stab1 ? (const T*)h->pres[cur] : nullptr;
    ca.pnext = stab1 ? (T*)h->pres[nxt] : nullptr;
    ca.tob = tob;
    ca.cfr = cfr ? 1 : 0;
    ca.cfr_target = h->forcing_value;
    ca.cfr_scale = g.hx * g.hy / g.area;
    double vf = g.area;
    if (coll) {
        double s = 0;
        for (int iz = 1; iz < g.NZ - 1; iz++) s += h->hm.cellh[iz];
        vf = s * g.hx * g.hy * g.NXY;
    }
    ca.cfr_volfac = g.area / vf;
    ca.ub_sum = h->red;
    ca.du_out = h->red + 1;
    ca.grad_only = 0;
    // the new level's diagnostics fused into the correction: forced, or (mode 2) while the
    // caller reads every step's diagnostics (the previous fused result was consumed)
    if (h->fused_valid && !h->fused_used) h->diag_follow = false;
    h->fused_valid = false;
    bool fuse = !coll && g.NX % 4 == 0 && (h->diag_fuse == 1 || (h->diag_fuse == 2 && h->diag_follow));
    if (fuse && !h->fdiag_part) {
        const size_t need = (size_t)g.NZ * correct_diag_chunks(g) * TC_DIAG_STRIDE * sizeof(double);
        if (cudaMalloc((void**)&h->fdiag_part, need) != cudaSuccess) {
            cudaGetLastError();
            h->fdiag_part = nullptr;
            fuse = false;
        }
    }
    if (fuse) {
        ca.dpart = h->fdiag_part;
        ca.nu_t = (h->nu_t && h->turb_kind != TC_TURB_NONE) ? (const T*)h->nu_t : nullptr;
        ca.dtau = tau;
        ca.dkv = g.visc_type != TC_VISC_CROSS ? 2.0 : 1.0;
    }
    launch_correct<T>(ca, h->st);
    h->launches += 1;
    if (fuse) {
        h->fused_valid = true;
        h->fused_used = false;
        h->fused_level = nxt;
        h->fused_tau = tau;
    }
    h->last_out = nxt;
    mark(h, 8, eb);
    if (h->timing) {
        h->ev_used += 9;
        h->timed_steps += 1;
    }
    h->last_tau = tau;
    h->last_bd0 = (double)bd0;
    return check_launch("tc_step");
}

extern "C" int tc_step(tc_handle* h, double t, double tau, int current_field, int bdf_order) {
    (void)t;
    if (!h) return fail(TC_E_ARG, "tc_step: null handle");
    if (bdf_order < 1 || bdf_order > 3) return fail(TC_E_ARG, "tc_step: wrong bdf_order");
    if (current_field < 0 || current_field > 3) return fail(TC_E_ARG, "tc_step: current_field out of range");
    if (!(tau > 0) || !std::isfinite(tau)) return fail(TC_E_ARG, "tc_step: tau must be positive");
    cudaSetDevice(h->prm.device);
    return TC_DISPATCH(h, step_impl, h, tau, current_field, bdf_order);
}

extern "C" int tc_phase_timing(tc_handle* h, int enable) {
    if (!h) return fail(TC_E_ARG, "tc_phase_timing: null handle");
    h->timing = enable != 0;
    return TC_OK;
}

extern "C" int tc_phase_times(tc_handle* h, double ms[TC_NPHASE], int* nsteps) {
    if (!h || !ms) return fail(TC_E_ARG, "tc_phase_times: null argument");
    cudaSetDevice(h->prm.device);
    TC_CUDA(cudaStreamSynchronize(h->st));
    double acc[TC_NPHASE] = {};
    for (int s = 0; s < h->timed_steps; s++)
        for (int k = 0; k < TC_NPHASE; k++) {
            float t = 0;
            TC_CUDA(cudaEventElapsedTime(&t, h->ev[(size_t)s * 9 + k], h->ev[(size_t)s * 9 + k + 1]));
            acc[k] += t;
        }
    for (int k = 0; k < TC_NPHASE; k++) ms[k] = acc[k];
    if (nsteps) *nsteps = h->timed_steps;
    h->timed_steps = 0;
    h->ev_used = 0;
    return TC_OK;
}

extern "C" int tc_launch_count(tc_handle* h, unsigned long long* n) {
    if (!h || !n) return fail(TC_E_ARG, "tc_launch_count: null argument");
    *n = h->launches;
    return TC_OK;
}

extern "C" int tc_set_forcing(tc_handle* h, int mode, double value) {
    if (!h || (mode != 0 && mode != 1)) return fail(TC_E_ARG, "tc_set_forcing: bad argument");
    h->forcing_mode = mode;
    if (mode == 0) {
        h->prm.sour_dpdx = value;
        h->g.sour_dpdx = value;
    } else {
        h->forcing_value = value;
    }
    return TC_OK;
}

extern "C" int tc_last_dpdx(tc_handle* h, double* dpdx) {
    if (!h || !dpdx) return fail(TC_E_ARG, "tc_last_dpdx: null argument");
    cudaSetDevice(h->prm.device);
    TC_CUDA(cudaStreamSynchronize(h->st));
    double du = 0;
    if (h->forcing_mode == 1) TC_CUDA(cudaMemcpy(&du, h->red + 1, sizeof(double), cudaMemcpyDeviceToHost));
    *dpdx = h->g.sour_dpdx + (h->last_tau > 0 ? du * h->last_bd0 / h->last_tau : 0.0);
    return TC_OK;
}

extern "C" int tc_set_turb_model(tc_handle* h, int kind, const void* weights) {
    if (!h) return fail(TC_E_ARG, "tc_set_turb_model: null handle");
    h->fused_valid = false;
    if (kind == TC_TURB_NONE) {
        h->turb_kind = kind;
        return TC_OK;
    }
    if (kind != TC_TURB_SMAGORINSKY && kind != TC_TURB_MLP) return fail(TC_E_ARG, "tc_set_turb_model: unknown model");
    if (h->g.visc_type == TC_VISC_CROSS) return fail(TC_E_ARG, "tc_set_turb_model: CROSS viscosity has no nu_t");
    cudaSetDevice(h->prm.device);
    if (kind == TC_TURB_MLP) {
        if (!weights) return fail(TC_E_ARG, "tc_set_turb_model: TC_TURB_MLP needs TC_MLP_NPAR float parameters");
        if (!h->mlp_params && cudaMalloc(&h->mlp_params, MLP_NPAR * sizeof(float)) != cudaSuccess)
            return fail(TC_E_NOMEM, "closure parameters");
        TC_CUDA(cudaMemcpy(h->mlp_params, weights, MLP_NPAR * sizeof(float), cudaMemcpyHostToDevice));
    }
    if (!h->nu_t) {
        if (cudaMalloc(&h->nu_t, (size_t)h->g.N * h->esz) != cudaSuccess) return fail(TC_E_NOMEM, "nu_t allocation");
        cudaMemsetAsync(h->nu_t, 0, (size_t)h->g.N * h->esz, h->st);
    }
    h->turb_kind = kind;
    h->g.turb = kind;
    return TC_OK;
}

// ---------------------------------------------------------------------------
// Diagnostics
// ---------------------------------------------------------------------------
template <typename T>
static int diag_run(tc_handle* h, int level, double tau) {
    if (h->fused_valid && level == h->fused_level && tau == h->fused_tau) {
        launch_diag_finish(h->fdiag_part, h->planes, h->g.NZ, correct_diag_chunks(h->g), h->st);
        h->fused_used = true;
        TC_CUDA(cudaGetLastError());
        TC_CUDA(cudaMemcpyAsync(h->planes_h, h->planes, (size_t)h->g.NZ * TC_DIAG_STRIDE * sizeof(double),
                                cudaMemcpyDeviceToHost, h->st));
        TC_CUDA(cudaStreamSynchronize(h->st));
        return TC_OK;
    }
    if (h->diag_fuse == 2 && level == h->last_out) h->diag_follow = true;
    DiagArgs<T> a;
    a.g = h->g;
    a.m = mesh_dev<T>(h);
    a.v = cvec<T>(h->vel[level], h->g.N);
    a.p = (const T*)h->pres[level];
    a.nu_t = (h->nu_t && h->turb_kind != TC_TURB_NONE) ? (const T*)h->nu_t : nullptr;
    a.tau = tau;
    a.planes = h->planes;
    a.part = h->diag_part;
    launch_diag<T>(a, h->st);
    TC_CUDA(cudaGetLastError());
    TC_CUDA(cudaMemcpyAsync(h->planes_h, h->planes, (size_t)h->g.NZ * TC_DIAG_STRIDE * sizeof(double),
                            cudaMemcpyDeviceToHost, h->st));
    TC_CUDA(cudaStreamSynchronize(h->st));
    return TC_OK;
}

// The diagnostics pass into h->planes without the copy to the host (time averaging).
template <typename T>
static int diag_device(tc_handle* h, int level) {
    if (h->fused_valid && level == h->fused_level) {
        launch_diag_finish(h->fdiag_part, h->planes, h->g.NZ, correct_diag_chunks(h->g), h->st);
        h->fused_used = true;
    } else {
        DiagArgs<T> a;
        a.g = h->g;
        a.m = mesh_dev<T>(h);
        a.v = cvec<T>(h->vel[level], h->g.N);
        a.p = (const T*)h->pres[level];
        a.nu_t = (h->nu_t && h->turb_kind != TC_TURB_NONE) ? (const T*)h->nu_t : nullptr;
        a.tau = 0.0;
        a.planes = h->planes;
        a.part = h->diag_part;
        launch_diag<T>(a, h->st);
    }
    TC_CUDA(cudaGetLastError());
    return TC_OK;
}

static void reduce_planes(const tc_handle* h, double integral[3], double* ke, double cfl[3], double* prof) {
    const Geom& g = h->g;
    const bool coll = g.scheme == TC_SCHEME_COLLOC;
    double I0 = 0, I1 = 0, I2 = 0, K = 0, c1 = 0, c2 = 0, c3 = 0;
    for (int z = 0; z < g.NZ; z++) {
        const double* s = h->planes_h + (size_t)z * TC_DIAG_STRIDE;
        const double wu = coll ? h->hm.cellh[z] : h->hm.DZ[z];
        const double ww = coll ? h->hm.cellh[z] : (z == 0 ? 0.0 : 0.5 * (h->hm.DZ[z] + h->hm.DZ[z - 1]));
        I0 += s[0] * wu;
        I1 += s[1] * wu;
        I2 += s[12] * ww;
        K += (s[3] + s[4]) * wu + s[13] * ww;
        c1 = std::max(c1, s[16]);
        c2 = std::max(c2, s[17]);
        c3 = std::max(c3, s[18]);
        if (prof)
            for (int k = 0; k < 12; k++) prof[z * 12 + k] = s[k] / g.NXY;
    }
    const double hxy = g.hx * g.hy;
    if (integral) {
        integral[0] = I0 * hxy;
        integral[1] = I1 * hxy;
        integral[2] = I2 * hxy;
    }
    if (ke) *ke = 0.5 * K * hxy;
    if (cfl) {
        cfl[0] = c1;
        cfl[1] = c2;
        cfl[2] = c3;
    }
}

// The plane sums of the diagnostics pass add every u, v, w, p (and nu_t) of the level,
// so a NaN or Inf anywhere in it makes one of them non-finite (the CFL maxima use fmax,
// which skips NaN, so they are not enough).  The outputs are still written.
static int check_planes_finite(const tc_handle* h, const char* who) {
    static const char* const names[NDIAG_SUMS] = {"sum u", "sum v", "sum w", "sum uu", "sum vv", "sum ww",
                                                  "sum uv", "sum uw", "sum vw", "sum nu_t", "sum p", "sum pp",
                                                  "sum w (raw)", "sum ww (raw)", "", ""};
    for (int z = 0; z < h->g.NZ; z++) {
        const double* s = h->planes_h + (size_t)z * TC_DIAG_STRIDE;
        for (int k = 0; k < NDIAG_SUMS; k++)
            if (!std::isfinite(s[k]))
                return fail(TC_E_NUMERIC, std::string(who) + ": non-finite value in the level (plane z = " +
                                              std::to_string(z) + ", " + names[k] + " = " + std::to_string(s[k]) + ")");
    }
    return TC_OK;
}

extern "C" int tc_diagnostics(tc_handle* h, int level, double tau, double integral[3], double* cfl, double* profiles) {
    if (!h || level < 0 || level > 3) return fail(TC_E_ARG, "tc_diagnostics: bad handle or level");
    cudaSetDevice(h->prm.device);
    int rc = TC_DISPATCH(h, diag_run, h, level, tau);
    if (rc) return rc;
    double c[3];
    reduce_planes(h, integral, nullptr, c, profiles);
    if (cfl) *cfl = c[2];
    return check_planes_finite(h, "tc_diagnostics");
}
extern "C" int tc_integral(tc_handle* h, int level, double out[3]) {
    return tc_diagnostics(h, level, 0.0, out, nullptr, nullptr);
}
extern "C" int tc_kinetic_energy(tc_handle* h, int level, double* out) {
    if (!h || !out || level < 0 || level > 3) return fail(TC_E_ARG, "tc_kinetic_energy: bad argument");
    cudaSetDevice(h->prm.device);
    int rc = TC_DISPATCH(h, diag_run, h, level, 0.0);
    if (rc) return rc;
    reduce_planes(h, nullptr, out, nullptr, nullptr);
    return check_planes_finite(h, "tc_kinetic_energy");
}
extern "C" int tc_cfl(tc_handle* h, int level, double tau, int mode, double* out) {
    if (!h || !out || level < 0 || level > 3 || mode < 1 || mode > 3) return fail(TC_E_ARG, "tc_cfl: bad argument");
    cudaSetDevice(h->prm.device);
    int rc = TC_DISPATCH(h, diag_run, h, level, tau);
    if (rc) return rc;
    double c[3];
    reduce_planes(h, nullptr, nullptr, c, nullptr);
    *out = c[mode - 1];
    return check_planes_finite(h, "tc_cfl");
}
extern "C" int tc_profiles(tc_handle* h, int level, double* out) {
    if (!out) return fail(TC_E_ARG, "tc_profiles: null output");
    return tc_diagnostics(h, level, 0.0, nullptr, nullptr, out);
}

// ---------------------------------------------------------------------------
// Operator-level entry points
// ---------------------------------------------------------------------------
template <typename T>
static int op_explicit(tc_handle* h, const double* v, double* f) {
    int rc = ensure_ops(h);
    if (!rc) rc = up_vec<T>(h, v, h->opv);
    if (rc) return rc;
    FluxArgs<T> fa{};
    fa.g = h->g;
    fa.m = mesh_dev<T>(h);
    fa.vel = cvec<T>(h->opv, h->g.N);
    fa.fout = vec<T>(h->opf, h->g.N);
    fa.nu_t = (h->nu_t && h->turb_kind != TC_TURB_NONE) ? (const T*)h->nu_t : nullptr;
    fa.order = 0;
    if (h->g.scheme == TC_SCHEME_COLLOC) launch_flux_coll<T>(fa, h->st);
    else launch_flux_stag<T>(fa, h->st);
    rc = check_launch("explicit_term");
    return rc ? rc : down_vec<T>(h, h->opf, f);
}
template <typename T>
static int op_grad(tc_handle* h, const double* p, double* g) {
    int rc = ensure_ops(h);
    if (!rc) rc = up_scal<T>(h, p, h->ops);
    if (rc) return rc;
    CorrArgs<T> ca{};
    ca.g = h->g;
    ca.m = mesh_dev<T>(h);
    ca.p = (const T*)h->ops;
    ca.vout = vec<T>(h->opv, h->g.N);
    ca.grad_only = 1;
    launch_correct<T>(ca, h->st);
    rc = check_launch("apply_gradient");
    return rc ? rc : down_vec<T>(h, h->opv, g);
}
template <typename T>
static int op_div(tc_handle* h, const double* v, double* dv) {
    int rc = ensure_ops(h);
    if (!rc) rc = up_vec<T>(h, v, h->opv);
    if (rc) return rc;
    DivArgs<T> a{h->g, mesh_dev<T>(h), cvec<T>(h->opv, h->g.N), (T*)h->ops};
    launch_divergence<T>(a, h->st);
    rc = check_launch("apply_divergence");
    return rc ? rc : down_scal<T>(h, h->ops, dv);
}
template <typename T>
static int op_unapply(tc_handle* h, const double* v, double* p) {
    int rc = ensure_ops(h);
    if (!rc) rc = up_vec<T>(h, v, h->opv);
    if (rc) return rc;
    poisson<T>(h, h->opv, nullptr, h->ops);
    rc = check_launch("unapply_gradient");
    return rc ? rc : down_scal<T>(h, h->ops, p);
}
template <typename T>
static int op_psolve(tc_handle* h, const double* rhs, double* p) {
    int rc = ensure_ops(h);
    if (!rc) rc = up_scal<T>(h, rhs, h->ops);
    if (rc) return rc;
    poisson<T>(h, nullptr, h->ops, h->ops);
    rc = check_launch("pressure_solve");
    return rc ? rc : down_scal<T>(h, h->ops, p);
}
template <typename T>
static int op_turb(tc_handle* h, const double* v, double* nt) {
    int rc = ensure_ops(h);
    if (!rc) rc = up_vec<T>(h, v, h->opv);
    if (rc) return rc;
    turb_visc<T>(h, h->opv);
    rc = check_launch("turb_visc");
    return rc ? rc : down_scal<T>(h, h->nu_t, nt);
}

#define TC_OPCHK(h, a, b)                                                  \
    if (!(h) || !(a) || !(b)) return fail(TC_E_ARG, "null argument");     \
    cudaSetDevice((h)->prm.device);

extern "C" int tc_op_explicit_term(tc_handle* h, const double* v, double* f) {
    TC_OPCHK(h, v, f);
    return TC_DISPATCH(h, op_explicit, h, v, f);
}
extern "C" int tc_op_apply_gradient(tc_handle* h, const double* p, double* g) {
    TC_OPCHK(h, p, g);
    return TC_DISPATCH(h, op_grad, h, p, g);
}
extern "C" int tc_op_apply_divergence(tc_handle* h, const double* v, double* dv) {
    TC_OPCHK(h, v, dv);
    return TC_DISPATCH(h, op_div, h, v, dv);
}
extern "C" int tc_op_unapply_gradient(tc_handle* h, const double* v, double* p) {
    TC_OPCHK(h, v, p);
    return TC_DISPATCH(h, op_unapply, h, v, p);
}
extern "C" int tc_op_pressure_solve(tc_handle* h, const double* rhs, double* p) {
    TC_OPCHK(h, rhs, p);
    return TC_DISPATCH(h, op_psolve, h, rhs, p);
}

// LinearSystemSolveFFT on device arrays (staggered/func_global.h:214-248): the same
// kernels as tc_op_pressure_solve without the host copies, asynchronous on the solver's
// stream; rhs and p in the working precision, cells [z][y][x]; rhs may equal p.
template <typename T>
static int dev_psolve(tc_handle* h, const void* rhs, void* p) {
    poisson<T>(h, nullptr, rhs, p);
    return check_launch("tc_pressure_solve_device");
}
extern "C" int tc_pressure_solve_device(tc_handle* h, const void* rhs, void* p) {
    TC_OPCHK(h, rhs, p);
    return TC_DISPATCH(h, dev_psolve, h, rhs, p);
}
// ---------------------------------------------------------------------------
// Segregated IMEX Runge-Kutta step of the collocated scheme (collocated_SRK/
// func_global.h:317-408, data::Step).  The reference's implicit part is empty
// (ImplicitTerm sets Ku = 0, ImplicitStage copies u*: func_global.h:310-315), so
// every Ku term is an exact zero and is left out.  Velocity and pressure live in ring
// level 0, dp/dt (StabType 1) in the pressure slot of level 1.  The explicit term is
// the collocated cross-viscosity flux with the source term, the same operator as
// collocated_AB3's CalcFluxTerm_FD (func_fluxes.h:86-117) and collocated_SRK's
// ExplicitTerm (func_global.h:270-307); gradient and divergence + pressure solve as in
// collocated_SRK/func_global.h:218-262.
// ---------------------------------------------------------------------------
struct SrkBufs {
    char *kuhat, *bufv, *nu1, *mujt, *qj, *bufs, *pjhat, *pj;
    size_t vb, sb;
};
static SrkBufs srk_bufs(tc_handle* h, size_t eb) {
    SrkBufs b;
    const int S = h->srk.S;
    b.vb = (size_t)3 * h->g.N * eb;
    b.sb = (size_t)h->g.N * eb;
    char* p = (char*)h->srk.buf;
    b.kuhat = p;
    p += S * b.vb;
    b.bufv = p;
    p += b.vb;
    b.nu1 = p;
    p += b.vb;
    b.mujt = p;
    p += S * b.sb;
    b.qj = p;
    p += S * b.sb;
    b.bufs = p;
    p += b.sb;
    b.pjhat = p;
    p += b.sb;
    b.pj = p;
    return b;
}
static size_t srk_bytes(const tc_handle* h, int S, size_t eb) {
    return ((size_t)(S + 2) * 3 + (size_t)2 * S + 3) * (size_t)h->g.N * eb;
}

template <typename T>
struct SrkOps {
    tc_handle* h;
    void lin(void* out, long long n, std::initializer_list<std::pair<double, const void*>> terms, double post = 1.0) {
        std::vector<std::pair<double, const void*>> v(terms);
        lin_v(out, n, v, post);
    }
    void lin_v(void* out, long long n, const std::vector<std::pair<double, const void*>>& v, double post = 1.0) {
        LinComb<T> a{};
        a.out = (T*)out;
        a.nt = (int)v.size();
        for (int k = 0; k < a.nt; k++) {
            a.c[k] = v[k].first;
            a.x[k] = (const T*)v[k].second;
        }
        a.post = post;
        a.n = n;
        launch_lincomb<T>(a, h->st);
        h->launches += 1;
    }
    void explicit_term(const void* v, void* out) {
        FluxArgs<T> fa{};
        fa.g = h->g;
        fa.m = mesh_dev<T>(h);
        fa.vel = cvec<T>((void*)v, h->g.N);
        fa.fout = vec<T>(out, h->g.N);
        fa.nu_t = nullptr;
        fa.order = 0;
        launch_flux_coll<T>(fa, h->st);
        h->launches += 1;
    }
    // out = rhs - G p (the correction kernel with tob = 1; out may alias rhs)
    void grad_sub(const void* rhs, const void* p, void* out) {
        CorrArgs<T> ca{};
        ca.g = h->g;
        ca.m = mesh_dev<T>(h);
        ca.rhs = cvec<T>((void*)rhs, h->g.N);
        ca.p = (const T*)p;
        ca.vout = vec<T>(out, h->g.N);
        ca.tob = (T)1;
        launch_correct<T>(ca, h->st);
        h->launches += 1;
    }
};

template <typename T>
static int srk_step_impl(tc_handle* h, double tau) {
    const auto& s = h->srk;
    const int S = s.S;
    const long long N = h->g.N, N3 = 3 * N;
    const SrkBufs b = srk_bufs(h, sizeof(T));
    auto KH = [&](int j) { return (void*)(b.kuhat + j * b.vb); };
    auto MT = [&](int j) { return (void*)(b.mujt + j * b.sb); };
    auto QJ = [&](int j) { return (void*)(b.qj + j * b.sb); };
    void* vel = h->vel[0];
    void* pres = h->pres[0];
    void* dpdt = h->pres[1];
    const double ass = s.BI[S * S - 1], inv_ass = 1. / ass, tau_stage = tau * ass, inv_tau_stage = 1. / tau_stage;
    const double alpha = s.alpha_tau / tau;
    const bool ck = s.type == TC_IMEX_CK, atype = s.type == TC_IMEX_A;
    SrkOps<T> op{h};
    if (!atype) {  // func_global.h:324-328
        op.explicit_term(vel, KH(0));
        op.grad_sub(KH(0), pres, KH(0));
    }
    if (ck) op.lin(b.nu1, N3, {{1.0, KH(0)}, {alpha, vel}});  // func_global.h:329-332
    const int j0 = atype ? 0 : 1;
    std::vector<std::pair<double, const void*>> t;
    for (int i = j0; i < S; i++) {
        // stage velocity u = u_n + tau sum_j aE_ij Kuhat_j (func_global.h:340-347)
        t.assign({{1.0, vel}});
        for (int j = 0; j < i; j++) t.push_back({tau * s.BE[i * S + j], KH(j)});
        op.lin_v(b.bufv, N3, t);
        op.explicit_term(b.bufv, KH(i));
        // right-hand side of the pressure system (func_global.h:356-380), one pass
        const double ck0 = ck ? (1. - s.alpha_tau * s.BI[i * S]) : 1.0;
        SrkScal<T> sc{};
        sc.stab = s.stab;
        sc.p = (const T*)pres;
        sc.dpdt = (const T*)dpdt;
        sc.n = N;
        sc.bufs = (T*)b.bufs;
        sc.pjhat = (T*)b.pjhat;
        sc.mode = 0;
        sc.nj = i - j0;
        for (int j = j0; j < i; j++) {
            sc.mujt[j - j0] = (const T*)MT(j);
            sc.qj[j - j0] = (const T*)QJ(j);
            sc.cm[j - j0] = inv_ass * s.BI[i * S + j];
            sc.cq[j - j0] = tau * s.BI[i * S + j];
        }
        sc.c0 = s.stab ? tau_stage * ck0 : ck0;
        sc.cpd = (s.stab && ck) ? tau * s.BI[i * S] : 0.0;
        sc.cb = s.stab ? alpha * tau_stage * tau_stage : alpha * tau_stage;
        launch_srk_scal<T>(sc, h->st);
        h->launches += 1;
        op.grad_sub(KH(i), b.bufs, b.bufv);  // func_global.h:381-386
        t.assign({{1.0, b.bufv}, {alpha, vel}});
        if (ck) t.push_back({-s.d[i], b.nu1});
        op.lin_v(b.bufv, N3, t);
        poisson<T>(h, b.bufv, nullptr, MT(i));  // UnapplyGradient
        sc.mode = 1;  // func_global.h:391-395: pj, mujt_i, qj_i in one pass
        sc.pj = (T*)b.pj;
        sc.mujt_i = (T*)MT(i);
        sc.qj_i = (T*)QJ(i);
        sc.inv = inv_tau_stage;
        launch_srk_scal<T>(sc, h->st);
        h->launches += 1;
        op.grad_sub(KH(i), b.pj, KH(i));
    }
    // final solution (func_global.h:400-407)
    t.assign({{1.0, vel}});
    for (int j = 0; j < S; j++) t.push_back({tau * s.BE[S * S + j], KH(j)});
    op.lin_v(vel, N3, t);
    TC_CUDA(cudaMemcpyAsync(pres, b.pj, b.sb, cudaMemcpyDeviceToDevice, h->st));
    if (s.stab) TC_CUDA(cudaMemcpyAsync(dpdt, QJ(S - 1), b.sb, cudaMemcpyDeviceToDevice, h->st));
    h->fused_valid = false;
    return check_launch("tc_srk_step");
}

extern "C" int tc_srk_init(tc_handle* h, int imex_type, int nstages, const double* butcher_e, const double* butcher_i,
                           int stab_type, double alpha_tau) {
    if (!h || !butcher_e || !butcher_i) return fail(TC_E_ARG, "tc_srk_init: null argument");
    if (h->g.scheme != TC_SCHEME_COLLOC || h->g.visc_type != TC_VISC_CROSS || h->nu_t)
        return fail(TC_E_ARG, "tc_srk_init: needs the collocated scheme with cross viscosity and no turbulence model");
    if (nstages < 1 || nstages > TC_SRK_MAX_STAGES || imex_type < TC_IMEX_A || imex_type > TC_IMEX_CK ||
        stab_type < 0 || stab_type > 1)
        return fail(TC_E_ARG, "tc_srk_init: bad method type, stage count or StabType");
    const int S = nstages;
    if (butcher_i[S * S - 1] == 0.0) return fail(TC_E_ARG, "tc_srk_init: a_ss of the implicit table is zero");
    cudaSetDevice(h->prm.device);
    const size_t eb = h->fp64 ? sizeof(double) : sizeof(float);
    if (h->srk.buf) {
        cudaFree(h->srk.buf);
        h->srk.buf = nullptr;
    }
    if (cudaMalloc(&h->srk.buf, srk_bytes(h, S, eb)) != cudaSuccess) {
        cudaGetLastError();
        h->srk.buf = nullptr;
        h->srk.S = 0;
        return fail(TC_E_NOMEM, "tc_srk_init: stage buffers");
    }
    TC_CUDA(cudaMemsetAsync(h->srk.buf, 0, srk_bytes(h, S, eb), h->st));
    auto& s = h->srk;
    s.S = S;
    s.type = imex_type;
    s.stab = stab_type;
    s.alpha_tau = alpha_tau;
    for (int k = 0; k < S * (S + 1); k++) {
        s.BE[k] = butcher_e[k];
        s.BI[k] = butcher_i[k];
    }
    // coefficients d of the CK formulation (collocated_SRK/imex.cpp:37-46)
    const double a_ss = s.BI[S * S - 1];
    s.d[0] = 1.;
    for (int j = 1; j < S; j++) {
        s.d[j] = 0.;
        for (int k = 0; k < j; k++) s.d[j] -= s.BI[j * S + k] * s.d[k] / a_ss;
    }
    h->g.norm_srk = 1;  // the SRK pressure normalisation (collocated_SRK/func_global.h:130-137)
    return TC_OK;
}

extern "C" int tc_srk_step(tc_handle* h, double t, double tau) {
    (void)t;  // the explicit term of the reference does not depend on time
    if (!h) return fail(TC_E_ARG, "tc_srk_step: null handle");
    if (h->srk.S == 0) return fail(TC_E_STATE, "tc_srk_step: tc_srk_init first");
    if (!(tau > 0)) return fail(TC_E_ARG, "tc_srk_step: tau must be positive");
    cudaSetDevice(h->prm.device);
    return TC_DISPATCH(h, srk_step_impl, h, tau);
}

extern "C" int tc_op_turb_visc(tc_handle* h, const double* v, double* nt) {
    if (h) h->fused_valid = false;
    TC_OPCHK(h, v, nt);
    if (!h->nu_t) return fail(TC_E_STATE, "tc_op_turb_visc: no turbulence model configured");
    return TC_DISPATCH(h, op_turb, h, v, nt);
}

// ---------------------------------------------------------------------------
// Seeded initial field
// ---------------------------------------------------------------------------
extern "C" void tc_mesh_tanh(int n, double gamma, double H, double* z) {
    for (int j = 0; j <= n; j++) z[j] = H * (1. + std::tanh(gamma * (2. * j / n - 1.)) / std::tanh(gamma));
}

template <typename T>
static int project_level(tc_handle* h, int level) {
    int rc = ensure_ops(h);
    if (rc) return rc;
    poisson<T>(h, h->vel[level], nullptr, h->ops);
    CorrArgs<T> ca{};
    ca.g = h->g;
    ca.m = mesh_dev<T>(h);
    ca.rhs = cvec<T>(h->vel[level], h->g.N);
    ca.p = (const T*)h->ops;
    ca.vout = vec<T>(h->vel[level], h->g.N);
    ca.tob = (T)1;
    launch_correct<T>(ca, h->st);
    return check_launch("projection");
}

extern "C" int tc_init_channel(tc_handle* h, int level, unsigned long long seed, double amp, int project) {
    if (!h || level < 0 || level > 3) return fail(TC_E_ARG, "tc_init_channel: bad handle or level");
    cudaSetDevice(h->prm.device);
    hist_plain(h, level);
    const Geom& g = h->g;
    const size_t N = (size_t)g.N;
    std::vector<double> v(3 * N), p(N, 0.0);
    std::mt19937_64 gen(seed);
    const bool coll = g.scheme == TC_SCHEME_COLLOC;
    const std::vector<double>& ZZ = h->hm.ZZ;
    const double H = coll ? 0.5 * (ZZ[g.NZ - 1] - ZZ[0]) : 0.5 * (ZZ[g.NZ] - ZZ[0]);
    for (size_t in = 0; in < N; in++) {
        const int iz = (int)(in / g.NXY);
        double r[3];
        for (int c = 0; c < 3; c++) r[c] = amp * (2. * (double)(gen() >> 11) * (1.0 / 9007199254740992.0) - 1.);
        const double zc = coll ? ZZ[iz] : 0.5 * (ZZ[iz] + ZZ[iz + 1]);
        const double y = (zc - ZZ[0]) / H - 1.;
        v[3 * in] = 1.5 * (1. - y * y) + r[0];
        v[3 * in + 1] = r[1];
        v[3 * in + 2] = r[2];
        if (coll) {
            if (iz == 0 || iz == g.NZ - 1) v[3 * in] = v[3 * in + 1] = v[3 * in + 2] = 0;
        } else if (iz == 0) {
            v[3 * in + 2] = 0;
        }
    }
    int rc = tc_upload_level(h, level, v.data(), p.data());
    if (rc) return rc;
    if (project) {
        rc = TC_DISPATCH(h, project_level, h, level);
        if (rc) return rc;
        TC_CUDA(cudaStreamSynchronize(h->st));
    }
    return TC_OK;
}

// ---------------------------------------------------------------------------
// Pressure solve on device buffers that allocates nothing at call time.
//
// tc_op_pressure_solve works on host arrays: on first use it allocates operator
// buffers and a staging buffer with cudaMalloc.  Some callers cannot do that: a host
// code that hands (nearly) all of HBM to its own pool or caching allocator up front
// has no device memory left for a library to allocate, and a latency-critical time
// loop cannot take cudaMalloc's implicit device-wide synchronisation.  This variant
// takes the right-hand side and the result as device pointers in the handle's working
// precision and runs the pressure solve's FFT launches around the z-solve that
// eliminates every mode on the fly (launch_zsolve; the step path uses the factors
// precomputed at creation instead); that elimination's coefficients live in a
// file-scope static device array (below), not in a buffer of the handle.
//
// * Setup: tc_create looks the array up with cudaGetSymbolAddress on the handle's
//   device.  With CUDA's lazy module loading that lookup is what loads this module into
//   the context, and loading it is what gives the 32 MiB array its device memory, so
//   the array is reserved when the handle is created, not inside the first
//   tc_op_pressure_solve_static call: create the handle before a caller's pool takes
//   the remaining HBM.  Every call looks the address up again (cheap once the module is
//   loaded), so no address outlives a context (e.g. after cudaDeviceReset).
// * Size limit: the z-solve needs (NX/2+1)*NY*NZ*c*8 bytes (c = 3 for VV4, 1
//   otherwise); problems above TC_STATIC_ZSCR_BYTES (32 MiB) are rejected with
//   TC_E_ARG.
// * Nothing in the array has to start at zero: the forward sweep writes every
//   coefficient of a mode before the backward sweep reads it.
// * The array is shared by every call on a device (every handle, stream and host
//   thread): calls whose launches overlap in time race on it.  Serialise them, e.g.
//   by issuing them on one stream.
// ---------------------------------------------------------------------------
static constexpr size_t TC_STATIC_ZSCR_BYTES = (size_t)32 << 20;
static __device__ __align__(256) unsigned char g_static_zscr[TC_STATIC_ZSCR_BYTES];

// Address of g_static_zscr on the current device.
static int static_zscr(void** out) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_static_zscr);
    if (e != cudaSuccess || !p)
        return fail(TC_E_CUDA, std::string("cudaGetSymbolAddress(static z-solve scratch): ") + cudaGetErrorString(e));
    *out = p;
    return TC_OK;
}

template <typename T>
static int poisson_static(tc_handle* h, const void* rhs, void* p_out, void* scratch) {
    const Geom& g = h->g;
    DivFftArgs<T> da;
    da.g = g;
    da.m = mesh_dev<T>(h);
    da.v = CV3<T>{{nullptr, nullptr, nullptr}};
    da.src_scalar = (const T*)rhs;
    da.spec = (cplx<T>*)h->spec;
    da.px = h->px;
    da.twx = twx<T>(h);
    const int ndx = launch_div_xfft<T>(da, h->st);
    YFftArgs<T> ya{g, (cplx<T>*)h->spec, h->py, twy<T>(h), -1};
    launch_yfft<T>(ya, h->st);
    ZSolveArgs<T> za{g, mesh_dev<T>(h), mode_tabs(h), (cplx<T>*)h->spec, scratch, h->err_flag};
    launch_zsolve<T>(za, h->st, h->side, h->ev_fork, h->ev_join);
    ya.sign = +1;
    launch_yfft<T>(ya, h->st);
    IxFftArgs<T> ia{g, (const cplx<T>*)h->spec, (T*)p_out, h->px, twx<T>(h), (T)(1.0 / ((double)g.NX * g.NY))};
    launch_ixfft<T>(ia, h->st);
    h->launches += ndx + 4 + (sizeof(T) == 4 ? 1 : 0);
    return check_launch("pressure_solve_static");
}

extern "C" int tc_op_pressure_solve_static(tc_handle* h, const void* rhs, void* p) {
    if (!h || !rhs || !p) return fail(TC_E_ARG, "tc_op_pressure_solve_static: null handle or buffer");
    const size_t need = zsolve_scratch_bytes(h->g, (int)h->esz);
    if (need > TC_STATIC_ZSCR_BYTES)
        return fail(TC_E_ARG, "tc_op_pressure_solve_static: the z-solve needs " + std::to_string(need) +
                                  " bytes of scratch ((NX/2+1)*NY*NZ*c*8, c = 3 for VV4, 1 otherwise), above the "
                                  "static array's " + std::to_string(TC_STATIC_ZSCR_BYTES) + " bytes");
    TC_CUDA(cudaSetDevice(h->prm.device));
    void* scr = nullptr;
    const int rc = static_zscr(&scr);
    if (rc) return rc;
    return TC_DISPATCH(h, poisson_static, h, rhs, p, scr);
}

// ---------------------------------------------------------------------------
// Learned LES closure: training data from a run (box filter), the network's training
// and inference, its parameters.  (include/turbch_les.h)
// ---------------------------------------------------------------------------
static_assert(MLP_NPAR == TC_MLP_NPAR, "parameter count of the closure");

static int les_scratch(tc_handle* h, size_t bytes) {
    if (h->les_bytes >= bytes) return TC_OK;
    if (h->les_buf) cudaFree(h->les_buf);
    h->les_buf = nullptr;
    h->les_bytes = 0;
    if (cudaMalloc((void**)&h->les_buf, bytes) != cudaSuccess) {
        cudaGetLastError();
        return fail(TC_E_NOMEM, "tc_les: scratch allocation failed");
    }
    h->les_bytes = bytes;
    return TC_OK;
}

static int les_check(tc_handle* h, int level, int width, int width_z, const char* who) {
    if (!h || level < 0 || level > 3) return fail(TC_E_ARG, std::string(who) + ": bad handle or level");
    if (h->g.scheme == TC_SCHEME_COLLOC) return fail(TC_E_ARG, std::string(who) + ": staggered schemes only");
    if (width < 1 || h->g.NX % width || h->g.NY % width)
        return fail(TC_E_ARG, std::string(who) + ": the filter width must divide NX and NY");
    if (width_z < 1 || h->g.NZ % width_z)
        return fail(TC_E_ARG, std::string(who) + ": the wall-normal filter width must divide NZ");
    return TC_OK;
}

template <typename T>
static void les_filter_run(tc_handle* h, int level, int width, int width_z, float* F) {
    const size_t N = (size_t)h->g.N;
    const T* v = (const T*)h->vel[level];
    launch_les_filter<T>(v, v + N, v + 2 * N, (const T*)h->pres[level], h->mesh_d, h->g, width, width_z, F, h->st);
}

extern "C" int tc_les_filter(tc_handle* h, int level, int width, int width_z, float* fields) {
    int rc = les_check(h, level, width, width_z, "tc_les_filter");
    if (rc) return rc;
    if (!fields) return fail(TC_E_ARG, "tc_les_filter: null output");
    cudaSetDevice(h->prm.device);
    const size_t M = (size_t)(h->g.NX / width) * (h->g.NY / width) * (h->g.NZ / width_z);
    if ((rc = les_scratch(h, 10 * M * sizeof(float)))) return rc;
    TC_DISPATCH(h, les_filter_run, h, level, width, width_z, h->les_buf);
    if ((rc = check_launch("tc_les_filter"))) return rc;
    TC_CUDA(cudaMemcpyAsync(fields, h->les_buf, 10 * M * sizeof(float), cudaMemcpyDeviceToHost, h->st));
    TC_CUDA(cudaStreamSynchronize(h->st));
    return TC_OK;
}

extern "C" int tc_les_samples(tc_handle* h, int level, int width, int width_z, float* features, float* targets) {
    int rc = les_check(h, level, width, width_z, "tc_les_samples");
    if (rc) return rc;
    if (!features || !targets) return fail(TC_E_ARG, "tc_les_samples: null output");
    cudaSetDevice(h->prm.device);
    const size_t M = (size_t)(h->g.NX / width) * (h->g.NY / width) * (h->g.NZ / width_z);
    if ((rc = les_scratch(h, 17 * M * sizeof(float)))) return rc;
    float* F = h->les_buf;
    float* X = F + 10 * M;
    float* Y = X + 6 * M;
    TC_DISPATCH(h, les_filter_run, h, level, width, width_z, F);
    launch_les_features(F, h->g, width, width_z, h->mesh_d, X, Y, h->st);
    if ((rc = check_launch("tc_les_samples"))) return rc;
    TC_CUDA(cudaMemcpyAsync(features, X, 6 * M * sizeof(float), cudaMemcpyDeviceToHost, h->st));
    TC_CUDA(cudaMemcpyAsync(targets, Y, M * sizeof(float), cudaMemcpyDeviceToHost, h->st));
    TC_CUDA(cudaStreamSynchronize(h->st));
    return TC_OK;
}

struct tc_mlp {
    int device = 0;
    cudaStream_t st = nullptr;
    float *P = nullptr, *M = nullptr, *V = nullptr, *grad = nullptr, *part = nullptr, *loss = nullptr;
    float *X = nullptr, *Y = nullptr;  // training data on the device
    long long n = 0, part_blocks = 0, loss_cap = 0;
    int step = 0;
};

static void mlp_free(tc_mlp* m) {
    float* ptrs[] = {m->P, m->M, m->V, m->grad, m->part, m->loss, m->X, m->Y};
    for (float* p : ptrs)
        if (p) cudaFree(p);
    if (m->st) cudaStreamDestroy(m->st);
}

// partial-gradient buffer for batches of up to n samples
static int mlp_parts(tc_mlp* m, long long n) {
    const long long nb = mlp_grad_blocks(n);
    if (nb <= m->part_blocks) return TC_OK;
    if (m->part) cudaFree(m->part);
    m->part = nullptr;
    m->part_blocks = 0;
    if (cudaMalloc((void**)&m->part, (size_t)nb * (MLP_NPAR + 1) * sizeof(float)) != cudaSuccess)
        return fail(TC_E_NOMEM, "tc_mlp: partial-gradient buffer");
    m->part_blocks = nb;
    return TC_OK;
}

extern "C" int tc_mlp_create(int device, unsigned long long seed, tc_mlp** out) {
    if (!out) return fail(TC_E_ARG, "tc_mlp_create: null output");
    *out = nullptr;
    TC_CUDA(cudaSetDevice(device));
    tc_mlp* m = new tc_mlp;
    m->device = device;
    bool ok = cudaStreamCreateWithFlags(&m->st, cudaStreamNonBlocking) == cudaSuccess;
    for (float** p : {&m->P, &m->M, &m->V, &m->grad})
        ok = ok && cudaMalloc((void**)p, (MLP_NPAR + 1) * sizeof(float)) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        mlp_free(m);
        delete m;
        return fail(TC_E_NOMEM, "tc_mlp_create: allocation failed");
    }
    // seeded initialisation: weights uniform in +-1/sqrt(fan_in), biases zero, b3 = -2
    std::vector<float> P(MLP_NPAR, 0.f);
    std::mt19937_64 gen(seed);
    auto uni = [&](double bound) { return (float)(bound * (2.0 * (double)(gen() >> 11) * (1.0 / 9007199254740992.0) - 1.0)); };
    for (int i = 0; i < MLP_IN * MLP_H; i++) P[MLP_OW1 + i] = uni(1.0 / std::sqrt((double)MLP_IN));
    for (int i = 0; i < MLP_H * MLP_H; i++) P[MLP_OW2 + i] = uni(1.0 / std::sqrt((double)MLP_H));
    for (int i = 0; i < MLP_H; i++) P[MLP_OW3 + i] = uni(1.0 / std::sqrt((double)MLP_H));
    P[MLP_OB3] = -2.f;
    cudaMemcpy(m->P, P.data(), MLP_NPAR * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemset(m->M, 0, (MLP_NPAR + 1) * sizeof(float));
    cudaMemset(m->V, 0, (MLP_NPAR + 1) * sizeof(float));
    *out = m;
    return TC_OK;
}

extern "C" int tc_mlp_destroy(tc_mlp* m) {
    if (!m) return TC_OK;
    cudaSetDevice(m->device);
    mlp_free(m);
    delete m;
    return TC_OK;
}

extern "C" int tc_mlp_get_params(tc_mlp* m, float* params) {
    if (!m || !params) return fail(TC_E_ARG, "tc_mlp_get_params: null argument");
    cudaSetDevice(m->device);
    TC_CUDA(cudaStreamSynchronize(m->st));
    TC_CUDA(cudaMemcpy(params, m->P, MLP_NPAR * sizeof(float), cudaMemcpyDeviceToHost));
    return TC_OK;
}

extern "C" int tc_mlp_set_params(tc_mlp* m, const float* params) {
    if (!m || !params) return fail(TC_E_ARG, "tc_mlp_set_params: null argument");
    cudaSetDevice(m->device);
    TC_CUDA(cudaStreamSynchronize(m->st));
    TC_CUDA(cudaMemcpy(m->P, params, MLP_NPAR * sizeof(float), cudaMemcpyHostToDevice));
    TC_CUDA(cudaMemset(m->M, 0, (MLP_NPAR + 1) * sizeof(float)));
    TC_CUDA(cudaMemset(m->V, 0, (MLP_NPAR + 1) * sizeof(float)));
    m->step = 0;
    return TC_OK;
}

extern "C" int tc_mlp_set_data(tc_mlp* m, const float* features, const float* targets, long long n) {
    if (!m || !features || !targets || n <= 0) return fail(TC_E_ARG, "tc_mlp_set_data: bad argument");
    cudaSetDevice(m->device);
    TC_CUDA(cudaStreamSynchronize(m->st));
    if (m->X) cudaFree(m->X);
    if (m->Y) cudaFree(m->Y);
    m->X = m->Y = nullptr;
    m->n = 0;
    if (cudaMalloc((void**)&m->X, (size_t)n * MLP_IN * sizeof(float)) != cudaSuccess ||
        cudaMalloc((void**)&m->Y, (size_t)n * sizeof(float)) != cudaSuccess) {
        cudaGetLastError();
        return fail(TC_E_NOMEM, "tc_mlp_set_data: allocation failed");
    }
    TC_CUDA(cudaMemcpy(m->X, features, (size_t)n * MLP_IN * sizeof(float), cudaMemcpyHostToDevice));
    TC_CUDA(cudaMemcpy(m->Y, targets, (size_t)n * sizeof(float), cudaMemcpyHostToDevice));
    m->n = n;
    return TC_OK;
}

extern "C" int tc_mlp_train(tc_mlp* m, int epochs, long long batch, float lr, float* epoch_loss) {
    if (!m || epochs < 1 || batch < 1 || !(lr > 0.f)) return fail(TC_E_ARG, "tc_mlp_train: bad argument");
    if (!m->X) return fail(TC_E_STATE, "tc_mlp_train: no training data (tc_mlp_set_data)");
    cudaSetDevice(m->device);
    const long long bsz = std::min(batch, m->n);
    int rc = mlp_parts(m, bsz);
    if (rc) return rc;
    if (m->loss_cap < epochs) {
        if (m->loss) cudaFree(m->loss);
        m->loss = nullptr;
        if (cudaMalloc((void**)&m->loss, (size_t)epochs * sizeof(float)) != cudaSuccess)
            return fail(TC_E_NOMEM, "tc_mlp_train: loss buffer");
        m->loss_cap = epochs;
    }
    TC_CUDA(cudaMemsetAsync(m->loss, 0, (size_t)epochs * sizeof(float), m->st));
    for (int e = 0; e < epochs; e++) {
        for (long long off = 0; off < m->n; off += bsz) {
            const long long nb = std::min(bsz, m->n - off);
            launch_mlp_grad(m->P, m->X + off * MLP_IN, m->Y + off, nb, m->part, m->grad, m->st);
            launch_mlp_loss_acc(m->loss + e, m->grad, m->st);
            launch_mlp_adam(m->P, m->M, m->V, m->grad, lr, ++m->step, m->st);
        }
    }
    if ((rc = check_launch("tc_mlp_train"))) return rc;
    if (epoch_loss) {
        std::vector<float> l(epochs);
        TC_CUDA(cudaMemcpyAsync(l.data(), m->loss, (size_t)epochs * sizeof(float), cudaMemcpyDeviceToHost, m->st));
        TC_CUDA(cudaStreamSynchronize(m->st));
        for (int e = 0; e < epochs; e++) epoch_loss[e] = l[e] / (float)m->n;
    }
    TC_CUDA(cudaStreamSynchronize(m->st));
    return TC_OK;
}

// one gradient evaluation on host data (no update): grad[TC_MLP_NPAR], loss = mean square error
extern "C" int tc_mlp_grad(tc_mlp* m, const float* features, const float* targets, long long n, float* grad, float* loss) {
    if (!m || !features || !targets || n <= 0 || !grad) return fail(TC_E_ARG, "tc_mlp_grad: bad argument");
    cudaSetDevice(m->device);
    int rc = mlp_parts(m, n);
    if (rc) return rc;
    float *X = nullptr, *Y = nullptr;
    if (cudaMalloc((void**)&X, (size_t)n * MLP_IN * sizeof(float)) != cudaSuccess ||
        cudaMalloc((void**)&Y, (size_t)n * sizeof(float)) != cudaSuccess) {
        cudaGetLastError();
        if (X) cudaFree(X);
        return fail(TC_E_NOMEM, "tc_mlp_grad: allocation failed");
    }
    cudaMemcpyAsync(X, features, (size_t)n * MLP_IN * sizeof(float), cudaMemcpyHostToDevice, m->st);
    cudaMemcpyAsync(Y, targets, (size_t)n * sizeof(float), cudaMemcpyHostToDevice, m->st);
    launch_mlp_grad(m->P, X, Y, n, m->part, m->grad, m->st);
    std::vector<float> gbuf(MLP_NPAR + 1);
    cudaMemcpyAsync(gbuf.data(), m->grad, (MLP_NPAR + 1) * sizeof(float), cudaMemcpyDeviceToHost, m->st);
    const cudaError_t e = cudaStreamSynchronize(m->st);
    cudaFree(X);
    cudaFree(Y);
    if (e != cudaSuccess) return fail(TC_E_CUDA, std::string("tc_mlp_grad: ") + cudaGetErrorString(e));
    std::copy(gbuf.begin(), gbuf.begin() + MLP_NPAR, grad);
    if (loss) *loss = gbuf[MLP_NPAR] / (float)n;
    return TC_OK;
}

extern "C" int tc_mlp_forward(tc_mlp* m, const float* features, long long n, float* out) {
    if (!m || !features || n <= 0 || !out) return fail(TC_E_ARG, "tc_mlp_forward: bad argument");
    cudaSetDevice(m->device);
    float *X = nullptr, *O = nullptr;
    if (cudaMalloc((void**)&X, (size_t)n * MLP_IN * sizeof(float)) != cudaSuccess ||
        cudaMalloc((void**)&O, (size_t)n * sizeof(float)) != cudaSuccess) {
        cudaGetLastError();
        if (X) cudaFree(X);
        return fail(TC_E_NOMEM, "tc_mlp_forward: allocation failed");
    }
    cudaMemcpyAsync(X, features, (size_t)n * MLP_IN * sizeof(float), cudaMemcpyHostToDevice, m->st);
    launch_mlp_forward(m->P, X, n, O, m->st);
    cudaMemcpyAsync(out, O, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost, m->st);
    const cudaError_t e = cudaStreamSynchronize(m->st);
    cudaFree(X);
    cudaFree(O);
    if (e != cudaSuccess) return fail(TC_E_CUDA, std::string("tc_mlp_forward: ") + cudaGetErrorString(e));
    return TC_OK;
}

extern "C" int tc_set_mlp_fusion(tc_handle* h, int mode) {
    if (!h || mode < 0 || mode > 1) return fail(TC_E_ARG, "tc_set_mlp_fusion: bad handle or mode");
    h->mlp_fuse = mode;
    return TC_OK;
}

extern "C" int tc_set_flux_staging(tc_handle* h, int mode) {
    if (!h || mode < 0 || mode > 1) return fail(TC_E_ARG, "tc_set_flux_staging: bad handle or mode");
    h->flux_staging = mode;
    return TC_OK;
}

extern "C" int tc_set_fft_fusion(tc_handle* h, int mode) {
    if (!h || mode < 0 || mode > 1) return fail(TC_E_ARG, "tc_set_fft_fusion: bad handle or mode");
    h->fft_plane = mode;
    return TC_OK;
}

extern "C" int tc_set_diag_fusion(tc_handle* h, int mode) {
    if (!h || mode < 0 || mode > 2) return fail(TC_E_ARG, "tc_set_diag_fusion: bad handle or mode");
    h->diag_fuse = mode;
    h->diag_follow = false;
    h->fused_valid = false;
    return TC_OK;
}

// ---------------------------------------------------------------------------
// Binary checkpoint of the whole step state: the four ring levels (velocity, flux,
// pressure, in the device layout) and the forcing state, so that a restarted run
// continues the SBDF history exactly.  The reference writes VTK ASCII fields of one
// level only (staggered/io.cpp:6-68), which loses the BDF history on restart.
// ---------------------------------------------------------------------------
namespace {
constexpr char TC_CKPT_MAGIC[8] = {'T', 'C', 'H', 'K', 'P', 'T', '0', '1'};
struct CkptHeader {
    char magic[8];
    int32_t version, scheme, precision, NX, NY, NZ, current_field, forcing_mode;
    double t, forcing_value, sour_dpdx, last_tau, last_bd0, last_du;
    int64_t N;
    double hist_it[4];  // version 2: the 1/tau baked into each flux level (A = F + it v / 2)
    char pad[256 - 8 - 8 * 4 - 6 * 8 - 8 - 4 * 8];
};
static_assert(sizeof(CkptHeader) == 256, "checkpoint header size");

struct FileCloser {
    FILE* f;
    ~FileCloser() {
        if (f) fclose(f);
    }
};

// Moves `bytes` between a device buffer and the file through a pinned bounce buffer.
int ckpt_stream(tc_handle* h, FILE* f, void* dev, size_t bytes, bool save, std::vector<char>& host) {
    const size_t chunk = host.size();
    for (size_t off = 0; off < bytes; off += chunk) {
        const size_t n = std::min(chunk, bytes - off);
        char* d = static_cast<char*>(dev) + off;
        if (save) {
            TC_CUDA(cudaMemcpyAsync(host.data(), d, n, cudaMemcpyDeviceToHost, h->st));
            TC_CUDA(cudaStreamSynchronize(h->st));
            if (fwrite(host.data(), 1, n, f) != n) return fail(TC_E_ARG, "tc_checkpoint_save: write failed");
        } else {
            if (fread(host.data(), 1, n, f) != n) return fail(TC_E_ARG, "tc_checkpoint_load: file too short");
            TC_CUDA(cudaMemcpyAsync(d, host.data(), n, cudaMemcpyHostToDevice, h->st));
            TC_CUDA(cudaStreamSynchronize(h->st));
        }
    }
    return TC_OK;
}

int ckpt_levels(tc_handle* h, FILE* f, bool save) {
    const size_t N = (size_t)h->g.N, E = h->esz;
    std::vector<char> host(std::min<size_t>((size_t)64 << 20, 3 * N * E));
    for (int l = 0; l < 4; l++) {
        int rc;
        if ((rc = ckpt_stream(h, f, h->vel[l], 3 * N * E, save, host))) return rc;
        if ((rc = ckpt_stream(h, f, h->flux[l], 3 * N * E, save, host))) return rc;
        if ((rc = ckpt_stream(h, f, h->pres[l], N * E, save, host))) return rc;
    }
    return TC_OK;
}
}  // namespace

extern "C" int tc_checkpoint_save(tc_handle* h, const char* path, int current_field, double t) {
    if (!h || !path || current_field < 0 || current_field > 3) return fail(TC_E_ARG, "tc_checkpoint_save: bad argument");
    cudaSetDevice(h->prm.device);
    TC_CUDA(cudaStreamSynchronize(h->st));
    CkptHeader hd;
    memset(&hd, 0, sizeof(hd));
    memcpy(hd.magic, TC_CKPT_MAGIC, 8);
    hd.version = 2;
    for (int l = 0; l < 4; l++) hd.hist_it[l] = h->hist_it[l];
    hd.scheme = h->prm.scheme;
    hd.precision = h->prm.precision;
    hd.NX = h->g.NX;
    hd.NY = h->g.NY;
    hd.NZ = h->g.NZ;
    hd.current_field = current_field;
    hd.forcing_mode = h->forcing_mode;
    hd.t = t;
    hd.forcing_value = h->forcing_value;
    hd.sour_dpdx = h->g.sour_dpdx;
    hd.last_tau = h->last_tau;
    hd.last_bd0 = h->last_bd0;
    double du = 0.0;
    TC_CUDA(cudaMemcpy(&du, h->red + 1, sizeof(double), cudaMemcpyDeviceToHost));
    hd.last_du = du;
    hd.N = h->g.N;
    FileCloser fc{fopen(path, "wb")};
    if (!fc.f) return fail(TC_E_ARG, std::string("tc_checkpoint_save: cannot open ") + path);
    if (fwrite(&hd, sizeof(hd), 1, fc.f) != 1) return fail(TC_E_ARG, "tc_checkpoint_save: write failed");
    int rc = ckpt_levels(h, fc.f, true);
    if (rc) return rc;
    if (fflush(fc.f) != 0) return fail(TC_E_ARG, "tc_checkpoint_save: write failed");
    return TC_OK;
}

extern "C" int tc_checkpoint_load(tc_handle* h, const char* path, int* current_field, double* t) {
    if (!h || !path) return fail(TC_E_ARG, "tc_checkpoint_load: bad argument");
    cudaSetDevice(h->prm.device);
    FileCloser fc{fopen(path, "rb")};
    if (!fc.f) return fail(TC_E_ARG, std::string("tc_checkpoint_load: cannot open ") + path);
    CkptHeader hd;
    if (fread(&hd, sizeof(hd), 1, fc.f) != 1 || memcmp(hd.magic, TC_CKPT_MAGIC, 8) != 0 || hd.version < 1 ||
        hd.version > 2)
        return fail(TC_E_ARG, "tc_checkpoint_load: not a checkpoint of this library");
    if (hd.scheme != h->prm.scheme || hd.precision != h->prm.precision || hd.NX != h->g.NX || hd.NY != h->g.NY ||
        hd.NZ != h->g.NZ || hd.N != h->g.N || hd.current_field < 0 || hd.current_field > 3)
        return fail(TC_E_ARG, "tc_checkpoint_load: the checkpoint's scheme, precision or grid differ from the solver's");
    TC_CUDA(cudaStreamSynchronize(h->st));
    int rc = ckpt_levels(h, fc.f, false);
    if (rc) return rc;
    h->forcing_mode = hd.forcing_mode;
    h->forcing_value = hd.forcing_value;
    h->prm.sour_dpdx = hd.sour_dpdx;
    h->g.sour_dpdx = hd.sour_dpdx;
    h->last_tau = hd.last_tau;
    h->last_bd0 = hd.last_bd0;
    for (int l = 0; l < 4; l++) h->hist_it[l] = hd.version >= 2 ? hd.hist_it[l] : 0.0;  // version 1: plain F
    TC_CUDA(cudaMemcpy(h->red + 1, &hd.last_du, sizeof(double), cudaMemcpyHostToDevice));
    h->fused_valid = false;
    if (current_field) *current_field = hd.current_field;
    if (t) *t = hd.t;
    return TC_OK;
}

// ---------------------------------------------------------------------------
// Time-averaged plane statistics kept on the device (the reference's driver adds the
// profiles of each step on the host, staggered/main.cpp:316-326): per call one
// diagnostics pass of the level and a weighted add into a device accumulator, no
// host synchronisation; a read returns the weighted means in tc_profiles' layout.
// ---------------------------------------------------------------------------
extern "C" int tc_stats_accumulate(tc_handle* h, int level, double weight) {
    if (!h || level < 0 || level > 3 || !(weight >= 0.0)) return fail(TC_E_ARG, "tc_stats_accumulate: bad argument");
    cudaSetDevice(h->prm.device);
    int rc = TC_DISPATCH(h, diag_device, h, level);
    if (rc) return rc;
    launch_stats_acc(h->planes, h->stats, h->g.NZ, 1.0 / (double)h->g.NXY, weight, h->st);
    TC_CUDA(cudaGetLastError());
    return TC_OK;
}

extern "C" int tc_stats_read(tc_handle* h, double* profiles, double* total_weight) {
    if (!h || !profiles) return fail(TC_E_ARG, "tc_stats_read: bad argument");
    cudaSetDevice(h->prm.device);
    const size_t n = (size_t)h->g.NZ * 12;
    std::vector<double> acc(n + 1);
    TC_CUDA(cudaMemcpyAsync(acc.data(), h->stats, (n + 1) * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    TC_CUDA(cudaStreamSynchronize(h->st));
    const double w = acc[n];
    for (size_t i = 0; i < n; i++) profiles[i] = w > 0.0 ? acc[i] / w : 0.0;
    if (total_weight) *total_weight = w;
    return TC_OK;
}

extern "C" int tc_stats_reset(tc_handle* h) {
    if (!h) return fail(TC_E_ARG, "tc_stats_reset: null handle");
    cudaSetDevice(h->prm.device);
    TC_CUDA(cudaMemsetAsync(h->stats, 0, ((size_t)h->g.NZ * 12 + 1) * sizeof(double), h->st));
    return TC_OK;
}

// ---------------------------------------------------------------------------
// Device-controlled runs: SBDF3 steps of a fixed tau replayed by a CUDA graph whose
// while-loop ends on the device when the CFL number leaves [cfl_min, cfl_max] (the
// reference's driver checks it on the host every 10 steps and halves or enlarges tau,
// staggered/main.cpp:361-370).  The body is `every` steps (a multiple of 4, so that the
// ring comes back to the same levels) followed by the diagnostics pass of the level just
// written and the condition kernel; the host waits once per run, not per step.
// ---------------------------------------------------------------------------
template <typename T>
static int run_capture_body(tc_handle* h, double tau, int cur, int every, int mode, cudaGraphConditionalHandle hnd) {
    for (int k = 0; k < every; k++) {
        int rc = step_impl<T>(h, tau, (cur + k) % 4, 3);
        if (rc) return rc;
    }
    DiagArgs<T> a;
    a.g = h->g;
    a.m = mesh_dev<T>(h);
    a.v = cvec<T>(h->vel[cur], h->g.N);
    a.p = (const T*)h->pres[cur];
    a.nu_t = (h->nu_t && h->turb_kind != TC_TURB_NONE) ? (const T*)h->nu_t : nullptr;
    a.tau = tau;
    a.planes = h->planes;
    a.part = h->diag_part;
    launch_diag<T>(a, h->st);
    launch_run_ctl(hnd, h->planes, h->g.NZ, mode, h->run_ctl, h->st);
    return check_launch("tc_run_graph");
}

static void run_graph_drop(tc_handle* h) {
    if (h->run_exec) cudaGraphExecDestroy(h->run_exec);
    if (h->run_graph) cudaGraphDestroy(h->run_graph);
    h->run_exec = nullptr;
    h->run_graph = nullptr;
    h->run_cur = -1;
}

static int run_graph_build(tc_handle* h, double tau, int cur, int every, int mode) {
    run_graph_drop(h);
    TC_CUDA(cudaGraphCreate(&h->run_graph, 0));
    cudaGraphConditionalHandle hnd;
    TC_CUDA(cudaGraphConditionalHandleCreate(&hnd, h->run_graph, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = hnd;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    TC_CUDA(cudaGraphAddNode(&node, h->run_graph, nullptr, 0, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    TC_CUDA(cudaStreamBeginCaptureToGraph(h->st, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    const int diag_fuse = h->diag_fuse;
    h->diag_fuse = 0;  // no lazily allocated fused-diagnostics buffer inside the capture
    int rc = TC_DISPATCH(h, run_capture_body, h, tau, cur, every, mode, hnd);
    h->diag_fuse = diag_fuse;
    cudaGraph_t captured = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(h->st, &captured);
    if (rc || ec != cudaSuccess) {
        cudaGetLastError();
        run_graph_drop(h);
        return rc ? rc : fail(TC_E_CUDA, std::string("tc_run_graph: capture failed: ") + cudaGetErrorString(ec));
    }
    TC_CUDA(cudaGraphInstantiate(&h->run_exec, h->run_graph, 0));
    h->run_tau = tau;
    h->run_cur = cur;
    h->run_every = every;
    h->run_mode = mode;
    return TC_OK;
}

extern "C" int tc_run_graph(tc_handle* h, double tau, int current_field, int nsteps, int check_every, int cfl_mode,
                            double cfl_min, double cfl_max, int* steps_done, double* cfl) {
    if (!h || current_field < 0 || current_field > 3 || cfl_mode < 1 || cfl_mode > 3)
        return fail(TC_E_ARG, "tc_run_graph: bad argument");
    if (!(tau > 0) || !std::isfinite(tau)) return fail(TC_E_ARG, "tc_run_graph: tau must be positive");
    if (check_every < 4 || check_every % 4 != 0 || nsteps < check_every)
        return fail(TC_E_ARG, "tc_run_graph: check_every must be a positive multiple of 4 and at most nsteps");
    if (h->timing) return fail(TC_E_STATE, "tc_run_graph: phase timing is on");
    cudaSetDevice(h->prm.device);
    if (!h->run_ctl && cudaMalloc((void**)&h->run_ctl, sizeof(RunCtl)) != cudaSuccess) {
        cudaGetLastError();
        return fail(TC_E_NOMEM, "tc_run_graph: allocation failed");
    }
    {
        // the graph's order-3 steps read flux levels current-1 and current-2 as written with
        // this tau: bring them there outside the graph
        const double itd = h->fp64 ? (double)(1. / tau) : (double)(float)(1. / tau);
        if (h->fp64) {
            rebase_hist<double>(h, (current_field + 3) % 4, itd);
            rebase_hist<double>(h, (current_field + 2) % 4, itd);
        } else {
            rebase_hist<float>(h, (current_field + 3) % 4, itd);
            rebase_hist<float>(h, (current_field + 2) % 4, itd);
        }
    }
    if (!h->run_exec || h->run_tau != tau || h->run_cur != current_field || h->run_every != check_every ||
        h->run_mode != cfl_mode) {
        int rc = run_graph_build(h, tau, current_field, check_every, cfl_mode);
        if (rc) return rc;
    }
    RunCtl c{0u, (unsigned)(nsteps / check_every), 0.0, cfl_min, cfl_max};
    TC_CUDA(cudaMemcpyAsync(h->run_ctl, &c, sizeof(c), cudaMemcpyHostToDevice, h->st));
    TC_CUDA(cudaGraphLaunch(h->run_exec, h->st));
    TC_CUDA(cudaMemcpyAsync(&c, h->run_ctl, sizeof(c), cudaMemcpyDeviceToHost, h->st));
    TC_CUDA(cudaStreamSynchronize(h->st));
    h->fused_valid = false;
    h->last_out = current_field;
    {  // every level was rewritten by the graph's steps (at least check_every >= 4 of them)
        const double itd = h->fp64 ? (double)(1. / tau) : (double)(float)(1. / tau);
        for (int l = 0; l < 4; l++) h->hist_it[l] = h->hist_a ? itd : 0.0;
    }
    if (steps_done) *steps_done = (int)c.iters * check_every;
    if (cfl) *cfl = c.cfl;
    return TC_OK;
}
