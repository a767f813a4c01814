// kernels.cuh -- argument blocks and host launchers of the sm_100a kernels.
// Internal to turbchannel_b200 (tc_api.cu is the only caller).
#pragma once
#include "tc_common.cuh"

namespace tc {

template <typename T>
struct V3 {
    T* c[3];
};
template <typename T>
struct CV3 {
    const T* c[3];
};

// Fused explicit flux + SBDF3 combine (one pass over v_n and the history).
//   F_n = (sour_dpdx,0,0) + Conv(v_n) + Visc(v_n)          -> fout
//   RHS = a0 F_n + a1 F_{n-1} + a2 F_{n-2} + inv_tau (b0 v_n + b1 v_{n-1} + b2 v_{n-2})
//         (staggered/func_global.h:910-932)                 -> rhs
//   collocated StabType 1 also subtracts grad p_n (collocated_AB3/func_global.h:436-437).
//   The weighted sum of RHS_x (bulk velocity of the result, up to tau/bd0) is
//   reduced deterministically into ub_out when ub_out != nullptr.
template <typename T>
struct FluxArgs {
    Geom g;
    MeshDev<T> m;
    // vel = v_n (stencil), velq = v_{n-2}; fp, fq = the flux ring's levels n-1, n-2, which
    // hold A_m = F_m + v_m / (2 tau) (sbdf_rhs); velp (v_{n-1}) is not read by the step
    CV3<T> vel, velp, velq, fp, fq;
    V3<T> fout, rhs;  // fout: A_n (orders 1..3) or F_n (order 0); rhs: the SBDF right-hand side
    const T* nu_t;
    const T* pcur;
    T inv_tau;
    int order;  // 0: F_n only (operator form), 1..3: SBDF order
    double* ub_partial;
    unsigned* ticket;
    double* ub_out;
    int* err_flag = nullptr;  // set to 2 when a bounded wait of the TMA staging gives up
    int staging = 0;          // float pair kernel: 0 cp.async ring fill, 1 TMA tensor tiles (interior tiles)
};

// SBDF right-hand side (staggered/func_global.h:910-932) with the flux history kept as
// A_m = F_m + v_m / (2 tau) instead of F_m: since
//   3 F_{n-1} + (3/2) v_{n-1} / tau = 3 A_{n-1} and F_{n-2} + v_{n-2} / (3 tau) =
//   A_{n-2} - v_{n-2} / (6 tau) (order 3), F_{n-1} + v_{n-1} / (2 tau) = A_{n-1} (order 2),
// the combination reads one array per history level plus v_{n-2} -- 3 words per cell
// fewer than F_{n-1}, F_{n-2}, v_{n-1}, v_{n-2} -- and the new level A_n = F_n + v_n/(2 tau)
// is written in place of F_n.  b = F_n + v_n / tau.
//   order 1: b;   order 2: 2 b - A_{n-1};   order 3: 3 b - 3 A_{n-1} + A_{n-2} - v_{n-2}/(6 tau)
// it = 1/tau, it6 = 1/(6 tau) (in the working precision).
template <int ORDER, typename V>
__device__ __forceinline__ V sbdf_rhs(V f, V vn, V ap, V aq, V vq, V it, V it6) {
    const V b = f + it * vn;
    if (ORDER == 1) return b;
    if (ORDER == 2) return V(2) * b - ap;
    return (V(3) * b - V(3) * ap) + (aq - it6 * vq);
}

// Divergence of the RHS fused with the forward real FFT along x.  Output: half
// spectrum spec[z][kx][y] (kx = 0..NX/2, y fastest).  src_scalar != nullptr: the
// input is a scalar field (already a divergence / a pressure RHS) instead.
template <typename T>
struct DivFftArgs {
    Geom g;
    MeshDev<T> m;
    CV3<T> v;
    const T* src_scalar;
    cplx<T>* spec;
    FftPlan px;
    const cplx<T>* twx;
    T* dtmp = nullptr;  // N-cell scratch for the divergence (the pressure output, free until the inverse FFT)
};

// In-place complex FFT along y of the lines spec[z][kx][0..NY).
template <typename T>
struct YFftArgs {
    Geom g;
    cplx<T>* spec;
    FftPlan py;
    const cplx<T>* twy;
    int sign;
};

// Rows of the z-solve factors (k_zfactor layout): four or two values of one mode.
template <typename T>
struct alignas(4 * sizeof(T)) Q4 {
    T x, y, z, w;
};
template <typename T>
struct alignas(2 * sizeof(T)) Q2 {
    T x, y;
};

// Banded wall-normal solve per (kx, ky) mode, in place on spec; normalisation of
// the mean mode (staggered/func_global.h:657-675) applied to mode (0, 0).
template <typename T>
struct ZSolveArgs {
    Geom g;
    MeshDev<T> m;
    ModeTabs tabs;
    cplx<T>* spec;
    void* scratch;  // per-mode elimination coefficients
    int* err_flag;  // set when a pivot underflows (the reference writes -1e50)
    void* fac = nullptr;  // precomputed factors (k_zfactor layout), zfactor_bytes()
    void* fac_low = nullptr;  // double factors of the low modes, zfactor_low_bytes()
};

// Inverse real FFT along x: p = scale * C2R(spec) (+ dest layout [z][y][x]).
template <typename T>
struct IxFftArgs {
    Geom g;
    const cplx<T>* spec;
    T* p;
    FftPlan px;
    const cplx<T>* twx;
    T scale;
};

// Velocity correction v_{n+1} = (RHS - G p) tau/bd0 (+ uniform flow-rate shift of u);
// collocated StabType 1 also p_{n+1} += p_n.
template <typename T>
struct CorrArgs {
    Geom g;
    MeshDev<T> m;
    CV3<T> rhs;
    const T* p;       // pressure (or pressure increment) whose gradient is removed
    V3<T> vout;
    const T* pcur;    // StabType 1: p_n
    T* pnext;         // StabType 1: p_{n+1} = p + p_n
    T tob;            // tau / bd0
    int cfr;          // 1: apply the flow-rate shift
    double cfr_target;
    double cfr_scale;      // hx hy / area: bulk velocity = ub_sum * cfr_scale * tob
    double cfr_volfac;     // area / fluid volume receiving the shift
    const double* ub_sum;  // sum of RHS_x weights from the flux kernel
    double* du_out;        // shift applied (for tc_last_dpdx)
    int grad_only;         // operator form: vout = G p
    // Diagnostics of the new level fused into the correction (staggered, NX % 4 == 0):
    // per (plane, xy-CTA) partial sums in the k_diag layout; nullptr: not fused.
    double* dpart = nullptr;
    const T* nu_t = nullptr;  // LES eddy viscosity (diagnostics only)
    double dtau = 0.0;        // time step of the CFL numbers
    double dkv = 1.0;         // viscous CFL factor of the scheme's viscosity
};

template <typename T>
struct TurbArgs {
    Geom g;
    MeshDev<T> m;
    CV3<T> v;
    T* nu_t;
};

template <typename T>
struct DivArgs {
    Geom g;
    MeshDev<T> m;
    CV3<T> v;
    T* dv;
};

// Per-plane diagnostics (profiles, integral, KE and CFL ingredients), double.
template <typename T>
struct DiagArgs {
    Geom g;
    MeshDev<T> m;
    CV3<T> v;
    const T* p;
    const T* nu_t;
    double tau;
    double* planes;  // NZ x TC_DIAG_STRIDE
    double* part;    // NZ x diag_chunks() x TC_DIAG_STRIDE partial sums
};
constexpr int TC_DIAG_STRIDE = 19;
constexpr int NDIAG_SUMS = 16;  // planes[z][0..15] are sums, [16..18] CFL maxima

template <typename T> void launch_flux_stag(const FluxArgs<T>& a, cudaStream_t s);
template <typename T> void launch_flux_coll(const FluxArgs<T>& a, cudaStream_t s);
bool launch_flux_stag_pair(const FluxArgs<float>& a, cudaStream_t s);  // k_flux_pair.cu; false: not covered
bool flux_pair_covers(const Geom& g);  // the float pair kernel takes the step (its history is plain F)
template <typename T> int launch_div_xfft(const DivFftArgs<T>& a, cudaStream_t s);  // returns launches
template <typename T> void launch_yfft(const YFftArgs<T>& a, cudaStream_t s);
template <typename T> void launch_zsolve(const ZSolveArgs<T>& a, cudaStream_t s, cudaStream_t side, cudaEvent_t fork,
                                       cudaEvent_t join);
// factored solve (step path): launch_zfactor once at creation, then launch_zsolve_fac
template <typename T> void launch_zfactor(const ZSolveArgs<T>& a, cudaStream_t s);
template <typename T> void launch_zsolve_fac(const ZSolveArgs<T>& a, cudaStream_t s, cudaStream_t side,
                                           cudaEvent_t fork, cudaEvent_t join);
template <typename T> void launch_ixfft(const IxFftArgs<T>& a, cudaStream_t s);
// two-pass register FFT versions (k_fft.cu); false when the length has none
template <typename T> int launch_div_xfft_reg(const DivFftArgs<T>& a, cudaStream_t s);  // 0: no such path
template <typename T> bool launch_yfft_reg(const YFftArgs<T>& a, cudaStream_t s);
template <typename T> bool launch_ixfft_reg(const IxFftArgs<T>& a, cudaStream_t s);
template <typename T> bool launch_div_quad(const DivFftArgs<T>& a, cudaStream_t s);  // divergence into a.dtmp
// Plane transforms (k_fft_plane.cu): the x- and y-FFTs of each z-plane in one kernel, one
// thread-block cluster per plane.  plane_fft_ok: whether (NX, NY) has a compiled plane
// kernel that fits this device; the launchers return 0 / false when it has none.
template <typename T> bool plane_fft_ok(const Geom& g);
template <typename T> int launch_div_xyfft_plane(const DivFftArgs<T>& a, const cplx<T>* twy, cudaStream_t s);
template <typename T> bool launch_ixyfft_plane(const IxFftArgs<T>& a, const cplx<T>* twy, cudaStream_t s);
template <typename T> void launch_correct(const CorrArgs<T>& a, cudaStream_t s);
template <typename T> void launch_turb(const TurbArgs<T>& a, cudaStream_t s);
template <typename T> void launch_divergence(const DivArgs<T>& a, cudaStream_t s);
template <typename T> void launch_diag(const DiagArgs<T>& a, cudaStream_t s);

// AoS double <-> SoA T conversions (host boundary), and misc.
template <typename T> void launch_aos_to_soa(const double* src, V3<T> dst, long long n, cudaStream_t s);
template <typename T> void launch_soa_to_aos(CV3<T> src, double* dst, long long n, cudaStream_t s);
template <typename T> void launch_d2t(const double* src, T* dst, long long n, cudaStream_t s);
template <typename T> void launch_t2d(const T* src, double* dst, long long n, cudaStream_t s);

// learned LES closure (k_les.cu, k_mlp.cu)
template <typename T>
void launch_les_filter(const T* u, const T* v, const T* w, const T* p, const double* ZZ, const Geom& g, int fw, int fz,
                       float* F, cudaStream_t s);
void launch_les_features(const float* F, const Geom& g, int fw, int fz, const double* ZZ, float* X, float* Y,
                         cudaStream_t s);
template <typename T> void launch_turb_mlp(const TurbArgs<T>& a, const float* P, cudaStream_t s);
// the staggered step flux (orders 1..3, NAIVE viscosity) with the learned closure's
// inference fused in; also writes nu_t of every cell to nu_out (k_flux_mlp.cu)
template <typename T> void launch_flux_mlp(const FluxArgs<T>& a, const float* P, T* nu_out, cudaStream_t s);
void launch_mlp_grad(const float* P, const float* X, const float* Y, long long n, float* part, float* grad,
                     cudaStream_t s);
void launch_mlp_adam(float* P, float* M, float* V, const float* grad, float lr, int step, cudaStream_t s);
void launch_mlp_forward(const float* P, const float* X, long long n, float* out, cudaStream_t s);
int mlp_grad_blocks(long long n);
void launch_mlp_loss_acc(float* acc, const float* grad, cudaStream_t s);  // acc += loss sum in grad

size_t zsolve_scratch_bytes(const Geom& g, int elem_bytes);
size_t zfactor_bytes(const Geom& g, int elem_bytes);
size_t zfactor_low_bytes(const Geom& g);
int diag_chunks(const Geom& g);
int correct_diag_chunks(const Geom& g);  // xy-CTAs per plane of the fused diagnostics
void launch_diag_finish(const double* part, double* planes, int NZ, int S, cudaStream_t s);
void launch_stats_acc(const double* planes, double* acc, int NZ, double inv_nxy, double w, cudaStream_t s);

// State of a device-controlled run (tc_run_graph): bodies done, their bound, the CFL
// number of the last check and the bounds that keep the loop going.
// out[i] = post * (c[0] x[0][i] + c[1] x[1][i] + ... + c[nt-1] x[nt-1][i]), summed left
// to right in T; x may alias out (elementwise).  The stage updates of the SRK step.
constexpr int TC_LIN_MAX = 8;
template <typename T>
struct LinComb {
    T* out;
    const T* x[TC_LIN_MAX];
    double c[TC_LIN_MAX];
    double post;
    int nt;
    long long n;
};
template <typename T> void launch_lincomb(const LinComb<T>& a, cudaStream_t s);

// Pressure bookkeeping of one SRK stage (collocated_SRK/func_global.h:356-380 and
// :391-395), one pass each.  rhs (mode 0): muj = c0 x + sum_j cm_j mujt_j with x = p
// (StabType 0) or dp/dt (1); StabType 1 also pjhat = p + cpd dp/dt + sum_j cq_j qj_j;
// bufs = muj + pjhat - cb dp/dt (1) or muj - cb p (0).  post (mode 1): pj = mujt_i +
// bufs; mujt_i -= cb (dp/dt or p); StabType 1 also qj_i = inv (pj - pjhat).
template <typename T>
struct SrkScal {
    int mode, stab, nj;
    const T* p;
    const T* dpdt;
    const T* mujt[TC_LIN_MAX];
    const T* qj[TC_LIN_MAX];
    double c0, cm[TC_LIN_MAX], cq[TC_LIN_MAX], cpd, cb, inv;
    T* bufs;
    T* pjhat;
    T* pj;
    T* mujt_i;
    T* qj_i;
    long long n;
};
template <typename T> void launch_srk_scal(const SrkScal<T>& a, cudaStream_t s);

struct RunCtl {
    unsigned iters, max_iters;
    double cfl, cfl_min, cfl_max;
};
void launch_run_ctl(cudaGraphConditionalHandle hnd, const double* planes, int NZ, int mode, RunCtl* ctl,
                    cudaStream_t s);
int flux_grid_blocks(const Geom& g);

}  // namespace tc
