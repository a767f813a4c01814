// k_misc.cu -- velocity correction, Smagorinsky viscosity, stand-alone operators,
// fused per-plane diagnostics and the host-boundary layout conversions.
#include <algorithm>

#include "kernels.cuh"
#include "stencil_div.cuh"
#include "stencil_stag.cuh"

namespace tc {

constexpr int KX = 32, KY = 8;

// ---------------------------------------------------------------------------
// Gradient + correction.  ApplyGradient: HW2 staggered/func_global.h:297-303,
// VV4 :316-322, collocated collocated_AB3/func_global.h:298-303; correction
// staggered/func_global.h:939-941, collocated_AB3/func_global.h:430-448.
// Each thread marches a column of z; x/y neighbours of p come through L1.
// ---------------------------------------------------------------------------
// Gradient of p at (ix, iy, z) from the column values p(z-2..z+1) and the x/y
// neighbours (plane z) loaded by the caller.
template <typename T, int SCHEME>
__device__ __forceinline__ void grad_at(const CorrArgs<T>& a, int z, int NZ, T p0, T pxm, T pxmm, T pxp, T pym, T pymm,
                                        T pyp, T pzm, T pzmm, T pzp, T gp[3]) {
    const T ihx = (T)a.g.inv_hx, ihy = (T)a.g.inv_hy;
    if (SCHEME == TC_SCHEME_HW2) {
        gp[0] = ihx * (p0 - pxm);
        gp[1] = ihy * (p0 - pym);
        gp[2] = z == 0 ? T(0) : (p0 - pzm) * (2 / (a.m.DZ[z] + a.m.DZ[z - 1]));
    } else if (SCHEME == TC_SCHEME_VV4) {
        const T g1 = a.m.GC1[z], g2 = a.m.GC2[z];
        gp[0] = ihx * (g1 * (p0 - pxm) + g2 * (pxp - pxmm));
        gp[1] = ihy * (g1 * (p0 - pym) + g2 * (pyp - pymm));
        if (z == 0) {
            gp[2] = 0;
        } else {
            const T pr = z == NZ - 1 ? -p0 : pzp;
            const T pll = z == 1 ? -pzm : pzmm;
            gp[2] = ((p0 - pzm) - T(0.03703703703703703703) * (pr - pll)) * a.m.GCZ[z];
        }
    } else {
        if (z == 0 || z == NZ - 1) {
            gp[0] = gp[1] = gp[2] = 0;
        } else {
            gp[0] = T(0.5) * ihx * (pxp - pxm);
            gp[1] = T(0.5) * ihy * (pyp - pym);
            gp[2] = T(0.5) * (pzp - pzm) / a.m.cellh[z];
        }
    }
}

// Each thread owns a column of ZC planes; all loads of the column are issued
// before any arithmetic so that they are in flight together.
constexpr int ZC = 4;

template <typename T, int SCHEME, bool STAB1, bool GRADONLY>
__global__ void __launch_bounds__(KX* KY) k_correct(CorrArgs<T> a, int tz) {
    const Geom& g = a.g;
    const int NX = g.NX, NY = g.NY, NZ = g.NZ;
    const size_t NXY = (size_t)NX * NY;
    const int ix = blockIdx.x * KX + threadIdx.x % KX, iy = blockIdx.y * KY + threadIdx.x / KX;
    if (ix >= NX || iy >= NY) return;
    const int zb = blockIdx.z * ZC;
    const int xm = wrapi(ix - 1, NX), xmm = wrapi(ix - 2, NX), xp = wrapi(ix + 1, NX);
    const int ym = wrapi(iy - 1, NY), ymm = wrapi(iy - 2, NY), yp = wrapi(iy + 1, NY);
    const T* __restrict__ p = a.p;
    T du = 0;
    if (!GRADONLY && a.cfr) {
        const double ub = (*a.ub_sum) * a.cfr_scale * (double)a.tob;
        const double d = (a.cfr_target - ub) * a.cfr_volfac;
        du = (T)d;
        if (blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0 && threadIdx.x == 0) *a.du_out = d;
    }
    // column values p(zb-2 .. zb+ZC) at (ix, iy); zero outside the domain (never used there)
    T col[ZC + 3];
#pragma unroll
    for (int k = 0; k < ZC + 3; k++) {
        const int z = zb - 2 + k;
        col[k] = (z >= 0 && z < NZ) ? __ldg(p + (size_t)z * NXY + (size_t)iy * NX + ix) : T(0);
    }
    T nb[ZC][6], rh[ZC][3], pc[ZC];
#pragma unroll
    for (int k = 0; k < ZC; k++) {
        const int z = zb + k;
        if (z >= NZ) break;
        const size_t pl = (size_t)z * NXY;
        nb[k][0] = __ldg(p + pl + (size_t)iy * NX + xm);
        nb[k][1] = __ldg(p + pl + (size_t)iy * NX + xmm);
        nb[k][2] = __ldg(p + pl + (size_t)iy * NX + xp);
        nb[k][3] = __ldg(p + pl + (size_t)ym * NX + ix);
        nb[k][4] = __ldg(p + pl + (size_t)ymm * NX + ix);
        nb[k][5] = __ldg(p + pl + (size_t)yp * NX + ix);
        if (!GRADONLY) {
            const size_t id = pl + (size_t)iy * NX + ix;
#pragma unroll
            for (int c = 0; c < 3; c++) rh[k][c] = __ldg(a.rhs.c[c] + id);
            if (STAB1) pc[k] = __ldg(a.pcur + id);
        }
    }
#pragma unroll
    for (int k = 0; k < ZC; k++) {
        const int z = zb + k;
        if (z >= NZ) break;
        const size_t id = (size_t)z * NXY + (size_t)iy * NX + ix;
        T gp[3];
        grad_at<T, SCHEME>(a, z, NZ, col[k + 2], nb[k][0], nb[k][1], nb[k][2], nb[k][3], nb[k][4], nb[k][5], col[k + 1],
                           col[k], col[k + 3], gp);
        if (GRADONLY) {
#pragma unroll
            for (int c = 0; c < 3; c++) a.vout.c[c][id] = gp[c];
        } else {
#pragma unroll
            for (int c = 0; c < 3; c++) a.vout.c[c][id] = (rh[k][c] - gp[c]) * a.tob;
            if (a.cfr && !(SCHEME == TC_SCHEME_COLLOC && (z == 0 || z == NZ - 1))) a.vout.c[0][id] += du;
            if (STAB1) a.pnext[id] = col[k + 2] + pc[k];
        }
    }
}

// The step's correction with four x-adjacent cells per thread (NX % 4 == 0): the
// pressure row x-4..x+7, the y-neighbour rows and the RHS are read as 16-byte
// vectors (the periodic wrap moves whole 4-cell chunks), so a thread issues about a
// quarter of the load instructions of k_correct.  Same expressions as k_correct.
constexpr int QX = 32, QY = 8;  // quads x rows per CTA
template <typename T>
__device__ __forceinline__ void st4(T* p, const T v[4]) {
    if constexpr (sizeof(T) == 4) {
        *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
    } else {
        reinterpret_cast<double2*>(p)[0] = make_double2(v[0], v[1]);
        reinterpret_cast<double2*>(p)[1] = make_double2(v[2], v[3]);
    }
}

// ZN planes per thread: 2 for float, 1 for double (register budget).
template <typename T>
constexpr int correct_quad_planes() { return sizeof(T) == 4 ? 2 : 1; }

// Three CTAs per SM (at most 85 registers; measured at 384x256x384: float 0.178 against
// 0.186 ms with 96 registers and two CTAs, double 0.362 against 0.367).
template <typename T, int SCHEME, bool STAB1>
__global__ void __launch_bounds__(QX* QY, 3) k_correct_quad(CorrArgs<T> a) {
    constexpr int ZN = correct_quad_planes<T>();
    const Geom& g = a.g;
    const int NX = g.NX, NY = g.NY, NZ = g.NZ, NQ = NX >> 2;
    const size_t NXY = (size_t)NX * NY;
    const int xq = blockIdx.x * QX + threadIdx.x % QX, iy = blockIdx.y * QY + threadIdx.x / QX;
    if (xq >= NQ || iy >= NY) return;
    // float: planes in descending z, so that the next step's flux kernel (marching up from
    // z = 0) finds the last-written low planes in L2; double keeps ascending planes, the
    // reverse of its descending inverse x-FFT
    const int x = 4 * xq, zb = (sizeof(T) == 4 ? (int)(gridDim.z - 1 - blockIdx.z) : (int)blockIdx.z) * ZN;
    const int xl = x == 0 ? NX - 4 : x - 4, xr = x + 4 == NX ? 0 : x + 4;
    const int ym = wrapi(iy - 1, NY), ymm = wrapi(iy - 2, NY), yp = wrapi(iy + 1, NY);
    const T* __restrict__ p = a.p;
    T du = 0;
    if (a.cfr) {
        const double ub = (*a.ub_sum) * a.cfr_scale * (double)a.tob;
        const double d = (a.cfr_target - ub) * a.cfr_volfac;
        du = (T)d;
        if (blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0 && threadIdx.x == 0) *a.du_out = d;
    }
    const size_t row = (size_t)iy * NX;
    Acc4<T> col[ZN + 3];  // p(zb-2 .. zb+ZN) at x..x+3; zero outside the domain (never used there)
#pragma unroll
    for (int k = 0; k < ZN + 3; k++) {
        const int z = zb - 2 + k;
        if (z >= 0 && z < NZ) col[k] = ld4(p + (size_t)z * NXY + row + x);
        else {
#pragma unroll
            for (int j = 0; j < 4; j++) col[k].v[j] = T(0);
        }
    }
    Acc4<T> pl4[ZN], pr4[ZN], pym[ZN], pymm[ZN], pyp[ZN], rh[ZN][3], pc[ZN];
#pragma unroll
    for (int k = 0; k < ZN; k++) {
        const int z = zb + k;
        if (z >= NZ) break;
        const size_t pl = (size_t)z * NXY;
        pl4[k] = ld4(p + pl + row + xl);
        pr4[k] = ld4(p + pl + row + xr);
        pym[k] = ld4(p + pl + (size_t)ym * NX + x);
        pymm[k] = ld4(p + pl + (size_t)ymm * NX + x);
        pyp[k] = ld4(p + pl + (size_t)yp * NX + x);
#pragma unroll
        for (int c = 0; c < 3; c++) rh[k][c] = ld4(a.rhs.c[c] + pl + row + x);
        if (STAB1) pc[k] = ld4(a.pcur + pl + row + x);
    }
#pragma unroll
    for (int k = 0; k < ZN; k++) {
        const int z = zb + k;
        if (z >= NZ) break;
        const size_t id = (size_t)z * NXY + row + x;
        T e[12];  // p at x-4 .. x+7 on plane z
#pragma unroll
        for (int j = 0; j < 4; j++) {
            e[j] = pl4[k].v[j];
            e[4 + j] = col[k + 2].v[j];
            e[8 + j] = pr4[k].v[j];
        }
        T o[3][4], pn[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            T gp[3];
            grad_at<T, SCHEME>(a, z, NZ, e[4 + j], e[3 + j], e[2 + j], e[5 + j], pym[k].v[j], pymm[k].v[j], pyp[k].v[j],
                               col[k + 1].v[j], col[k].v[j], col[k + 3].v[j], gp);
#pragma unroll
            for (int c = 0; c < 3; c++) o[c][j] = (rh[k][c].v[j] - gp[c]) * a.tob;
            if (a.cfr && !(SCHEME == TC_SCHEME_COLLOC && (z == 0 || z == NZ - 1))) o[0][j] += du;
            if (STAB1) pn[j] = col[k + 2].v[j] + pc[k].v[j];
        }
#pragma unroll
        for (int c = 0; c < 3; c++) st4(a.vout.c[c] + id, o[c]);
        if (STAB1) st4(a.pnext + id, pn);
    }
}

template <typename T, int SCHEME>
void launch_correct_diag(const CorrArgs<T>& a, cudaStream_t s);

static void column_shape(const Geom& g, dim3& grid, int& tz) {
    tz = ZC;
    grid = dim3((g.NX + KX - 1) / KX, (g.NY + KY - 1) / KY, (g.NZ + tz - 1) / tz);
}

template <typename T, int SCHEME>
static void correct_scheme(const CorrArgs<T>& a, cudaStream_t s) {
    if constexpr (SCHEME != TC_SCHEME_COLLOC) {
        if (a.dpart && !a.grad_only && !a.pnext && a.g.NX % 4 == 0) {
            launch_correct_diag<T, SCHEME>(a, s);
            return;
        }
    }
    if (!a.grad_only && a.g.NX % 4 == 0) {
        constexpr int ZN = correct_quad_planes<T>();
        const dim3 gq((a.g.NX / 4 + QX - 1) / QX, (a.g.NY + QY - 1) / QY, (a.g.NZ + ZN - 1) / ZN);
        if (a.pnext) k_correct_quad<T, SCHEME, true><<<gq, QX * QY, 0, s>>>(a);
        else k_correct_quad<T, SCHEME, false><<<gq, QX * QY, 0, s>>>(a);
        return;
    }
    dim3 grid;
    int tz;
    column_shape(a.g, grid, tz);
    if (a.grad_only) k_correct<T, SCHEME, false, true><<<grid, KX * KY, 0, s>>>(a, tz);
    else if (a.pnext) k_correct<T, SCHEME, true, false><<<grid, KX * KY, 0, s>>>(a, tz);
    else k_correct<T, SCHEME, false, false><<<grid, KX * KY, 0, s>>>(a, tz);
}

template <typename T>
void launch_correct(const CorrArgs<T>& a, cudaStream_t s) {
    if (a.g.scheme == TC_SCHEME_VV4) correct_scheme<T, TC_SCHEME_VV4>(a, s);
    else if (a.g.scheme == TC_SCHEME_HW2) correct_scheme<T, TC_SCHEME_HW2>(a, s);
    else correct_scheme<T, TC_SCHEME_COLLOC>(a, s);
}

// ---------------------------------------------------------------------------
// Smagorinsky-van Driest eddy viscosity.  Staggered: per cell,
// staggered/func_global.h:875-890 with |S| of :823-870.  Collocated: per element
// (lower-corner node index), collocated_AB3/func_global.h:342-384.
// ---------------------------------------------------------------------------
template <typename T>
struct GAcc {
    const T* v[3];
    int ix, iy, iz, NX, NY;
    size_t NXY;
    __device__ __forceinline__ T operator()(int c, int dx, int dy, int dz) const {
        const int x = wrapi(ix + dx, NX), y = wrapi(iy + dy, NY);
        return __ldg(v[c] + (size_t)(iz + dz) * NXY + (size_t)y * NX + x);
    }
};

template <typename T>
__device__ __forceinline__ T smag_nut(T AbsS, T dist, T vol, T inv_ls) {
    const T yp = dist * inv_ls;
    const T C_SMAG = T(0.1), C_exp = T(0.04 * 0.04 * 0.04);
    const T fvd = 1 - exp(-C_exp * yp * yp * yp);
    T Dl = C_SMAG * pow(vol, T(0.33333333333333333333));
    if (Dl > T(0.41) * dist) Dl = T(0.41) * dist;
    return fvd * Dl * Dl * AbsS;
}

template <typename T>
__global__ void __launch_bounds__(256) k_turb_stag(TurbArgs<T> a) {
    const Geom& g = a.g;
    const long long in = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (in >= g.N) return;
    const int ix = (int)(in % g.NX), iy = (int)((in / g.NX) % g.NY), iz = (int)(in / g.NXY);
    GAcc<T> A{{a.v.c[0], a.v.c[1], a.v.c[2]}, ix, iy, iz, g.NX, g.NY, (size_t)g.NXY};
    StagZ<T> mz{iz, g.NZ, a.m.DZ, a.m.DZW, (T)g.hx, (T)g.hy, (T)g.inv_hx, (T)g.inv_hy, (T)g.visc, {}};
#pragma unroll
    for (int k = 0; k < 6; k++) mz.pc[k] = a.m.PC[TC_PC * iz + k];
    const T S = abs_strain(A, mz);
    const T* ZZ = a.m.ZZ;
    const T H = T(0.5) * (ZZ[g.NZ] - ZZ[0]);
    const T Z = T(0.5) * (ZZ[iz] + ZZ[iz + 1]) - ZZ[0];
    const T d = (Z < H) ? Z : 2 * H - Z;
    a.nu_t[in] = smag_nut(S, d, (T)g.hx * (T)g.hy * a.m.DZ[iz], (T)g.inv_ls);
}

template <typename T>
__global__ void __launch_bounds__(256) k_turb_coll(TurbArgs<T> a) {
    const Geom& g = a.g;
    const long long ie = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (ie >= g.N) return;
    const int ix = (int)(ie % g.NX), iy = (int)((ie / g.NX) % g.NY), iz = (int)(ie / g.NXY);
    if (iz >= g.NZ - 1) return;
    GAcc<T> A{{a.v.c[0], a.v.c[1], a.v.c[2]}, ix, iy, iz, g.NX, g.NY, (size_t)g.NXY};
    const T hz = (T)a.m.dDZ[iz];
    const T ihx = (T)g.inv_hx, ihy = (T)g.inv_hy;
    T gr[3][3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        const T q = A(c, 0, 0, 0), qx = A(c, 1, 0, 0), qy = A(c, 0, 1, 0), qxy = A(c, 1, 1, 0);
        const T qz = A(c, 0, 0, 1), qxz = A(c, 1, 0, 1), qyz = A(c, 0, 1, 1), qxyz = A(c, 1, 1, 1);
        gr[0][c] = ((qx + qxy + qxz + qxyz) - (q + qy + qz + qyz)) * (T(0.25) * ihx);
        gr[1][c] = ((qy + qxy + qyz + qxyz) - (q + qx + qz + qxz)) * (T(0.25) * ihy);
        gr[2][c] = ((qz + qxz + qyz + qxyz) - (q + qx + qy + qxy)) / (4 * hz);
    }
    gr[0][1] = T(0.5) * (gr[0][1] + gr[1][0]);
    gr[0][2] = T(0.5) * (gr[0][2] + gr[2][0]);
    gr[1][2] = T(0.5) * (gr[1][2] + gr[2][1]);
    T S = gr[0][0] * gr[0][0] + gr[1][1] * gr[1][1] + gr[2][2] * gr[2][2] +
          2 * (gr[0][1] * gr[0][1] + gr[0][2] * gr[0][2] + gr[1][2] * gr[1][2]);
    S = sqrt(2 * S);
    const double* ZZ = a.m.dZZ;
    const T H = (T)(0.5 * (ZZ[g.NZ - 1] - ZZ[0]));
    const T Z = (T)(0.5 * (ZZ[iz] + ZZ[iz + 1]));
    const T d = (Z < H) ? Z : 2 * H - Z;
    a.nu_t[ie] = smag_nut(S, d, (T)g.hx * (T)g.hy * hz, (T)g.inv_ls);
}

template <typename T>
void launch_turb(const TurbArgs<T>& a, cudaStream_t s) {
    const unsigned nb = (unsigned)((a.g.N + 255) / 256);
    if (a.g.scheme == TC_SCHEME_COLLOC) k_turb_coll<T><<<nb, 256, 0, s>>>(a);
    else k_turb_stag<T><<<nb, 256, 0, s>>>(a);
}

// ---------------------------------------------------------------------------
// Stand-alone divergence (operator form of ApplyDivergence)
// ---------------------------------------------------------------------------
template <typename T, int SCHEME>
__global__ void __launch_bounds__(256) k_divergence(DivArgs<T> a) {
    const Geom& g = a.g;
    const long long in = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (in >= g.N) return;
    const int ix = (int)(in % g.NX), iy = (int)((in / g.NX) % g.NY), iz = (int)(in / g.NXY);
    a.dv[in] = div_at<T, SCHEME, false>(g, a.m, a.v, nullptr, ix, iy, iz);
}

template <typename T>
void launch_divergence(const DivArgs<T>& a, cudaStream_t s) {
    const unsigned nb = (unsigned)((a.g.N + 255) / 256);
    if (a.g.scheme == TC_SCHEME_VV4) k_divergence<T, TC_SCHEME_VV4><<<nb, 256, 0, s>>>(a);
    else if (a.g.scheme == TC_SCHEME_HW2) k_divergence<T, TC_SCHEME_HW2><<<nb, 256, 0, s>>>(a);
    else k_divergence<T, TC_SCHEME_COLLOC><<<nb, 256, 0, s>>>(a);
}

// ---------------------------------------------------------------------------
// Per-plane diagnostics in double: one CTA per z-plane.
// planes[z*TC_DIAG_STRIDE + k]: 0..2 sum u, v, w_c; 3..8 sum uu, vv, w_cw_c, uv, uw_c,
// vw_c; 9 sum nu_t; 10 sum p; 11 sum pp; 12 sum w (raw); 13 sum w^2 (raw); 14..15
// unused (0); 16..18 max CFL convective / viscous / both.  (CalcProfiles,
// CalcIntegral, CalcKineticEnergy, CalcCFL: staggered/func_global.h:678-808.)
// ---------------------------------------------------------------------------
constexpr int NDIAG = NDIAG_SUMS;
static_assert(NDIAG + 3 == TC_DIAG_STRIDE, "diagnostics layout");

// Stage 1: CTA (z, s) reduces chunk s of plane z into part[(z*S + s)*STRIDE + k];
// stage 2 sums the S chunks of every (z, k) in index order (deterministic).  Chunks
// are multiples of 4 cells (NX*NY is), read as 16-byte vectors of 4 cells, so each
// thread keeps 5-6 vector loads in flight per iteration.
template <typename T>
__global__ void __launch_bounds__(256) k_diag(DiagArgs<T> a, double* part, int S) {
    const Geom& g = a.g;
    const int z = blockIdx.x, s = blockIdx.y;
    const int NX = g.NX, NZ = g.NZ;
    const size_t NXY = (size_t)NX * g.NY;
    const size_t per = ((NXY + 4 * S - 1) / (4 * S)) * 4, j0 = (size_t)s * per, j1 = min(NXY, j0 + per);
    const bool coll = g.scheme == TC_SCHEME_COLLOC;
    double sm[NDIAG];
#pragma unroll
    for (int k = 0; k < NDIAG; k++) sm[k] = 0;
    // per-cell arithmetic and this thread's sums over its chunk (8 groups of 4 cells at
    // most) in the working type T, promoted to double once; the plane sums across threads
    // stay double
    T mconv = 0, mvisc = 0, mboth = 0;
    const T ihx = (T)g.inv_hx, ihy = (T)g.inv_hy;
    const T ihz = coll ? T(1) / a.m.cellh[z] : T(1) / a.m.DZ[z];
    const T kv = coll ? (g.visc_type == TC_VISC_GALERKIN ? T(2) : T(1)) : (g.visc_type != TC_VISC_CROSS ? T(2) : T(1));
    const T lap = ihx * ihx + ihy * ihy + ihz * ihz;
    const T tau = (T)a.tau, visc = (T)g.visc;
    const size_t pl = (size_t)z * NXY;
    const bool wtop = !coll && z == NZ - 1;  // staggered: w above the top cell is the wall (0)
    T s4[NDIAG];
#pragma unroll
    for (int k = 0; k < NDIAG; k++) s4[k] = 0;
    for (size_t j = j0 + 4 * threadIdx.x; j < j1; j += 4 * blockDim.x) {
        const size_t id = pl + j;
        const Acc4<T> U = ld4(a.v.c[0] + id), V = ld4(a.v.c[1] + id), W = ld4(a.v.c[2] + id);
        Acc4<T> WN, P, NT;
        if (!coll && !wtop) WN = ld4(a.v.c[2] + id + NXY);
        if (a.p) P = ld4(a.p + id);
        if (a.nu_t) NT = ld4(a.nu_t + id);
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const T u = U.v[q], v = V.v[q], w = W.v[q];
            const T wc = coll ? w : T(0.5) * (w + (wtop ? T(0) : WN.v[q]));
            s4[0] += u; s4[1] += v; s4[2] += wc;
            s4[3] += u * u; s4[4] += v * v; s4[5] += wc * wc; s4[6] += u * v; s4[7] += u * wc; s4[8] += v * wc;
            T nt = 0;
            if (a.nu_t) {
                s4[9] += NT.v[q];
                if (!coll) nt = NT.v[q];
                else if (z != 0 && z != NZ - 1) {
                    const size_t jj = j + q;
                    const int ix = (int)(jj % NX), iy = (int)(jj / NX);
                    const int xm = ix == 0 ? NX - 1 : ix - 1, ym = iy == 0 ? g.NY - 1 : iy - 1;
                    const T* n = a.nu_t;
                    const size_t p0 = pl, p1 = p0 - NXY;
                    nt = T(0.125) * (n[p0 + iy * NX + ix] + n[p0 + iy * NX + xm] + n[p0 + ym * NX + ix] + n[p0 + ym * NX + xm] +
                                     n[p1 + iy * NX + ix] + n[p1 + iy * NX + xm] + n[p1 + ym * NX + ix] + n[p1 + ym * NX + xm]);
                }
            }
            const T p = a.p ? P.v[q] : T(0);
            s4[10] += p; s4[11] += p * p; s4[12] += w; s4[13] += w * w;
            const T cc = tau * (fabs(u) * ihx + fabs(v) * ihy + fabs(w) * ihz);
            const T cv = 4 * kv * tau * (visc + nt) * lap;
            mconv = fmax(mconv, cc);
            mvisc = fmax(mvisc, cv);
            mboth = fmax(mboth, cc + cv);
        }
    }
#pragma unroll
    for (int k = 0; k < NDIAG; k++) sm[k] = (double)s4[k];
    __shared__ double sb[NDIAG + 3][8];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NDIAG; k++) {
        const double r = warp_sum(sm[k]);
        if (lane == 0) sb[k][wid] = r;
    }
    const double m0 = warp_max((double)mconv), m1 = warp_max((double)mvisc), m2 = warp_max((double)mboth);
    if (lane == 0) {
        sb[NDIAG][wid] = m0;
        sb[NDIAG + 1][wid] = m1;
        sb[NDIAG + 2][wid] = m2;
    }
    __syncthreads();
    if (threadIdx.x < NDIAG + 3) {
        const int k = threadIdx.x;
        double r = sb[k][0];
        for (int w2 = 1; w2 < (int)(blockDim.x >> 5); w2++) r = k < NDIAG ? r + sb[k][w2] : fmax(r, sb[k][w2]);
        part[((size_t)z * S + s) * TC_DIAG_STRIDE + k] = r;
    }
}

__global__ void k_diag_finish(const double* part, double* planes, int NZ, int S) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= NZ * TC_DIAG_STRIDE) return;
    const int z = t / TC_DIAG_STRIDE, k = t - z * TC_DIAG_STRIDE;
    double r = part[((size_t)z * S) * TC_DIAG_STRIDE + k];
    for (int s = 1; s < S; s++) {
        const double x = part[((size_t)z * S + s) * TC_DIAG_STRIDE + k];
        r = k < NDIAG ? r + x : fmax(r, x);
    }
    planes[(size_t)z * TC_DIAG_STRIDE + k] = r;
}

int diag_chunks(const Geom& g) {
    // about 8 warps per SM worth of CTAs in total, at most one chunk per 2048 cells
    const long long nxy = (long long)g.NX * g.NY;
    int S = (int)std::min<long long>(64, std::max<long long>(1, nxy / 2048));
    while (S > 1 && (long long)S * g.NZ > 148 * 32) S--;
    // at most 8 groups of 4 cells per thread (256 threads): k_diag's per-thread sums in
    // the working type stay short
    return (int)std::max<long long>(S, (nxy + 8191) / 8192);
}

// ---------------------------------------------------------------------------
// Correction with the diagnostics of the new level fused in (staggered schemes).
// Same correction as k_correct_quad; each thread also corrects w on the plane above
// its chunk (the centred w of its top plane needs it), accumulates the k_diag sums of
// its 4 x ZN cells per plane in double, and each CTA writes one partial per plane
// (layout of k_diag's part[z][chunk][k], chunk = the CTA's xy index) for
// k_diag_finish.
// ---------------------------------------------------------------------------
int correct_diag_chunks(const Geom& g) {
    return ((g.NX / 4 + QX - 1) / QX) * ((g.NY + QY - 1) / QY);
}

template <typename T, int SCHEME>
__global__ void __launch_bounds__(QX* QY) k_correct_diag(CorrArgs<T> a) {
    constexpr int ZN = correct_quad_planes<T>();
    const Geom& g = a.g;
    const int NX = g.NX, NY = g.NY, NZ = g.NZ, NQ = NX >> 2;
    const size_t NXY = (size_t)NX * NY;
    const int xq = blockIdx.x * QX + threadIdx.x % QX, iy = blockIdx.y * QY + threadIdx.x / QX;
    const bool act = xq < NQ && iy < NY;
    const int x = 4 * (act ? xq : 0), zb = blockIdx.z * ZN, yy = act ? iy : 0;
    const int xl = x == 0 ? NX - 4 : x - 4, xr = x + 4 == NX ? 0 : x + 4;
    const int ym = wrapi(yy - 1, NY), ymm = wrapi(yy - 2, NY), yp = wrapi(yy + 1, NY);
    const T* __restrict__ p = a.p;
    T du = 0;
    if (a.cfr) {
        const double ub = (*a.ub_sum) * a.cfr_scale * (double)a.tob;
        const double d = (a.cfr_target - ub) * a.cfr_volfac;
        du = (T)d;
        if (blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0 && threadIdx.x == 0) *a.du_out = d;
    }
    const size_t row = (size_t)yy * NX;
    Acc4<T> col[ZN + 4];  // p(zb-2 .. zb+ZN+1)
#pragma unroll
    for (int k = 0; k < ZN + 4; k++) {
        const int z = zb - 2 + k;
        if (act && z >= 0 && z < NZ) col[k] = ld4(p + (size_t)z * NXY + row + x);
        else {
#pragma unroll
            for (int j = 0; j < 4; j++) col[k].v[j] = T(0);
        }
    }
    T o[ZN][3][4];
    T wtop[4] = {T(0), T(0), T(0), T(0)};  // corrected w on plane zb+ZN (0 at the top wall)
#pragma unroll
    for (int k = 0; k < ZN; k++) {
        const int z = zb + k;
        if (!act || z >= NZ) continue;
        const size_t pl = (size_t)z * NXY;
        const Acc4<T> pl4 = ld4(p + pl + row + xl), pr4 = ld4(p + pl + row + xr);
        const Acc4<T> pym = ld4(p + pl + (size_t)ym * NX + x), pymm = ld4(p + pl + (size_t)ymm * NX + x),
                      pyp = ld4(p + pl + (size_t)yp * NX + x);
        Acc4<T> rh[3];
#pragma unroll
        for (int c = 0; c < 3; c++) rh[c] = ld4(a.rhs.c[c] + pl + row + x);
        T e[12];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            e[j] = pl4.v[j];
            e[4 + j] = col[k + 2].v[j];
            e[8 + j] = pr4.v[j];
        }
#pragma unroll
        for (int j = 0; j < 4; j++) {
            T gp[3];
            grad_at<T, SCHEME>(a, z, NZ, e[4 + j], e[3 + j], e[2 + j], e[5 + j], pym.v[j], pymm.v[j], pyp.v[j],
                               col[k + 1].v[j], col[k].v[j], col[k + 3].v[j], gp);
#pragma unroll
            for (int c = 0; c < 3; c++) o[k][c][j] = (rh[c].v[j] - gp[c]) * a.tob;
            if (a.cfr) o[k][0][j] += du;
        }
#pragma unroll
        for (int c = 0; c < 3; c++) st4(a.vout.c[c] + pl + row + x, o[k][c]);
    }
    if (act && zb + ZN < NZ) {  // w on the plane above: the z-component of the gradient only
        const int z = zb + ZN;
        const Acc4<T> rw = ld4(a.rhs.c[2] + (size_t)z * NXY + row + x);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            T gp[3];
            grad_at<T, SCHEME>(a, z, NZ, col[ZN + 2].v[j], T(0), T(0), T(0), T(0), T(0), T(0), col[ZN + 1].v[j],
                               col[ZN].v[j], col[ZN + 3].v[j], gp);
            wtop[j] = (rw.v[j] - gp[2]) * a.tob;
        }
    }
    // per-plane sums (k_diag's definitions) and the CTA reduction
    __shared__ double sb[NDIAG + 3][QX * QY / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int S = gridDim.x * gridDim.y, sidx = blockIdx.y * gridDim.x + blockIdx.x;
    const double ihx = g.inv_hx, ihy = g.inv_hy;
#pragma unroll
    for (int k = 0; k < ZN; k++) {
        const int z = zb + k;
        if (z >= NZ) break;  // uniform over the CTA
        // this thread's 4 cells in the working precision T (float in the mixed mode), the
        // warp and CTA sums in double
        T sm[NDIAG];
#pragma unroll
        for (int q = 0; q < NDIAG; q++) sm[q] = T(0);
        T mconv = 0, mvisc = 0, mboth = 0;
        const T ihz = T(1) / a.m.DZ[z], tihx = (T)ihx, tihy = (T)ihy;
        const T lap = tihx * tihx + tihy * tihy + ihz * ihz, tau = (T)a.dtau, kv4 = (T)(4 * a.dkv);
        if (act) {
            const size_t id = (size_t)z * NXY + row + x;
            Acc4<T> NT;
            if (a.nu_t) NT = ld4(a.nu_t + id);
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const T u = o[k][0][j], v = o[k][1][j], w = o[k][2][j];
                const T wn = k + 1 < ZN ? o[k + 1][2][j] : wtop[j];
                const T wc = T(0.5) * (w + (z == NZ - 1 ? T(0) : wn));
                sm[0] += u; sm[1] += v; sm[2] += wc;
                sm[3] += u * u; sm[4] += v * v; sm[5] += wc * wc; sm[6] += u * v; sm[7] += u * wc; sm[8] += v * wc;
                T nt = 0;
                if (a.nu_t) {
                    nt = NT.v[j];
                    sm[9] += nt;
                }
                const T pv = col[k + 2].v[j];
                sm[10] += pv; sm[11] += pv * pv; sm[12] += w; sm[13] += w * w;
                const T cc = tau * (fabs(u) * tihx + fabs(v) * tihy + fabs(w) * ihz);
                const T cv = kv4 * tau * ((T)g.visc + nt) * lap;
                mconv = fmax(mconv, cc);
                mvisc = fmax(mvisc, cv);
                mboth = fmax(mboth, cc + cv);
            }
        }
#pragma unroll
        for (int q = 0; q < NDIAG; q++) {
            const double r = warp_sum((double)sm[q]);
            if (lane == 0) sb[q][wid] = r;
        }
        const double m0 = warp_max((double)mconv), m1 = warp_max((double)mvisc), m2 = warp_max((double)mboth);
        if (lane == 0) {
            sb[NDIAG][wid] = m0;
            sb[NDIAG + 1][wid] = m1;
            sb[NDIAG + 2][wid] = m2;
        }
        __syncthreads();
        if (threadIdx.x < NDIAG + 3) {
            const int q = threadIdx.x;
            double r = sb[q][0];
            for (int w2 = 1; w2 < QX * QY / 32; w2++) r = q < NDIAG ? r + sb[q][w2] : fmax(r, sb[q][w2]);
            a.dpart[((size_t)z * S + sidx) * TC_DIAG_STRIDE + q] = r;
        }
        __syncthreads();
    }
}

template <typename T, int SCHEME>
void launch_correct_diag(const CorrArgs<T>& a, cudaStream_t s) {
    constexpr int ZN = correct_quad_planes<T>();
    const dim3 gq((a.g.NX / 4 + QX - 1) / QX, (a.g.NY + QY - 1) / QY, (a.g.NZ + ZN - 1) / ZN);
    k_correct_diag<T, SCHEME><<<gq, QX * QY, 0, s>>>(a);
}

// Time averaging on the device: acc[z][k] += w * planes[z][k] / NXY for the 12 profile
// sums of a plane, acc[NZ*12] += w (the total weight).
__global__ void k_stats_acc(const double* __restrict__ planes, double* __restrict__ acc, int NZ, double inv_nxy,
                            double w) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < NZ * 12) acc[e] += w * planes[(e / 12) * TC_DIAG_STRIDE + e % 12] * inv_nxy;
    else if (e == NZ * 12) acc[e] += w;
}

// The loop condition of a device-controlled run: the CFL number (maximum over the
// planes of the chosen estimate, slots 16..18 of the diagnostics) of the level just
// written, then continue while bodies remain and the CFL lies in [cfl_min, cfl_max]
// (a NaN stops the loop).  One CTA.
__global__ void __launch_bounds__(256) k_run_ctl(cudaGraphConditionalHandle hnd, const double* __restrict__ planes,
                                                 int NZ, int mode, RunCtl* ctl) {
    __shared__ double sb[8];
    double m = 0.0;
    bool nan = false;
    for (int z = threadIdx.x; z < NZ; z += blockDim.x) {
        const double c = planes[(size_t)z * TC_DIAG_STRIDE + 15 + mode];
        nan |= !(c == c);
        m = fmax(m, c);
    }
    nan = __syncthreads_or(nan);
    m = warp_max(m);
    if ((threadIdx.x & 31) == 0) sb[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); w++) m = fmax(m, sb[w]);
        m = fmax(m, sb[0]);
        const double cfl = nan ? __longlong_as_double(0x7ff8000000000000LL) : m;
        const unsigned it = ctl->iters + 1;
        ctl->iters = it;
        ctl->cfl = cfl;
        const bool go = it < ctl->max_iters && cfl >= ctl->cfl_min && cfl <= ctl->cfl_max;
        cudaGraphSetConditional(hnd, go ? 1u : 0u);
    }
}

void launch_run_ctl(cudaGraphConditionalHandle hnd, const double* planes, int NZ, int mode, RunCtl* ctl,
                    cudaStream_t s) {
    k_run_ctl<<<1, 256, 0, s>>>(hnd, planes, NZ, mode, ctl);
}

void launch_stats_acc(const double* planes, double* acc, int NZ, double inv_nxy, double w, cudaStream_t s) {
    const int n = NZ * 12 + 1;
    k_stats_acc<<<(n + 255) / 256, 256, 0, s>>>(planes, acc, NZ, inv_nxy, w);
}

void launch_diag_finish(const double* part, double* planes, int NZ, int S, cudaStream_t s) {
    const int n = NZ * TC_DIAG_STRIDE;
    k_diag_finish<<<(n + 255) / 256, 256, 0, s>>>(part, planes, NZ, S);
}

template <typename T>
void launch_diag(const DiagArgs<T>& a, cudaStream_t s) {
    const int S = diag_chunks(a.g);
    k_diag<T><<<dim3(a.g.NZ, S), 256, 0, s>>>(a, a.part, S);
    const int n = a.g.NZ * TC_DIAG_STRIDE;
    k_diag_finish<<<(n + 255) / 256, 256, 0, s>>>(a.part, a.planes, a.g.NZ, S);
}

// ---------------------------------------------------------------------------
// Layout conversions at the host boundary.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_aos_to_soa(const double* __restrict__ src, V3<T> dst, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        dst.c[0][i] = (T)src[3 * i];
        dst.c[1][i] = (T)src[3 * i + 1];
        dst.c[2][i] = (T)src[3 * i + 2];
    }
}
template <typename T>
__global__ void k_soa_to_aos(CV3<T> src, double* __restrict__ dst, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        dst[3 * i] = (double)src.c[0][i];
        dst[3 * i + 1] = (double)src.c[1][i];
        dst[3 * i + 2] = (double)src.c[2][i];
    }
}
template <typename T>
__global__ void k_d2t(const double* __restrict__ src, T* __restrict__ dst, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[i] = (T)src[i];
}
template <typename T>
__global__ void k_t2d(const T* __restrict__ src, double* __restrict__ dst, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[i] = (double)src[i];
}

static unsigned conv_blocks(long long n) { return (unsigned)std::min<long long>((n + 255) / 256, 148 * 32); }

template <typename T>
void launch_aos_to_soa(const double* src, V3<T> dst, long long n, cudaStream_t s) {
    k_aos_to_soa<T><<<conv_blocks(n), 256, 0, s>>>(src, dst, n);
}
template <typename T>
void launch_soa_to_aos(CV3<T> src, double* dst, long long n, cudaStream_t s) {
    k_soa_to_aos<T><<<conv_blocks(n), 256, 0, s>>>(src, dst, n);
}
template <typename T>
void launch_d2t(const double* src, T* dst, long long n, cudaStream_t s) {
    k_d2t<T><<<conv_blocks(n), 256, 0, s>>>(src, dst, n);
}
template <typename T>
void launch_t2d(const T* src, double* dst, long long n, cudaStream_t s) {
    k_t2d<T><<<conv_blocks(n), 256, 0, s>>>(src, dst, n);
}

#define TC_INST(T)                                                                 \
    template void launch_correct<T>(const CorrArgs<T>&, cudaStream_t);            \
    template void launch_turb<T>(const TurbArgs<T>&, cudaStream_t);               \
    template void launch_divergence<T>(const DivArgs<T>&, cudaStream_t);          \
    template void launch_diag<T>(const DiagArgs<T>&, cudaStream_t);               \
    template void launch_aos_to_soa<T>(const double*, V3<T>, long long, cudaStream_t); \
    template void launch_soa_to_aos<T>(CV3<T>, double*, long long, cudaStream_t); \
    template void launch_d2t<T>(const double*, T*, long long, cudaStream_t);      \
    template void launch_t2d<T>(const T*, double*, long long, cudaStream_t);
TC_INST(double)
TC_INST(float)
#undef TC_INST

// ---------------------------------------------------------------------------
// Linear combinations of device arrays (SRK stage updates)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_lincomb(LinComb<T> a) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride) {
        T acc = (T)a.c[0] * a.x[0][i];
        for (int k = 1; k < a.nt; k++) acc += (T)a.c[k] * a.x[k][i];
        if (a.post != 1.0) acc = (T)a.post * acc;
        a.out[i] = acc;
    }
}

// The same combination over 16-byte vectors (n a multiple of the vector width, every
// pointer 16-byte aligned): identical arithmetic per element, a quarter (float) or half
// (double) of the load instructions.
template <typename T>
__global__ void __launch_bounds__(256) k_lincomb_v(LinComb<T> a) {
    constexpr int W = 16 / sizeof(T);
    using V = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
    const long long nv = a.n / W;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += stride) {
        T acc[W];
        {
            const V x = reinterpret_cast<const V*>(a.x[0])[i];
            const T* xe = reinterpret_cast<const T*>(&x);
#pragma unroll
            for (int w = 0; w < W; w++) acc[w] = (T)a.c[0] * xe[w];
        }
        for (int k = 1; k < a.nt; k++) {
            const V x = reinterpret_cast<const V*>(a.x[k])[i];
            const T* xe = reinterpret_cast<const T*>(&x);
            const T c = (T)a.c[k];
#pragma unroll
            for (int w = 0; w < W; w++) acc[w] += c * xe[w];
        }
        if (a.post != 1.0) {
#pragma unroll
            for (int w = 0; w < W; w++) acc[w] = (T)a.post * acc[w];
        }
        V o;
        T* oe = reinterpret_cast<T*>(&o);
#pragma unroll
        for (int w = 0; w < W; w++) oe[w] = acc[w];
        reinterpret_cast<V*>(a.out)[i] = o;
    }
}

template <typename T>
void launch_lincomb(const LinComb<T>& a, cudaStream_t s) {
    constexpr int W = 16 / sizeof(T);
    bool vec = a.n % W == 0 && (reinterpret_cast<uintptr_t>(a.out) & 15) == 0;
    for (int k = 0; k < a.nt; k++) vec = vec && (reinterpret_cast<uintptr_t>(a.x[k]) & 15) == 0;
    if (vec) {
        const long long nb = std::min<long long>((a.n / W + 255) / 256, 148LL * 16);
        k_lincomb_v<T><<<(unsigned)std::max<long long>(nb, 1), 256, 0, s>>>(a);
        return;
    }
    const long long nb = std::min<long long>((a.n + 255) / 256, 148LL * 16);
    k_lincomb<T><<<(unsigned)std::max<long long>(nb, 1), 256, 0, s>>>(a);
}
template void launch_lincomb<double>(const LinComb<double>&, cudaStream_t);
template void launch_lincomb<float>(const LinComb<float>&, cudaStream_t);

template <typename T>
__global__ void __launch_bounds__(256) k_srk_scal(SrkScal<T> a) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride) {
        const T x = a.stab ? a.dpdt[i] : a.p[i];
        if (a.mode == 0) {
            T muj = (T)a.c0 * x;
            for (int j = 0; j < a.nj; j++) muj += (T)a.cm[j] * a.mujt[j][i];
            if (a.stab) {
                T pjhat = a.p[i];
                if (a.cpd != 0.0) pjhat += (T)a.cpd * x;
                for (int j = 0; j < a.nj; j++) pjhat += (T)a.cq[j] * a.qj[j][i];
                a.pjhat[i] = pjhat;
                a.bufs[i] = muj + pjhat - (T)a.cb * x;
            } else {
                a.bufs[i] = muj - (T)a.cb * x;
            }
        } else {
            const T m = a.mujt_i[i];
            const T pj = m + a.bufs[i];
            a.pj[i] = pj;
            a.mujt_i[i] = m - (T)a.cb * x;
            if (a.stab) a.qj_i[i] = (T)a.inv * (pj - a.pjhat[i]);
        }
    }
}

template <typename T>
void launch_srk_scal(const SrkScal<T>& a, cudaStream_t s) {
    const long long nb = std::min<long long>((a.n + 255) / 256, 148LL * 16);
    k_srk_scal<T><<<(unsigned)std::max<long long>(nb, 1), 256, 0, s>>>(a);
}
template void launch_srk_scal<double>(const SrkScal<double>&, cudaStream_t);
template void launch_srk_scal<float>(const SrkScal<float>&, cudaStream_t);

}  // namespace tc
