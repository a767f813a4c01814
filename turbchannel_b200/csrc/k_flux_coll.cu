// k_flux_coll.cu -- fused explicit-flux kernel of the collocated scheme.
//
// Same structure as k_flux_stag.cu (32 x 8 tile, z-marching shared-memory ring of
// 4 node planes fed by cp.async, SBDF3 combine in the epilogue) with the
// collocated arithmetic of collocated_AB3/func_fluxes.h:21-120: skew-symmetric
// convection -(div + adv)/2 and either the 7-point "cross" viscosity or the
// 27-point Galerkin viscosity with nu_t on the 8 surrounding elements.  Wall nodes
// (iz = 0, NZ-1) carry no flux.  For StabType 1 the gradient of p_n is subtracted
// from the RHS in the same pass (collocated_AB3/func_global.h:436-437).
#include <algorithm>

#include "flux_ring.cuh"
#include "kernels.cuh"

namespace tc {

constexpr int CPLANES = 128;  // planes whose constants a CTA keeps in shared memory

// Galerkin viscous term, collocated_AB3/func_fluxes.h:21-85 (without the final
// 1/(hx hy hz) factor).  NUT(ex, ey, ez) = nu_t of the element with lower corner at
// the displaced node (ex, ey, ez in {-1, 0}).
template <typename T, typename ACC, typename NUT>
__device__ __forceinline__ void visc_galerkin(const ACC& A, const NUT& nut, int iz, const double* cDZ, T hx, T hy,
                                              T ihx, T ihy, T visc, T s[3]) {
    const T C9 = T(0.11111111111111111111), C18 = T(0.05555555555555555555), C36 = T(0.02777777777777777777);
    const T C3 = T(0.33333333333333333333), C6 = T(0.16666666666666666666);
    s[0] = s[1] = s[2] = 0;
#pragma unroll
    for (int oz = 0; oz <= 1; oz++) {
        const int sz = oz ? 1 : -1;
        const T hz = (T)(oz == 0 ? cDZ[iz == 0 ? 0 : iz - 1] : cDZ[iz]);
        const T inv_hz = (T)(1. / hz);
#pragma unroll
        for (int oy = 0; oy <= 1; oy++) {
            const int sy = oy ? 1 : -1;
#pragma unroll
            for (int ox = 0; ox <= 1; ox++) {
                const int sx = ox ? 1 : -1;
                const T mx = ihx * hy * hz, my = ihy * hx * hz, mz = inv_hz * hx * hy;
                T q0[3], qx[3], qy[3], qz[3], qxy[3], qxz[3], qyz[3], qxyz[3], g[3];
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    q0[c] = A(c, 0, 0, 0);
                    qx[c] = A(c, sx, 0, 0);
                    qy[c] = A(c, 0, sy, 0);
                    qz[c] = A(c, 0, 0, sz);
                    qxy[c] = A(c, sx, sy, 0);
                    qxz[c] = A(c, sx, 0, sz);
                    qyz[c] = A(c, 0, sy, sz);
                    qxyz[c] = A(c, sx, sy, sz);
                    g[c] = (C9 * (qx[c] - q0[c]) + C18 * (qxy[c] - qy[c]) + C18 * (qxz[c] - qz[c]) + C36 * (qxyz[c] - qyz[c])) * mx +
                           (C9 * (qy[c] - q0[c]) + C18 * (qxy[c] - qx[c]) + C18 * (qyz[c] - qz[c]) + C36 * (qxyz[c] - qxz[c])) * my +
                           (C9 * (qz[c] - q0[c]) + C18 * (qxz[c] - qx[c]) + C18 * (qyz[c] - qy[c]) + C36 * (qxyz[c] - qxy[c])) * mz;
                }
                T gxx = C9 * (qx[0] - q0[0]) + C18 * (qxy[0] - qy[0]) + C18 * (qxz[0] - qz[0]) + C36 * (qxyz[0] - qyz[0]);
                T gxy = T(0.25) * (C3 * (qx[1] - q0[1] + qxy[1] - qy[1]) + C6 * (qxz[1] - qz[1] + qxyz[1] - qyz[1]));
                T gxz = T(0.25) * (C3 * (qx[2] - q0[2] + qxz[2] - qz[2]) + C6 * (qxy[2] - qy[2] + qxyz[2] - qyz[2]));
                T gyy = C9 * (qy[1] - q0[1]) + C18 * (qxy[1] - qx[1]) + C18 * (qyz[1] - qz[1]) + C36 * (qxyz[1] - qxz[1]);
                T gyx = T(0.25) * (C3 * (qy[0] - q0[0] + qxy[0] - qx[0]) + C6 * (qyz[0] - qz[0] + qxyz[0] - qxz[0]));
                T gyz = T(0.25) * (C3 * (qy[2] - q0[2] + qyz[2] - qz[2]) + C6 * (qxy[2] - qx[2] + qxyz[2] - qxz[2]));
                T gzz = C9 * (qz[2] - q0[2]) + C18 * (qyz[2] - qy[2]) + C18 * (qxz[2] - qx[2]) + C36 * (qxyz[2] - qxy[2]);
                T gzx = T(0.25) * (C3 * (qz[0] - q0[0] + qxz[0] - qx[0]) + C6 * (qyz[0] - qy[0] + qxyz[0] - qxy[0]));
                T gzy = T(0.25) * (C3 * (qz[1] - q0[1] + qyz[1] - qy[1]) + C6 * (qxz[1] - qx[1] + qxyz[1] - qxy[1]));
                const T sxy = (ox ^ oy) ? T(-1) : T(1), sxz = (ox ^ oz) ? T(-1) : T(1), syz = (oy ^ oz) ? T(-1) : T(1);
                gxx *= mx;
                gxy *= hz * sxy;
                gxz *= hy * sxz;
                gyy *= my;
                gyx *= hz * sxy;
                gyz *= hx * syz;
                gzz *= mz;
                gzx *= hy * sxz;
                gzy *= hx * syz;
                g[0] += gxx + gxy + gxz;
                g[1] += gyy + gyx + gyz;
                g[2] += gzz + gzx + gzy;
                const T vc = visc + nut(ox ? 0 : -1, oy ? 0 : -1, oz ? 0 : -1);
                s[0] += g[0] * vc;
                s[1] += g[1] * vc;
                s[2] += g[2] * vc;
            }
        }
    }
}

// CY: nodes per thread along y (the tile is 32 x 8 CY nodes): two for float, one for double.
template <typename T, int VISC, bool LES, int ORDER, bool STAB1, bool VEC, int CY>
__global__ void __launch_bounds__(STX* STY, 2) k_flux_coll(FluxArgs<T> a, int tz) {
    using ACC = RingAcc<T, 1, CY>;
    constexpr int RS = ACC::RS;
    extern __shared__ __align__(16) unsigned char smraw[];
    T* ring = reinterpret_cast<T*>(smraw);
    __shared__ double sbuf[32];

    const Geom& g = a.g;
    const int NX = g.NX, NY = g.NY, NZ = g.NZ;
    const size_t NXY = (size_t)NX * NY;
    const int tx = threadIdx.x % STX, tyt = threadIdx.x / STX;
    const int x0 = blockIdx.x * STX, y0 = blockIdx.y * (STY * CY);
    const int zb = blockIdx.z * tz, ze = min(NZ, zb + tz);
    const int ix = x0 + tx;

    TileCopy<T, 1, CY, VEC> cp;
    cp.init(x0, y0, NX, NY, g.N);
    const T* vbase = a.vel.c[0];  // the three components are consecutive blocks of N
    for (int z = max(0, zb - 1); z <= min(NZ - 1, zb + 1); z++) cp.load(ring, vbase, z, NXY);
    cp_async_commit();

    const int xm = wrapi(ix - 1, NX), xp = wrapi(ix + 1, NX);
    const T hx = (T)g.hx, hy = (T)g.hy, ihx = (T)g.inv_hx, ihy = (T)g.inv_hy, visc = (T)g.visc;
    const T inv_tau = a.inv_tau, it2 = T(0.5) * a.inv_tau, it6 = a.inv_tau * T(0.16666666666666666667);
    const double* cDZ = a.m.dDZ;
    double ub = 0.0;
    // per-plane constants of the CTA's planes, once in double: 2 / (DZ[z-1] + DZ[z]),
    // visc inv_hz / DZ[z], visc inv_hz / DZ[z-1] (cross viscosity); the per-node work
    // then has no double arithmetic
    __shared__ T pc[3][CPLANES];
    for (int k = threadIdx.x; k < ze - zb && k < CPLANES; k += blockDim.x) {
        const int z = zb + k;
        if (z == 0 || z == NZ - 1) {
            pc[0][k] = pc[1][k] = pc[2][k] = T(0);
        } else {
            const double ihz = 2. / (cDZ[z - 1] + cDZ[z]);
            pc[0][k] = (T)ihz;
            pc[1][k] = (T)(g.visc * ihz / cDZ[z]);
            pc[2][k] = (T)(g.visc * ihz / cDZ[z - 1]);
        }
    }

    for (int z = zb; z < ze; z++) {
        if (z + 1 < ze && z + 2 < NZ) cp.load(ring, vbase, z + 2, NXY);
        cp_async_commit();
        const bool wall = (z == 0 || z == NZ - 1);
        // history (and, for StabType 1, p_n around the node) issued before the stencil so
        // its latency overlaps it
        T hp[CY][3], hq[CY][3], vq[CY][3], pn[CY][6];
#pragma unroll
        for (int q = 0; q < CY; q++) {
            const int iy = y0 + tyt * CY + q;
            if (ix >= NX || iy >= NY) continue;
            const size_t id = (size_t)z * NXY + (size_t)iy * NX + ix;
            if (ORDER >= 2) {
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    hp[q][c] = __ldg(a.fp.c[c] + id);
                    if (ORDER == 3) {
                        hq[q][c] = __ldg(a.fq.c[c] + id);
                        vq[q][c] = __ldg(a.velq.c[c] + id);
                    }
                }
            }
            if (STAB1 && ORDER > 0 && !wall) {
                const T* p = a.pcur + (size_t)z * NXY;
                const int ym = wrapi(iy - 1, NY), yp = wrapi(iy + 1, NY);
                pn[q][0] = __ldg(p + (size_t)iy * NX + xp);
                pn[q][1] = __ldg(p + (size_t)iy * NX + xm);
                pn[q][2] = __ldg(p + (size_t)yp * NX + ix);
                pn[q][3] = __ldg(p + (size_t)ym * NX + ix);
                pn[q][4] = __ldg(a.pcur + id + NXY);
                pn[q][5] = __ldg(a.pcur + id - NXY);
            }
        }
        cp_async_wait<1>();
        __syncthreads();
        const int kz = z - zb;
        const T inv_hz = wall ? T(0) : (kz < CPLANES ? pc[0][kz] : (T)(2. / (cDZ[z - 1] + cDZ[z])));
        ACC A0;
        A0.set(ring, z & (RS - 1), tx, tyt * CY);
#pragma unroll
        for (int q = 0; q < CY; q++) {
            const int iy = y0 + tyt * CY + q;
            if (ix >= NX || iy >= NY) continue;
            ACC A = A0;
            A.shift_rows(q);
            const size_t id = (size_t)z * NXY + (size_t)iy * NX + ix;
            T f[3] = {0, 0, 0};
            if (!wall) {
                const T invh[3] = {ihx, ihy, inv_hz};
#pragma unroll
                for (int d = 0; d < 3; d++) {
                    const int ex = d == 0, ey = d == 1, ez = d == 2;
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        const T ukc = A(c, ex, ey, ez), ujc = A(c, -ex, -ey, -ez);
                        const T ukd = A(d, ex, ey, ez), ujd = A(d, -ex, -ey, -ez);
                        const T cd = T(0.5) * (ukc * ukd - ujc * ujd);
                        const T ca = A(d, 0, 0, 0) * (T(0.5) * (ukc - ujc));
                        f[c] -= T(0.5) * (cd + ca) * invh[d];
                    }
                }
                if (VISC == TC_VISC_GALERKIN) {
                    const int ym = wrapi(iy - 1, NY);
                    auto nut = [&](int ex, int ey, int ez) -> T {
                        if (!LES) return T(0);
                        const int xx = ex < 0 ? xm : ix, yy = ey < 0 ? ym : iy;
                        return __ldg(a.nu_t + (size_t)(z + ez) * NXY + (size_t)yy * NX + xx);
                    };
                    T gv[3];
                    visc_galerkin(A, nut, z, cDZ, hx, hy, ihx, ihy, visc, gv);
#pragma unroll
                    for (int c = 0; c < 3; c++) f[c] += gv[c] * ihx * ihy * inv_hz;
                } else {
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        const T u0 = A(c, 0, 0, 0);
                        f[c] += visc * ihx * ihx * (A(c, 1, 0, 0) + A(c, -1, 0, 0) - T(2.) * u0);
                        f[c] += visc * ihy * ihy * (A(c, 0, 1, 0) + A(c, 0, -1, 0) - T(2.) * u0);
                        if (kz < CPLANES)
                            f[c] += pc[1][kz] * (A(c, 0, 0, 1) - u0) - pc[2][kz] * (u0 - A(c, 0, 0, -1));
                        else
                            f[c] += visc * (T)(((double)A(c, 0, 0, 1) - u0) / cDZ[z] - ((double)u0 - A(c, 0, 0, -1)) / cDZ[z - 1]) * inv_hz;
                    }
                }
                f[0] += (T)g.sour_dpdx;
            }
            if (ORDER == 0) {
#pragma unroll
                for (int c = 0; c < 3; c++) a.fout.c[c][id] = f[c];
            } else {
                T gp[3] = {0, 0, 0};
                if (STAB1 && !wall) {
                    gp[0] = T(0.5) * ihx * (pn[q][0] - pn[q][1]);
                    gp[1] = T(0.5) * ihy * (pn[q][2] - pn[q][3]);
                    gp[2] = T(0.5) * (pn[q][4] - pn[q][5]) / a.m.cellh[z];
                }
                T r[3];
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    const T vn = A(c, 0, 0, 0);
                    r[c] = sbdf_rhs<ORDER, T>(f[c], vn, ORDER >= 2 ? hp[q][c] : T(0), ORDER == 3 ? hq[q][c] : T(0),
                                              ORDER == 3 ? vq[q][c] : T(0), inv_tau, it6);
                    if (STAB1) r[c] -= gp[c];
                    a.fout.c[c][id] = f[c] + it2 * vn;  // A_n
                    a.rhs.c[c][id] = r[c];
                }
                ub += (double)r[0] * (double)a.m.cellh[z];
            }
        }
        __syncthreads();
    }
    if (ORDER > 0 && a.ub_out) {
        const double s = block_sum(ub, sbuf);
        grid_sum_finish(s, a.ub_partial, a.ticket, a.ub_out, sbuf);
    }
}

// nodes per thread along y: two for float, one for double (register budget of 2 CTAs/SM)
template <typename T>
constexpr int coll_cy() { return sizeof(T) == 4 ? 2 : 1; }

static void flux_coll_shape(const Geom& g, int cy, dim3& grid, int& tz) {
    const int ty = STY * cy;
    const int tiles = ((g.NX + STX - 1) / STX) * ((g.NY + ty - 1) / ty);
    int nch = std::max(1, (148 * 8 + tiles - 1) / tiles);
    tz = std::max(4, (g.NZ + nch - 1) / nch);
    grid = dim3((g.NX + STX - 1) / STX, (g.NY + ty - 1) / ty, (g.NZ + tz - 1) / tz);
}

template <typename T, int VISC, bool LES, int ORDER, bool STAB1>
static void run(const FluxArgs<T>& a, cudaStream_t s) {
    constexpr int CY = coll_cy<T>();
    constexpr size_t smem = sizeof(T) * 4 * 3 * RingAcc<T, 1, CY>::PL;
    const bool vec = a.g.NX % (16 / (int)sizeof(T)) == 0;
    auto kern = vec ? k_flux_coll<T, VISC, LES, ORDER, STAB1, true, CY> : k_flux_coll<T, VISC, LES, ORDER, STAB1, false, CY>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    dim3 grid;
    int tz;
    flux_coll_shape(a.g, CY, grid, tz);
    kern<<<grid, STX * STY, smem, s>>>(a, tz);
}

template <typename T, int VISC, bool LES>
static void run_order(const FluxArgs<T>& a, cudaStream_t s) {
    const bool st = a.pcur != nullptr;
    switch (a.order) {
        case 0: run<T, VISC, LES, 0, false>(a, s); break;
        case 1: st ? run<T, VISC, LES, 1, true>(a, s) : run<T, VISC, LES, 1, false>(a, s); break;
        case 2: st ? run<T, VISC, LES, 2, true>(a, s) : run<T, VISC, LES, 2, false>(a, s); break;
        default: st ? run<T, VISC, LES, 3, true>(a, s) : run<T, VISC, LES, 3, false>(a, s); break;
    }
}

template <typename T>
void launch_flux_coll(const FluxArgs<T>& a, cudaStream_t s) {
    if (a.g.visc_type == TC_VISC_GALERKIN) {
        if (a.nu_t) run_order<T, TC_VISC_GALERKIN, true>(a, s);
        else run_order<T, TC_VISC_GALERKIN, false>(a, s);
    } else {
        run_order<T, TC_VISC_CROSS, false>(a, s);
    }
}

template void launch_flux_coll<double>(const FluxArgs<double>&, cudaStream_t);
template void launch_flux_coll<float>(const FluxArgs<float>&, cudaStream_t);

}  // namespace tc
