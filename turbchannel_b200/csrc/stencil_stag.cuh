// stencil_stag.cuh -- per-cell arithmetic of the staggered schemes, written against
// an accessor A(c, dx, dy, dz) that returns velocity component c at the cell
// displaced by (dx, dy, dz) from the current one.  Shared by the fused flux kernel
// (reads a shared-memory ring of z-planes) and the stand-alone operator kernels.
//
//   conv_hw2   : staggered/func_global.h:345-370   (Harlow-Welch)
//   conv_vv4   : staggered/func_global.h:374-529   (Verstappen-Veldman, 'bar' x16,
//                'barbar' x16/9 scaling as in the reference)
//   visc_cross : staggered/func_global.h:533-562
//   visc_naive : staggered/func_global.h:564-625   (stress divergence, mu = visc+nu_t,
//                including the reference's mu(XR(YR)) weight in sxy_190)
//   abs_strain : staggered/func_global.h:823-870
// The INT template flag compiles a plane-interior copy: every wall special case of
// the reference is a test on iz, and for 3 <= iz <= NZ-4 (VV4) or 1 <= iz <= NZ-2
// (HW2) all of them are false, so INT = true drops them at compile time.
#pragma once
#include "tc_common.cuh"

namespace tc {

template <typename T>
struct StagZ {  // wall-normal metric at the current plane
    int iz, NZ;
    const T* DZ;
    const T* DZW;
    T hx, hy, ihx, ihy, visc;
    T pc[6];  // MeshDev::PC[TC_PC * iz + 0..5], loaded once per plane
};

template <typename T, typename ACC, bool INT = false, typename VT = T>
__device__ __forceinline__ void conv_hw2(const ACC& A, const StagZ<T>& m, VT s[3]) {
#define U(a, b, c) A(0, a, b, c)
#define V(a, b, c) A(1, a, b, c)
#define W(a, b, c) A(2, a, b, c)
    const int iz = m.iz, NZ = m.NZ;
    const T* DZ = m.DZ;
    const T inv_hz = m.pc[0];
    const T inv_hz_alt = m.pc[1];
    const VT U0 = U(0, 0, 0), V0 = V(0, 0, 0), W0 = W(0, 0, 0);
    s[0] = s[1] = s[2] = 0;
    VT a = U0 + U(1, 0, 0), c = U0 + U(-1, 0, 0);
    s[0] -= (a * a - c * c) * m.ihx;
    s[0] -= ((U0 + U(0, 1, 0)) * (V(0, 1, 0) + V(-1, 1, 0)) - (U0 + U(0, -1, 0)) * (V0 + V(-1, 0, 0))) * m.ihy;
    if ((INT || iz != NZ - 1)) s[0] -= (U0 + U(0, 0, 1)) * (W(0, 0, 1) + W(-1, 0, 1)) * inv_hz;
    if ((INT || iz != 0)) s[0] += (U0 + U(0, 0, -1)) * (W0 + W(-1, 0, 0)) * inv_hz;

    s[1] -= ((V0 + V(1, 0, 0)) * (U(1, 0, 0) + U(1, -1, 0)) - (V0 + V(-1, 0, 0)) * (U0 + U(0, -1, 0))) * m.ihx;
    a = V0 + V(0, 1, 0);
    c = V0 + V(0, -1, 0);
    s[1] -= (a * a - c * c) * m.ihy;
    if ((INT || iz != NZ - 1)) s[1] -= (V0 + V(0, 0, 1)) * (W(0, 0, 1) + W(0, -1, 1)) * inv_hz;
    if ((INT || iz != 0)) s[1] += (V0 + V(0, 0, -1)) * (W0 + W(0, -1, 0)) * inv_hz;

    if ((INT || iz != 0)) {
        s[2] -= ((W0 + W(1, 0, 0)) * (U(1, 0, 0) * DZ[iz] + U(1, 0, -1) * DZ[iz - 1]) -
                 (W0 + W(-1, 0, 0)) * (U0 * DZ[iz] + U(0, 0, -1) * DZ[iz - 1])) * m.ihx * inv_hz_alt;
        s[2] -= ((W0 + W(0, 1, 0)) * (V(0, 1, 0) * DZ[iz] + V(0, 1, -1) * DZ[iz - 1]) -
                 (W0 + W(0, -1, 0)) * (V0 * DZ[iz] + V(0, 0, -1) * DZ[iz - 1])) * m.ihy * inv_hz_alt;
        a = W0 + ((!INT && iz == NZ - 1) ? VT(0) : W(0, 0, 1));
        s[2] -= a * a * inv_hz_alt;
        a = W0 + W(0, 0, -1);
        s[2] += a * a * inv_hz_alt;
    }
    s[0] *= T(0.25);
    s[1] *= T(0.25);
    s[2] *= T(0.25);
}

template <typename T, typename ACC, bool INT = false, typename VT = T>
__device__ __forceinline__ void conv_vv4(const ACC& A, const StagZ<T>& m, T gcz, VT s[3]) {
    const int iz = m.iz, NZ = m.NZ;
    const T *DZ = m.DZ, *DZW = m.DZW;
    const T hx = m.hx, hy = m.hy, dz = DZ[iz], dzw = DZW[iz], hxhy = hx * hy;
    const T C27 = T(0.03703703703703703703), C9 = T(0.11111111111111111111);
    const VT U0 = U(0, 0, 0), V0 = V(0, 0, 0), W0 = W(0, 0, 0);
    s[0] = s[1] = s[2] = 0;
    {  // u: x-faces
        VT br = dz * hy * (9 * (U0 + U(1, 0, 0)) - (U(-1, 0, 0) + U(2, 0, 0)));
        VT bl = dz * hy * (9 * (U(-1, 0, 0) + U0) - (U(-2, 0, 0) + U(1, 0, 0)));
        VT bbr = dzw * hy * (9 * (U(1, 0, 0) + U(2, 0, 0)) - (U0 + U(3, 0, 0)));
        VT bbl = dzw * hy * (9 * (U(-2, 0, 0) + U(-1, 0, 0)) - (U(-3, 0, 0) + U0));
        s[0] += br * (U0 + U(1, 0, 0)) - C27 * bbr * (U0 + U(3, 0, 0)) - bl * (U(-1, 0, 0) + U0) + C27 * bbl * (U(-3, 0, 0) + U0);
    }
    {  // u: y-faces
        VT br = dz * hx * (9 * (V(0, 1, 0) + V(-1, 1, 0)) - (V(-2, 1, 0) + V(1, 1, 0)));
        VT bl = dz * hx * (9 * (V0 + V(-1, 0, 0)) - (V(-2, 0, 0) + V(1, 0, 0)));
        VT bbr = dzw * hx * (9 * (V(0, 2, 0) + V(-1, 2, 0)) - (V(-2, 2, 0) + V(1, 2, 0)));
        VT bbl = dzw * hx * (9 * (V(0, -1, 0) + V(-1, -1, 0)) - (V(-2, -1, 0) + V(1, -1, 0)));
        s[0] += br * (U0 + U(0, 1, 0)) - C27 * bbr * (U0 + U(0, 3, 0)) - bl * (U(0, -1, 0) + U0) + C27 * bbl * (U(0, -3, 0) + U0);
    }
    {  // u: z-faces
        VT wzl, wzr, wbzl, wbzr;
        if ((!INT && iz == 0)) wzl = 0;
        else wzl = hxhy * (9 * (W0 + W(-1, 0, 0)) - (W(-2, 0, 0) + W(1, 0, 0)));
        if ((!INT && iz == NZ - 1)) wzr = 0;
        else wzr = hxhy * (9 * (W(0, 0, 1) + W(-1, 0, 1)) - (W(-2, 0, 1) + W(1, 0, 1)));
        if ((!INT && iz == 1)) wbzl = 0;
        else if ((!INT && iz == 0)) wbzl = wzr;
        else wbzl = hxhy * (9 * (W(0, 0, -1) + W(-1, 0, -1)) - (W(-2, 0, -1) + W(1, 0, -1)));
        if ((!INT && iz == NZ - 2)) wbzr = 0;
        else if ((!INT && iz == NZ - 1)) wbzr = wzl;
        else wbzr = hxhy * (9 * (W(0, 0, 2) + W(-1, 0, 2)) - (W(-2, 0, 2) + W(1, 0, 2)));
        VT uzr = (!INT && iz == NZ - 1) ? VT(0) : U0 + U(0, 0, 1);
        VT uzrr = U0 + ((!INT && iz == NZ - 3) ? -U(0, 0, 2) : (!INT && iz == NZ - 2) ? VT(0) : (!INT && iz == NZ - 1) ? U(0, 0, -2) : U(0, 0, 3));
        VT uzl = (!INT && iz == 0) ? VT(0) : U(0, 0, -1) + U0;
        VT uzll = U0 + ((!INT && iz == 2) ? -U(0, 0, -2) : (!INT && iz == 1) ? VT(0) : (!INT && iz == 0) ? U(0, 0, 2) : U(0, 0, -3));
        s[0] += wzr * uzr - C27 * wbzr * uzrr - wzl * uzl + C27 * wbzl * uzll;
    }
    {  // v: x-faces
        VT br = dz * hy * (9 * (U(1, 0, 0) + U(1, -1, 0)) - (U(1, -2, 0) + U(1, 1, 0)));
        VT bl = dz * hy * (9 * (U0 + U(0, -1, 0)) - (U(0, -2, 0) + U(0, 1, 0)));
        VT bbr = dzw * hy * (9 * (U(2, 0, 0) + U(2, -1, 0)) - (U(2, -2, 0) + U(2, 1, 0)));
        VT bbl = dzw * hy * (9 * (U(-1, 0, 0) + U(-1, -1, 0)) - (U(-1, -2, 0) + U(-1, 1, 0)));
        s[1] += br * (V0 + V(1, 0, 0)) - C27 * bbr * (V0 + V(3, 0, 0)) - bl * (V(-1, 0, 0) + V0) + C27 * bbl * (V(-3, 0, 0) + V0);
    }
    {  // v: y-faces
        VT br = dz * hx * (9 * (V0 + V(0, 1, 0)) - (V(0, -1, 0) + V(0, 2, 0)));
        VT bl = dz * hx * (9 * (V(0, -1, 0) + V0) - (V(0, -2, 0) + V(0, 1, 0)));
        VT bbr = dzw * hx * (9 * (V(0, 1, 0) + V(0, 2, 0)) - (V0 + V(0, 3, 0)));
        VT bbl = dzw * hx * (9 * (V(0, -2, 0) + V(0, -1, 0)) - (V(0, -3, 0) + V0));
        s[1] += br * (V0 + V(0, 1, 0)) - C27 * bbr * (V0 + V(0, 3, 0)) - bl * (V(0, -1, 0) + V0) + C27 * bbl * (V(0, -3, 0) + V0);
    }
    {  // v: z-faces
        VT wzl, wzr, wbzl, wbzr;
        if ((!INT && iz == 0)) wzl = 0;
        else wzl = hxhy * (9 * (W0 + W(0, -1, 0)) - (W(0, -2, 0) + W(0, 1, 0)));
        if ((!INT && iz == NZ - 1)) wzr = 0;
        else wzr = hxhy * (9 * (W(0, 0, 1) + W(0, -1, 1)) - (W(0, -2, 1) + W(0, 1, 1)));
        if ((!INT && iz == 1)) wbzl = 0;
        else if ((!INT && iz == 0)) wbzl = wzr;
        else wbzl = hxhy * (9 * (W(0, 0, -1) + W(0, -1, -1)) - (W(0, -2, -1) + W(0, 1, -1)));
        if ((!INT && iz == NZ - 2)) wbzr = 0;
        else if ((!INT && iz == NZ - 1)) wbzr = wzl;
        else wbzr = hxhy * (9 * (W(0, 0, 2) + W(0, -1, 2)) - (W(0, -2, 2) + W(0, 1, 2)));
        VT vzr = (!INT && iz == NZ - 1) ? VT(0) : V0 + V(0, 0, 1);
        VT vzrr = V0 + ((!INT && iz == NZ - 3) ? -V(0, 0, 2) : (!INT && iz == NZ - 2) ? VT(0) : (!INT && iz == NZ - 1) ? V(0, 0, -2) : V(0, 0, 3));
        VT vzl = (!INT && iz == 0) ? VT(0) : V(0, 0, -1) + V0;
        VT vzll = V0 + ((!INT && iz == 2) ? -V(0, 0, -2) : (!INT && iz == 1) ? VT(0) : (!INT && iz == 0) ? V(0, 0, 2) : V(0, 0, -3));
        s[1] += wzr * vzr - C27 * wbzr * vzrr - wzl * vzl + C27 * wbzl * vzll;
    }
    if ((INT || iz != 0)) {
        {  // w: x-faces, mass flux averaged to the w-face in z
            VT br, bl, bbr, bbl;
            br = 9 * (U(1, 0, 0) * DZ[iz] + U(1, 0, -1) * DZ[iz - 1]);
            br -= ((!INT && iz == 1)) ? -U(1, 0, -1) * DZ[0] : U(1, 0, -2) * DZ[iz - 2];
            br -= ((!INT && iz == NZ - 1)) ? -U(1, 0, 0) * DZ[NZ - 1] : U(1, 0, 1) * DZ[iz + 1];
            br *= hy;
            bl = 9 * (U0 * DZ[iz] + U(0, 0, -1) * DZ[iz - 1]);
            bl -= ((!INT && iz == 1)) ? -U(0, 0, -1) * DZ[0] : U(0, 0, -2) * DZ[iz - 2];
            bl -= ((!INT && iz == NZ - 1)) ? -U0 * DZ[NZ - 1] : U(0, 0, 1) * DZ[iz + 1];
            bl *= hy;
            bbr = 9 * (U(2, 0, 0) * DZW[iz] + U(2, 0, -1) * DZW[iz - 1]);
            bbr -= ((!INT && iz == 1)) ? -U(2, 0, -1) * DZW[0] : U(2, 0, -2) * DZW[iz - 2];
            bbr -= ((!INT && iz == NZ - 1)) ? -U(2, 0, 0) * DZW[NZ - 1] : U(2, 0, 1) * DZW[iz + 1];
            bbr *= hy;
            bbl = 9 * (U(-1, 0, 0) * DZW[iz] + U(-1, 0, -1) * DZW[iz - 1]);
            bbl -= ((!INT && iz == 1)) ? -U(-1, 0, -1) * DZW[0] : U(-1, 0, -2) * DZW[iz - 2];
            bbl -= ((!INT && iz == NZ - 1)) ? -U(-1, 0, 0) * DZW[NZ - 1] : U(-1, 0, 1) * DZW[iz + 1];
            bbl *= hy;
            s[2] += br * (W0 + W(1, 0, 0)) - C27 * bbr * (W0 + W(3, 0, 0)) - bl * (W(-1, 0, 0) + W0) + C27 * bbl * (W(-3, 0, 0) + W0);
        }
        {  // w: y-faces (scaled by hy as in staggered/func_global.h:475-487)
            VT br, bl, bbr, bbl;
            br = 9 * (V(0, 1, 0) * DZ[iz] + V(0, 1, -1) * DZ[iz - 1]);
            br -= ((!INT && iz == 1)) ? -V(0, 1, -1) * DZ[0] : V(0, 1, -2) * DZ[iz - 2];
            br -= ((!INT && iz == NZ - 1)) ? -V(0, 1, 0) * DZ[NZ - 1] : V(0, 1, 1) * DZ[iz + 1];
            br *= hy;
            bl = 9 * (V0 * DZ[iz] + V(0, 0, -1) * DZ[iz - 1]);
            bl -= ((!INT && iz == 1)) ? -V(0, 0, -1) * DZ[0] : V(0, 0, -2) * DZ[iz - 2];
            bl -= ((!INT && iz == NZ - 1)) ? -V0 * DZ[NZ - 1] : V(0, 0, 1) * DZ[iz + 1];
            bl *= hy;
            bbr = 9 * (V(0, 2, 0) * DZW[iz] + V(0, 2, -1) * DZW[iz - 1]);
            bbr -= ((!INT && iz == 1)) ? -V(0, 2, -1) * DZW[0] : V(0, 2, -2) * DZW[iz - 2];
            bbr -= ((!INT && iz == NZ - 1)) ? -V(0, 2, 0) * DZW[NZ - 1] : V(0, 2, 1) * DZW[iz + 1];
            bbr *= hy;
            bbl = 9 * (V(0, -1, 0) * DZW[iz] + V(0, -1, -1) * DZW[iz - 1]);
            bbl -= ((!INT && iz == 1)) ? -V(0, -1, -1) * DZW[0] : V(0, -1, -2) * DZW[iz - 2];
            bbl -= ((!INT && iz == NZ - 1)) ? -V(0, -1, 0) * DZW[NZ - 1] : V(0, -1, 1) * DZW[iz + 1];
            bbl *= hy;
            s[2] += br * (W0 + W(0, 1, 0)) - C27 * bbr * (W0 + W(0, 3, 0)) - bl * (W(0, -1, 0) + W0) + C27 * bbl * (W(0, -3, 0) + W0);
        }
        {  // w: z-faces
            VT wzl = W(0, 0, -1);
            VT wzr = (!INT && iz == NZ - 1) ? VT(0) : W(0, 0, 1);
            VT wzll = (!INT && iz == 1) ? W0 : W(0, 0, -2);
            VT wzrr = (!INT && iz == NZ - 2) ? VT(0) : (!INT && iz == NZ - 1) ? W0 : W(0, 0, 2);
            VT wzlll = (!INT && iz == 1) ? W(0, 0, 1) : (!INT && iz == 2) ? W(0, 0, -1) : W(0, 0, -3);
            VT wzrrr = (!INT && iz == NZ - 3) ? VT(0) : (!INT && iz == NZ - 2) ? W(0, 0, 1) : (!INT && iz == NZ - 1) ? W(0, 0, -1) : W(0, 0, 3);
            VT bl = hxhy * (9 * (wzl + W0) - (wzll + wzr));
            VT br = hxhy * (9 * (W0 + wzr) - (wzl + wzrr));
            VT bbl = hxhy * (9 * (wzll + wzl) - (wzlll + W0));
            VT bbr = hxhy * (9 * (wzr + wzrr) - (W0 + wzrrr));
            s[2] += br * (W0 + wzr) - bl * (wzl + W0);
            if ((INT || iz < NZ - 2)) s[2] -= C27 * bbr * (W0 + wzrrr);
            else if ((!INT && iz == NZ - 2)) s[2] -= C27 * bbr * (-W(0, 0, 1) + W0);
            else s[2] -= C27 * bbr * (W(0, 0, -1) + W0);
            if ((INT || iz > 2)) s[2] += C27 * bbl * (wzlll + W0);
            else if ((!INT && iz == 2)) s[2] += C27 * bbl * (-W(0, 0, -1) + W0);
            else s[2] += C27 * bbl * (W(0, 0, 1) + W0);
        }
    }
    const T miv = m.pc[4];
    s[0] *= miv;
    s[1] *= miv;
    s[2] *= m.pc[5];
}

template <typename T, typename ACC, bool INT = false, typename VT = T>
__device__ __forceinline__ void visc_cross(const ACC& A, const StagZ<T>& m, VT s[3]) {
    const int iz = m.iz, NZ = m.NZ;
    const T* DZ = m.DZ;
    const T inv_hz = m.pc[0];
    const T inv_hz_alt = m.pc[1];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        const VT v0 = A(c, 0, 0, 0);
        s[c] = m.ihx * m.ihx * (A(c, 1, 0, 0) + A(c, -1, 0, 0) - T(2.) * v0);
        s[c] += m.ihy * m.ihy * (A(c, 0, 1, 0) + A(c, 0, -1, 0) - T(2.) * v0);
    }
    const VT U0 = U(0, 0, 0), V0 = V(0, 0, 0), W0 = W(0, 0, 0);
    if ((INT || iz != NZ - 1)) {
        const T up = m.pc[2];
        s[0] += (U(0, 0, 1) - U0) * up * inv_hz;
        s[1] += (V(0, 0, 1) - V0) * up * inv_hz;
        s[2] += (W(0, 0, 1) - W0) * inv_hz * inv_hz_alt;
    } else {
        const T up = m.pc[2];
        s[0] += (-U0) * up * inv_hz;
        s[1] += (-V0) * up * inv_hz;
        s[2] += (-W0) * inv_hz * inv_hz_alt;
    }
    if ((INT || iz != 0)) {
        s[0] += (U(0, 0, -1) - U0) * inv_hz_alt * inv_hz;
        s[1] += (V(0, 0, -1) - V0) * inv_hz_alt * inv_hz;
        s[2] += (W(0, 0, -1) - W0) * m.pc[3] * inv_hz_alt;
    } else {
        s[0] += (-U0) * inv_hz_alt * inv_hz;
        s[1] += (-V0) * inv_hz_alt * inv_hz;
    }
    s[0] *= m.visc;
    s[1] *= m.visc;
    s[2] *= m.visc;
}

// MUF(dx, dy, dz) returns visc + nu_t at the displaced cell (or visc for DNS).
template <typename T, typename ACC, typename MUF, bool INT = false>
__device__ __forceinline__ void visc_naive(const ACC& A, const MUF& MU, const StagZ<T>& m, T s[3]) {
    const int iz = m.iz, NZ = m.NZ;
    const T *DZ = m.DZ, ihx = m.ihx, ihy = m.ihy, visc = m.visc;
    const T inv_hz = m.pc[0];
    const T up = m.pc[2];
    const T dn = m.pc[1];
    const T U0 = U(0, 0, 0), V0 = V(0, 0, 0), W0 = W(0, 0, 0);
    const T q = T(0.25);
    const T mu0 = MU(0, 0, 0), muxl = MU(-1, 0, 0), muyl = MU(0, -1, 0);
    s[0] = s[1] = s[2] = 0;
    const T sxx000 = 2 * (U(1, 0, 0) - U0) * ihx * mu0;
    const T sxx800 = 2 * (U0 - U(-1, 0, 0)) * ihx * muxl;
    s[0] += (sxx000 - sxx800) * ihx;
    const T sxy910 = ((U(0, 1, 0) - U0) * ihy + (V(0, 1, 0) - V(-1, 1, 0)) * ihx) * q * (mu0 + muxl + MU(0, 1, 0) + MU(-1, 1, 0));
    const T sxy990 = ((U0 - U(0, -1, 0)) * ihy + (V0 - V(-1, 0, 0)) * ihx) * q * (muyl + MU(-1, -1, 0) + mu0 + muxl);
    s[0] += (sxy910 - sxy990) * ihy;
    const T sxz901 = ((!INT && iz == NZ - 1)) ? (-2 * U0 * inv_hz * visc)
                                    : ((U(0, 0, 1) - U0) * up + (W(0, 0, 1) - W(-1, 0, 1)) * ihx) * q * (mu0 + muxl + MU(0, 0, 1) + MU(-1, 0, 1));
    const T sxz909 = ((!INT && iz == 0)) ? (2 * U0 * inv_hz * visc)
                               : ((U0 - U(0, 0, -1)) * dn + (W0 - W(-1, 0, 0)) * ihx) * q * (MU(0, 0, -1) + MU(-1, 0, -1) + mu0 + muxl);
    s[0] += (sxz901 - sxz909) * inv_hz;

    const T sxy190 = ((U(1, 0, 0) - U(1, -1, 0)) * ihy + (V(1, 0, 0) - V0) * ihx) * q * (mu0 + MU(1, 0, 0) + muyl + MU(1, 1, 0));
    s[1] += (sxy190 - sxy990) * ihx;
    const T syy000 = 2 * (V(0, 1, 0) - V0) * ihy * mu0;
    const T syy080 = 2 * (V0 - V(0, -1, 0)) * ihy * muyl;
    s[1] += (syy000 - syy080) * ihy;
    const T syz091 = ((!INT && iz == NZ - 1)) ? (-2 * V0 * inv_hz * visc)
                                    : ((V(0, 0, 1) - V0) * up + (W(0, 0, 1) - W(0, -1, 1)) * ihy) * q * (mu0 + muyl + MU(0, 0, 1) + MU(0, -1, 1));
    const T syz099 = ((!INT && iz == 0)) ? (2 * V0 * inv_hz * visc)
                               : ((V0 - V(0, 0, -1)) * dn + (W0 - W(0, -1, 0)) * ihy) * q * (MU(0, 0, -1) + MU(0, -1, -1) + mu0 + muyl);
    s[1] += (syz091 - syz099) * inv_hz;

    if ((!INT && iz == 0)) return;
    const T sxz109 = ((U(1, 0, 0) - U(1, 0, -1)) * dn + (W(1, 0, 0) - W0) * ihx) * q * (MU(0, 0, -1) + MU(1, 0, -1) + mu0 + MU(1, 0, 0));
    s[2] += (sxz109 - sxz909) * ihx;
    const T syz019 = ((V(0, 1, 0) - V(0, 1, -1)) * dn + (W(0, 1, 0) - W0) * ihy) * q * (MU(0, 0, -1) + MU(0, 1, -1) + mu0 + MU(0, 1, 0));
    s[2] += (syz019 - syz099) * ihy;
    const T szz000 = 2 * (((!INT && iz == NZ - 1) ? T(0) : W(0, 0, 1)) - W0) * inv_hz * mu0;
    const T szz008 = 2 * (W0 - W(0, 0, -1)) * MU(0, 0, -1) / DZ[iz - 1];
    s[2] += (szz000 - szz008) * dn;
}

template <typename T, typename ACC>
__device__ __forceinline__ T abs_strain(const ACC& A, const StagZ<T>& m) {
    const int iz = m.iz, NZ = m.NZ;
    const T *DZ = m.DZ, ihx = m.ihx, ihy = m.ihy;
    const T inv_hz = m.pc[0];
    const T up = m.pc[2];
    const T dn = m.pc[1];
    const T U0 = U(0, 0, 0), V0 = V(0, 0, 0), W0 = W(0, 0, 0);
    const T sxx = (U(1, 0, 0) - U0) * ihx;
    const T syy = (V(0, 1, 0) - V0) * ihy;
    const T szz = ((iz == NZ - 1 ? T(0) : W(0, 0, 1)) - W0) * inv_hz;
    T S = sxx * sxx + syy * syy + szz * szz;
    {
        T a = (U(0, 1, 0) - U0) * ihy + (V(0, 1, 0) - V(-1, 1, 0)) * ihx;
        T c = (U0 - U(0, -1, 0)) * ihy + (V0 - V(-1, 0, 0)) * ihx;
        T d = (U(1, 1, 0) - U(1, 0, 0)) * ihy + (V(1, 1, 0) - V(0, 1, 0)) * ihx;
        T e = (U(1, 0, 0) - U(1, -1, 0)) * ihy + (V(1, 0, 0) - V0) * ihx;
        S += T(0.125) * (a * a + c * c + d * d + e * e);
    }
    {
        T a = (iz == NZ - 1) ? (-2 * U0 * inv_hz) : (U(0, 0, 1) - U0) * up + (W(0, 0, 1) - W(-1, 0, 1)) * ihx;
        T c = (iz == 0) ? (2 * U0 * inv_hz) : (U0 - U(0, 0, -1)) * dn + (W0 - W(-1, 0, 0)) * ihx;
        T d = (iz == NZ - 1) ? (-2 * U(1, 0, 0) * inv_hz) : (U(1, 0, 1) - U(1, 0, 0)) * up + (W(1, 0, 1) - W(0, 0, 1)) * ihx;
        T e = (iz == 0) ? (2 * U(1, 0, 0) * inv_hz) : (U(1, 0, 0) - U(1, 0, -1)) * dn + (W(1, 0, 0) - W0) * ihx;
        S += T(0.125) * (a * a + c * c + d * d + e * e);
    }
    {
        T a = (iz == NZ - 1) ? (-2 * V0 * inv_hz) : (V(0, 0, 1) - V0) * up + (W(0, 0, 1) - W(0, -1, 1)) * ihy;
        T c = (iz == 0) ? (2 * V0 * inv_hz) : (V0 - V(0, 0, -1)) * dn + (W0 - W(0, -1, 0)) * ihy;
        T d = (iz == NZ - 1) ? (-2 * V(0, 1, 0) * inv_hz) : (V(0, 1, 1) - V(0, 1, 0)) * up + (W(0, 1, 1) - W(0, 0, 1)) * ihy;
        T e = (iz == 0) ? (2 * V(0, 1, 0) * inv_hz) : (V(0, 1, 0) - V(0, 1, -1)) * dn + (W(0, 1, 0) - W0) * ihy;
        S += T(0.125) * (a * a + c * c + d * d + e * e);
    }
    return sqrt(2 * S);
}
#undef U
#undef V
#undef W

}  // namespace tc
