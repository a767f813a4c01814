// stencil_vv4_int.cuh -- the VV4 convection and CROSS viscosity of interior planes in the
// regrouped form of the flux kernels' fast path, for any value type VT with +, -, * and a
// vfma(a, b, c) = a b + c found by argument-dependent lookup (the packed float pair of
// k_flux_pair.cu) or declared here (double).
#pragma once
#include "tc_common.cuh"

namespace tc {

// Interior planes of VV4 with the CROSS viscosity (3 <= z <= NZ-4): the arithmetic of
// conv_vv4 / visc_cross (INT = true) regrouped for FMAs, with the 24 plane constants K
// (host-computed in double, see fill_flux_plane_consts in tc_api.cu; float2 pairs in the
// float pair kernel, doubles in the FP64 kernel):
// every fourth-order interpolant 9 s - t is formed negated, t - 9 s (one FMA, no
// negation needed), a face pair's fluxes Ir pr - Il pl as nl pl - nr pr, and each
// direction's narrow and wide pairs are accumulated with their scale factors (the
// reference's dz hy, C27 dzw hy, ... times the plane's momentum or w scale) folded
// into K.  Same stencils and face fluxes as the reference (staggered/func_global.h:
// 374-529 and 533-562); only the rounding order differs.

__device__ __forceinline__ double vfma(double a, double b, double c) { return __fma_rn(a, b, c); }
// t - 9 s
template <class VT>
__device__ __forceinline__ VT ni(VT s, VT t) { return vfma(VT(-9.f), s, t); }
// nl pl - nr pr
template <class VT>
__device__ __forceinline__ VT pd(VT nl, VT pl, VT nr, VT pr) { return nl * pl - nr * pr; }

#define U(a, b, c) A(0, a, b, c)
#define V(a, b, c) A(1, a, b, c)
#define W(a, b, c) A(2, a, b, c)
template <class VT, class ACC>
__device__ __forceinline__ void visc_cross_int(const ACC& A, const VT* K, VT s[3]) {
#pragma unroll
    for (int c = 0; c < 3; c++) {
        const VT v0 = A(c, 0, 0, 0);
        const VT tx = vfma(VT(-2.f), v0, A(c, 1, 0, 0) + A(c, -1, 0, 0));
        const VT ty = vfma(VT(-2.f), v0, A(c, 0, 1, 0) + A(c, 0, -1, 0));
        VT r = vfma(K[22], tx, s[c]);
        r = vfma(K[23], ty, r);
        r = vfma(K[c < 2 ? 18 : 20], A(c, 0, 0, 1) - v0, r);
        s[c] = vfma(K[c < 2 ? 19 : 21], A(c, 0, 0, -1) - v0, r);
    }
}

template <class VT, class ACC>
__device__ __forceinline__ void conv_vv4_int(const ACC& A, const VT* K, VT s[3]) {
    {  // u: x-faces
        const VT U0 = U(0, 0, 0), Um1 = U(-1, 0, 0), Up1 = U(1, 0, 0), Um2 = U(-2, 0, 0), Up2 = U(2, 0, 0);
        const VT a = U0 + Up1, c = Um1 + U0;
        const VT dn = pd(ni(c, Um2 + Up1), c, ni(a, Um1 + Up2), a);
        const VT ppr = U0 + U(3, 0, 0), ppl = U(-3, 0, 0) + U0;
        const VT dw = pd(ni(Um2 + Um1, ppl), ppl, ni(Up1 + Up2, ppr), ppr);
        s[0] = vfma(K[0], dn, s[0]);
        s[0] = vfma(K[1], dw, s[0]);
    }
    {  // u: y-faces, v interpolated in x to the rows -1..2
        const VT U0 = U(0, 0, 0);
        auto J = [&](int r) { return ni(V(0, r, 0) + V(-1, r, 0), V(-2, r, 0) + V(1, r, 0)); };
        const VT dn = pd(J(0), U(0, -1, 0) + U0, J(1), U0 + U(0, 1, 0));
        const VT dw = pd(J(-1), U(0, -3, 0) + U0, J(2), U0 + U(0, 3, 0));
        s[0] = vfma(K[2], dn, s[0]);
        s[0] = vfma(K[3], dw, s[0]);
    }
    {  // u: z-faces, w interpolated in x to the planes -1..2
        const VT U0 = U(0, 0, 0);
        auto Kx = [&](int p) { return ni(W(0, 0, p) + W(-1, 0, p), W(-2, 0, p) + W(1, 0, p)); };
        const VT dn = pd(Kx(0), U(0, 0, -1) + U0, Kx(1), U0 + U(0, 0, 1));
        const VT dw = pd(Kx(-1), U0 + U(0, 0, -3), Kx(2), U0 + U(0, 0, 3));
        s[0] = vfma(K[4], dn, s[0]);
        s[0] = vfma(K[5], dw, s[0]);
    }
    {  // v: x-faces, u interpolated in y to the columns -1..2
        const VT V0 = V(0, 0, 0);
        auto L = [&](int c) { return ni(U(c, 0, 0) + U(c, -1, 0), U(c, -2, 0) + U(c, 1, 0)); };
        const VT dn = pd(L(0), V(-1, 0, 0) + V0, L(1), V0 + V(1, 0, 0));
        const VT dw = pd(L(-1), V(-3, 0, 0) + V0, L(2), V0 + V(3, 0, 0));
        s[1] = vfma(K[0], dn, s[1]);
        s[1] = vfma(K[1], dw, s[1]);
    }
    {  // v: y-faces
        const VT V0 = V(0, 0, 0), Vm1 = V(0, -1, 0), Vp1 = V(0, 1, 0), Vm2 = V(0, -2, 0), Vp2 = V(0, 2, 0);
        const VT a = V0 + Vp1, c = Vm1 + V0;
        const VT dn = pd(ni(c, Vm2 + Vp1), c, ni(a, Vm1 + Vp2), a);
        const VT ppr = V0 + V(0, 3, 0), ppl = V(0, -3, 0) + V0;
        const VT dw = pd(ni(Vm2 + Vm1, ppl), ppl, ni(Vp1 + Vp2, ppr), ppr);
        s[1] = vfma(K[2], dn, s[1]);
        s[1] = vfma(K[3], dw, s[1]);
    }
    {  // v: z-faces, w interpolated in y to the planes -1..2
        const VT V0 = V(0, 0, 0);
        auto Ky = [&](int p) { return ni(W(0, 0, p) + W(0, -1, p), W(0, -2, p) + W(0, 1, p)); };
        const VT dn = pd(Ky(0), V(0, 0, -1) + V0, Ky(1), V0 + V(0, 0, 1));
        const VT dw = pd(Ky(-1), V0 + V(0, 0, -3), Ky(2), V0 + V(0, 0, 3));
        s[1] = vfma(K[4], dn, s[1]);
        s[1] = vfma(K[5], dw, s[1]);
    }
    {  // w: x-faces, u interpolated in z (cell-height weights) to the w-face, columns -1..2
        const VT W0 = W(0, 0, 0);
        auto M = [&](int c) {
            return vfma(K[11], U(c, 0, -1), vfma(K[10], U(c, 0, 0), vfma(K[13], U(c, 0, 1), K[12] * U(c, 0, -2))));
        };
        auto MW = [&](int c) {
            return vfma(K[15], U(c, 0, -1), vfma(K[14], U(c, 0, 0), vfma(K[17], U(c, 0, 1), K[16] * U(c, 0, -2))));
        };
        const VT dn = pd(M(0), W(-1, 0, 0) + W0, M(1), W0 + W(1, 0, 0));
        const VT dw = pd(MW(-1), W(-3, 0, 0) + W0, MW(2), W0 + W(3, 0, 0));
        s[2] = vfma(K[6], dn, s[2]);
        s[2] = vfma(K[7], dw, s[2]);
    }
    {  // w: y-faces, v interpolated in z to the w-face, rows -1..2
        const VT W0 = W(0, 0, 0);
        auto M = [&](int r) {
            return vfma(K[11], V(0, r, -1), vfma(K[10], V(0, r, 0), vfma(K[13], V(0, r, 1), K[12] * V(0, r, -2))));
        };
        auto MW = [&](int r) {
            return vfma(K[15], V(0, r, -1), vfma(K[14], V(0, r, 0), vfma(K[17], V(0, r, 1), K[16] * V(0, r, -2))));
        };
        const VT dn = pd(M(0), W(0, -1, 0) + W0, M(1), W0 + W(0, 1, 0));
        const VT dw = pd(MW(-1), W(0, -3, 0) + W0, MW(2), W0 + W(0, 3, 0));
        s[2] = vfma(K[6], dn, s[2]);
        s[2] = vfma(K[7], dw, s[2]);
    }
    {  // w: z-faces
        const VT W0 = W(0, 0, 0), Wm1 = W(0, 0, -1), Wp1 = W(0, 0, 1), Wm2 = W(0, 0, -2), Wp2 = W(0, 0, 2);
        const VT pr = W0 + Wp1, pl = Wm1 + W0;
        const VT dn = pd(ni(pl, Wm2 + Wp1), pl, ni(pr, Wm1 + Wp2), pr);
        const VT ppr = W0 + W(0, 0, 3), ppl = W(0, 0, -3) + W0;
        const VT dw = pd(ni(Wm2 + Wm1, ppl), ppl, ni(Wp1 + Wp2, ppr), ppr);
        s[2] = vfma(K[8], dn, s[2]);
        s[2] = vfma(K[9], dw, s[2]);
    }
}
#undef U
#undef V
#undef W

}  // namespace tc
