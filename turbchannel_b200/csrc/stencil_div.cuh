// stencil_div.cuh -- discrete divergence (times the cell height) of a face/node
// velocity field: HW2 staggered/func_global.h:306-312, VV4 :325-333, collocated
// collocated_AB3/func_global.h:310-325.  Used by the fused divergence + FFT kernel
// and by the stand-alone operator.
#pragma once
#include "kernels.cuh"

namespace tc {

template <typename T, int SCHEME, bool SCALAR>
__device__ __forceinline__ T div_at(const Geom& g, const MeshDev<T>& mesh, const CV3<T>& vel, const T* src_scalar, int x, int y, int z) {
    const int NX = g.NX, NY = g.NY, NZ = g.NZ;
    const size_t NXY = (size_t)NX * NY;
    const size_t id = (size_t)z * NXY + (size_t)y * NX + x;
    if (SCALAR) return src_scalar[id];
    const T *u = vel.c[0], *v = vel.c[1], *w = vel.c[2];
    const size_t row = (size_t)z * NXY + (size_t)y * NX;
    const int xp = x + 1 == NX ? 0 : x + 1, xm = x == 0 ? NX - 1 : x - 1;
    const int yp = y + 1 == NY ? 0 : y + 1, ym = y == 0 ? NY - 1 : y - 1;
    const T ihx = (T)g.inv_hx, ihy = (T)g.inv_hy;
    if (SCHEME == TC_SCHEME_HW2) {
        const T hz = mesh.DZ[z];
        return (__ldg(u + row + xp) - __ldg(u + id)) * ihx * hz +
               (__ldg(v + (size_t)z * NXY + (size_t)yp * NX + x) - __ldg(v + id)) * ihy * hz +
               ((z < NZ - 1) ? (__ldg(w + id + NXY) - __ldg(w + id)) : (-__ldg(w + id)));
    } else if (SCHEME == TC_SCHEME_VV4) {
        const T C27 = T(0.03703703703703703703);
        const int xpp = xp + 1 == NX ? 0 : xp + 1, ypp = yp + 1 == NY ? 0 : yp + 1;
        const T dz = mesh.DZ[z], dzw = mesh.DZW[z];
        const T dudx = ihx * (dz * (__ldg(u + row + xp) - __ldg(u + id)) - C27 * dzw * (__ldg(u + row + xpp) - __ldg(u + row + xm)));
        const size_t pl = (size_t)z * NXY;
        const T dvdy = ihy * (dz * (__ldg(v + pl + (size_t)yp * NX + x) - __ldg(v + id)) -
                              C27 * dzw * (__ldg(v + pl + (size_t)ypp * NX + x) - __ldg(v + pl + (size_t)ym * NX + x)));
        const T w0 = __ldg(w + id);
        const T wr = (z == NZ - 1) ? T(0) : __ldg(w + id + NXY);
        const T wrr = (z == NZ - 1) ? w0 : (z == NZ - 2) ? T(0) : __ldg(w + id + 2 * NXY);
        const T wll = (z == 0) ? __ldg(w + id + NXY) : (z == 1) ? T(0) : __ldg(w + id - NXY);
        return dudx + dvdy + (wr - w0) - C27 * (wrr - wll);
    } else {
        const T hz = mesh.cellh[z], hx = (T)g.hx, hy = (T)g.hy;
        const size_t pl = (size_t)z * NXY;
        T d = 0;
        d += T(0.5) * (__ldg(u + row + xp) - __ldg(u + row + xm)) * hy * hz;
        d += T(0.5) * (__ldg(v + pl + (size_t)yp * NX + x) - __ldg(v + pl + (size_t)ym * NX + x)) * hx * hz;
        if (z == 0) d += T(0.5) * (__ldg(w + id + NXY) - __ldg(w + id)) * hx * hy;
        else if (z == NZ - 1) d += T(0.5) * (__ldg(w + id) - __ldg(w + id - NXY)) * hx * hy;
        else d += T(0.5) * (__ldg(w + id + NXY) - __ldg(w + id - NXY)) * hx * hy;
        return d;
    }
}

}  // namespace tc
