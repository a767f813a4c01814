// k_flux_stag.cu -- fused explicit-flux kernel of the staggered schemes (HW2, VV4).
//
// One CTA owns a 32 x 8 (x, y) tile and marches a chunk of z-planes.  The velocity
// planes z-H .. z+H (H = 3 for VV4, 1 for HW2) of the tile plus an H-wide periodic
// halo live in a shared-memory ring of 2H+2 slots; the next plane is fetched with
// LDGSTS (cp.async) while the current one is computed, so every v_n value crosses
// HBM once and the halo re-reads hit L2.  The epilogue fuses the SBDF3 history
// combination (staggered/func_global.h:910-932) and the weighted sum of RHS_x
// used by the constant-flow-rate forcing, so the kernel reads v_n, v_{n-1},
// v_{n-2}, F_{n-1}, F_{n-2} and writes F_n and the RHS exactly once.
// Arithmetic: stencil_stag.cuh (staggered/func_global.h:345-625).
#include <algorithm>

#include "flux_ring.cuh"
#include "kernels.cuh"
#include "stencil_stag.cuh"
#include "stencil_vv4_int.cuh"

namespace tc {

template <typename T, int SCHEME, int VISC, bool LES, bool INT, int CY, int TY>
__device__ __forceinline__ void flux_cell(const RingAcc<T, SCHEME == TC_SCHEME_VV4 ? 3 : 1, CY, TY>& A, const StagZ<T>& mz,
                                          T gcz, const FluxArgs<T>& a, int ix, int iy, int xm, int xp, int ym,
                                          int yp, size_t NXY, T f[3]) {
    using ACC = RingAcc<T, SCHEME == TC_SCHEME_VV4 ? 3 : 1, CY, TY>;
    T cf[3], vf[3];
    if constexpr (SCHEME == TC_SCHEME_VV4) conv_vv4<T, ACC, INT>(A, mz, gcz, cf);
    else conv_hw2<T, ACC, INT>(A, mz, cf);
    if constexpr (VISC == TC_VISC_CROSS) {
        visc_cross<T, ACC, INT>(A, mz, vf);
    } else {
        const T* nt = a.nu_t;
        const int z = mz.iz;
        const T visc = mz.visc;
        auto MU = [&](int dx, int dy, int dz) -> T {
            if (!LES) return visc;
            const int xx = dx < 0 ? xm : (dx > 0 ? xp : ix);
            const int yy = dy < 0 ? ym : (dy > 0 ? yp : iy);
            return visc + __ldg(nt + (size_t)(z + dz) * NXY + (size_t)yy * a.g.NX + xx);
        };
        visc_naive<T, ACC, decltype(MU), INT>(A, MU, mz, vf);
    }
    f[0] = ((T)a.g.sour_dpdx + cf[0]) + vf[0];
    f[1] = (T(0) + cf[1]) + vf[1];
    f[2] = (T(0) + cf[2]) + vf[2];
}

template <typename T, int SCHEME, int VISC, bool LES, int ORDER, bool VEC, int CY, int TY>
__global__ void __launch_bounds__(STX* TY, 2) k_flux_stag(FluxArgs<T> a, int tz) {
    constexpr int H = SCHEME == TC_SCHEME_VV4 ? 3 : 1;
    using ACC = RingAcc<T, H, CY, TY>;
    constexpr int RS = ACC::RS;
    extern __shared__ __align__(16) unsigned char smraw[];
    T* ring = reinterpret_cast<T*>(smraw);
    __shared__ double sbuf[32];
    // FP64 VV4 DNS: interior planes take the regrouped stencils of stencil_vv4_int.cuh with
    // the plane constants FK64 of z and z+1 staged here
    constexpr bool FAST = sizeof(T) == 8 && SCHEME == TC_SCHEME_VV4 && VISC == TC_VISC_CROSS && !LES;
    __shared__ __align__(16) double fks[FAST ? 2 : 1][TC_FK64];

    const Geom& g = a.g;
    const int NX = g.NX, NY = g.NY, NZ = g.NZ;
    const size_t NXY = (size_t)NX * NY;
    const int tx = threadIdx.x % STX, tyt = threadIdx.x / STX;
    const int x0 = blockIdx.x * STX, y0 = blockIdx.y * (TY * CY);
    const int zb = blockIdx.z * tz, ze = min(NZ, zb + tz);
    const int ix = x0 + tx;
    // interior planes: no wall special case of the scheme applies
    const int zlo = SCHEME == TC_SCHEME_VV4 ? 3 : 1, zhi = SCHEME == TC_SCHEME_VV4 ? NZ - 4 : NZ - 2;

    TileCopy<T, H, CY, VEC, TY> cp;
    cp.init(x0, y0, NX, NY, g.N);
    const T* vbase = a.vel.c[0];  // the three components are consecutive blocks of N
    for (int z = max(0, zb - H); z <= min(NZ - 1, zb + H); z++) cp.load(ring, vbase, z, NXY);
    if (FAST && threadIdx.x < TC_FK64 / 2 && zb < NZ)
        cp_async<16>(&fks[zb & 1][2 * threadIdx.x], a.m.FK64 + (size_t)TC_FK64 * zb + 2 * threadIdx.x);
    cp_async_commit();

    StagZ<T> mz;
    mz.NZ = NZ;
    mz.DZ = a.m.DZ;
    mz.DZW = a.m.DZW;
    mz.hx = (T)g.hx;
    mz.hy = (T)g.hy;
    mz.ihx = (T)g.inv_hx;
    mz.ihy = (T)g.inv_hy;
    mz.visc = (T)g.visc;
    const int xm = wrapi(ix - 1, NX), xp = wrapi(ix + 1, NX);
    const T inv_tau = a.inv_tau, it2 = T(0.5) * a.inv_tau, it6 = a.inv_tau * T(0.16666666666666666667);
    double ub = 0.0;

    for (int z = zb; z < ze; z++) {
        if (z + 1 < ze && z + H + 1 < NZ) cp.load(ring, vbase, z + H + 1, NXY);
        if (FAST && z + 1 < ze && threadIdx.x < TC_FK64 / 2)
            cp_async<16>(&fks[(z + 1) & 1][2 * threadIdx.x], a.m.FK64 + (size_t)TC_FK64 * (z + 1) + 2 * threadIdx.x);
        cp_async_commit();
        // history of this thread's cells, issued before the stencil so its latency overlaps it
        T hp[CY][3], hq[CY][3], vq[CY][3];
        if (ORDER >= 2) {
#pragma unroll
            for (int q = 0; q < CY; q++) {
                const int iy = y0 + tyt * CY + q;
                if (ix < NX && iy < NY) {
                    const size_t id = (size_t)z * NXY + (size_t)iy * NX + ix;
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        hp[q][c] = __ldg(a.fp.c[c] + id);
                        if (ORDER == 3) {
                            hq[q][c] = __ldg(a.fq.c[c] + id);
                            vq[q][c] = __ldg(a.velq.c[c] + id);
                        } else {
                            hq[q][c] = vq[q][c] = T(0);
                        }
                    }
                }
            }
        }
        cp_async_wait<1>();
        __syncthreads();
        mz.iz = z;
#pragma unroll
        for (int k = 0; k < 6; k++) mz.pc[k] = a.m.PC[TC_PC * z + k];
        const T gcz = SCHEME == TC_SCHEME_VV4 ? a.m.GCZ[z] : T(0);
        const bool inner = z >= zlo && z <= zhi;
        ACC A0;
        A0.set(ring, z & (RS - 1), tx, tyt * CY);
#pragma unroll
        for (int q = 0; q < CY; q++) {
            const int ty = tyt * CY + q, iy = y0 + ty;
            if (ix >= NX || iy >= NY) continue;
            const int ym = wrapi(iy - 1, NY), yp = wrapi(iy + 1, NY);
            ACC A = A0;
            A.shift_rows(q);
            T f[3];
            bool done = false;
            if constexpr (FAST) {
                if (inner) {
                    f[0] = (T)a.g.sour_dpdx;
                    f[1] = f[2] = T(0);
                    visc_cross_int(A, fks[z & 1], f);
                    conv_vv4_int(A, fks[z & 1], f);
                    done = true;
                }
            }
            if (done) {
            } else if (inner) flux_cell<T, SCHEME, VISC, LES, true, CY, TY>(A, mz, gcz, a, ix, iy, xm, xp, ym, yp, NXY, f);
            else flux_cell<T, SCHEME, VISC, LES, false, CY, TY>(A, mz, gcz, a, ix, iy, xm, xp, ym, yp, NXY, f);
            if (z == 0) f[2] = 0;
            const size_t id = (size_t)z * NXY + (size_t)iy * NX + ix;
            if (ORDER == 0) {
#pragma unroll
                for (int c = 0; c < 3; c++) a.fout.c[c][id] = f[c];
            } else {
                T r[3];
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    const T vn = A(c, 0, 0, 0);
                    r[c] = sbdf_rhs<ORDER, T>(f[c], vn, ORDER >= 2 ? hp[q][c] : T(0), ORDER == 3 ? hq[q][c] : T(0),
                                              ORDER == 3 ? vq[q][c] : T(0), inv_tau, it6);
                    a.fout.c[c][id] = f[c] + it2 * vn;  // A_n
                    a.rhs.c[c][id] = r[c];
                }
                ub += (double)r[0] * (double)a.m.DZ[z];
            }
        }
        __syncthreads();
    }
    if (ORDER > 0 && a.ub_out) {
        const double s = block_sum(ub, sbuf);
        grid_sum_finish(s, a.ub_partial, a.ticket, a.ub_out, sbuf);
    }
}

// cells per thread along y: two for float (more reuse per shared-memory load),
// one for double (register budget of 2 CTAs/SM)
template <typename T>
constexpr int flux_cy() { return sizeof(T) == 4 ? 2 : 1; }
// threads along y: 8 (256 threads per CTA)
template <typename T>
constexpr int flux_ty() { return STY; }

static void flux_stag_shape(const Geom& g, int tile_rows, dim3& grid, int& tz) {
    const int ty = tile_rows;
    const int tiles = ((g.NX + STX - 1) / STX) * ((g.NY + ty - 1) / ty);
    int nch = std::max(1, (148 * 8 + tiles - 1) / tiles);
    tz = std::max(4, (g.NZ + nch - 1) / nch);
    grid = dim3((g.NX + STX - 1) / STX, (g.NY + ty - 1) / ty, (g.NZ + tz - 1) / tz);
}

// upper bound of the flux kernels' grid sizes (sizes the partial-sum buffer)
int flux_grid_blocks(const Geom& g) {
    dim3 gr;
    int tz;
    flux_stag_shape(g, STY, gr, tz);  // the smallest tile of the kernels
    return (int)(gr.x * gr.y * gr.z);
}

template <typename T, int SCHEME, int VISC, bool LES, int ORDER>
static void run(const FluxArgs<T>& a, cudaStream_t s) {
    constexpr int H = SCHEME == TC_SCHEME_VV4 ? 3 : 1;
    constexpr int CY = flux_cy<T>(), TY = flux_ty<T>();
    constexpr size_t smem = sizeof(T) * (2 * H + 2) * 3 * RingAcc<T, H, CY, TY>::PL;
    const bool vec = a.g.NX % (16 / (int)sizeof(T)) == 0;
    auto kern = vec ? k_flux_stag<T, SCHEME, VISC, LES, ORDER, true, CY, TY>
                    : k_flux_stag<T, SCHEME, VISC, LES, ORDER, false, CY, TY>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    dim3 grid;
    int tz;
    flux_stag_shape(a.g, TY * CY, grid, tz);
    kern<<<grid, STX * TY, smem, s>>>(a, tz);
}

template <typename T, int SCHEME, int VISC, bool LES>
static void run_order(const FluxArgs<T>& a, cudaStream_t s) {
    switch (a.order) {
        case 0: run<T, SCHEME, VISC, LES, 0>(a, s); break;
        case 1: run<T, SCHEME, VISC, LES, 1>(a, s); break;
        case 2: run<T, SCHEME, VISC, LES, 2>(a, s); break;
        default: run<T, SCHEME, VISC, LES, 3>(a, s); break;
    }
}

template <typename T, int SCHEME>
static void run_visc(const FluxArgs<T>& a, cudaStream_t s) {
    if (a.g.visc_type == TC_VISC_CROSS) run_order<T, SCHEME, TC_VISC_CROSS, false>(a, s);
    else if (a.nu_t) run_order<T, SCHEME, TC_VISC_NAIVE, true>(a, s);
    else run_order<T, SCHEME, TC_VISC_NAIVE, false>(a, s);
}

template <typename T>
void launch_flux_stag(const FluxArgs<T>& a, cudaStream_t s) {
    if constexpr (sizeof(T) == 4) {
        if (launch_flux_stag_pair(a, s)) return;
    }
    if (a.g.scheme == TC_SCHEME_VV4) run_visc<T, TC_SCHEME_VV4>(a, s);
    else run_visc<T, TC_SCHEME_HW2>(a, s);
}

template void launch_flux_stag<double>(const FluxArgs<double>&, cudaStream_t);
template void launch_flux_stag<float>(const FluxArgs<float>&, cudaStream_t);

}  // namespace tc
