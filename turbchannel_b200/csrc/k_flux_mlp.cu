// k_flux_mlp.cu -- the staggered explicit-flux kernel with the learned closure's
// inference fused in (LES with TC_TURB_MLP and tc_set_mlp_fusion(h, 1)).
//
// The NAIVE stress divergence (staggered/func_global.h:564-625) reads mu = visc + nu_t
// at the cell and at its +-1 neighbours in x, y and z.  One CTA owns a 32 x 8 (x, y)
// tile and marches a chunk of z-planes like k_flux_stag; besides the velocity ring it
// keeps three planes of nu_t over the tile plus a one-cell halo (34 x 10) in shared
// memory.  At plane z it evaluates the closure for plane z+1 from the velocity planes it
// has staged anyway (features from the centred-velocity gradient exactly as k_turb_mlp
// forms them, the network on the tensor cores), then computes the flux of plane z
// reading nu_t from that ring.  Halo cells are evaluated by both neighbouring CTAs
// (34 x 10 / (32 x 8) = 1.33 evaluations per cell, plus two planes per z-chunk); in
// exchange the separate pass's launch, its nu_t write and re-read and its gathers of
// the velocity from HBM go.  The tile's own cells of each nu_t plane are written to the
// nu_t array as well, so diagnostics and tc_get_nu_t see the same nu_t as with the
// separate pass (the same arithmetic, up to how the compiler fuses multiply-adds).
// Measured on the 96 x 64 x 96 LES (FP64 / mixed, ms per step): separate pass 0.206 /
// 0.174, fused 0.289 / 0.257 -- the 1.33x (plus chunk-start) evaluations of the network
// cost more than the nu_t round trip saves, so the separate pass stays the default.
#include <algorithm>

#include "kernels.cuh"
#include "mlp.cuh"
#include "stencil_stag.cuh"

namespace tc {

constexpr int FMX = 32, FMY = 8;       // tile / threads per CTA: 32 x 8, one cell per thread
constexpr int FMSG = 4;                // x-halo of the velocity tile (whole 16-byte chunks)
constexpr int NRX = FMX + 2, NRY = FMY + 2, NRC = NRX * NRY;  // nu_t plane: tile + 1-cell halo
constexpr int NRB = (NRC + 31) / 32;   // batches of 32 nu_t cells per plane

// Velocity ring of RS planes (z mod RS), each [3][PH][PW] with PW = 32 + 2*4 columns
// (tile x-coordinate X at column X + 4) and PH = 8 + YL + YH rows (Y at row Y + YL).
// The closure's gradients at the nu_t halo reach 2 cells below and 3 above the tile
// (u at x+2, v at y+2 of the halo cell 32 / 8), the stencils H cells both ways.
template <typename T, int H>
struct MRing {
    static constexpr int YL = H > 2 ? H : 2, YH = H > 3 ? H : 3;
    static constexpr int PW = FMX + 2 * FMSG, PH = FMY + YL + YH, PL = PW * PH;
    static constexpr int RS = H + 5;  // planes z-H .. z+4 (the last one in flight)
    static constexpr int ZL = H > 2 ? H : 2;  // lowest plane the chunk's prologue needs: zb - ZL
    static __device__ __forceinline__ int slot(int z) { return ((z % RS) + RS) % RS; }
};

// The stencil accessor of one cell: pointers to (component 0, this cell) in the slots
// of planes z-H .. z+H.
template <typename T, int H>
struct MAcc {
    using R = MRing<T, H>;
    const T* p[2 * H + 1];
    __device__ __forceinline__ void set(const T* ring, int z, int tx, int ty) {
        const T* c = ring + (ty + R::YL) * R::PW + tx + FMSG;
#pragma unroll
        for (int dz = -H; dz <= H; dz++) p[dz + H] = c + R::slot(z + dz) * 3 * R::PL;
    }
    __device__ __forceinline__ T operator()(int c, int dx, int dy, int dz) const {
        return p[dz + H][c * R::PL + dy * R::PW + dx];
    }
};

// This thread's share of copying one velocity plane (3 components) of the tile and its
// halo into a ring slot: shared offsets and global offsets without the z term, computed
// once.  VEC: 16-byte chunks (NX a multiple of the chunk: the x-halo is chunk aligned).
template <typename T, int H, bool VEC>
struct MCopy {
    using R = MRing<T, H>;
    static constexpr int CH = VEC ? 16 / sizeof(T) : 1, NCH = R::PW / CH, PER = R::PH * NCH;
    static constexpr int TOTAL = 3 * PER, NK = (TOTAL + FMX * FMY - 1) / (FMX * FMY);
    int sofs[NK];
    unsigned gofs[NK];  // < 2^32: 3 N is checked on the host
    __device__ __forceinline__ void init(int x0, int y0, int NX, int NY, long long N) {
#pragma unroll
        for (int k = 0; k < NK; k++) {
            const int e = threadIdx.x + k * FMX * FMY;
            if (e < TOTAL) {
                const int c = e / PER, r = e - c * PER, py = r / NCH, ch = r - py * NCH;
                const int gy = wrapi(y0 - R::YL + py, NY), gx = wrapi(x0 - FMSG + ch * CH, NX);
                sofs[k] = c * R::PL + py * R::PW + ch * CH;
                gofs[k] = (unsigned)((long long)c * N + (long long)gy * NX + gx);
            } else {
                sofs[k] = -1;
                gofs[k] = 0;
            }
        }
    }
    __device__ __forceinline__ void load(T* ring, const T* base, int z, size_t NXY) const {
        T* dst = ring + R::slot(z) * 3 * R::PL;
        const T* src = base + (size_t)z * NXY;
#pragma unroll
        for (int k = 0; k < NK; k++)
            if (sofs[k] >= 0) cp_async<CH * sizeof(T)>(dst + sofs[k], src + gofs[k]);
    }
};

// nu_t of plane zc over the tile and its one-cell halo, into the nu_t ring slot zc % 3;
// the tile's own cells also to the nu_t array.  Every warp takes batches of 32 cells:
// each lane forms its cell's features (the centred-velocity gradient of k_turb_mlp,
// differences in T, then float), then two 16-row tiles go through the network.
template <typename T, int H>
__device__ __forceinline__ void nut_plane(const Geom& g, const double* ZZ, const T* ring, T* nts, float (*Xs)[MLP_IN],
                                          const MlpSmem& S, int zc, int x0, int y0, T* nu_out) {
    using R = MRing<T, H>;
    const int NX = g.NX, NY = g.NY, NZ = g.NZ;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, gq = lane >> 2, t = lane & 3;
    const double nu = g.visc, utau = g.inv_ls * g.visc;
    const float sc = (float)(nu / (utau * utau));
    const float gx = (float)(0.25 * g.inv_hx), gy = (float)(0.25 * g.inv_hy);
    const bool lo = zc > 0, hi = zc + 1 < NZ, hi2 = zc + 2 < NZ;
    const double zm = lo ? 0.5 * (ZZ[zc - 1] + ZZ[zc]) : ZZ[0];
    const double zp = hi ? 0.5 * (ZZ[zc + 1] + ZZ[zc + 2]) : ZZ[NZ];
    const float gz = (float)(0.5 / (zp - zm));
    const double zcc = 0.5 * (ZZ[zc] + ZZ[zc + 1]);
    const float yplus = (float)(fmin(zcc - ZZ[0], ZZ[NZ] - zcc) * utau / nu);
    // plane pointers of component c at z-offset dz (planes outside the channel are never read)
    auto P = [&](int c, int dz) -> const T* { return ring + R::slot(zc + dz) * 3 * R::PL + c * R::PL; };
    const T *u0 = P(0, 0), *v0 = P(1, 0), *w0 = P(2, 0);
    const T *um = P(0, -1), *vm = P(1, -1), *wm = P(2, -1);
    const T *up = P(0, 1), *vp = P(1, 1), *wp = P(2, 1), *wpp = P(2, 2);
    T* nslot = nts + (zc % 3) * NRC;
    for (int b = wid; b < NRB; b += FMX * FMY / 32) {
        const int r = 32 * b + lane;
        if (r < NRC) {
            const int X = r % NRX - 1, Y = r / NRX - 1;
            auto at = [&](const T* q, int dx, int dy) -> T { return q[(Y + R::YL + dy) * R::PW + X + FMSG + dx]; };
            float G[3][3];
            G[0][0] = (float)((at(u0, 2, 0) + at(u0, 1, 0)) - (at(u0, 0, 0) + at(u0, -1, 0))) * gx;
            G[0][1] = (float)((at(u0, 0, 1) + at(u0, 1, 1)) - (at(u0, 0, -1) + at(u0, 1, -1))) * gy;
            G[1][0] = (float)((at(v0, 1, 0) + at(v0, 1, 1)) - (at(v0, -1, 0) + at(v0, -1, 1))) * gx;
            G[1][1] = (float)((at(v0, 0, 2) + at(v0, 0, 1)) - (at(v0, 0, 0) + at(v0, 0, -1))) * gy;
            const T w0c = at(w0, 0, 0), w1c = hi ? at(wp, 0, 0) : T(0);
            G[2][0] = (float)((at(w0, 1, 0) + (hi ? at(wp, 1, 0) : T(0))) - (at(w0, -1, 0) + (hi ? at(wp, -1, 0) : T(0)))) * gx;
            G[2][1] = (float)((at(w0, 0, 1) + (hi ? at(wp, 0, 1) : T(0))) - (at(w0, 0, -1) + (hi ? at(wp, 0, -1) : T(0)))) * gy;
            const T uzp = hi ? at(up, 0, 0) + at(up, 1, 0) : T(0);
            const T uzm = lo ? at(um, 0, 0) + at(um, 1, 0) : T(0);
            const T vzp = hi ? at(vp, 0, 0) + at(vp, 0, 1) : T(0);
            const T vzm = lo ? at(vm, 0, 0) + at(vm, 0, 1) : T(0);
            const T wzp = hi ? w1c + (hi2 ? at(wpp, 0, 0) : T(0)) : T(0);
            const T wzm = lo ? at(wm, 0, 0) + w0c : T(0);
            G[0][2] = (float)(uzp - uzm) * gz;
            G[1][2] = (float)(vzp - vzm) * gz;
            G[2][2] = (float)(wzp - wzm) * gz;
            les_features_f(G, sc, yplus, Xs[32 * wid + lane]);
        }
        __syncwarp();
#pragma unroll 1
        for (int hh = 0; hh < 2; hh++) {
            const int nr = min(16, NRC - (32 * b + 16 * hh));
            if (nr <= 0) break;
            unsigned ax[4];
            feature_fragment(&Xs[32 * wid + 16 * hh][0], MLP_IN, nr, ax);
            Acc64 z1, z2;
            unsigned h1a[4][4];
            float z3[2];
            mlp_forward_tile(S, ax, z1, z2, h1a, z3);
            if (t == 0) {
#pragma unroll
                for (int k = 0; k < 2; k++) {
                    const int row = gq + 8 * k;
                    if (row < nr) {
                        const int rr = 32 * b + 16 * hh + row;
                        const T val = (T)(nu * softplus(z3[k]));
                        nslot[rr] = val;
                        const int X = rr % NRX - 1, Y = rr / NRX - 1;
                        const int ix = x0 + X, iy = y0 + Y;
                        if (X >= 0 && X < FMX && Y >= 0 && Y < FMY && ix < NX && iy < NY)
                            nu_out[(size_t)zc * NX * NY + (size_t)iy * NX + ix] = val;
                    }
                }
            }
        }
        __syncwarp();
    }
}

template <typename T, int SCHEME, int ORDER, bool VEC>
__global__ void __launch_bounds__(FMX* FMY, 1) k_flux_mlp(FluxArgs<T> a, const float* __restrict__ P, T* nu_out,
                                                          int tz) {
    constexpr int H = SCHEME == TC_SCHEME_VV4 ? 3 : 1;
    using R = MRing<T, H>;
    using ACC = MAcc<T, H>;
    extern __shared__ __align__(16) unsigned char smraw[];
    T* ring = reinterpret_cast<T*>(smraw);
    T* nts = ring + R::RS * 3 * R::PL;                                   // [3][NRC]
    float(*Xs)[MLP_IN] = reinterpret_cast<float(*)[MLP_IN]>(nts + 3 * NRC);  // [8 warps x 32][6]
    __shared__ MlpSmem S;
    __shared__ double sbuf[32];
    mlp_load_smem(S, P);

    const Geom& g = a.g;
    const int NX = g.NX, NY = g.NY, NZ = g.NZ;
    const size_t NXY = (size_t)NX * NY;
    const int tx = threadIdx.x % FMX, ty = threadIdx.x / FMX;
    const int x0 = blockIdx.x * FMX, y0 = blockIdx.y * FMY;
    const int zb = blockIdx.z * tz, ze = min(NZ, zb + tz);
    const int ix = x0 + tx, iy = y0 + ty;
    const bool own = ix < NX && iy < NY;
    const int zlo = SCHEME == TC_SCHEME_VV4 ? 3 : 1, zhi = SCHEME == TC_SCHEME_VV4 ? NZ - 4 : NZ - 2;
    const double* ZZ = a.m.dZZ;

    MCopy<T, H, VEC> cp;
    cp.init(x0, y0, NX, NY, g.N);
    const T* vbase = a.vel.c[0];  // the three components are consecutive blocks of N
    for (int z = max(0, zb - R::ZL); z <= min(NZ - 1, zb + 3); z++) cp.load(ring, vbase, z, NXY);
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();  // also publishes the network's shared-memory image
    if (zb - 1 >= 0) nut_plane<T, H>(g, ZZ, ring, nts, Xs, S, zb - 1, x0, y0, nu_out);
    nut_plane<T, H>(g, ZZ, ring, nts, Xs, S, zb, x0, y0, nu_out);
    __syncthreads();  // the ring slot of plane zb - 2 is refilled by the first iteration

    StagZ<T> mz;
    mz.NZ = NZ;
    mz.DZ = a.m.DZ;
    mz.DZW = a.m.DZW;
    mz.hx = (T)g.hx;
    mz.hy = (T)g.hy;
    mz.ihx = (T)g.inv_hx;
    mz.ihy = (T)g.inv_hy;
    mz.visc = (T)g.visc;
    const T inv_tau = a.inv_tau, it2 = T(0.5) * a.inv_tau, it6 = a.inv_tau * T(0.16666666666666666667);
    const T visc = (T)g.visc;
    double ub = 0.0;

    for (int z = zb; z < ze; z++) {
        if (z + 1 < ze && z + 4 < NZ) cp.load(ring, vbase, z + 4, NXY);
        cp_async_commit();
        T hp[3], hq[3], vq[3];
        if (ORDER >= 2 && own) {
            const size_t id = (size_t)z * NXY + (size_t)iy * NX + ix;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                hp[c] = __ldg(a.fp.c[c] + id);
                if (ORDER == 3) {
                    hq[c] = __ldg(a.fq.c[c] + id);
                    vq[c] = __ldg(a.velq.c[c] + id);
                }
            }
        }
        cp_async_wait<1>();
        __syncthreads();  // plane z+3 staged; nu_t slot (z+1) % 3 free (plane z-2 done)
        if (z + 1 < NZ) nut_plane<T, H>(g, ZZ, ring, nts, Xs, S, z + 1, x0, y0, nu_out);
        __syncthreads();
        mz.iz = z;
#pragma unroll
        for (int k = 0; k < 6; k++) mz.pc[k] = a.m.PC[TC_PC * z + k];
        const T gcz = SCHEME == TC_SCHEME_VV4 ? a.m.GCZ[z] : T(0);
        if (own) {
            ACC A;
            A.set(ring, z, tx, ty);
            auto MU = [&](int dx, int dy, int dz) -> T {
                return visc + nts[((z + dz + 3) % 3) * NRC + (ty + 1 + dy) * NRX + tx + 1 + dx];
            };
            T cf[3], vf[3];
            const bool inner = z >= zlo && z <= zhi;
            if (inner) {
                if constexpr (SCHEME == TC_SCHEME_VV4) conv_vv4<T, ACC, true>(A, mz, gcz, cf);
                else conv_hw2<T, ACC, true>(A, mz, cf);
                visc_naive<T, ACC, decltype(MU), true>(A, MU, mz, vf);
            } else {
                if constexpr (SCHEME == TC_SCHEME_VV4) conv_vv4<T, ACC, false>(A, mz, gcz, cf);
                else conv_hw2<T, ACC, false>(A, mz, cf);
                visc_naive<T, ACC, decltype(MU), false>(A, MU, mz, vf);
            }
            T f[3];
            f[0] = ((T)g.sour_dpdx + cf[0]) + vf[0];
            f[1] = (T(0) + cf[1]) + vf[1];
            f[2] = (T(0) + cf[2]) + vf[2];
            if (z == 0) f[2] = 0;
            const size_t id = (size_t)z * NXY + (size_t)iy * NX + ix;
            {
                T r[3];
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    const T vn = A(c, 0, 0, 0);
                    r[c] = sbdf_rhs<ORDER, T>(f[c], vn, ORDER >= 2 ? hp[c] : T(0), ORDER == 3 ? hq[c] : T(0),
                                              ORDER == 3 ? vq[c] : T(0), inv_tau, it6);
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

template <typename T, int SCHEME>
static size_t flux_mlp_smem() {
    using R = MRing<T, SCHEME == TC_SCHEME_VV4 ? 3 : 1>;
    return sizeof(T) * ((size_t)R::RS * 3 * R::PL + 3 * NRC) + sizeof(float) * FMX * FMY * MLP_IN;
}

template <typename T, int SCHEME, int ORDER>
static void run_mlp(const FluxArgs<T>& a, const float* P, T* nu_out, cudaStream_t s) {
    const size_t smem = flux_mlp_smem<T, SCHEME>();
    const bool vec = a.g.NX % (16 / (int)sizeof(T)) == 0;
    auto kern = vec ? k_flux_mlp<T, SCHEME, ORDER, true> : k_flux_mlp<T, SCHEME, ORDER, false>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    // z-chunks: one wave of resident CTAs (whole chunks per SM slot), at least 8 planes
    // each (a chunk evaluates the closure on two planes below its own)
    int dev = 0, sms = 148, occ = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, FMX * FMY, smem);
    const int tiles = ((a.g.NX + FMX - 1) / FMX) * ((a.g.NY + FMY - 1) / FMY);
    const int nch = std::max(1, sms * std::max(1, occ) / tiles);
    const int tz = std::max(8, (a.g.NZ + nch - 1) / nch);
    const dim3 grid((a.g.NX + FMX - 1) / FMX, (a.g.NY + FMY - 1) / FMY, (a.g.NZ + tz - 1) / tz);
    kern<<<grid, FMX * FMY, smem, s>>>(a, P, nu_out, tz);
}

// The flux of a step with the closure fused in (orders 1..3, staggered NAIVE viscosity).
// The grid never has more CTAs than flux_grid_blocks(g) (the flow-rate partial sums).
template <typename T>
void launch_flux_mlp(const FluxArgs<T>& a, const float* P, T* nu_out, cudaStream_t s) {
    const bool vv = a.g.scheme == TC_SCHEME_VV4;
    switch (a.order) {
        case 1: vv ? run_mlp<T, TC_SCHEME_VV4, 1>(a, P, nu_out, s) : run_mlp<T, TC_SCHEME_HW2, 1>(a, P, nu_out, s); break;
        case 2: vv ? run_mlp<T, TC_SCHEME_VV4, 2>(a, P, nu_out, s) : run_mlp<T, TC_SCHEME_HW2, 2>(a, P, nu_out, s); break;
        default: vv ? run_mlp<T, TC_SCHEME_VV4, 3>(a, P, nu_out, s) : run_mlp<T, TC_SCHEME_HW2, 3>(a, P, nu_out, s); break;
    }
}

template void launch_flux_mlp<double>(const FluxArgs<double>&, const float*, double*, cudaStream_t);
template void launch_flux_mlp<float>(const FluxArgs<float>&, const float*, float*, cudaStream_t);

}  // namespace tc
