// k_flux_pair.cu -- float flux kernel of the staggered schemes with two x-adjacent
// cells per thread and packed fp32x2 arithmetic (sm_100 FFMA2 / FADD2 / FMUL2).
//
// Same algorithm and data flow as k_flux_stag (z-marching shared-memory ring of
// velocity planes fetched with LDGSTS, fused SBDF3 epilogue, deterministic RHS_x
// sum), but the CTA tile is 64 x 8 cells and thread (tx, ty) owns the pair of cells
// x = 2 tx, 2 tx + 1.  Every stencil access then reads an aligned pair of floats
// (one 8-byte shared load; odd displacements combine two neighbouring pairs, which
// the other accesses load anyway), the arithmetic of both cells is one packed
// instruction, and the history/outputs move as 8-byte global accesses.  The
// stencils are the ones of stencil_stag.cuh, instantiated with the pair type F2.
// Used for the CROSS (DNS) viscosity; every other variant keeps k_flux_stag.  Its flux
// history is the reference's F_n (the other flux kernels keep A_n = F_n + v_n/(2 tau), see
// sbdf_rhs): measured at 384x384x256, reading A_{n-1}, A_{n-2}, v_{n-2} instead of F_{n-1},
// F_{n-2}, v_{n-1}, v_{n-2} moved 20% fewer bytes but took 0.741 against 0.702 ms -- at 254
// registers the compiler re-read stencil values from shared memory (+24% shared loads,
// +8% instructions), and staging the history in shared memory instead took 0.987 ms.
#include <algorithm>

#include "kernels.cuh"
#include "stencil_stag.cuh"
#include "stencil_vv4_int.cuh"

namespace tc {

// Two cells' values; every operation is the IEEE round-to-nearest operation per lane.
struct F2 {
    float2 v;
    F2() = default;
    __device__ __forceinline__ F2(float s) : v(make_float2(s, s)) {}
    __device__ __forceinline__ explicit F2(float2 a) : v(a) {}
};
__device__ __forceinline__ F2 operator+(F2 a, F2 b) { return F2(__fadd2_rn(a.v, b.v)); }
__device__ __forceinline__ F2 operator-(F2 a, F2 b) { return F2(__ffma2_rn(b.v, make_float2(-1.f, -1.f), a.v)); }
__device__ __forceinline__ F2 operator*(F2 a, F2 b) { return F2(__fmul2_rn(a.v, b.v)); }
__device__ __forceinline__ F2 operator-(F2 a) { return F2(make_float2(-a.v.x, -a.v.y)); }
__device__ __forceinline__ F2& operator+=(F2& a, F2 b) { return a = a + b; }
__device__ __forceinline__ F2& operator-=(F2& a, F2 b) { return a = a - b; }
__device__ __forceinline__ F2& operator*=(F2& a, F2 b) { return a = a * b; }

constexpr int PTX = 32;        // threads along x (two cells each)
constexpr int PTR = 8;         // tile rows along y (RY rows per thread)
constexpr int PCX = 2 * PTX;   // cells per tile along x
constexpr int PSG = 4;         // x-halo (whole 16-byte chunks)

template <int H>
struct RingX2 {
    static constexpr int PW = PCX + 2 * PSG, PH = PTR + 2 * H, PL = PW * PH, RS = 2 * H + 2;
    const float* p[2 * H + 1];  // (slot of plane z+dz, component 0, this pair)
    __device__ __forceinline__ void set(const float* r, int zs, int tx, int ty) {
        const float* c = r + (ty + H) * PW + 2 * tx + PSG;
#pragma unroll
        for (int dz = -H; dz <= H; dz++) p[dz + H] = c + ((zs + dz) & (RS - 1)) * 3 * PL;
    }
    __device__ __forceinline__ F2 operator()(int c, int dx, int dy, int dz) const {
        const float* q = p[dz + H] + c * PL + dy * PW + dx;
        if ((dx & 1) == 0) return F2(*reinterpret_cast<const float2*>(q));
        const float2 lo = *reinterpret_cast<const float2*>(q - 1), hi = *reinterpret_cast<const float2*>(q + 1);
        return F2(make_float2(lo.y, hi.x));
    }
};

// This thread's share (NT threads) of the 16-byte chunks of one plane of the tile
// (3 components, PH rows, PW/4 chunks per row, periodic wrap in x and y).
template <int H, int NT>
struct TileCopyX2 {
    using ACC = RingX2<H>;
    static constexpr int NCH = ACC::PW / 4, PER = ACC::PH * NCH, TOTAL = 3 * PER;
    static constexpr int NK = (TOTAL + NT - 1) / NT;
    int sofs[NK];
    unsigned gofs[NK];  // < 2^32: checked on the host (3 N elements)
    __device__ __forceinline__ void init(int x0, int y0, int NX, int NY, long long N) {
#pragma unroll
        for (int k = 0; k < NK; k++) {
            const int e = threadIdx.x + k * NT;
            if (e < TOTAL) {
                const int c = e / PER, r = e - c * PER, py = r / NCH, ch = r - py * NCH;
                const int gy = wrapi(y0 - H + py, NY), gx = wrapi(x0 - PSG + ch * 4, NX);
                sofs[k] = c * ACC::PL + py * ACC::PW + ch * 4;
                gofs[k] = (unsigned)((long long)c * N + (long long)gy * NX + gx);
            } else {
                sofs[k] = -1;
                gofs[k] = 0;
            }
        }
    }
    __device__ __forceinline__ void load(float* ring, const float* base, int z, size_t NXY) const {
        float* dst = ring + (z & (ACC::RS - 1)) * 3 * ACC::PL;
        const float* src = base + (size_t)z * NXY;
#pragma unroll
        for (int k = 0; k < NK; k++)
            if (sofs[k] >= 0) cp_async<16>(dst + sofs[k], src + gofs[k]);
    }
};

__device__ __forceinline__ F2 ld2(const float* p) { return F2(__ldg(reinterpret_cast<const float2*>(p))); }
__device__ __forceinline__ void st2(float* p, F2 v) { *reinterpret_cast<float2*>(p) = v.v; }
__device__ __forceinline__ F2 fma2(F2 a, F2 b, F2 c) { return F2(__ffma2_rn(a.v, b.v, c.v)); }

// the interior-plane stencils of the fast path (the packed pair's vfma below)
__device__ __forceinline__ F2 vfma(F2 a, F2 b, F2 c) { return fma2(a, b, c); }

// RY: tile rows per thread (1: 256 threads; 2: 128 threads whose two rows share the
// loads of their y-stencils, which the compiler merges as equal shared addresses).
template <int SCHEME, int ORDER, int RY>
__global__ void __launch_bounds__(PTX * PTR / RY, 2) k_flux_pair(FluxArgs<float> a, int tz) {
    constexpr int H = SCHEME == TC_SCHEME_VV4 ? 3 : 1;
    constexpr int NT = PTX * PTR / RY;
    using ACC = RingX2<H>;
    constexpr int RS = ACC::RS;
    extern __shared__ __align__(16) unsigned char smraw[];
    float* ring = reinterpret_cast<float*>(smraw);
    __shared__ double sbuf[32];
    __shared__ __align__(16) float fks[2][TC_FK];  // plane constants of z and z+1 (VV4)
    constexpr bool FAST = SCHEME == TC_SCHEME_VV4;

    const Geom& g = a.g;
    const int NX = g.NX, NY = g.NY, NZ = g.NZ;
    const size_t NXY = (size_t)NX * NY;
    const int tx = threadIdx.x % PTX, ty = threadIdx.x / PTX;
    const int x0 = blockIdx.x * PCX, y0 = blockIdx.y * PTR;
    const int zb = blockIdx.z * tz, ze = min(NZ, zb + tz);
    const int ix = x0 + 2 * tx;
    int iy[RY];
    bool act[RY];  // NX is even: both cells of a pair or neither
#pragma unroll
    for (int r = 0; r < RY; r++) {
        iy[r] = y0 + RY * ty + r;
        act[r] = ix < NX && iy[r] < NY;
    }
    const int zlo = SCHEME == TC_SCHEME_VV4 ? 3 : 1, zhi = SCHEME == TC_SCHEME_VV4 ? NZ - 4 : NZ - 2;

    TileCopyX2<H, NT> cp;
    cp.init(x0, y0, NX, NY, g.N);
    const float* vbase = a.vel.c[0];
    for (int z = max(0, zb - H); z <= min(NZ - 1, zb + H); z++) cp.load(ring, vbase, z, NXY);
    if (FAST && threadIdx.x < TC_FK / 4 && zb < NZ)
        cp_async<16>(&fks[zb & 1][4 * threadIdx.x], a.m.FK + (size_t)TC_FK * zb + 4 * threadIdx.x);
    cp_async_commit();

    StagZ<float> mz;
    mz.NZ = NZ;
    mz.DZ = a.m.DZ;
    mz.DZW = a.m.DZW;
    mz.hx = (float)g.hx;
    mz.hy = (float)g.hy;
    mz.ihx = (float)g.inv_hx;
    mz.ihy = (float)g.inv_hy;
    mz.visc = (float)g.visc;
    const F2 inv_tau(a.inv_tau);
    const float sour = (float)g.sour_dpdx;
    const F2 it3(3.f * a.inv_tau), itm15(-1.5f * a.inv_tau), it13(a.inv_tau * 0.33333333333333333333f);
    double ub = 0.0;

    for (int z = zb; z < ze; z++) {
        if (z + 1 < ze && z + H + 1 < NZ) cp.load(ring, vbase, z + H + 1, NXY);
        if (FAST && z + 1 < ze && threadIdx.x < TC_FK / 4)
            cp_async<16>(&fks[(z + 1) & 1][4 * threadIdx.x], a.m.FK + (size_t)TC_FK * (z + 1) + 4 * threadIdx.x);
        cp_async_commit();
        size_t id[RY];
        F2 hp[RY][3], hq[RY][3], vp[RY][3], vq[RY][3];
#pragma unroll
        for (int r = 0; r < RY; r++) {
            id[r] = (size_t)z * NXY + (size_t)iy[r] * NX + ix;
            if (ORDER >= 2 && act[r]) {
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    hp[r][c] = ld2(a.fp.c[c] + id[r]);
                    vp[r][c] = ld2(a.velp.c[c] + id[r]);
                    if (ORDER == 3) {
                        hq[r][c] = ld2(a.fq.c[c] + id[r]);
                        vq[r][c] = ld2(a.velq.c[c] + id[r]);
                    }
                }
            }
        }
        cp_async_wait<1>();
        __syncthreads();
        const bool inner = z >= zlo && z <= zhi;
        ACC A[RY];
        F2 f[RY][3];
#pragma unroll
        for (int r = 0; r < RY; r++) A[r].set(ring, z & (RS - 1), tx, RY * ty + r);
        if (FAST && inner) {
            const F2* K = reinterpret_cast<const F2*>(fks[z & 1]);
#pragma unroll
            for (int r = 0; r < RY; r++) {
                f[r][0] = F2(sour);
                f[r][1] = f[r][2] = F2(0.f);
                visc_cross_int(A[r], K, f[r]);
                conv_vv4_int(A[r], K, f[r]);
            }
        } else {
            mz.iz = z;
#pragma unroll
            for (int k = 0; k < 6; k++) mz.pc[k] = a.m.PC[TC_PC * z + k];
            const float gcz = SCHEME == TC_SCHEME_VV4 ? a.m.GCZ[z] : 0.f;
#pragma unroll
            for (int r = 0; r < RY; r++) {
                F2 cf[3], vf[3];
                if (inner) {
                    if constexpr (SCHEME == TC_SCHEME_VV4) conv_vv4<float, ACC, true, F2>(A[r], mz, gcz, cf);
                    else conv_hw2<float, ACC, true, F2>(A[r], mz, cf);
                    visc_cross<float, ACC, true, F2>(A[r], mz, vf);
                } else {
                    if constexpr (SCHEME == TC_SCHEME_VV4) conv_vv4<float, ACC, false, F2>(A[r], mz, gcz, cf);
                    else conv_hw2<float, ACC, false, F2>(A[r], mz, cf);
                    visc_cross<float, ACC, false, F2>(A[r], mz, vf);
                }
                f[r][0] = (F2(sour) + cf[0]) + vf[0];
                f[r][1] = (F2(0.f) + cf[1]) + vf[1];
                f[r][2] = (F2(0.f) + cf[2]) + vf[2];
                if (z == 0) f[r][2] = F2(0.f);
            }
        }
#pragma unroll
        for (int r = 0; r < RY; r++) {
            if (!act[r]) continue;
#pragma unroll
            for (int c = 0; c < 3; c++) st2(a.fout.c[c] + id[r], f[r][c]);
            if (ORDER > 0) {
                F2 rh[3];
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    const F2 vn = A[r](c, 0, 0, 0);
                    if (ORDER == 1) rh[c] = f[r][c] + inv_tau * vn;
                    else if (ORDER == 2)
                        rh[c] = (F2(2.f) * f[r][c] - hp[r][c]) + inv_tau * (F2(2.f) * vn - F2(0.5f) * vp[r][c]);
                    else  // (3 f - 3 f_p + f_q) + (3 v - 3/2 v_p + 1/3 v_q) / tau as FMA chains
                        rh[c] = fma2(F2(3.f), f[r][c], fma2(F2(-3.f), hp[r][c], hq[r][c])) +
                                fma2(it3, vn, fma2(itm15, vp[r][c], it13 * vq[r][c]));
                    st2(a.rhs.c[c] + id[r], rh[c]);
                }
                const double dz = (double)a.m.DZ[z];
                ub += (double)rh[0].v.x * dz;
                ub += (double)rh[0].v.y * dz;
            }
        }
        __syncthreads();
    }
    if (ORDER > 0 && a.ub_out) {
        const double s = block_sum(ub, sbuf);
        grid_sum_finish(s, a.ub_partial, a.ticket, a.ub_out, sbuf);
    }
}

constexpr int PAIR_RY = 2;  // rows per thread of the launched variant (measured faster than 1)

template <int SCHEME, int ORDER>
static void run_pair(const FluxArgs<float>& a, cudaStream_t s) {
    constexpr int H = SCHEME == TC_SCHEME_VV4 ? 3 : 1;
    constexpr size_t smem = sizeof(float) * (2 * H + 2) * 3 * RingX2<H>::PL;
    auto kern = k_flux_pair<SCHEME, ORDER, PAIR_RY>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const int tiles = ((a.g.NX + PCX - 1) / PCX) * ((a.g.NY + PTR - 1) / PTR);
    // z-chunks: about one CTA per resident slot (2 per SM; measured at 384x384x256:
    // 0.699 ms against 0.710 ms with 8 slots per SM, shorter chunks)
    const int nch = std::max(1, (148 * 2 + tiles - 1) / tiles);
    const int tz = std::max(4, (a.g.NZ + nch - 1) / nch);
    const dim3 grid((a.g.NX + PCX - 1) / PCX, (a.g.NY + PTR - 1) / PTR, (a.g.NZ + tz - 1) / tz);
    kern<<<grid, PTX * PTR / PAIR_RY, smem, s>>>(a, tz);
}

template <int SCHEME>
static void run_pair_order(const FluxArgs<float>& a, cudaStream_t s) {
    switch (a.order) {
        case 0: run_pair<SCHEME, 0>(a, s); break;
        case 1: run_pair<SCHEME, 1>(a, s); break;
        case 2: run_pair<SCHEME, 2>(a, s); break;
        default: run_pair<SCHEME, 3>(a, s); break;
    }
}

// The pair kernel covers the CROSS viscosity with NX % 4 == 0 (16-byte tile chunks);
// returns false for every other case.
bool flux_pair_covers(const Geom& g) {
    return g.scheme != TC_SCHEME_COLLOC && g.visc_type == TC_VISC_CROSS && g.NX % 4 == 0;
}

bool launch_flux_stag_pair(const FluxArgs<float>& a, cudaStream_t s) {
    if (!flux_pair_covers(a.g)) return false;
    if (a.g.scheme == TC_SCHEME_VV4) run_pair_order<TC_SCHEME_VV4>(a, s);
    else run_pair_order<TC_SCHEME_HW2>(a, s);
    return true;
}

}  // namespace tc
