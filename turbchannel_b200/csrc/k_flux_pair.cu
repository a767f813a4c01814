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
#include <cuda.h>  // CUtensorMap (the tensor map is encoded through the runtime's driver entry point)
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstring>

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

// PLP: the component stride of a ring slot, PL rounded up to 128 bytes (a TMA box
// destination is 128-byte aligned).
template <int H>
struct RingX2 {
    static constexpr int PW = PCX + 2 * PSG, PH = PTR + 2 * H, PL = PW * PH, RS = 2 * H + 2;
    static constexpr int PLP = (PL + 31) / 32 * 32;
    const float* p[2 * H + 1];  // (slot of plane z+dz, component 0, this pair)
    __device__ __forceinline__ void set(const float* r, int zs, int tx, int ty) {
        const float* c = r + (ty + H) * PW + 2 * tx + PSG;
#pragma unroll
        for (int dz = -H; dz <= H; dz++) p[dz + H] = c + ((zs + dz) & (RS - 1)) * 3 * PLP;
    }
    __device__ __forceinline__ F2 operator()(int c, int dx, int dy, int dz) const {
        const float* q = p[dz + H] + c * PLP + dy * PW + dx;
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
                sofs[k] = c * ACC::PLP + py * ACC::PW + ch * 4;
                gofs[k] = (unsigned)((long long)c * N + (long long)gy * NX + gx);
            } else {
                sofs[k] = -1;
                gofs[k] = 0;
            }
        }
    }
    __device__ __forceinline__ void load(float* ring, const float* base, int z, size_t NXY) const {
        float* dst = ring + (z & (ACC::RS - 1)) * 3 * ACC::PLP;
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
// TMA: the velocity ring is filled by one thread with 3-D tensor-map boxes (one per
// component and plane) completed on an mbarrier per ring slot, instead of 16-byte
// cp.async chunks from every thread; launched on tiles whose halo does not wrap.
// tmode: 0 all tiles (grid = tile grid), 1 interior tiles (tile = block + (1, 1)),
// 2 border tiles (blockIdx.x indexes the tiles of the first and last tile rows, then
// the first and last tile of the rows between).  The flow-rate sum takes block
// bid_off + (block index) of nb_total over the launches of one step.
template <int SCHEME, int ORDER, int RY, bool TMA>
__global__ void __launch_bounds__(PTX * PTR / RY, 2)
    k_flux_pair(FluxArgs<float> a, int tz, int tmode, int bid_off, int nb_total, const __grid_constant__ CUtensorMap tmap) {
    constexpr int H = SCHEME == TC_SCHEME_VV4 ? 3 : 1;
    constexpr int NT = PTX * PTR / RY;
    using ACC = RingX2<H>;
    constexpr int RS = ACC::RS, PLP = ACC::PLP;
    extern __shared__ __align__(16) unsigned char smraw[];
    float* ring = reinterpret_cast<float*>(smraw + ((128u - (smem_u32(smraw) & 127u)) & 127u));  // 128-byte aligned
    __shared__ double sbuf[32];
    __shared__ __align__(16) float fks[2][TC_FK];  // plane constants of z and z+1 (VV4)
    __shared__ __align__(8) unsigned long long bars[TMA ? RS : 1];
    constexpr bool FAST = SCHEME == TC_SCHEME_VV4;

    const Geom& g = a.g;
    const int NX = g.NX, NY = g.NY, NZ = g.NZ;
    const size_t NXY = (size_t)NX * NY;
    const int tx = threadIdx.x % PTX, ty = threadIdx.x / PTX;
    int btx = blockIdx.x, bty = blockIdx.y;
    if (tmode == 1) {
        btx += 1;
        bty += 1;
    } else if (tmode == 2) {
        const int ntx = (NX + PCX - 1) / PCX, nty = (NY + PTR - 1) / PTR;
        int i = blockIdx.x;
        if (i < ntx) {
            btx = i;
            bty = 0;
        } else if (i < 2 * ntx) {
            btx = i - ntx;
            bty = nty - 1;
        } else {
            i -= 2 * ntx;
            btx = (i & 1) ? ntx - 1 : 0;
            bty = 1 + (i >> 1);
        }
    }
    const int x0 = btx * PCX, y0 = bty * PTR;
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

    const float* vbase = a.vel.c[0];
    TileCopyX2<H, NT> cp;
    unsigned ph = 0, pend = 0;  // TMA: per slot the parity awaited next, and the slots with a box in flight
    auto issue = [&](int zz) {  // TMA: the three component boxes of plane zz
        const int sl = zz & (RS - 1);
        if (threadIdx.x == 0) {
            float* dst = ring + sl * 3 * PLP;
            fence_proxy_async_smem();
            mbar_expect_tx(&bars[sl], 3u * ACC::PW * ACC::PH * (unsigned)sizeof(float));
#pragma unroll
            for (int c = 0; c < 3; c++) tma_load_3d(dst + c * PLP, &tmap, x0 - PSG, y0 - H, c * NZ + zz, &bars[sl]);
        }
        pend |= 1u << sl;
    };
    auto wait_plane = [&](int zz) {  // TMA: false when the bounded wait gave up
        const int sl = zz & (RS - 1);
        const bool ok = mbar_wait_bounded(&bars[sl], (ph >> sl) & 1u);
        ph ^= 1u << sl;
        pend &= ~(1u << sl);
        return ok;
    };
    if constexpr (TMA) {
        if (threadIdx.x == 0) {
            for (int k = 0; k < RS; k++) mbar_init(&bars[k], 1);
            mbar_fence_init();
        }
        __syncthreads();
        for (int z = max(0, zb - H); z <= min(NZ - 1, zb + H); z++) issue(z);
    } else {
        cp.init(x0, y0, NX, NY, g.N);
        for (int z = max(0, zb - H); z <= min(NZ - 1, zb + H); z++) cp.load(ring, vbase, z, NXY);
    }
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

    bool failed = false;
    for (int z = zb; z < ze; z++) {
        if (z + 1 < ze && z + H + 1 < NZ) {
            if constexpr (TMA) issue(z + H + 1);
            else cp.load(ring, vbase, z + H + 1, NXY);
        }
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
        if constexpr (TMA) {
            bool ok = true;
            if (z == zb) {
                for (int zz = max(0, zb - H); zz <= min(NZ - 1, zb + H); zz++) ok = wait_plane(zz) && ok;
            } else if (z + H < NZ) {
                ok = wait_plane(z + H);
            }
            if (__syncthreads_or(!ok)) {  // a box never arrived: record it, drain what is in flight, stop
                for (int sl = 0; sl < RS; sl++)
                    if (pend & (1u << sl)) mbar_wait_bounded(&bars[sl], (ph >> sl) & 1u);
                cp_async_wait<0>();
                if (threadIdx.x == 0 && a.err_flag) atomicExch(a.err_flag, 2);
                failed = true;
                __syncthreads();
                break;
            }
        } else {
            __syncthreads();
        }
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
    if (failed) ub = 0.0;
    if (ORDER > 0 && a.ub_out) {
        const double s = block_sum(ub, sbuf);
        grid_sum_finish_at(s, a.ub_partial, a.ticket, a.ub_out, sbuf,
                           (unsigned)bid_off + blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z),
                           (unsigned)nb_total);
    }
}

constexpr int PAIR_RY = 2;  // rows per thread of the launched variant (measured faster than 1)

// cuTensorMapEncodeTiled through the runtime (no link against the driver library);
// null when the driver does not provide it.
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        else
            cudaGetLastError();
    }
    return fn;
}

// The velocity level as a 3-D float tensor (x, y, component-major z: plane c NZ + z) with
// the ring's box (PW x PH x 1).  False when it cannot be encoded.
template <int H>
static bool velocity_tensor_map(const FluxArgs<float>& a, CUtensorMap* tm) {
    auto enc = tensor_map_encoder();
    if (!enc) return false;
    const Geom& g = a.g;
    const cuuint64_t dims[3] = {(cuuint64_t)g.NX, (cuuint64_t)g.NY, (cuuint64_t)3 * g.NZ};
    const cuuint64_t strides[2] = {(cuuint64_t)g.NX * sizeof(float), (cuuint64_t)g.NX * g.NY * sizeof(float)};
    const cuuint32_t box[3] = {(cuuint32_t)RingX2<H>::PW, (cuuint32_t)RingX2<H>::PH, 1u};
    const cuuint32_t es[3] = {1u, 1u, 1u};
    return enc(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(a.vel.c[0]), dims, strides, box, es,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int SCHEME, int ORDER>
static void run_pair(const FluxArgs<float>& a, cudaStream_t s) {
    constexpr int H = SCHEME == TC_SCHEME_VV4 ? 3 : 1;
    constexpr size_t smem = sizeof(float) * (2 * H + 2) * 3 * RingX2<H>::PLP + 128;  // + alignment slack
    const int ntx = (a.g.NX + PCX - 1) / PCX, nty = (a.g.NY + PTR - 1) / PTR, tiles = ntx * nty;
    // z-chunks: as many as still fit the 2 resident CTAs per SM in one wave (measured at
    // 384x384x256, 288 tiles: one chunk 0.703 ms, two chunks (two waves) 0.708, chunks for
    // 8 slots per SM 0.710)
    const int nch = std::max(1, (148 * 2) / tiles);
    const int tz = std::max(4, (a.g.NZ + nch - 1) / nch);
    const int nzc = (a.g.NZ + tz - 1) / tz;
    auto plain = k_flux_pair<SCHEME, ORDER, PAIR_RY, false>;
    cudaFuncSetAttribute(plain, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    CUtensorMap tm;
    memset(&tm, 0, sizeof(tm));
    // TMA staging: interior tiles (whole tiles whose halo does not wrap) by tensor boxes,
    // the border tiles by cp.async in a second launch
    const bool tma = a.staging == 1 && a.g.NX % PCX == 0 && a.g.NY % PTR == 0 && ntx >= 3 && nty >= 3 &&
                     velocity_tensor_map<H>(a, &tm);
    if (!tma) {
        plain<<<dim3(ntx, nty, nzc), PTX * PTR / PAIR_RY, smem, s>>>(a, tz, 0, 0, tiles * nzc, tm);
        return;
    }
    auto boxed = k_flux_pair<SCHEME, ORDER, PAIR_RY, true>;
    cudaFuncSetAttribute(boxed, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const int ni = (ntx - 2) * (nty - 2) * nzc;
    boxed<<<dim3(ntx - 2, nty - 2, nzc), PTX * PTR / PAIR_RY, smem, s>>>(a, tz, 1, 0, tiles * nzc, tm);
    plain<<<dim3(2 * ntx + 2 * (nty - 2), 1, nzc), PTX * PTR / PAIR_RY, smem, s>>>(a, tz, 2, ni, tiles * nzc, tm);
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
