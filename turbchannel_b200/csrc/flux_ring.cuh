// flux_ring.cuh -- the z-marching shared-memory ring of velocity planes used by the
// fused flux kernels (k_flux_stag.cu, k_flux_coll.cu): a CTA owns a 32 x (8 CY) (x, y)
// tile, the planes z-H .. z+H of the tile plus an H-wide periodic halo (x-halo 4 wide, so
// the periodic wrap moves whole 16-byte chunks) sit in a ring of 2H+2 slots, and the next
// plane is fetched with LDGSTS (cp.async) while the current one is computed.
#pragma once
#include "tc_common.cuh"

namespace tc {

constexpr int STX = 32, STY = 8;  // threads per CTA: 32 x 8
constexpr int SG = 4;              // x-halo of the shared tile (a whole 16-byte chunk for float and double)

// CY: cells per thread along y, TY: threads along y (the tile is 32 x TY*CY cells).
// The offsets of the 2H+1 planes around the current one are computed once per plane,
// so every stencil access is one of them plus a compile-time displacement.
template <typename T, int H, int CY, int TY = STY>
struct RingAcc {
    static constexpr int PW = STX + 2 * SG, PH = TY * CY + 2 * H, PL = PW * PH, RS = 2 * H + 2;
    const T* p[2 * H + 1];  // (slot of plane z+dz, component 0, this cell)
    __device__ __forceinline__ void set(const T* r, int zs, int tx, int ty) {  // ty: cell row inside the tile
        const T* c = r + (ty + H) * PW + tx + SG;
#pragma unroll
        for (int dz = -H; dz <= H; dz++) p[dz + H] = c + ((zs + dz) & (RS - 1)) * 3 * PL;
    }
    __device__ __forceinline__ void shift_rows(int q) {
#pragma unroll
        for (int k = 0; k < 2 * H + 1; k++) p[k] += q * PW;
    }
    __device__ __forceinline__ T operator()(int c, int dx, int dy, int dz) const {
        return p[dz + H][c * PL + dy * PW + dx];
    }
};

// Plane-invariant part of this thread's share of the tile copy: for chunk k, the
// shared-memory offset inside a ring slot and the global element offset without
// the z term.  VEC: 16-byte chunks (the x-halo is chunk aligned, so the periodic
// wrap moves whole chunks); otherwise single elements.
template <typename T, int H, int CY, bool VEC, int TY = STY>
struct TileCopy {
    using ACC = RingAcc<T, H, CY, TY>;
    static constexpr int NT = STX * TY;  // threads of the CTA
    static constexpr int CH = VEC ? 16 / sizeof(T) : 1, NCH = ACC::PW / CH, PER = ACC::PH * NCH;
    static constexpr int TOTAL = 3 * PER, NK = (TOTAL + NT - 1) / NT;
    int sofs[NK];
    unsigned gofs[NK];  // < 2^32: checked on the host (3 N elements)
    __device__ __forceinline__ void init(int x0, int y0, int NX, int NY, long long N) {
#pragma unroll
        for (int k = 0; k < NK; k++) {
            const int e = threadIdx.x + k * NT;
            if (e < TOTAL) {
                const int c = e / PER, r = e - c * PER, py = r / NCH, ch = r - py * NCH;
                const int gy = wrapi(y0 - H + py, NY), gx = wrapi(x0 - SG + ch * CH, NX);
                sofs[k] = c * ACC::PL + py * ACC::PW + ch * CH;
                gofs[k] = (unsigned)((long long)c * N + (long long)gy * NX + gx);
            } else {
                sofs[k] = -1;
                gofs[k] = 0;
            }
        }
    }
    __device__ __forceinline__ void load(T* ring, const T* base, int z, size_t NXY) const {
        T* dst = ring + (z & (ACC::RS - 1)) * 3 * ACC::PL;
        const T* src = base + (size_t)z * NXY;
#pragma unroll
        for (int k = 0; k < NK; k++)
            if (sofs[k] >= 0) cp_async<CH * sizeof(T)>(dst + sofs[k], src + gofs[k]);
    }
};

}  // namespace tc
