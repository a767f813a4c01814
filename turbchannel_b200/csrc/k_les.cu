// k_les.cu -- data for the learned LES closure and its use in a run (staggered grids).
//
//   k_les_filter    box filter of width fw in x and y (the periodic directions) and fz
//                   cells in z (volume-weighted over the fz cell heights, so the coarse
//                   cells are those of the grid with every fz-th z-face) of one ring
//                   level: per coarse cell the cell-centred means of u, v, w, p and of
//                   the six products u_i u_j (10 fields) -- the snapshot and the
//                   sub-filter stresses tau_ij = <u_i u_j> - <u_i><u_j>;
//   k_les_features  per coarse cell the closure's 6 inputs (les_features) from the
//                   filtered gradient, and its training target nu*/nu, the
//                   least-squares eddy viscosity -tau^d_ij S_ij / (2 S_kl S_kl) (of
//                   either sign);
//   k_turb_mlp      a run's nu_t = nu * MLP(features of the resolved field), one warp
//                   per 32 cells (staggered) or elements (collocated): features by
//                   every lane in float, the network on the tensor cores as two 16-row
//                   tiles (inference of mlp.cuh).
// Cell-centred velocities: u_c = (u_x + u_{x+1})/2 etc. (u on the lower x-face,
// v on the lower y-face, w on the lower z-face, w = 0 on the top wall).  Gradients:
// central differences; at the walls the no-slip value 0 at the wall plane is the
// missing neighbour.
#include "kernels.cuh"
#include "mlp.cuh"

namespace tc {

// The closure's inputs from the velocity gradient G[i][j] = du_i/dx_j: with S, O the
// symmetric and antisymmetric parts in wall units (times nu/u_tau^2), asinh of
// tr(S^2), tr(O^2), tr(S^3), tr(O^2 S), tr(O^2 S^2), and log(1 + y+)/4.
__device__ __forceinline__ void les_features(const double G[3][3], double nu, double utau, double d, float f[6]) {
    const double sc = nu / (utau * utau);
    double S[3][3], O[3][3];
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            S[i][j] = 0.5 * (G[i][j] + G[j][i]) * sc;
            O[i][j] = 0.5 * (G[i][j] - G[j][i]) * sc;
        }
    double S2[3][3], O2[3][3];
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            S2[i][j] = S[i][0] * S[0][j] + S[i][1] * S[1][j] + S[i][2] * S[2][j];
            O2[i][j] = O[i][0] * O[0][j] + O[i][1] * O[1][j] + O[i][2] * O[2][j];
        }
    double l1 = 0, l2 = 0, l3 = 0, l4 = 0, l5 = 0;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            l1 += S[i][j] * S[j][i];
            l2 += O[i][j] * O[j][i];
            l3 += S2[i][j] * S[j][i];
            l4 += O2[i][j] * S[j][i];
            l5 += O2[i][j] * S2[j][i];
        }
    f[0] = (float)asinh(l1);
    f[1] = (float)asinh(l2);
    f[2] = (float)asinh(l3);
    f[3] = (float)asinh(l4);
    f[4] = (float)asinh(l5);
    f[5] = (float)(0.25 * log1p(d * utau / nu));
}

// z-derivative of a cell-centred column value at plane z of a grid with NZ cells and
// z-faces ZZ[0], ZZ[zs], ..., ZZ[zs NZ] from the values at z-1, z, z+1 (the wall value 0
// replaces a missing neighbour).
__device__ __forceinline__ double ddz(const double* ZZ, int zs, int NZ, int z, double qm, double qp) {
    const double zm = z > 0 ? 0.5 * (ZZ[zs * (z - 1)] + ZZ[zs * z]) : ZZ[0];
    const double zp = z < NZ - 1 ? 0.5 * (ZZ[zs * (z + 1)] + ZZ[zs * (z + 2)]) : ZZ[zs * NZ];
    return ((z < NZ - 1 ? qp : 0.0) - (z > 0 ? qm : 0.0)) / (zp - zm);
}

template <typename T>
__global__ void __launch_bounds__(256) k_les_filter(const T* __restrict__ u, const T* __restrict__ v,
                                                    const T* __restrict__ w, const T* __restrict__ p,
                                                    const double* __restrict__ ZZ, int NX, int NY, int NZ, int fw,
                                                    int fz, float* __restrict__ F) {
    const int NXc = NX / fw, NYc = NY / fw, NZc = NZ / fz;
    const long long M = (long long)NXc * NYc * NZc;
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= M) return;
    const int X = (int)(c % NXc), Y = (int)((c / NXc) % NYc), Z = (int)(c / ((long long)NXc * NYc));
    const size_t NXY = (size_t)NX * NY;
    double s[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int dz = 0; dz < fz; dz++) {
        const int z = fz * Z + dz;
        const size_t pl = (size_t)z * NXY;
        double t[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int dy = 0; dy < fw; dy++) {
            const int iy = fw * Y + dy, iyp = iy + 1 == NY ? 0 : iy + 1;
            for (int dx = 0; dx < fw; dx++) {
                const int ix = fw * X + dx, ixp = ix + 1 == NX ? 0 : ix + 1;
                const size_t id = pl + (size_t)iy * NX + ix;
                const double uc = 0.5 * ((double)u[id] + (double)u[pl + (size_t)iy * NX + ixp]);
                const double vc = 0.5 * ((double)v[id] + (double)v[pl + (size_t)iyp * NX + ix]);
                const double wc = 0.5 * ((double)w[id] + (z + 1 < NZ ? (double)w[id + NXY] : 0.0));
                t[0] += uc; t[1] += vc; t[2] += wc; t[3] += p ? (double)p[id] : 0.0;
                t[4] += uc * uc; t[5] += vc * vc; t[6] += wc * wc;
                t[7] += uc * vc; t[8] += uc * wc; t[9] += vc * wc;
            }
        }
        const double hz = ZZ[z + 1] - ZZ[z];
#pragma unroll
        for (int k = 0; k < 10; k++) s[k] += hz * t[k];
    }
    const double inv = 1.0 / ((double)(fw * fw) * (ZZ[fz * (Z + 1)] - ZZ[fz * Z]));
#pragma unroll
    for (int k = 0; k < 10; k++) F[k * M + c] = (float)(s[k] * inv);
}

// F: the 10 filtered fields of k_les_filter (layout [k][z][Y][X]) on the coarse grid of
// NXc x NYc x NZ cells whose z-faces are ZZ[0], ZZ[zs], ..., ZZ[zs NZ].  X: M x 6, Y: M.
__global__ void __launch_bounds__(256) k_les_features(const float* __restrict__ F, int NXc, int NYc, int NZ, double dxc,
                                                      double dyc, const double* __restrict__ ZZ, int zs, double nu,
                                                      double utau, float* __restrict__ Xo, float* __restrict__ Yo) {
    const long long M = (long long)NXc * NYc * NZ;
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= M) return;
    const int X = (int)(c % NXc), Y = (int)((c / NXc) % NYc), z = (int)(c / ((long long)NXc * NYc));
    const long long pl = (long long)NXc * NYc;
    const int Xp = X + 1 == NXc ? 0 : X + 1, Xm = X == 0 ? NXc - 1 : X - 1;
    const int Yp = Y + 1 == NYc ? 0 : Y + 1, Ym = Y == 0 ? NYc - 1 : Y - 1;
    auto at = [&](int k, int xx, int yy, int zz) -> double {
        return (double)F[k * M + (long long)zz * pl + (long long)yy * NXc + xx];
    };
    double G[3][3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
        G[i][0] = (at(i, Xp, Y, z) - at(i, Xm, Y, z)) / (2 * dxc);
        G[i][1] = (at(i, X, Yp, z) - at(i, X, Ym, z)) / (2 * dyc);
        G[i][2] = ddz(ZZ, zs, NZ, z, z > 0 ? at(i, X, Y, z - 1) : 0.0, z < NZ - 1 ? at(i, X, Y, z + 1) : 0.0);
    }
    const double zc = 0.5 * (ZZ[zs * z] + ZZ[zs * (z + 1)]);
    const double d = fmin(zc - ZZ[0], ZZ[zs * NZ] - zc);
    float f[6];
    les_features(G, nu, utau, d, f);
#pragma unroll
    for (int k = 0; k < 6; k++) Xo[c * 6 + k] = f[k];
    // target: least-squares eddy viscosity of the sub-filter stress
    const double ub[3] = {at(0, X, Y, z), at(1, X, Y, z), at(2, X, Y, z)};
    double tau[3][3];
    tau[0][0] = at(4, X, Y, z) - ub[0] * ub[0];
    tau[1][1] = at(5, X, Y, z) - ub[1] * ub[1];
    tau[2][2] = at(6, X, Y, z) - ub[2] * ub[2];
    tau[0][1] = tau[1][0] = at(7, X, Y, z) - ub[0] * ub[1];
    tau[0][2] = tau[2][0] = at(8, X, Y, z) - ub[0] * ub[2];
    tau[1][2] = tau[2][1] = at(9, X, Y, z) - ub[1] * ub[2];
    const double tr = (tau[0][0] + tau[1][1] + tau[2][2]) / 3.0;
    double num = 0, den = 0;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            const double Sij = 0.5 * (G[i][j] + G[j][i]);
            num -= (tau[i][j] - (i == j ? tr : 0.0)) * Sij;
            den += 2 * Sij * Sij;
        }
    // not clipped at zero: the backscatter points (negative nu*) stay in the training data,
    // so the network (softplus output, >= 0) learns the conditional mean; clipping them
    // to 0 biased it upward and over-dissipated the LES near the walls
    const double nus = den > 1e-300 ? num / den : 0.0;
    Yo[c] = (float)(nus / nu);
}

// nu_t of a run from the learned closure.  P: packed FP32 parameters.  Each warp takes
// 32 cells at a time: every lane gathers its cell's velocity gradient (differences in
// T, then float) and features, then two 16-row tiles go through the network on the
// tensor cores.  Staggered (COLL = false): the centred-velocity gradient of the cell.
// Collocated (COLL = true): the elements between 8 nodes, where that scheme keeps nu_t
// (iz < NZ-1, the top plane untouched as in the Smagorinsky kernel), with the element
// gradient of the nodal velocity -- the network's inputs are invariants of the resolved
// gradient in wall units and y+, the same physical quantities for both schemes.
template <typename T, bool COLL>
__global__ void __launch_bounds__(128, 4) k_turb_mlp(TurbArgs<T> a, const float* __restrict__ P) {
    __shared__ MlpSmem S;
    __shared__ float Xs[4][32][MLP_IN];
    mlp_load_smem(S, P);
    __syncthreads();
    const Geom& g = a.g;
    const int NX = g.NX, NY = g.NY, NZ = g.NZ;
    const size_t NXY = (size_t)NX * NY;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, gq = lane >> 2, t = lane & 3;
    const double nu = g.visc, utau = g.inv_ls * g.visc;
    const float sc = (float)(nu / (utau * utau));
    const float gx = (float)(0.25 * g.inv_hx), gy = (float)(0.25 * g.inv_hy);
    const T* __restrict__ u = a.v.c[0];
    const T* __restrict__ v = a.v.c[1];
    const T* __restrict__ w = a.v.c[2];
    const double* ZZ = a.m.dZZ;
    const long long N = g.N, ngrp = (N + 31) / 32;
    for (long long grp = (long long)blockIdx.x * 4 + wid; grp < ngrp; grp += (long long)gridDim.x * 4) {
        const long long c0 = grp * 32;
        const int nrow = (int)min(32LL, N - c0);
        if (COLL && lane < nrow && (c0 + lane) / (long long)NXY >= NZ - 1) {
#pragma unroll
            for (int k = 0; k < MLP_IN; k++) Xs[wid][lane][k] = 0.f;  // top node plane: no element
        } else if (COLL && lane < nrow) {
            const long long c = c0 + lane;
            const int ix = (int)(c % NX), iy = (int)((c / NX) % NY), iz = (int)(c / NXY);
            const int xp = ix + 1 == NX ? 0 : ix + 1, yp = iy + 1 == NY ? 0 : iy + 1;
            const size_t p0 = (size_t)iz * NXY, p1 = p0 + NXY;
            const size_t i00 = (size_t)iy * NX + ix, i10 = (size_t)iy * NX + xp, i01 = (size_t)yp * NX + ix,
                         i11 = (size_t)yp * NX + xp;
            const float ghx = (float)(0.25 * g.inv_hx), ghy = (float)(0.25 * g.inv_hy);
            const float ghz = (float)(0.25 / (a.m.dZZ[iz + 1] - a.m.dZZ[iz]));
            float G[3][3];
#pragma unroll
            for (int cc = 0; cc < 3; cc++) {
                const T* q = a.v.c[cc];
                const T q000 = q[p0 + i00], q100 = q[p0 + i10], q010 = q[p0 + i01], q110 = q[p0 + i11];
                const T q001 = q[p1 + i00], q101 = q[p1 + i10], q011 = q[p1 + i01], q111 = q[p1 + i11];
                G[cc][0] = (float)((q100 + q110 + q101 + q111) - (q000 + q010 + q001 + q011)) * ghx;
                G[cc][1] = (float)((q010 + q110 + q011 + q111) - (q000 + q100 + q001 + q101)) * ghy;
                G[cc][2] = (float)((q001 + q101 + q011 + q111) - (q000 + q100 + q010 + q110)) * ghz;
            }
            const double* ZZ = a.m.dZZ;
            const double zc = 0.5 * (ZZ[iz] + ZZ[iz + 1]);
            const double d = fmin(zc - ZZ[0], ZZ[NZ - 1] - zc);
            les_features_f(G, sc, (float)(d * utau / nu), Xs[wid][lane]);
        } else if (lane < nrow) {
            const long long c = c0 + lane;
            const int ix = (int)(c % NX), iy = (int)((c / NX) % NY), iz = (int)(c / NXY);
            const int xm = ix == 0 ? NX - 1 : ix - 1, xp = ix + 1 == NX ? 0 : ix + 1;
            const int xpp = xp + 1 == NX ? 0 : xp + 1;
            const int ym = iy == 0 ? NY - 1 : iy - 1, yp = iy + 1 == NY ? 0 : iy + 1;
            const int ypp = yp + 1 == NY ? 0 : yp + 1;
            const size_t pl = (size_t)iz * NXY;
            const size_t r0 = pl + (size_t)iy * NX, rm = pl + (size_t)ym * NX, rp = pl + (size_t)yp * NX,
                         rpp = pl + (size_t)ypp * NX;
            const bool lo = iz > 0, hi = iz + 1 < NZ;
            const size_t dm = lo ? NXY : 0, dp = hi ? NXY : 0;
            // cell-centred values: u_c = (u_x + u_{x+1})/2, v_c = (v_y + v_{y+1})/2,
            // w_c = (w_z + w_{z+1})/2 (w_NZ = 0); central differences, the wall value 0
            // replacing a missing z-neighbour
            float G[3][3];
            G[0][0] = (float)((u[r0 + xpp] + u[r0 + xp]) - (u[r0 + ix] + u[r0 + xm])) * gx;
            G[0][1] = (float)((u[rp + ix] + u[rp + xp]) - (u[rm + ix] + u[rm + xp])) * gy;
            G[1][0] = (float)((v[r0 + xp] + v[rp + xp]) - (v[r0 + xm] + v[rp + xm])) * gx;
            G[1][1] = (float)((v[rpp + ix] + v[rp + ix]) - (v[r0 + ix] + v[rm + ix])) * gy;
            const T w0 = w[r0 + ix], w1 = hi ? w[r0 + ix + NXY] : T(0);
            G[2][0] = (float)((w[r0 + xp] + (hi ? w[r0 + xp + NXY] : T(0))) -
                              (w[r0 + xm] + (hi ? w[r0 + xm + NXY] : T(0)))) * gx;
            G[2][1] = (float)((w[rp + ix] + (hi ? w[rp + ix + NXY] : T(0))) -
                              (w[rm + ix] + (hi ? w[rm + ix + NXY] : T(0)))) * gy;
            // z: (q(z+1) - q(z-1)) / (zc(z+1) - zc(z-1)) with zc the wall plane at a wall
            const double zm = lo ? 0.5 * (ZZ[iz - 1] + ZZ[iz]) : ZZ[0];
            const double zp = hi ? 0.5 * (ZZ[iz + 1] + ZZ[iz + 2]) : ZZ[NZ];
            const float gz = (float)(0.5 / (zp - zm));
            const T uzp = hi ? u[r0 + ix + dp] + u[r0 + xp + dp] : T(0);
            const T uzm = lo ? u[r0 + ix - dm] + u[r0 + xp - dm] : T(0);
            const T vzp = hi ? v[r0 + ix + dp] + v[rp + ix + dp] : T(0);
            const T vzm = lo ? v[r0 + ix - dm] + v[rp + ix - dm] : T(0);
            const T wzp = hi ? w1 + (iz + 2 < NZ ? w[r0 + ix + 2 * NXY] : T(0)) : T(0);
            const T wzm = lo ? w[r0 + ix - NXY] + w0 : T(0);
            G[0][2] = (float)(uzp - uzm) * gz;
            G[1][2] = (float)(vzp - vzm) * gz;
            G[2][2] = (float)(wzp - wzm) * gz;
            const double zc = 0.5 * (ZZ[iz] + ZZ[iz + 1]);
            const double d = fmin(zc - ZZ[0], ZZ[NZ] - zc);
            les_features_f(G, sc, (float)(d * utau / nu), Xs[wid][lane]);
        }
        __syncwarp();
#pragma unroll 1
        for (int h = 0; h < 2; h++) {
            const int nr = min(16, nrow - 16 * h);
            if (nr <= 0) break;
            unsigned ax[4];
            feature_fragment(&Xs[wid][16 * h][0], MLP_IN, nr, ax);
            Acc64 z1, z2;
            unsigned h1a[4][4];
            float z3[2];
            mlp_forward_tile(S, ax, z1, z2, h1a, z3);
            if (t == 0) {
                const long long cb = c0 + 16 * h;
                const long long top = COLL ? (long long)(NZ - 1) * (long long)NXY : N;  // first cell without element
                if (gq < nr && cb + gq < top) a.nu_t[cb + gq] = (T)(nu * softplus(z3[0]));
                if (gq + 8 < nr && cb + gq + 8 < top) a.nu_t[cb + gq + 8] = (T)(nu * softplus(z3[1]));
            }
        }
        __syncwarp();
    }
}

template <typename T>
void launch_les_filter(const T* u, const T* v, const T* w, const T* p, const double* ZZ, const Geom& g, int fw, int fz,
                       float* F, cudaStream_t s) {
    const long long M = (long long)(g.NX / fw) * (g.NY / fw) * (g.NZ / fz);
    k_les_filter<T><<<(unsigned)((M + 255) / 256), 256, 0, s>>>(u, v, w, p, ZZ, g.NX, g.NY, g.NZ, fw, fz, F);
}

void launch_les_features(const float* F, const Geom& g, int fw, int fz, const double* ZZ, float* X, float* Y,
                         cudaStream_t s) {
    const int NXc = g.NX / fw, NYc = g.NY / fw, NZc = g.NZ / fz;
    const long long M = (long long)NXc * NYc * NZc;
    k_les_features<<<(unsigned)((M + 255) / 256), 256, 0, s>>>(F, NXc, NYc, NZc, fw * g.hx, fw * g.hy, ZZ, fz, g.visc,
                                                              g.inv_ls * g.visc, X, Y);
}

template <typename T>
void launch_turb_mlp(const TurbArgs<T>& a, const float* P, cudaStream_t s) {
    const long long ngrp = (a.g.N + 31) / 32;
    const int nb = (int)std::max<long long>(1, std::min<long long>((ngrp + 3) / 4, 148 * 6));
    if (a.g.scheme == TC_SCHEME_COLLOC) k_turb_mlp<T, true><<<nb, 128, 0, s>>>(a, P);
    else k_turb_mlp<T, false><<<nb, 128, 0, s>>>(a, P);
}

template void launch_les_filter<double>(const double*, const double*, const double*, const double*, const double*,
                                        const Geom&, int, int, float*, cudaStream_t);
template void launch_les_filter<float>(const float*, const float*, const float*, const float*, const double*,
                                       const Geom&, int, int, float*, cudaStream_t);
template void launch_turb_mlp<double>(const TurbArgs<double>&, const float*, cudaStream_t);
template void launch_turb_mlp<float>(const TurbArgs<float>&, const float*, cudaStream_t);

}  // namespace tc
