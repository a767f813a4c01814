"""CPU oracle of the learned LES closure (test infrastructure only: imported by tests/
and never by the library).

The closure has no counterpart in the reference (its subgrid model is the algebraic
Smagorinsky-van Driest one, staggered/func_global.h:815-890), so this module restates
the library's own definitions in numpy (float64 unless a rounding is stated) as the
checker of the CUDA kernels:

* box_filter        k_les_filter  (turbchannel_b200/csrc/k_les.cu)
* features_targets  k_les_features / les_features
* mlp_forward, mlp_grad   the network of turbchannel_b200/csrc/mlp.cuh, with its BF16
                    roundings (weights, inputs, hidden activations, backward factors)
* smagorinsky_nut   the reference's algebraic model in the same wall units, as the
                    baseline the learned closure is compared with
* adam_step         the optimiser of k_mlp_adam

Staggered layout: u on the lower x-face, v on the lower y-face, w on the lower z-face
of a cell (w = 0 on both walls); cell-centred values are the two-face means.
"""
import numpy as np

MLP_IN, MLP_H = 6, 64
OW1 = 0
OB1 = OW1 + MLP_IN * MLP_H
OW2 = OB1 + MLP_H
OB2 = OW2 + MLP_H * MLP_H
OW3 = OB2 + MLP_H
OB3 = OW3 + MLP_H
NPAR = OB3 + 1


# ----------------------------------------------------------------------------- filter
def cell_centred(vel, NX, NY, NZ):
    """vel: (N, 3) staggered field, index ix + NX (iy + NY iz) -> (3, NZ, NY, NX) centred."""
    u = vel[:, 0].reshape(NZ, NY, NX)
    v = vel[:, 1].reshape(NZ, NY, NX)
    w = vel[:, 2].reshape(NZ, NY, NX)
    uc = 0.5 * (u + np.roll(u, -1, axis=2))
    vc = 0.5 * (v + np.roll(v, -1, axis=1))
    wn = np.concatenate([w[1:], np.zeros((1, NY, NX))], axis=0)
    wc = 0.5 * (w + wn)
    return np.stack([uc, vc, wc])


def box_filter(vel, p, NX, NY, NZ, fw, fz=1, ZZ=None):
    """The 10 filtered fields [k][Z][Y][X] of k_les_filter (float64): means over fw x fw
    cells in x, y and, weighted by the cell heights ZZ[z+1] - ZZ[z], over fz cells in z."""
    c = cell_centred(vel, NX, NY, NZ)
    pp = p.reshape(NZ, NY, NX)
    q = [c[0], c[1], c[2], pp, c[0] * c[0], c[1] * c[1], c[2] * c[2], c[0] * c[1], c[0] * c[2], c[1] * c[2]]
    hz = np.ones(NZ) if ZZ is None else np.diff(np.asarray(ZZ, dtype=np.float64))
    wz = hz.reshape(NZ // fz, fz)
    wz = wz / wz.sum(axis=1, keepdims=True)
    out = []
    for a in q:
        b = a.reshape(NZ // fz, fz, NY // fw, fw, NX // fw, fw).mean(axis=(3, 5))
        out.append(np.einsum("zkyx,zk->zyx", b, wz))
    return np.stack(out)


def _ddz(F, ZZ):
    """d/dz of cell-centred columns F[..., z, Y, X] with wall value 0 at ZZ[0], ZZ[NZ]."""
    NZ = F.shape[-3]
    zc = 0.5 * (ZZ[:-1] + ZZ[1:])
    zm = np.concatenate([[ZZ[0]], zc[:-1]])
    zp = np.concatenate([zc[1:], [ZZ[NZ]]])
    Fm = np.concatenate([np.zeros_like(F[..., :1, :, :]), F[..., :-1, :, :]], axis=-3)
    Fp = np.concatenate([F[..., 1:, :, :], np.zeros_like(F[..., :1, :, :])], axis=-3)
    return (Fp - Fm) / (zp - zm)[:, None, None]


def gradient(U, dx, dy, ZZ):
    """U: (3, NZ, NYc, NXc) centred velocities -> G[i][j] (3, 3, NZ, NYc, NXc)."""
    G = np.zeros((3, 3) + U.shape[1:])
    for i in range(3):
        G[i, 0] = (np.roll(U[i], -1, axis=2) - np.roll(U[i], 1, axis=2)) / (2 * dx)
        G[i, 1] = (np.roll(U[i], -1, axis=1) - np.roll(U[i], 1, axis=1)) / (2 * dy)
        G[i, 2] = _ddz(U[i], ZZ)
    return G


def features_from_gradient(G, nu, utau, d):
    """les_features: G (3, 3, ...) physical gradient, d wall distance (broadcast) -> (..., 6)."""
    sc = nu / (utau * utau)
    S = 0.5 * (G + np.swapaxes(G, 0, 1)) * sc
    O = 0.5 * (G - np.swapaxes(G, 0, 1)) * sc
    S2 = np.einsum("ik...,kj...->ij...", S, S)
    O2 = np.einsum("ik...,kj...->ij...", O, O)
    tr = lambda A, B: np.einsum("ij...,ji...->...", A, B)
    lam = [tr(S, S), tr(O, O), tr(S2, S), tr(O2, S), tr(O2, S2)]
    f = [np.arcsinh(l) for l in lam] + [0.25 * np.log1p(d * utau / nu) * np.ones_like(lam[0])]
    return np.stack(f, axis=-1)


def features_targets(F, NXc, NYc, NZ, dx, dy, ZZ, nu, utau):
    """k_les_features: (M, 6) features and (M,) targets nu*/nu from the filtered fields."""
    U = F[0:3]
    G = gradient(U, dx, dy, ZZ)
    zc = 0.5 * (ZZ[:-1] + ZZ[1:])
    d = np.minimum(zc - ZZ[0], ZZ[NZ] - zc)[:, None, None]
    X = features_from_gradient(G, nu, utau, d).reshape(-1, 6)
    tau = np.zeros((3, 3) + U.shape[1:])
    idx = {(0, 0): 4, (1, 1): 5, (2, 2): 6, (0, 1): 7, (0, 2): 8, (1, 2): 9}
    for (i, j), k in idx.items():
        tau[i, j] = F[k] - U[i] * U[j]
        tau[j, i] = tau[i, j]
    trc = (tau[0, 0] + tau[1, 1] + tau[2, 2]) / 3.0
    for i in range(3):
        tau[i, i] -= trc
    S = 0.5 * (G + np.swapaxes(G, 0, 1))
    num = -np.einsum("ij...,ij...->...", tau, S)
    den = 2 * np.einsum("ij...,ij...->...", S, S)
    nus = np.where(den > 1e-300, num / np.where(den > 1e-300, den, 1.0), 0.0)
    return X, (nus / nu).reshape(-1)


def element_features(vel, NX, NY, NZ, hx, hy, ZZ, nu, utau):
    """k_turb_mlp's collocated inputs: per element between the 8 nodes (ix..ix+1, iy..iy+1,
    iz..iz+1), iz < NZ-1, the element gradient of the nodal velocity (vel: (N, 3) at the
    nodes, ZZ the NZ node heights) and the wall distance of the element centre ->
    ((NZ-1) NY NX, 6) features, elements in node-index order."""
    ZZ = np.asarray(ZZ, dtype=np.float64)
    q = vel.reshape(NZ, NY, NX, 3).transpose(3, 0, 1, 2)
    xp = lambda a: np.roll(a, -1, axis=-1)
    yp = lambda a: np.roll(a, -1, axis=-2)
    lo, hi = q[:, :-1], q[:, 1:]
    c = [lo, xp(lo), yp(lo), xp(yp(lo)), hi, xp(hi), yp(hi), xp(yp(hi))]  # 000 100 010 110 001 101 011 111
    hz = np.diff(ZZ)[:, None, None]
    G = np.zeros((3, 3) + lo.shape[1:])
    G[:, 0] = ((c[1] + c[3] + c[5] + c[7]) - (c[0] + c[2] + c[4] + c[6])) / (4 * hx)
    G[:, 1] = ((c[2] + c[3] + c[6] + c[7]) - (c[0] + c[1] + c[4] + c[5])) / (4 * hy)
    G[:, 2] = ((c[4] + c[5] + c[6] + c[7]) - (c[0] + c[1] + c[2] + c[3])) / (4 * hz)
    zc = 0.5 * (ZZ[:-1] + ZZ[1:])
    d = np.minimum(zc - ZZ[0], ZZ[-1] - zc)[:, None, None]
    return features_from_gradient(G, nu, utau, d).reshape(-1, 6)


def smagorinsky_nut(X, hx, hy, dz_local, utau, nu, cs=0.1):
    """The reference's Smagorinsky-van Driest model (staggered/func_global.h:875-890, as in
    k_turb_stag's smag_nut) as nu_t/nu from the features: |S| = sqrt(2 S:S) from tr(S^2),
    y+ from the last feature, Delta = min(cs (hx hy dz)^(1/3), 0.41 d), damping
    1 - exp(-(0.04 y+)^3)."""
    l1 = np.sinh(X[:, 0].astype(np.float64))
    Splus = np.sqrt(np.maximum(2.0 * l1, 0.0))
    yplus = np.expm1(4.0 * X[:, 5].astype(np.float64))
    d = yplus * nu / utau
    dl = np.minimum(cs * (hx * hy * dz_local) ** (1.0 / 3.0), 0.41 * d)
    fvd = 1.0 - np.exp(-(0.04 * yplus) ** 3)
    return fvd * (dl * utau / nu) ** 2 * Splus


# ----------------------------------------------------------------------------- network
def bf16(x):
    """Round to bfloat16 (nearest even), returned as float32."""
    b = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).reshape(np.shape(x))


def unpack(P):
    P = np.asarray(P)
    return (P[OW1:OB1].reshape(MLP_IN, MLP_H), P[OB1:OW2], P[OW2:OB2].reshape(MLP_H, MLP_H), P[OB2:OW3],
            P[OW3:OB3], P[OB3])


def _sig(z):
    return 1.0 / (1.0 + np.exp(-z))


def _silu(z):
    return z * _sig(z)


def _dsilu(z):
    s = _sig(z)
    return s * (1.0 + z * (1.0 - s))


def _softplus(z):
    return np.where(z > 20.0, z, np.log1p(np.exp(np.minimum(z, 20.0))))


def _f64(x):
    return np.asarray(x, dtype=np.float64)


def mlp_forward(P, X, return_cache=False, rnd=bf16):
    """rnd: the rounding applied where the kernels round to bf16 (identity: exact math)."""
    W1, b1, W2, b2, w3, b3 = [_f64(a) for a in unpack(P)]
    r = (lambda a: _f64(rnd(a))) if rnd is not None else _f64
    xb = r(X)
    z1 = xb @ r(W1) + b1
    h1b = r(_silu(z1))
    z2 = h1b @ r(W2) + b2
    h2b = r(_silu(z2))
    z3 = h2b @ r(w3) + float(b3)
    out = _softplus(z3)
    if return_cache:
        return out, (xb, z1, h1b, z2, h2b, z3)
    return out


def mlp_grad(P, X, Y, rnd=bf16):
    """Gradient (packed like P) and loss of mean((out - Y)^2), k_mlp_grad's roundings."""
    W1, b1, W2, b2, w3, b3 = [_f64(a) for a in unpack(P)]
    r = (lambda a: _f64(rnd(a))) if rnd is not None else _f64
    n = len(Y)
    out, (xb, z1, h1b, z2, h2b, z3) = mlp_forward(P, X, True, rnd)
    d = out - np.asarray(Y, dtype=np.float64)
    loss = float(np.mean(d * d))
    gz3 = 2.0 * d / n * _sig(z3)
    g = np.zeros(NPAR)
    w3b = r(w3)
    g[OW3:OB3] = gz3 @ h2b
    g[OB3] = gz3.sum()
    gz2b = r(gz3[:, None] * w3b[None, :] * _dsilu(z2))
    g[OW2:OB2] = (h1b.T @ gz2b).reshape(-1)
    g[OB2:OW3] = gz2b.sum(axis=0)
    gh1 = gz2b @ r(W2).T
    gz1b = r(gh1 * _dsilu(z1))
    g[OW1:OB1] = (xb.T @ gz1b).reshape(-1)
    g[OB1:OW2] = gz1b.sum(axis=0)
    return g, loss


def adam_step(P, M, V, g, lr, step, b1=0.9, b2=0.999, eps=1e-8):
    M = b1 * M + (1 - b1) * g
    V = b2 * V + (1 - b2) * g * g
    c1, c2 = 1 - b1 ** step, 1 - b2 ** step
    return P - lr * (M / c1) / (np.sqrt(V / c2) + eps), M, V
