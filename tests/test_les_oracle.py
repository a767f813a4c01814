"""CPU checks of the learned-closure oracle (oracle/les_oracle.py): BF16 rounding,
the analytic MLP gradient against finite differences (roundings off), and the
filter/feature/target definitions on fields with known answers."""
import numpy as np

import les_oracle as lo


def test_bf16_rounding_known_values():
    x = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -9, -2.5, 0.0, 1e-3], dtype=np.float32)
    got = lo.bf16(x)
    # 1 + 2^-8 is halfway between 1 and 1 + 2^-7: ties to even -> 1; 1 + 3*2^-9 rounds up
    want = np.array([1.0, 1.0, 1.0 + 2.0 ** -7, -2.5, 0.0, np.float32(0.00099945068359375)], dtype=np.float32)
    assert np.array_equal(got, want)


def _random_net(seed):
    rng = np.random.default_rng(seed)
    P = np.zeros(lo.NPAR)
    P[lo.OW1:lo.OB1] = rng.uniform(-0.4, 0.4, lo.OB1 - lo.OW1)
    P[lo.OB1:lo.OW2] = rng.uniform(-0.1, 0.1, lo.MLP_H)
    P[lo.OW2:lo.OB2] = rng.uniform(-0.125, 0.125, lo.MLP_H * lo.MLP_H)
    P[lo.OB2:lo.OW3] = rng.uniform(-0.1, 0.1, lo.MLP_H)
    P[lo.OW3:lo.OB3] = rng.uniform(-0.125, 0.125, lo.MLP_H)
    P[lo.OB3] = -0.5
    X = rng.normal(size=(40, 6))
    Y = np.abs(rng.normal(size=40))
    return P, X, Y


def test_mlp_gradient_matches_finite_differences():
    P, X, Y = _random_net(1)
    g, loss = lo.mlp_grad(P, X, Y, rnd=None)
    rng = np.random.default_rng(2)
    idx = np.concatenate([rng.choice(np.arange(lo.OW1, lo.OB1), 6), rng.choice(np.arange(lo.OB1, lo.OW2), 3),
                          rng.choice(np.arange(lo.OW2, lo.OB2), 8), rng.choice(np.arange(lo.OB2, lo.OW3), 3),
                          rng.choice(np.arange(lo.OW3, lo.OB3), 4), [lo.OB3]])
    h = 1e-6
    for k in idx:
        Pp, Pm = P.copy(), P.copy()
        Pp[k] += h
        Pm[k] -= h
        lp = np.mean((lo.mlp_forward(Pp, X, rnd=None) - Y) ** 2)
        lm = np.mean((lo.mlp_forward(Pm, X, rnd=None) - Y) ** 2)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(fd)), (k, fd, g[k])


def test_linear_shear_filters_to_zero_subfilter_stress():
    NX, NY, NZ, fw = 16, 8, 12, 4
    ZZ = 1.0 + np.tanh(1.8 * (2.0 * np.arange(NZ + 1) / NZ - 1.0)) / np.tanh(1.8)
    zc = 0.5 * (ZZ[:-1] + ZZ[1:])
    vel = np.zeros((NX * NY * NZ, 3))
    vel[:, 0] = np.repeat(3.0 * zc, NX * NY)  # u depends on z only: the x/y filter changes nothing
    p = np.zeros(NX * NY * NZ)
    F = lo.box_filter(vel, p, NX, NY, NZ, fw)
    assert np.allclose(F[0], np.broadcast_to(3.0 * zc[:, None, None], F[0].shape))
    X, Y = lo.features_targets(F, NX // fw, NY // fw, NZ, fw * 0.1, fw * 0.2, ZZ, 1e-3, 0.05)
    assert X.shape == ((NX // fw) * (NY // fw) * NZ, 6) and np.all(Y == 0.0)
    # tr(O^2) = -tr(S^2) for a pure shear; y+ feature from the wall distance
    assert np.allclose(X[:, 1], -X[:, 0])
    d = np.minimum(zc - ZZ[0], ZZ[NZ] - zc)
    assert np.allclose(X.reshape(NZ, -1, 6)[:, 0, 5], 0.25 * np.log1p(d * 0.05 / 1e-3))


def test_wall_normal_filter_is_volume_weighted():
    """fz > 1: each coarse cell holds the volume-weighted mean of its fz x fw x fw fine
    cells (domain integrals are kept), a z-only field gets the variance within the coarse
    cell as its uu sub-filter stress, and fz = 1 is the x-y filter alone."""
    NX, NY, NZ, fw, fz = 8, 8, 12, 2, 4
    ZZ = 1.0 + np.tanh(1.8 * (2.0 * np.arange(NZ + 1) / NZ - 1.0)) / np.tanh(1.8)
    hz = np.diff(ZZ)
    rng = np.random.default_rng(3)
    vel = rng.normal(size=(NX * NY * NZ, 3))
    vel[:NX * NY, 2] = 0.0  # w = 0 on the bottom wall
    p = rng.normal(size=NX * NY * NZ)
    F = lo.box_filter(vel, p, NX, NY, NZ, fw, fz, ZZ)
    assert F.shape == (10, NZ // fz, NY // fw, NX // fw)
    c = lo.cell_centred(vel, NX, NY, NZ)
    Hc = hz.reshape(-1, fz).sum(axis=1)
    for k in range(3):
        fine = np.sum(c[k] * hz[:, None, None])
        coarse = np.sum(F[k] * Hc[:, None, None]) * fw * fw
        assert abs(fine - coarse) <= 1e-12 * max(1.0, abs(fine))
    assert np.allclose(lo.box_filter(vel, p, NX, NY, NZ, fw, 1, ZZ), lo.box_filter(vel, p, NX, NY, NZ, fw))
    zc = 0.5 * (ZZ[:-1] + ZZ[1:])
    v2 = np.zeros_like(vel)
    v2[:, 0] = np.repeat(zc, NX * NY)
    F2 = lo.box_filter(v2, np.zeros(len(p)), NX, NY, NZ, fw, fz, ZZ)
    wz = (hz / np.repeat(Hc, fz)).reshape(-1, fz)
    m = (zc.reshape(-1, fz) * wz).sum(axis=1)
    var = ((zc.reshape(-1, fz) - m[:, None]) ** 2 * wz).sum(axis=1)
    assert np.allclose(F2[0][:, 0, 0], m) and np.allclose(F2[4][:, 0, 0] - m * m, var)
