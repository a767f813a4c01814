"""GPU checks of the learned LES closure against its CPU oracle (oracle/les_oracle.py).

Tolerances:
  filtered fields and features: 1e-5 relative (double arithmetic on the GPU, float32 output);
  targets: 1e-4 of their maximum (a ratio of small numbers near zero strain);
  network forward: 2e-3 relative, gradients: 2e-2 relative in the 2-norm per block -- the
  BF16 roundings of the kernels and of the oracle agree except where an FP32 value sits
  next to a rounding boundary;
  nu_t of a run: 1e-2 relative in the 2-norm.
"""
import numpy as np
import pytest

import les_oracle as lo
from cases import HW2, VV4, make_case, rel_err

pytestmark = pytest.mark.gpu


def _solver(scheme, NX, NY, NZ, precision, turb=0, steps=3):
    import turbchannel_b200 as tb

    prod, _, zz = make_case(scheme=scheme, NX=NX, NY=NY, NZ=NZ, precision=precision, turb=turb)
    S = tb.Solver(prod, zz)
    S.init_channel(0, seed=12345, amp=0.1, project=True)
    tau = 2e-3
    for it in range(steps):
        S.Step(it * tau, tau, it % 4, min(it + 1, 3))
    return S, prod, zz, steps % 4


@pytest.mark.parametrize("fz", [1, 4])
@pytest.mark.parametrize("precision", [0, 1])
def test_filter_and_samples_match_oracle(precision, fz):
    S, p, zz, lev = _solver(VV4, 32, 16, 24, precision)
    fw = 4
    vel, pr = S.download_level(lev)
    F = S.les_filter(lev, fw, fz)
    Fo = lo.box_filter(vel, pr, 32, 16, 24, fw, fz, np.asarray(zz))
    for k in range(10):
        assert rel_err(F[k], Fo[k]) < 1e-5, k
    X, Y = S.les_samples(lev, fw, fz)
    utau = p["inv_length_scale"] * p["visc"]
    Xo, Yo = lo.features_targets(Fo, 8, 4, 24 // fz, fw * p["hx"], fw * p["hy"], np.asarray(zz)[::fz], p["visc"],
                                 utau)
    for k in range(6):
        assert rel_err(X[:, k], Xo[:, k]) < 1e-5, k
    assert np.max(np.abs(Y - Yo)) <= 1e-4 * max(np.max(np.abs(Yo)), 1e-30)
    S.close()


def _teacher_data(n, seed):
    rng = np.random.default_rng(seed)
    X = rng.normal(size=(n, 6)).astype(np.float32)
    P = np.zeros(lo.NPAR, dtype=np.float32)
    P[lo.OW1:lo.OB1] = rng.uniform(-0.4, 0.4, lo.OB1 - lo.OW1)
    P[lo.OW2:lo.OB2] = rng.uniform(-0.125, 0.125, lo.MLP_H * lo.MLP_H)
    P[lo.OW3:lo.OB3] = rng.uniform(-0.5, 0.5, lo.MLP_H)
    P[lo.OB3] = 0.2
    return X, P


def test_mlp_forward_and_gradient_match_oracle():
    import turbchannel_b200 as tb

    m = tb.Mlp(seed=7)
    P = m.params
    X, _ = _teacher_data(1000, 3)
    Y = np.abs(np.random.default_rng(4).normal(size=1000)).astype(np.float32)
    out = m.forward(X)
    assert rel_err(out, lo.mlp_forward(P, X)) < 2e-3
    g, loss = m.grad(X, Y)
    go, lo_loss = lo.mlp_grad(P, X, Y)
    assert abs(loss - lo_loss) <= 2e-3 * lo_loss
    blocks = [(lo.OW1, lo.OB1), (lo.OB1, lo.OW2), (lo.OW2, lo.OB2), (lo.OB2, lo.OW3), (lo.OW3, lo.OB3), (lo.OB3, lo.NPAR)]
    for a, b in blocks:
        err = np.linalg.norm(g[a:b] - go[a:b]) / max(np.linalg.norm(go[a:b]), 1e-30)
        assert err < 2e-2, (a, b, err)
    m.close()


def test_adam_step_matches_oracle():
    import turbchannel_b200 as tb

    m = tb.Mlp(seed=11)
    P0 = m.params.astype(np.float64)
    X, _ = _teacher_data(512, 5)
    Y = np.abs(np.random.default_rng(6).normal(size=512)).astype(np.float32)
    g, _ = m.grad(X, Y)
    m.set_data(X, Y)
    m.train(1, 512, 1e-3)  # one batch = one Adam step from zero moments
    P1 = m.params
    Po, _, _ = lo.adam_step(P0, np.zeros(lo.NPAR), np.zeros(lo.NPAR), g.astype(np.float64), 1e-3, 1)
    assert np.max(np.abs(P1 - Po)) < 1e-6
    m.close()


def test_training_fits_a_teacher_network():
    import turbchannel_b200 as tb

    X, Pt = _teacher_data(20000, 8)
    Y = lo.mlp_forward(Pt, X).astype(np.float32)
    m = tb.Mlp(seed=9)
    m.set_data(X, Y)
    loss = m.train(60, 1000, 3e-3)
    assert np.all(np.isfinite(loss))
    assert loss[-1] < 0.1 * loss[0], (loss[0], loss[-1])
    m.close()


def test_learned_closure_beats_no_model_and_smagorinsky():
    """On held-out filtered-DNS samples the trained closure predicts the sub-filter eddy
    viscosity better than no model (nu_t = 0) and than Smagorinsky-van Driest."""
    import turbchannel_b200 as tb

    prod, _, zz = make_case(scheme=HW2, NX=64, NY=32, NZ=48, precision=1, Re_b=5600.0)
    S = tb.Solver(prod, zz)
    S.init_channel(0, seed=12345, amp=0.3, project=True)
    S.set_forcing(1, 1.0)
    tau, cur = 2e-3, 0
    Xs, Ys = [], []
    for it in range(400):
        S.Step(it * tau, tau, cur, min(it + 1, 3))
        cur = (cur + 1) % 4
        if it >= 200 and it % 40 == 0:
            X, Y = S.les_samples(cur, 4)
            Xs.append(X)
            Ys.append(Y)
    S.close()
    Xtr, Ytr = np.concatenate(Xs[:-1]), np.concatenate(Ys[:-1])
    Xte, Yte = Xs[-1], Ys[-1]
    rng = np.random.default_rng(0)
    perm = rng.permutation(len(Ytr))
    m = tb.Mlp(seed=3)
    m.set_data(Xtr[perm], Ytr[perm])
    m.train(150, 1024, 2e-3)
    pred = m.forward(Xte)
    m.close()
    mse = lambda a: float(np.mean((a - Yte) ** 2))
    zc = 0.5 * (zz[:-1] + zz[1:])
    dz = np.diff(zz)
    dzl = np.broadcast_to(dz[:, None], (48, (64 // 4) * (32 // 4))).reshape(-1)
    utau = prod["inv_length_scale"] * prod["visc"]
    smag = lo.smagorinsky_nut(Xte, 4 * prod["hx"], 4 * prod["hy"], dzl, utau, prod["visc"])
    e_mlp, e_none, e_smag = mse(pred), mse(np.zeros_like(Yte)), mse(smag)
    assert e_mlp < 0.9 * e_none, (e_mlp, e_none, e_smag)
    assert e_mlp < e_smag, (e_mlp, e_none, e_smag)


def test_run_with_learned_closure_matches_oracle_nu_t():
    import turbchannel_b200 as tb

    prod, _, zz = make_case(scheme=HW2, NX=32, NY=16, NZ=24, precision=0, turb=1)
    S = tb.Solver(prod, zz)
    m = tb.Mlp(seed=21)
    P = m.params
    m.close()
    S.set_turb_model(tb.TURB_MLP, P)
    S.init_channel(0, seed=5, amp=0.2, project=True)
    v, _ = S.download_level(0)
    nt = S.RecalcTurbVisc(v)
    Fo = lo.box_filter(v, np.zeros(len(v)), 32, 16, 24, 1)
    utau = prod["inv_length_scale"] * prod["visc"]
    G = lo.gradient(Fo[0:3], prod["hx"], prod["hy"], np.asarray(zz))
    zc = 0.5 * (zz[:-1] + zz[1:])
    d = np.minimum(zc - zz[0], zz[-1] - zc)[:, None, None]
    X = lo.features_from_gradient(G, prod["visc"], utau, d).reshape(-1, 6).astype(np.float32)
    want = prod["visc"] * lo.mlp_forward(P, X)
    assert np.all(nt >= 0) and np.all(np.isfinite(nt))
    assert np.linalg.norm(nt - want) / np.linalg.norm(want) < 1e-2
    tau = 2e-3
    for it in range(10):
        S.Step(it * tau, tau, it % 4, min(it + 1, 3))
    v2, p2 = S.download_level(10 % 4)
    assert np.all(np.isfinite(v2)) and np.all(np.isfinite(p2))
    S.close()


def test_collocated_run_with_learned_closure_matches_oracle_nu_t():
    """The closure on the collocated scheme: nu_t on the elements from the element
    gradient of the nodal velocity, against the oracle's features and network; the top
    node plane (no element) keeps nu_t = 0; a short run stays finite."""
    import turbchannel_b200 as tb
    from cases import COLLOC

    NX, NY, NZ = 32, 16, 25
    prod, _, zz = make_case(scheme=COLLOC, NX=NX, NY=NY, NZ=NZ, precision=0, turb=1)
    S = tb.Solver(prod, zz)
    m = tb.Mlp(seed=23)
    P = m.params
    m.close()
    S.set_turb_model(tb.TURB_MLP, P)
    S.init_channel(0, seed=5, amp=0.2, project=True)
    v, _ = S.download_level(0)
    nt = S.RecalcTurbVisc(v)
    utau = prod["inv_length_scale"] * prod["visc"]
    X = lo.element_features(v, NX, NY, NZ, prod["hx"], prod["hy"], np.asarray(zz), prod["visc"], utau)
    want = prod["visc"] * lo.mlp_forward(P, X.astype(np.float32))
    ne = NX * NY * (NZ - 1)
    assert np.all(np.isfinite(nt)) and np.all(nt[:ne] >= 0)
    assert np.linalg.norm(nt[:ne] - want) / np.linalg.norm(want) < 1e-2
    assert not nt[ne:].any()
    tau = 1e-3
    S.set_forcing(1, 1.0)
    for it in range(10):
        S.Step(it * tau, tau, it % 4, min(it + 1, 3))
    v2, p2 = S.download_level(10 % 4)
    assert np.all(np.isfinite(v2)) and np.all(np.isfinite(p2))
    S.close()


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("shape", [(HW2, 32, 16, 24), (HW2, 54, 18, 9), (VV4, 36, 18, 20), (HW2, 64, 24, 40)])
def test_closure_fused_into_flux_matches_separate_pass(shape, precision):
    """tc_set_mlp_fusion(h, 1): the flux kernel evaluates the network for the planes it
    stages (tile plus a one-cell halo).  Against the separate pass (k_turb_mlp, then the
    flux kernel) over six steps.  The arithmetic is the same, but the compiler may fuse
    multiply-adds differently in the two kernels, and in either precision a float-rounding
    difference in a feature can move it across a BF16 rounding boundary of the network
    (measured: 2 of 61 440 cells, 2e-5 relative, in FP64), so nu_t agrees to 1e-3 in the
    2-norm and the fields to 1e-7 (FP64) or the mixed step tolerance (2e-4 velocity, 4e-3
    pressure), relative to the max-norm.  nu_t of the first step also against the oracle's features and network
    (1e-2 in the 2-norm, as the separate-pass test).  Shapes cover partial tiles in x and
    y (54 x 18, 36 x 18), one z-chunk (9 planes) and several (40), and VV4's wider
    stencil."""
    import turbchannel_b200 as tb

    scheme, NX, NY, NZ = shape
    prod, _, zz = make_case(scheme=scheme, NX=NX, NY=NY, NZ=NZ, precision=precision, turb=1)
    m = tb.Mlp(seed=21)
    P = m.params
    m.close()
    runs = []
    for fuse in (0, 1):
        S = tb.Solver(prod, zz)
        S.set_turb_model(tb.TURB_MLP, P)
        S.set_mlp_fusion(fuse)
        S.init_channel(0, seed=5, amp=0.2, project=True)
        tau, cur = 2e-3, 0
        nts = []
        for it in range(6):
            S.Step(it * tau, tau, cur, min(it + 1, 3))
            cur = (cur + 1) % 4
            nts.append(S.get_nu_t())
        v, p = S.download_level(cur)
        runs.append((v, p, nts))
        S.close()
    (v0, p0, n0), (v1, p1, n1) = runs
    for a, b in zip(n0, n1):
        assert np.linalg.norm(b - a) / np.linalg.norm(a) < 1e-3
    tv, tp = (1e-7, 1e-7) if precision == 0 else (2e-4, 4e-3)
    assert rel_err(v1, v0) < tv and rel_err(p1, p0) < tp
    # the first step's nu_t is the closure of the initial field: against the oracle
    S = tb.Solver(prod, zz)
    S.init_channel(0, seed=5, amp=0.2, project=True)
    v, _ = S.download_level(0)
    S.close()
    Fo = lo.box_filter(v, np.zeros(len(v)), NX, NY, NZ, 1)
    utau = prod["inv_length_scale"] * prod["visc"]
    G = lo.gradient(Fo[0:3], prod["hx"], prod["hy"], np.asarray(zz))
    zc = 0.5 * (zz[:-1] + zz[1:])
    d = np.minimum(zc - zz[0], zz[-1] - zc)[:, None, None]
    X = lo.features_from_gradient(G, prod["visc"], utau, d).reshape(-1, 6).astype(np.float32)
    want = prod["visc"] * lo.mlp_forward(P, X)
    assert np.linalg.norm(n1[0] - want) / np.linalg.norm(want) < 1e-2
