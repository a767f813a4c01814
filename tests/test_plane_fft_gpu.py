"""The pressure solve's plane kernels (csrc/k_fft_plane.cu: the x- and y-FFTs of each
z-plane in one thread-block cluster) against the separate x- and y-FFT kernels and the
oracle, for the scalar solve (tc_op_pressure_solve) and through full steps (the
divergence of the vector RHS feeding the forward plane kernel)."""
import numpy as np
import pytest

from cases import COLLOC, HW2, VV4, make_case, rel_err, seeded_field, within

# (NX, NY) pairs with plane kernels, staggered and collocated; the last grid has none
# (both settings take the separate kernels)
GRIDS = {
    "vv4_32x16": dict(scheme=VV4, NX=32, NY=16, NZ=12),
    "hw2_64x64": dict(scheme=HW2, NX=64, NY=64, NZ=64),
    "coll_64x32": dict(scheme=COLLOC, NX=64, NY=32, NZ=9),
    "vv4_32x32": dict(scheme=VV4, NX=32, NY=32, NZ=20),
    "hw2_128x128": dict(scheme=HW2, NX=128, NY=128, NZ=6),
}
PLANE = {"vv4_32x16", "hw2_64x64", "coll_64x32", "vv4_32x32"}
# plane vs separate kernels on the same inputs: the same arithmetic, FMA contraction aside
SAME = {0: 1e-13, 1: 2e-6}


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("name", list(GRIDS))
def test_plane_pressure_solve(name, precision):
    import oracle_py as op
    import turbchannel_b200 as tb

    prod, orc, zz = make_case(precision=precision, **GRIDS[name])
    S = tb.Solver(prod, zz)
    O = op.Oracle(orc, zz, "f64")
    NXY = S.NX * S.NY
    coll = GRIDS[name]["scheme"] == COLLOC
    v = seeded_field(S.N, NXY, seed=3, wall_w_zero=not coll)
    if coll:
        v[:NXY] = 0.0
        v[-NXY:] = 0.0
    rhs = O.apply_divergence(v)
    want = O.pressure_solve(rhs)
    S.set_fft_fusion(1)
    fused = S.LinearSystemSolveFFT(rhs)
    S.set_fft_fusion(0)
    sep = S.LinearSystemSolveFFT(rhs)
    L = f"plane/{name}/p{precision}"
    if name not in PLANE:
        assert np.array_equal(fused, sep)
    assert within(L + "/same", rel_err(fused, sep), SAME[precision]), rel_err(fused, sep)
    # mixed: float transforms, whose round-off grows with the line lengths (2.2e-6 measured at 192 x 192)
    tol = 1e-10 if precision == 0 else 6e-6
    assert within(L + "/oracle", rel_err(fused, want), tol), rel_err(fused, want)
    with pytest.raises(tb.TcError):
        S.set_fft_fusion(2)
    S.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("name", ["vv4_32x16", "coll_64x32", "hw2_64x64"])
def test_plane_steps(name, precision):
    """Three SBDF steps (orders 1-3) from the oracle's seeded, projected channel field with
    the plane kernels and with the separate kernels, and against the oracle."""
    import oracle_py as op
    import turbchannel_b200 as tb

    prod, orc, zz = make_case(precision=precision, **GRIDS[name])
    O = op.Oracle(orc, zz, "f64")
    O.init_channel(0, seed=12345, amp=0.1, project=True)
    v0, p0 = O.get_level(0)
    tau = 1e-3
    runs = []
    for mode in (1, 0):
        S = tb.Solver(prod, zz)
        S.set_fft_fusion(mode)
        for lvl in range(4):
            S.upload_level(lvl, np.zeros_like(v0), np.zeros_like(p0))
        S.upload_level(0, v0, p0)
        cur = 0
        for it in range(3):
            S.Step(it * tau, tau, cur, it + 1)
            cur = (cur + 1) % 4
        runs.append(S.download_level(cur))
        S.close()
    cur = 0
    for it in range(3):
        O.step(it * tau, tau, cur, it + 1)
        cur = (cur + 1) % 4
    vo, po = O.get_level(cur)
    (vf, pf), (vs, ps) = runs
    L = f"plane_step/{name}/p{precision}"
    assert within(L + "/same_vel", rel_err(vf, vs), SAME[precision]), rel_err(vf, vs)
    assert within(L + "/same_pres", rel_err(pf, ps), 1e-12 if precision == 0 else 2e-4), rel_err(pf, ps)
    assert within(L + "/vel", rel_err(vf, vo), 1e-10 if precision == 0 else 3e-6), rel_err(vf, vo)
    assert within(L + "/pres", rel_err(pf, po), 2e-9 if precision == 0 else 4.5e-3), rel_err(pf, po)
