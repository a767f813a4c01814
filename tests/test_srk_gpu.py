"""GPU parity of the segregated IMEX Runge-Kutta step of the collocated scheme
(tc_srk_step, collocated_SRK/func_global.h:317-408) against the oracle's restatement
(oracle/srk_oracle.py, itself checked against the reference's CPU solver), for methods of
both formulations (ARS, CK) and both StabTypes.

Tolerances (relative to the max-norm of the oracle result), after three steps:
  FP64 : velocity 1e-10, pressure and dp/dt 1e-8 (round-off from FMA contraction,
         FFT ordering and summation order);
  MIXED: float storage and arithmetic against the FP64 oracle, velocity 2e-4,
         pressure 5e-2 (the pressure of a stage is a difference of nearly equal terms
         of size p / tau_stage).
"""
import os
import sys

import numpy as np
import pytest

from cases import COLLOC, make_case, rel_err, seeded_field

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))

pytestmark = pytest.mark.gpu

CASES = [("ARS_343", 1), ("ARS_232", 0), ("ARK3", 1), ("ARK4", 0), ("BHR_553", 1), ("MARS_343", 0), ("ARS_232:A", 1)]
TOL = {0: dict(v=1e-10, p=1e-8), 1: dict(v=2e-4, p=5e-2)}


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("name,stab", CASES)
def test_srk_steps_match_oracle(name, stab, precision):
    _srk_case(name, stab, precision, 32, 16, 17)


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("name,stab", [("ARS_343", 1), ("ARK3", 0)])
def test_srk_steps_match_oracle_ragged(name, stab, precision):
    """NX, NY = 36, 18: a y-length without a compiled register transform (the pressure
    solve's fallback kernels) and a non-power-of-two x-length."""
    _srk_case(name, stab, precision, 36, 18, 11)


def _srk_case(name, stab, precision, NX, NY, NZ):
    import oracle_py as op
    from srk_oracle import SrkOracle

    import turbchannel_b200 as tb
    from turbchannel_b200 import imex

    prod, orc, zz = make_case(scheme=COLLOC, NX=NX, NY=NY, NZ=NZ, precision=precision)
    N, NXY = NX * NY * NZ, NX * NY
    v = 0.3 * seeded_field(N, NXY, seed=31, wall_w_zero=False)
    v[:, 0] += 1.0
    v[:NXY] = 0.0
    v[-NXY:] = 0.0
    rng = np.random.default_rng(32)
    p = 1e-2 * rng.standard_normal(N)
    q = 1e-2 * rng.standard_normal(N) if stab else np.zeros(N)
    base, _, kind = name.partition(":")
    m = imex.METHODS[base]()
    if kind == "A":  # the type-A formulation (no explicit pre-stage)
        m.kind = imex.A
    O = op.Oracle(orc, zz, "f64")
    so = SrkOracle(O, orc, zz, m.kind, m.S, m.E, m.I, stab, m.alpha_tau(stab))
    S = tb.Solver(prod, zz)
    S.srk_init(m, stab)
    S.upload_level(0, v, p)
    S.upload_level(1, np.zeros((N, 3)), q)
    tau = 2e-3
    want = (v, p, q)
    for k in range(3):
        S.srk_step(k * tau, tau)
        want = so.step(tau, *want)
    gv, gp = S.download_level(0)
    _, gq = S.download_level(1)
    tol = TOL[precision]
    assert np.all(np.isfinite(gv)) and np.all(np.isfinite(gp))
    assert rel_err(gv, want[0]) < tol["v"]
    assert rel_err(gp, want[1]) < tol["p"]
    if stab:
        assert rel_err(gq, want[2]) < tol["p"]
    S.close()


def test_srk_init_rejects_unsupported_handles():
    import turbchannel_b200 as tb
    from turbchannel_b200 import imex

    prod, _, zz = make_case(scheme=COLLOC, NX=32, NY=16, NZ=17, turb=1)
    S = tb.Solver(prod, zz)
    with pytest.raises(tb.TcError):
        S.srk_init(imex.ARS_343(), 1)
    S.close()
    prod, _, zz = make_case(scheme=COLLOC, NX=32, NY=16, NZ=17)
    S = tb.Solver(prod, zz)
    with pytest.raises(tb.TcError):
        S.srk_step(0.0, 1e-3)  # before srk_init
    S.close()
