"""The segregated IMEX Runge-Kutta step of the collocated scheme on the CPU: the method
tables (order conditions, collocated_SRK/imex.cpp:7-33) and the oracle's restatement of
data::Step (collocated_SRK/func_global.h:317-408) against the reference's own CPU solver
compiled from its sources (oracle/_ref/libref_srk_f64.so, NX = 128, NY = 64)."""
import os
import sys

import numpy as np
import pytest

from cases import COLLOC, make_case, rel_err, seeded_field

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))

from turbchannel_b200 import imex  # noqa: E402

ORDERS = {"ARS_121": 1, "ARS_232": 2, "ARS_343": 3, "MARS_343": 3, "ARK3": 3, "ARK4": 3, "MARK3": 3, "BHR_553": 3}
REF_LIB = os.path.join(os.path.dirname(__file__), "..", "oracle", "_ref", "libref_srk_f64.so")


@pytest.mark.parametrize("name", list(imex.METHODS))
def test_tables_meet_their_order_conditions(name):
    m = imex.METHODS[name]()
    assert len(m.E) == len(m.I) == m.S * (m.S + 1)
    order = ORDERS[name]
    for table in (m.E, m.I):
        s = imex.order_sums(m.S, table)
        conds = [s[0]] + ([s[1]] if order >= 2 else []) + (list(s[2:]) if order >= 3 else [])
        assert max(abs(c) for c in conds) < 1e-12, (name, s)
    # both tables share their weights, the implicit one is stiffly accurate (last row = b)
    S = m.S
    assert np.allclose(m.I[S * S:], m.I[(S - 1) * S:S * S])


def srk_case(NZ=13, precision=0):
    prod, orc, zz = make_case(scheme=COLLOC, NX=128, NY=64, NZ=NZ, precision=precision)
    N = 128 * 64 * NZ
    NXY = 128 * 64
    v = 0.3 * seeded_field(N, NXY, seed=21, wall_w_zero=False)
    v[:NXY] = 0.0
    v[-NXY:] = 0.0
    v[:, 0] += 1.0
    v[:NXY, 0] = 0.0
    v[-NXY:, 0] = 0.0
    rng = np.random.default_rng(22)
    p = 1e-2 * rng.standard_normal(N)
    q = 1e-2 * rng.standard_normal(N)
    return prod, orc, zz, v, p, q


CASES = [("ARS_343", 1), ("ARS_232", 0), ("ARS_121", 1), ("MARS_343", 0), ("ARK3", 1), ("ARK4", 0), ("MARK3", 1),
         ("BHR_553", 0), ("ARS_232:A", 1), ("ARS_343:A", 0)]


def method(name):
    """A table of turbchannel_b200.imex; "X:A" runs X's tables in the type-A formulation
    (no explicit pre-stage, func_global.h:324 and :333), which no published method uses."""
    base, _, kind = name.partition(":")
    m = imex.METHODS[base]()
    if kind == "A":
        m.kind = imex.A
    return m


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="reference SRK build absent (make -C oracle ref)")
@pytest.mark.parametrize("name,stab", CASES)
def test_oracle_step_matches_reference(name, stab):
    import oracle_py as op
    from srk_oracle import RefSrk, SrkOracle

    prod, orc, zz, v, p, q = srk_case()
    m = method(name)
    at = m.alpha_tau(stab)
    O = op.Oracle(orc, zz, "f64")
    so = SrkOracle(O, orc, zz, m.kind, m.S, m.E, m.I, stab, at)
    ref = RefSrk(orc, zz, m.kind, m.S, m.E, m.I, stab, at)
    tau = 2e-3
    a = (v, p, q)
    b = (v, p, q)
    for k in range(2):
        a = so.step(tau, *a)
        b = ref.step(k * tau, tau, *b)
    assert rel_err(a[0], b[0]) < 1e-12
    assert rel_err(a[1], b[1]) < 1e-10
    if stab:
        assert rel_err(a[2], b[2]) < 1e-9
