"""tc_op_pressure_solve_static: the pressure solve on device buffers whose z-solve
scratch is a static device array (no allocation at call time), against the host-buffer
entry point tc_op_pressure_solve on the same right-hand sides.

Tolerances (relative to the max-norm of tc_op_pressure_solve's result): FP64 1e-10,
MIXED 1e-4 (both run the same launches; only where the z-solve keeps its coefficients
differs).  Two calls in a row check that nothing left in the shared array from one
call leaks into the next.  This file is collected last, so it also runs after every
other GPU test in the same process.
"""
import ctypes as C

import numpy as np
import pytest

from cases import COLLOC, HW2, VV4, make_case, rel_err

pytestmark = pytest.mark.gpu

CASES = {
    "vv4": dict(scheme=VV4, NX=64, NY=32, NZ=48),
    "hw2": dict(scheme=HW2, NX=48, NY=24, NZ=20),
    "coll": dict(scheme=COLLOC, NX=32, NY=16, NZ=25),
}
TOL = {0: 1e-10, 1: 1e-4}


def _static_solve(S, level, rhs):
    """Upload rhs as the pressure of ring level `level`, solve in place on the device."""
    S.upload_level(level, p=rhs)
    _, p_dev = S.device_level(level)
    S._check(S.L.tc_op_pressure_solve_static(S.h, C.c_void_p(p_dev), C.c_void_p(p_dev)))
    S.sync()
    return S.download_level(level)[1]


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("name", list(CASES))
def test_static_scratch_matches_pressure_solve(name, precision):
    import turbchannel_b200 as tb

    prod, _, zz = make_case(precision=precision, **CASES[name])
    S = tb.Solver(prod, zz)
    rng = np.random.default_rng(11)
    for call in range(2):
        rhs = rng.standard_normal(S.N)
        want = S.LinearSystemSolveFFT(rhs)
        got = _static_solve(S, 1 + call, rhs)
        assert np.all(np.isfinite(got))
        assert rel_err(got, want) < TOL[precision], (name, precision, call)
    S.close()


def test_static_scratch_rejects_oversized_problem():
    import turbchannel_b200 as tb

    # (192/2+1)*128*128*3*8 bytes = 38 MB > 32 MiB
    prod, _, zz = make_case(scheme=VV4, NX=192, NY=128, NZ=128, precision=1)
    S = tb.Solver(prod, zz)
    _, p_dev = S.device_level(0)
    rc = S.L.tc_op_pressure_solve_static(S.h, C.c_void_p(p_dev), C.c_void_p(p_dev))
    assert rc == -1
    assert b"static array" in S.L.tc_last_error()
    S.close()
