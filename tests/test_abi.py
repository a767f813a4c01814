"""The C-ABI library loads and exports every entry point include/turbch.h declares;
host-side argument validation works without a GPU (no compute calls here)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "turbch.h")


HEADER_LES = os.path.join(ROOT, "include", "turbch_les.h")


def _declared(path=HEADER):
    src = open(path).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(tc_[a-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    import turbchannel_b200 as tb
    from turbchannel_b200 import build

    build.build()
    return tb.load_library()


def test_exports_every_declared_symbol(lib):
    import turbchannel_b200 as tb

    names = _declared()
    assert len(names) >= 25
    for n in names:
        assert hasattr(lib, n), n
    assert sorted(tb.EXPORTS) == names
    les = _declared(HEADER_LES)
    for n in les:
        assert hasattr(lib, n), n
    assert sorted(tb.EXPORTS_LES) == les


def test_version_and_error_strings(lib):
    assert b"sm_100a" in lib.tc_version()
    assert isinstance(lib.tc_last_error(), bytes)


def _params(**over):
    import turbchannel_b200 as tb
    from cases import make_case

    prod, _, zz = make_case(1, 32, 16, 24)
    prod.update(over)
    s = tb.TcParams()
    for k, _t in tb.TcParams._fields_:
        setattr(s, k, prod.get(k, 0))
    return s, np.ascontiguousarray(zz)


@pytest.mark.parametrize("over,needle", [
    (dict(NX=30), b"NX and NY"),
    (dict(NY=10), b"NX and NY"),
    (dict(NX=33), b"NX and NY"),
    (dict(NZ=4), b"NZ"),
    (dict(scheme=7), b"scheme"),
    (dict(precision=5), b"precision"),
    (dict(visc_type=2), b"Galerkin"),
    (dict(turb_model=1, visc_type=0), b"turbulence model"),
    (dict(hx=-1.0), b"mesh steps"),
])
def test_create_rejects_bad_params(lib, over, needle):
    s, zz = _params(**over)
    h = C.c_void_p()
    rc = lib.tc_create(C.byref(s), zz.ctypes.data_as(C.POINTER(C.c_double)), C.byref(h))
    assert rc == -1
    assert needle in lib.tc_last_error()
    assert not h.value


def test_create_rejects_non_monotone_mesh(lib):
    s, zz = _params()
    zz = zz.copy()
    zz[5] = zz[4]
    h = C.c_void_p()
    rc = lib.tc_create(C.byref(s), zz.ctypes.data_as(C.POINTER(C.c_double)), C.byref(h))
    assert rc == -1 and b"increase" in lib.tc_last_error()


def test_calls_reject_null_handle(lib):
    assert lib.tc_step(None, 0.0, 0.001, 0, 1) == -1
    assert lib.tc_sync(None) == -1
    out = np.zeros(3)
    assert lib.tc_integral(None, 0, out.ctypes.data_as(C.c_void_p)) == -1
    assert lib.tc_destroy(None) == 0


def test_mesh_tanh_matches_formula(lib):
    import turbchannel_b200 as tb

    z = tb.mesh_tanh(16, 1.8)
    j = np.arange(17)
    ref = 1 + np.tanh(1.8 * (2 * j / 16 - 1)) / np.tanh(1.8)
    assert np.allclose(z, ref, rtol=0, atol=1e-15)
    assert z[0] == 0.0 and abs(z[-1] - 2.0) < 1e-15
