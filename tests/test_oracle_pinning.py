"""Pin the CPU oracle to the reference itself.

1. Golden vectors: tests/golden/ref_<variant>.npz were produced by running the
   reference's own CPU solver (compiled from its sources, see
   tests/golden/make_golden.py).  The oracle must reproduce them: bit-for-bit on
   the explicit term / gradient / turbulent viscosity, to round-off on anything
   that goes through the FFT.
2. Live comparison with oracle/_ref (when it has been built here).
3. The reference's start-up self-tests (staggered/selftest.cpp:345-356) reproduce
   their known-answer levels on the reference's own default mesh.
"""
import glob
import os

import numpy as np
import pytest

from cases import rel_err

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = sorted(glob.glob(os.path.join(HERE, "golden", "ref_*.npz")))


def _golden_case(path):
    import make_golden as mg

    variant = os.path.basename(path)[4:-4]
    d = np.load(path)
    NX, NY, NZ = (int(x) for x in d["shape"])
    scheme, turb, stab, fd = mg.VARIANTS[variant]
    from cases import make_case

    _, orc, zz = make_case(scheme, NX, NY, NZ, turb=turb, stab_type=stab, fd_mode=fd)
    assert np.array_equal(zz, d["zz"])
    return variant, d, orc, zz, scheme, turb


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_oracle_matches_reference_golden(path):
    import sys

    sys.path.insert(0, os.path.join(HERE, "golden"))
    import make_golden as mg
    import oracle_py as op

    variant, d, orc, zz, scheme, turb = _golden_case(path)
    O = op.Oracle(orc, zz, "f64")
    out = mg.outputs(O, orc, zz, scheme, turb)
    k = int(d["stride"])
    exact = ["explicit", "grad"] + (["nu_t"] if turb else [])
    for name in exact:
        got = np.ascontiguousarray(out[name]).reshape(-1)[::k]
        assert rel_err(got, d[name]) <= 1e-15, name
    for name, tol in (("unapply", 1e-12), ("step_v", 1e-12), ("step_p", 1e-9), ("profiles", 1e-12), ("integral", 1e-12)):
        got = np.ascontiguousarray(out[name]).reshape(-1)[::k]
        assert rel_err(got, d[name]) < tol, name


# The *_w48 / *_w36 variants are built with the index-wrap generalisation
# (oracle/ref/index_wrap.h) at sizes that are not powers of two (48 x 24, 36 x 18).
REF_VARIANTS = ["stag_hw2_dns_f64", "stag_hw2_les_f64", "stag_vv4_dns_f64", "stag_vv4_les_f64", "coll_gal_f64",
                "coll_cross_f64", "stag_vv4_les_f32", "coll_gal_f32", "stag_vv4_dns_w48_f64", "stag_hw2_les_w36_f64"]


@pytest.mark.parametrize("variant", REF_VARIANTS)
def test_oracle_matches_live_reference(variant):
    import oracle_py as op
    from cases import make_case

    if not op.ref_available(variant):
        pytest.skip("oracle/_ref not built (reference sources unavailable)")
    R = op.RefLib(variant)
    f32 = variant.endswith("f32")
    scheme = 2 if variant.startswith("coll") else (1 if "vv4" in variant else 0)
    turb = 1 if ("les" in variant or "gal" in variant) else 0
    for stab in ([0, 1] if scheme == 2 else [0]):
        _, orc, zz = make_case(scheme, R.NX, R.NY, R.NZMAX, turb=turb, stab_type=stab)
        R.setup(orc, zz)
        O = op.Oracle(orc, zz, "f32" if f32 else "f64")
        tol_exact = 1e-6 if f32 else 1e-15
        for nm in ["DZ", "DZW", "GC1", "GC2", "MAT_A", "MAT_D", "KERG", "cMAT_A"]:
            b = R.mesh(nm)
            if len(b):
                assert rel_err(O.mesh(nm), b) <= (0 if not f32 else 1e-7), nm
        O.init_channel(0, 12345, 0.1, True)
        v, q = O.get_level(0)
        nt = 1e-3 * np.abs(np.random.default_rng(1).standard_normal(O.N))
        O.set_nu_t(nt)
        R.set_nu_t(nt)
        assert rel_err(O.explicit_term(v), R.explicit_term(v)) <= tol_exact
        pp = np.random.default_rng(2).standard_normal(O.N)
        assert rel_err(O.apply_gradient(pp), R.apply_gradient(pp)) <= tol_exact
        assert rel_err(O.apply_divergence(v), R.apply_divergence(v)) <= tol_exact
        assert rel_err(O.unapply_gradient(v), R.unapply_gradient(v)) < (1e-5 if f32 else 1e-13)
        for lvl in range(4):
            O.set_level(lvl, v * 0, q * 0)
            R.set_level(lvl, v * 0, q * 0)
        O.set_level(0, v, q)
        R.set_level(0, v, q)
        cur = 0
        for it in range(6):
            O.step(it * 0.002, 0.002, cur, min(it + 1, 3))
            R.step(it * 0.002, 0.002, cur, min(it + 1, 3))
            cur = (cur + 1) % 4
        vo, po = O.get_level(cur)
        vr, pr = R.get_level(cur)
        assert rel_err(vo, vr) < (1e-5 if f32 else 1e-13)
        assert rel_err(po, pr) < (1e-2 if f32 else 1e-10)
        assert rel_err(O.integral(cur), R.integral(cur)) < (1e-5 if f32 else 1e-12)
        ncol = 10 if scheme == 2 else 12
        assert rel_err(O.profiles(cur)[:, :ncol], R.profiles(cur)[:, :ncol]) < (1e-5 if f32 else 1e-13)


def _default_reference_case():
    """staggered/main.cpp:200-242 defaults: Re_tau 395, 4pi x 2pi x 2, sinh mesh (6.5), 64x32x32."""
    NX, NY, NZ = 64, 32, 32
    visc = 1.0 / 395
    H, stretch = 1.0, 6.5
    zz = np.zeros(NZ + 1)
    for i in range(NZ // 2 + 1):
        zz[i] = H * np.sinh(stretch * i / NZ) / np.sinh(0.5 * stretch)
        zz[NZ - i] = 2 * H - zz[i]
    Hx, Hy = 4 * np.pi, 2 * np.pi
    orc = dict(scheme=1, visc_type=1, turb=1, stab_type=0, fd_mode=0, NX=NX, NY=NY, NZ=NZ, visc=visc,
               sour_dpdx=1.0, inv_length_scale=1.0 / visc, xmin=0.0, ymin=-0.5 * Hy, hx=Hx / NX, hy=Hy / NY,
               area=Hx * Hy * 2.0)
    return orc, zz


def test_reference_selftest_levels():
    """Known-answer levels printed by the reference self-tests on its default case
    (gradient kernel 9e-15, projection 6e-17, skew part 0, pressure matrix 3e-14,
    pressure solver 3e-13 / 8e-14, projected divergence 4e-15, K 8e-13 3e-13 2e-14)."""
    import oracle_py as op

    orc, zz = _default_reference_case()
    O = op.Oracle(orc, zz, "f64")
    assert O.check("gradient_kernel") < 1e-13
    assert O.check("normalization_projection") < 1e-15
    assert O.check("matrix_symmetry") == 0.0
    assert O.check("pressure_matrix") < 1e-12
    assert O.check("pressure_solver", 0) < 1e-11
    assert O.check("pressure_solver", 1) < 1e-11
    ediv, K = O.check_conservation()
    assert ediv < 1e-13
    assert np.all(np.abs(K) < 1e-10)
