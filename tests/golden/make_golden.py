"""Generate tests/golden/ref_<variant>.npz by running the reference's own CPU solver
(compiled from its sources into oracle/_ref/ by `make -C oracle ref`).

Inputs are deterministic formula fields in the style of the reference self-tests
(staggered/selftest.cpp:89,220: sin(in*in + ...)), so no RNG stream is involved.
Outputs are stored at every k-th element (a strided sample, k >= 5) to keep the fixtures
small; the test recomputes everything with the oracle and compares the samples.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

VARIANTS = {
    # variant: (scheme, turb, stab_type, fd_mode)
    "stag_hw2_dns_f64": (0, 0, 0, 1),
    "stag_hw2_les_f64": (0, 1, 0, 1),
    "stag_vv4_dns_f64": (1, 0, 0, 1),
    "stag_vv4_les_f64": (1, 1, 0, 1),
    "coll_gal_f64": (2, 1, 1, 1),
    "coll_cross_f64": (2, 0, 0, 1),
}
MAX_SAMPLES = 2500  # per field: stride = max(5, N // MAX_SAMPLES)


def formula_fields(N, NXY, scheme):
    i = np.arange(N, dtype=np.float64)
    v = np.stack([0.1 * np.sin(i * i + np.cos(10.0 * c)) for c in range(3)], axis=1)
    v[:, 0] += 1.0
    if scheme == 2:
        v[:NXY] = 0.0
        v[-NXY:] = 0.0
    else:
        v[:NXY, 2] = 0.0
    p = np.sin(i * i + 87.0)
    nt = 1e-3 * (1.0 + np.sin(i * i + 5.0))
    return v, p, nt


def case_for(variant, R):
    from cases import make_case

    scheme, turb, stab, fd = VARIANTS[variant]
    NZ = R.NZMAX
    prod, orc, zz = make_case(scheme, R.NX, R.NY, NZ, turb=turb, stab_type=stab, fd_mode=fd)
    return orc, zz


def outputs(S, orc, zz, scheme, turb):
    """Same sequence for RefLib and Oracle objects (duck-typed)."""
    N = orc["NX"] * orc["NY"] * orc["NZ"]
    NXY = orc["NX"] * orc["NY"]
    v, p, nt = formula_fields(N, NXY, scheme)
    out = {}
    if turb:
        S.set_nu_t(nt)
    out["explicit"] = S.explicit_term(v)
    out["grad"] = S.apply_gradient(p)
    out["unapply"] = S.unapply_gradient(v)
    if turb:
        S.recalc_turb_visc(v)
        out["nu_t"] = S.get_nu_t()
    # projected initial field, 6 steps with the order ramp
    q = S.unapply_gradient(v)
    v0 = v - S.apply_gradient(q)
    z = np.zeros_like(v0)
    for lvl in range(4):
        S.set_level(lvl, z, np.zeros(N))
    S.set_level(0, v0, np.zeros(N))
    cur = 0
    for it in range(6):
        S.step(it * 0.002, 0.002, cur, min(it + 1, 3))
        cur = (cur + 1) % 4
    vs, ps = S.get_level(cur)
    out["step_v"], out["step_p"] = vs, ps
    prof = S.profiles(cur)
    # the collocated reference profile has no pressure columns (collocated_AB3/real3.h:39-50)
    out["profiles"] = prof[:, :10] if scheme == 2 else prof
    out["integral"] = S.integral(cur)
    return out


def main():
    import oracle_py as op

    for variant, (scheme, turb, stab, fd) in VARIANTS.items():
        if not op.ref_available(variant):
            raise SystemExit(f"oracle/_ref/libref_{variant}.so missing: run `make -C oracle ref`")
        R = op.RefLib(variant)
        orc, zz = case_for(variant, R)
        R.setup(orc, zz)
        out = outputs(R, orc, zz, scheme, turb)
        stride = max(5, (R.NX * R.NY * R.NZMAX) // MAX_SAMPLES)
        save = {k: np.ascontiguousarray(a).reshape(-1)[::stride] for k, a in out.items()}
        save["zz"] = zz
        save["stride"] = np.array(stride)
        save["shape"] = np.array([R.NX, R.NY, R.NZMAX])
        np.savez_compressed(os.path.join(HERE, f"ref_{variant}.npz"), **save)
        print("wrote", variant)


if __name__ == "__main__":
    main()
