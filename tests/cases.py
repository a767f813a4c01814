"""Shared case construction for the parity tests: one spec -> identical inputs
for the product (turbchannel_b200) and the oracle (oracle/oracle_py.py)."""
import numpy as np

HW2, VV4, COLLOC = 0, 1, 2
CROSS, NAIVE, GALERKIN = 0, 1, 2


def make_case(scheme, NX, NY, NZ, Lx=2 * np.pi, Ly=np.pi, Re_b=5600.0, gamma=1.8, turb=0, visc_type=None,
              stab_type=0, fd_mode=1, precision=0, low_modes=0):
    visc = 2.0 / Re_b
    if visc_type is None:
        visc_type = (GALERKIN if turb else CROSS) if scheme == COLLOC else (NAIVE if turb else CROSS)
    re_tau = 0.09 * Re_b ** 0.88
    u_tau = re_tau * visc
    n_int = NZ - 1 if scheme == COLLOC else NZ
    j = np.arange(n_int + 1)
    zz = 1.0 + np.tanh(gamma * (2.0 * j / n_int - 1.0)) / np.tanh(gamma)
    area = Lx * Ly * (zz[-1] - zz[0])
    common = dict(scheme=scheme, visc_type=visc_type, stab_type=stab_type, fd_mode=fd_mode, NX=NX, NY=NY, NZ=NZ,
                  visc=visc, sour_dpdx=u_tau * u_tau, inv_length_scale=u_tau / visc, xmin=0.0, ymin=0.0,
                  hx=Lx / NX, hy=Ly / NY, area=area)
    prod = dict(common, precision=precision, turb_model=turb, device=0, low_modes=low_modes)
    orc = dict(common, turb=turb)
    return prod, orc, zz


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def seeded_field(N, NXY, seed=7, amp=1.0, wall_w_zero=True):
    rng = np.random.default_rng(seed)
    v = amp * rng.standard_normal((N, 3))
    if wall_w_zero:
        v[:NXY, 2] = 0.0
    return v


def within(label, err, tol):
    """err < tol as a test check; with TC_ERROR_LOG set, also appends the measured error
    (label, err, tol) to that file as a JSON line (how the tolerances were sized)."""
    import json
    import os

    path = os.environ.get("TC_ERROR_LOG")
    if path:
        with open(path, "a") as f:
            f.write(json.dumps({"label": label, "err": float(err), "tol": float(tol)}) + "\n")
    return err < tol
