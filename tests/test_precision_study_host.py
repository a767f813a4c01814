"""Host logic of the mixed-vs-FP64 study (turbchannel_b200/precision_study.py): the turbulence
statistics derived from time-averaged plane means, and the comparison of two runs."""
import numpy as np


def _profiles(NZ, rng, scale=1.0):
    z = (np.arange(NZ) + 0.5) / NZ
    U = 1.2 * (1 - (2 * z - 1) ** 2) ** 0.3 * scale
    prof = np.zeros((NZ, 12))
    prof[:, 0] = U
    prof[:, 3] = U * U + 0.01 + 0.001 * rng.random(NZ)
    prof[:, 4] = 0.005
    prof[:, 5] = 0.004
    prof[:, 7] = U * 0.0 - 0.002 * (1 - 2 * z)  # <uw>, odd about the centre (W = 0)
    prof[:, 10] = 0.1
    prof[:, 11] = 0.1 ** 2 + 0.003
    return prof


def test_derived_statistics():
    from turbchannel_b200 import precision_study as ps

    NZ = 32
    zz = 1 + np.tanh(2.2 * (2 * np.arange(NZ + 1) / NZ - 1)) / np.tanh(2.2)
    prof = _profiles(NZ, np.random.default_rng(0))
    d = ps.derived(prof, zz, visc=2 / 21900)
    assert np.allclose(d["uu"], prof[:, 3] - prof[:, 0] ** 2)
    assert np.allclose(d["p_rms"], np.sqrt(0.003))
    dz0 = zz[1] - zz[0]
    ut = np.sqrt(2 / 21900 * prof[0, 0] / (0.5 * dz0))
    assert abs(d["Re_tau_walls"][0] - ut * 1.0 / (2 / 21900)) < 1e-9 * d["Re_tau"]


def test_compare_identical_and_scaled():
    from turbchannel_b200 import precision_study as ps

    NZ = 32
    zz = 1 + np.tanh(2.2 * (2 * np.arange(NZ + 1) / NZ - 1)) / np.tanh(2.2)
    rng = np.random.default_rng(1)
    prof = _profiles(NZ, rng)
    a = ps.derived(prof, zz, visc=1e-4)
    c = ps.compare(a, a)
    assert all(c[k]["max_rel"] == 0 for k in ps.STATS) and c["Re_tau"] == 0
    b = ps.derived(_profiles(NZ, np.random.default_rng(1), scale=1.01), zz, visc=1e-4)
    c = ps.compare(b, a)
    assert abs(c["U"]["max_rel"] - 0.01) < 1e-12
    assert abs(c["Re_tau"] - (np.sqrt(1.01) - 1)) < 1e-12


def test_report_renders():
    from turbchannel_b200 import precision_study as ps

    NZ = 16
    zz = 1 + np.tanh(2.2 * (2 * np.arange(NZ + 1) / NZ - 1)) / np.tanh(2.2)
    runs = []
    for name, seed, sc in (("fp64", 1, 1.0), ("mixed", 1, 1.001), ("fp64", 2, 0.999), ("mixed", 2, 1.0)):
        d = ps.derived(_profiles(NZ, np.random.default_rng(seed), sc), zz, 1e-4)
        w = {k: (v.tolist() if isinstance(v, np.ndarray) else v) for k, v in d.items()}
        runs.append({"name": f"{name}_seed{seed}", "seed": seed, "steps": 10, "wall_ms_per_step": 1.0,
                     "windows": {"5": w, "10": w}})
    long_res = {"kind": "long", "runs": runs, "windows": [5], "stat_steps": 10, "dt": 8e-4, "dt_transition": 6e-4,
                "spinup": [1, 1], "grid": [8, 8, NZ], "stat_every": 1}
    txt = ps.report(None, long_res)
    assert "mixed_seed1 vs fp64_seed1" in txt and "fp64_seed2 vs fp64_seed1" in txt
    assert "mixed_pooled vs fp64_pooled" in txt

    # the JSON summary carries the same comparisons, rounded, for both windows
    sm = ps._round(ps.summary(None, long_res))
    assert set(sm["long"]["windows"]) == {"5", "10"}
    pr = sm["long"]["windows"]["10"]["pairs"]
    assert set(pr) == {"mixed_seed1 vs fp64_seed1", "mixed_seed2 vs fp64_seed2", "fp64_seed2 vs fp64_seed1",
                       "mixed_seed2 vs mixed_seed1", "mixed_pooled vs fp64_pooled"}
    assert abs(pr["mixed_seed1 vs fp64_seed1"]["U"]["max_rel"] - 0.001) < 1e-6
    assert sm["long"]["failed"] == {}
