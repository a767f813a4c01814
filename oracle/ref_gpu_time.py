#!/usr/bin/env python
"""Time the reference's own GPU path on this GPU: its data_cuda solver object (lambda
Forall kernels, cuFFT D2Z/Z2D, Thrust reductions; staggered/func_cuda.cpp,
collocated_AB3/main.cpp:114-178), compiled from the reference's sources by
``make -C oracle ref`` into oracle/_ref/libref_<variant>.so.

Timing infrastructure for the comparison only (like the oracle): the product never loads these
libraries; bench.py runs this script in a child process for its ``reference_gpu``
figures, so the reference's CUDA context, allocations and exit-on-error handling
(staggered/func_cuda.cpp:23-35) stay out of the benchmark process.

    python oracle/ref_gpu_time.py --config vv4_c4 --precision f64 [--sync] --steps K --warmup W

prints one JSON line.  Inputs: the configuration's seeded field (u = 1.5(1 - y^2) plus
MT19937-64(12345) uniform noise of amplitude 0.1, 3 draws per cell in index order, the
same definition as the product's tc_init_channel), projected divergence-free with the
reference's own GPU operators (UnapplyGradient, ApplyGradient: staggered/selftest.cpp:
224-226).  Forcing is the reference's own constant sour_dpdx (it has no constant flow
rate).  Times: CUDA events on the default stream the reference launches on, K steps
after W warm-up steps (order ramp 1, 2, 3 as staggered/main.cpp:308), without and
with the time loop's per-step diagnostics (main.cpp:313-338).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
REF_DIR = os.path.join(HERE, "_ref")

# name -> solver kind, library stem (precision / sync suffix added), grid and flow parameters
CONFIGS = {
    # staggered VV4 DNS, 384 x 256 x 384 cells (x, wall-normal, span), Re_b 21900, tanh 2.2
    "vv4_c4": dict(kind="stag", stem="stag_vv4_dns_c4", scheme=1, NX=384, NY=384, NZ=256, Lx=2 * math.pi,
                   Ly=math.pi, Re_b=21900.0, gamma=2.2, tau=0.0008),
    # staggered HW2 DNS, 64 x 64 x 64 cells, 4 pi x 2 x 4/3 pi, Re_b 5600, tanh 1.8
    "hw2_c1": dict(kind="stag", stem="stag_hw2_dns", sync_stem="stag_hw2_dns_c1sync", scheme=0, NX=64, NY=64, NZ=64,
                   Lx=4 * math.pi, Ly=4 * math.pi / 3, Re_b=5600.0, gamma=1.8, tau=0.002),
    # collocated DNS, 256 x 192 x 256 nodes, 2 pi x 2 x pi, Re_b 13750, tanh 2.0, cross viscosity
    "coll_c3": dict(kind="coll", stem="coll_cross_c3", scheme=2, NX=256, NY=256, NZ=192, Lx=2 * math.pi,
                    Ly=math.pi, Re_b=13750.0, gamma=2.0, tau=0.001),
}


def library(cfg: dict, precision: str, sync: bool) -> str:
    stem = cfg.get("sync_stem", cfg["stem"] + "sync") if sync else cfg["stem"]
    return os.path.join(REF_DIR, f"libref_{stem}_{precision}.so")


def seeded_field(p: dict, zz: np.ndarray, scheme: int, seed: int = 12345, amp: float = 0.1) -> np.ndarray:
    """Raw seeded field, AoS (N, 3) double, before the projection."""
    import oracle_py as op

    NX, NY, NZ = p["NX"], p["NY"], p["NZ"]
    NXY, N = NX * NY, NX * NY * NZ
    r = op.mt64(seed, 3 * N)
    r = amp * (2.0 * (r >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0) - 1.0)
    v = r.reshape(N, 3)
    if scheme == 2:
        zc, H, z0 = zz, 0.5 * (zz[-1] - zz[0]), zz[0]
    else:
        zc, H, z0 = 0.5 * (zz[:-1] + zz[1:]), 0.5 * (zz[-1] - zz[0]), zz[0]
    y = (zc - z0) / H - 1.0
    v[:, 0] += np.repeat(1.5 * (1.0 - y * y), NXY)
    if scheme == 2:
        v[:NXY] = 0.0
        v[-NXY:] = 0.0
    else:
        v[:NXY, 2] = 0.0
    return v


def run(config: str, precision: str, sync: bool, steps: int, warmup: int, device: int = 0) -> dict:
    import oracle_py as op

    cfg = CONFIGS[config]
    path = library(cfg, precision, sync)
    if not os.path.exists(path):
        return {"unavailable": f"{os.path.basename(path)} not built (make -C oracle ref)"}
    L = C.CDLL(path)
    dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int)
    L.refgpu_set_level.argtypes = [C.c_int, C.c_void_p, C.c_void_p]
    L.refgpu_project.argtypes = [C.c_int]
    L.refgpu_run.argtypes = [C.c_int, C.c_double, C.c_int, ip, ip]
    L.refgpu_run.restype = C.c_double
    L.refgpu_integral.argtypes = [C.c_int, dp]
    L.refgpu_free.restype = None
    p, zz = op.channel_params(cfg["scheme"], cfg["NX"], cfg["NY"], cfg["NZ"], cfg["Lx"], cfg["Ly"], cfg["Re_b"],
                              cfg["gamma"])
    zz = np.ascontiguousarray(zz, dtype=np.float64)
    if cfg["kind"] == "coll":
        L.refgpu_setup_colloc.argtypes = [C.c_int, dp] + [C.c_double] * 6 + [C.c_int] * 4
        rc = L.refgpu_setup_colloc(p["NZ"], zz.ctypes.data_as(dp), p["visc"], p["sour_dpdx"], p["inv_length_scale"],
                                   p["hx"], p["hy"], p["area"], 0, 0, 1, device)
    else:
        L.refgpu_setup.argtypes = [C.c_int, dp] + [C.c_double] * 6 + [C.c_int]
        rc = L.refgpu_setup(p["NZ"], zz.ctypes.data_as(dp), p["visc"], p["sour_dpdx"], p["inv_length_scale"], p["hx"],
                            p["hy"], p["area"], device)
    if rc:
        return {"unavailable": f"reference GPU setup failed ({rc})"}
    v = seeded_field(p, zz, cfg["scheme"])
    q = np.zeros(v.shape[0])
    if L.refgpu_set_level(0, v.ctypes.data, q.ctypes.data) or L.refgpu_project(0):
        return {"unavailable": "reference GPU upload/projection failed"}
    del v, q
    tau = cfg["tau"]
    cur, it = C.c_int(0), C.c_int(0)
    if L.refgpu_run(warmup, tau, 0, C.byref(cur), C.byref(it)) < 0:
        return {"unavailable": "reference GPU warm-up failed"}
    ms = L.refgpu_run(steps, tau, 0, C.byref(cur), C.byref(it))
    ms_diag = L.refgpu_run(steps, tau, 1, C.byref(cur), C.byref(it))
    integ = np.zeros(3)
    L.refgpu_integral(cur.value, integ.ctypes.data_as(dp))
    L.refgpu_free()
    if ms < 0 or ms_diag < 0:
        return {"unavailable": "reference GPU step failed"}
    N = cfg["NX"] * cfg["NY"] * cfg["NZ"]
    grid = f"{cfg['NX']}x{cfg['NZ']}x{cfg['NY']}"  # x, wall-normal, span
    return {"impl": "reference_gpu", "config": config, "grid": grid, "cells": N, "dtype": precision,
            "sync_after_each_kernel": sync, "steps": steps, "warmup": warmup,
            "ms_per_step": ms / steps, "value": N * steps / (ms * 1e-3), "unit": "cell-steps/s",
            "ms_per_step_with_diagnostics": ms_diag / steps,
            "bulk_velocity_after": float(integ[0] / p["area"]),
            "library": os.path.basename(path),
            "timing": "CUDA events on the default stream around K steps (reference's own launches)"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", default="vv4_c4", choices=list(CONFIGS))
    ap.add_argument("--precision", default="f64", choices=["f64", "f32"])
    ap.add_argument("--sync", action="store_true", help="the reference's SYNC_AFTER_EACH_KERNEL build")
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args()
    print(json.dumps(run(a.config, a.precision, a.sync, a.steps, max(3, a.warmup), a.device)), flush=True)


if __name__ == "__main__":
    main()
