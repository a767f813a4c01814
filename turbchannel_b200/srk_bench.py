"""Timing of the segregated IMEX Runge-Kutta step of the collocated scheme (tc_srk_step).

    python -m turbchannel_b200.srk_bench [--sizes 128x49x64 384x257x384] [--methods ARS_343 ARK3]
        [--precisions fp64 mixed] [--steps 20] [--warmup 3]

Sizes are x by wall-normal nodes by span (NX x NZ x NY); the collocated channel of
the reference's SRK driver (collocated_SRK/main.cpp:303-335: Re_tau 180, domain
4 pi x 2 x 4 pi/3), here on a tanh mesh (stretching 1.8) with the seeded divergence-free
field of tc_init_channel and the driver's source term u_tau^2 / H.  StabType 1 and
alpha_tau = alpha_tau_max / 2 as the driver sets them; tau = min(2e-3, 0.2 hz_min^2 / visc)
(the step treats viscosity explicitly).  Each line: ms per step (CUDA
events on the solver's stream after warm-up), node-steps per second, launches per step.
"""
from __future__ import annotations

import argparse
import json
import math

import numpy as np

import turbchannel_b200 as tb
from turbchannel_b200 import imex


def run_one(name: str, precision: int, NX: int, NZ: int, NY: int, steps: int, warmup: int):
    import torch

    re_tau, H = 180.0, 1.0
    visc = 1.0 / re_tau
    u_tau = re_tau * visc
    Lx, Ly = 4 * math.pi * H, 4 * math.pi * H / 3
    j = np.arange(NZ)
    zz = H * (1.0 + np.tanh(1.8 * (2.0 * j / (NZ - 1) - 1.0)) / np.tanh(1.8))
    # the step is explicit in the viscous term as well (the reference's implicit part is
    # empty): tau within the wall-normal diffusion limit, at most the driver's 2e-3
    tau = min(2e-3, 0.2 * float(np.min(np.diff(zz))) ** 2 / visc)
    p = dict(scheme=tb.COLLOC, visc_type=tb.VISC_CROSS, stab_type=1, fd_mode=1, NX=NX, NY=NY, NZ=NZ, visc=visc,
             sour_dpdx=u_tau * u_tau / H, inv_length_scale=u_tau / visc, xmin=0.0, ymin=0.0, hx=Lx / NX, hy=Ly / NY,
             area=Lx * Ly * (zz[-1] - zz[0]), precision=precision, turb_model=0, device=0, low_modes=0)
    S = tb.Solver(p, zz)
    m = imex.METHODS[name]()
    S.srk_init(m, 1)
    S.init_channel(0, seed=12345, amp=0.1, project=True)
    dev = torch.device("cuda")
    stream = torch.cuda.ExternalStream(S.stream(), device=dev)
    for k in range(warmup):
        S.srk_step(k * tau, tau)
    S.sync()
    l0 = S.launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for k in range(steps):
        S.srk_step((warmup + k) * tau, tau)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / steps
    launches = (S.launch_count() - l0) / steps
    v, _ = S.download_level(0)
    finite = bool(np.all(np.isfinite(v)))
    S.close()
    N = NX * NY * NZ
    return {"method": name, "stages": m.S, "precision": "fp64" if precision == tb.FP64 else "mixed",
            "grid": [NX, NZ, NY], "nodes": N, "tau": tau, "ms_per_step": round(ms, 4), "node_steps_per_s": N / (ms * 1e-3),
            "launches_per_step": launches, "finite": finite}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--sizes", nargs="+", default=["128x49x64", "384x257x384"])
    ap.add_argument("--methods", nargs="+", default=["ARS_343", "ARK3"])
    ap.add_argument("--precisions", nargs="+", default=["fp64", "mixed"])
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    args = ap.parse_args()
    for size in args.sizes:
        NX, NZ, NY = (int(v) for v in size.split("x"))
        for name in args.methods:
            for prec in args.precisions:
                r = run_one(name, tb.FP64 if prec == "fp64" else tb.MIXED, NX, NZ, NY, args.steps, args.warmup)
                print(json.dumps(r), flush=True)


if __name__ == "__main__":
    main()
