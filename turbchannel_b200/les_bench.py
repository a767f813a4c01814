"""Step time of the LES configuration with each closure: staggered HW2 + NAIVE viscosity,
96 x 64 x 96 cells (x, wall-normal, span), Re_b 21900, 2pi x 2 x pi, tanh 2.2, constant
flow rate, from the seeded field (a seeded network stands in for a trained one: the cost
does not depend on the weights).

    python -m turbchannel_b200.les_bench [--grid 96 96 64] [--steps 500] [--warmup 20]

Per precision, ms per step (CUDA events on the solver's stream, K order-3 steps after W
warm-up steps) and ns per cell-step for: no model, Smagorinsky-van Driest, the learned
closure as a separate pass (k_turb_mlp, then the flux kernel) and fused into the flux
kernel (tc_set_mlp_fusion), next to the FP64 DNS step of the 384 x 256 x 384 workload
per cell-step (--dns).
"""
from __future__ import annotations

import argparse
import json
import math

import turbchannel_b200 as tb

LX, LY, RE_B, GAMMA = 2 * math.pi, math.pi, 21900.0, 2.2


def time_les(grid, precision, model, fuse, steps, warmup, tau=0.002):
    import torch

    p, zz = tb.channel_params(tb.HW2, grid[0], grid[1], grid[2], LX, LY, RE_B, GAMMA, precision=precision,
                              visc_type=tb.VISC_NAIVE, turb=tb.TURB_SMAGORINSKY)
    S = tb.Solver(p, zz)
    if model == "mlp":
        m = tb.Mlp(seed=21)
        S.set_turb_model(tb.TURB_MLP, m.params)
        m.close()
        S.set_mlp_fusion(fuse)
    elif model == "none":
        S.set_turb_model(tb.TURB_NONE)
    S.init_channel(0, seed=12345, amp=0.1, project=True)
    S.set_forcing(1, 1.0)
    cur, it = 0, 0
    for _ in range(warmup):
        S.Step(it * tau, tau, cur, min(it + 1, 3))
        cur, it = (cur + 1) % 4, it + 1
    stream = torch.cuda.ExternalStream(S.stream())
    S.sync()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        S.Step(it * tau, tau, cur, 3)
        cur, it = (cur + 1) % 4, it + 1
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / steps
    S.close()
    return ms


def time_dns(precision, steps, warmup):
    import torch

    p, zz = tb.channel_params(tb.VV4, 384, 384, 256, LX, LY, RE_B, GAMMA, precision=precision)
    S = tb.Solver(p, zz)
    S.init_channel(0, seed=12345, amp=0.1, project=True)
    S.set_forcing(1, 1.0)
    tau, cur, it = 0.0008, 0, 0
    for _ in range(warmup):
        S.Step(it * tau, tau, cur, min(it + 1, 3))
        cur, it = (cur + 1) % 4, it + 1
    stream = torch.cuda.ExternalStream(S.stream())
    S.sync()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        S.Step(it * tau, tau, cur, 3)
        cur, it = (cur + 1) % 4, it + 1
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / steps
    S.close()
    return ms


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--grid", type=int, nargs=3, default=[96, 96, 64], help="NX (x), NY (span), NZ (wall-normal)")
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--dns", action="store_true", help="also the FP64 DNS step of the 384x256x384 workload")
    a = ap.parse_args()
    cells = a.grid[0] * a.grid[1] * a.grid[2]
    for prec in (tb.FP64, tb.MIXED):
        row = {"grid": a.grid, "precision": "fp64" if prec == tb.FP64 else "mixed"}
        for name, model, fuse in (("none", "none", 0), ("smagorinsky", "smag", 0), ("mlp_separate", "mlp", 0),
                                  ("mlp_fused", "mlp", 1)):
            ms = time_les(a.grid, prec, model, fuse, a.steps, a.warmup)
            row[name] = {"ms_per_step": round(ms, 5), "ns_per_cell_step": round(ms * 1e6 / cells, 4)}
        print(json.dumps(row), flush=True)
    if a.dns:
        ms = time_dns(tb.FP64, 50, 5)
        print(json.dumps({"dns_fp64_384x256x384": {"ms_per_step": round(ms, 4),
                                                   "ns_per_cell_step": round(ms * 1e6 / (384 * 384 * 256), 4)}}))


if __name__ == "__main__":
    main()
