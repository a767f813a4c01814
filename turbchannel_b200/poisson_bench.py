"""Poisson microbenchmark: the pressure solve alone (forward x- and y-FFTs, the banded
z-solve per (kx, ky) mode, inverse FFTs) on device buffers, at the sizes of the
Poisson configuration of the channel workloads.

    python -m turbchannel_b200.poisson_bench [--sizes 128x128x128 256x192x256 ...]
        [--schemes hw2 vv4] [--precisions fp64 mixed] [--solves 20] [--warmup 3]

Sizes are x by wall-normal by span cells (NX x NZ x NY), tanh stretching 1.8 in the
wall-normal direction, domain 2 pi x 2 x pi.  The right-hand side is N(0, 1) drawn on
the device with a seeded generator (12345), its mean removed.  Each line reports the
time per solve (CUDA events on the solver's stream after warm-up), cells per second and
the fraction of the HBM roofline of the 10-word model (read the RHS, write the half
spectrum; read and write it in the y-FFT, the z-solve and the inverse y-FFT; read it
and write p in the inverse x-FFT: 10 words of the working precision per cell).  The
solver holds the full step state (about 32 words per cell), so the largest size in
FP64 (137 GB) runs only with --allow-large.
"""
from __future__ import annotations

import argparse
import json
import math

import numpy as np

import turbchannel_b200 as tb

DEFAULT_SIZES = ["128x128x128", "256x192x256", "512x256x512", "1024x512x1024"]
WORDS = 10


def run_one(scheme: int, precision: int, NX: int, NZ: int, NY: int, solves: int, warmup: int, peak_gbs: float):
    import torch

    p, zz = tb.channel_params(scheme, NX, NY, NZ, 2 * math.pi, math.pi, 5600.0, 1.8, precision=precision)
    S = tb.Solver(p, zz)
    dt = torch.float64 if precision == tb.FP64 else torch.float32
    dev = torch.device("cuda")
    gen = torch.Generator(device=dev)
    gen.manual_seed(12345)
    N = NX * NY * NZ
    rhs = torch.randn(N, generator=gen, device=dev, dtype=dt)
    rhs -= rhs.mean()
    out = torch.empty_like(rhs)
    stream = torch.cuda.ExternalStream(S.stream(), device=dev)
    torch.cuda.synchronize()
    for _ in range(warmup):
        S.pressure_solve_device(rhs.data_ptr(), out.data_ptr())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(solves):
        S.pressure_solve_device(rhs.data_ptr(), out.data_ptr())
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / solves
    finite = bool(torch.isfinite(out).all().item())
    S.close()
    w = 8 if precision == tb.FP64 else 4
    gbs = WORDS * w * N / (ms * 1e-3) / 1e9
    return {"scheme": "vv4" if scheme == tb.VV4 else "hw2", "precision": "fp64" if precision == tb.FP64 else "mixed",
            "grid": [NX, NZ, NY], "cells": N, "ms_per_solve": round(ms, 4), "cells_per_s": N / (ms * 1e-3),
            "achieved_gbs": round(gbs, 1), "peak_gbs": peak_gbs, "frac": round(gbs / peak_gbs, 4),
            "l2": "inputs larger than L2" if w * N > 126e6 else "inputs fit in L2", "finite": finite}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--sizes", nargs="+", default=DEFAULT_SIZES)
    ap.add_argument("--schemes", nargs="+", default=["hw2", "vv4"])
    ap.add_argument("--precisions", nargs="+", default=["fp64", "mixed"])
    ap.add_argument("--solves", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--allow-large", action="store_true")
    ap.add_argument("--peak-gbs", type=float, default=0.0,
                    help="HBM bandwidth for the roofline fraction (default: MEASURED_PEAKS.json, else 6650)")
    args = ap.parse_args()
    peak = args.peak_gbs
    if peak <= 0:
        import os

        path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "MEASURED_PEAKS.json")
        peak = 6650.0
        if os.path.exists(path):
            with open(path) as f:
                peak = float(json.load(f).get("hbm_gbs", peak))
    for size in args.sizes:
        NX, NZ, NY = (int(v) for v in size.split("x"))
        for sch in args.schemes:
            for prec in args.precisions:
                precision = tb.FP64 if prec == "fp64" else tb.MIXED
                words = 32 * NX * NY * NZ * (8 if precision == tb.FP64 else 4)
                if words > 100e9 and not args.allow_large:
                    print(json.dumps({"scheme": sch, "precision": prec, "grid": [NX, NZ, NY],
                                      "skipped": f"the solver would hold about {words / 1e9:.0f} GB (use --allow-large)"}),
                          flush=True)
                    continue
                r = run_one(tb.VV4 if sch == "vv4" else tb.HW2, precision, NX, NZ, NY, args.solves, args.warmup, peak)
                print(json.dumps(r), flush=True)


if __name__ == "__main__":
    main()
