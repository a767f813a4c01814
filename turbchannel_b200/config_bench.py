"""Throughput of the step at the other flow configurations, beside the reference's own
GPU path on the same GPU:

* config 1: staggered HW2 DNS, 64 x 64 x 64 cells, 4 pi x 2 x 4/3 pi, Re_b 5600, tanh 1.8,
  dt 0.002 (the reference's CPU-runnable case);
* config 3: collocated DNS (cross viscosity, StabType 0, FDmode 1), 256 x 192 x 256
  nodes (x, wall-normal, span), 2 pi x 2 x pi, Re_b 13750, tanh 2.0, dt 0.001;
* config 4 (the headline workload) for completeness.

    python -m turbchannel_b200.config_bench [--configs c1 c3] [--steps 200] [--warmup 10]
        [--no-reference]

Per configuration and precision: ms per step and cell-steps/s (CUDA events on the
solver's stream, K order-3 steps after W warm-up steps, constant flow rate), the phase
split of the step (tc_phase_timing), the fraction of the HBM roofline of the 40-word
step model, and the reference's GPU step (oracle/ref_gpu_time.py in a child process, the
reference's own build at that size; its forcing is its constant dp/dx).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys

import numpy as np

import turbchannel_b200 as tb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STEP_WORDS = 40
CONFIGS = {
    "c1": dict(ref="hw2_c1", scheme=tb.HW2, NX=64, NY=64, NZ=64, Lx=4 * math.pi, Ly=4 * math.pi / 3, Re_b=5600.0,
               gamma=1.8, tau=0.002, what="staggered HW2 DNS 64x64x64 cells"),
    "c3": dict(ref="coll_c3", scheme=tb.COLLOC, NX=256, NY=256, NZ=192, Lx=2 * math.pi, Ly=math.pi, Re_b=13750.0,
               gamma=2.0, tau=0.001, what="collocated DNS 256x192x256 nodes (x, wall-normal, span)"),
    "c4": dict(ref="vv4_c4", scheme=tb.VV4, NX=384, NY=384, NZ=256, Lx=2 * math.pi, Ly=math.pi, Re_b=21900.0,
               gamma=2.2, tau=0.0008, what="staggered VV4 DNS 384x256x384 cells (x, wall-normal, span)"),
}


def peak_gbs() -> tuple[float, str]:
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def time_ours(c: dict, precision: int, steps: int, warmup: int) -> dict:
    import torch

    p, zz = tb.channel_params(c["scheme"], c["NX"], c["NY"], c["NZ"], c["Lx"], c["Ly"], c["Re_b"], c["gamma"],
                              precision=precision)
    S = tb.Solver(p, zz)
    S.init_channel(0, seed=12345, amp=0.1, project=True)
    S.set_forcing(1, 1.0)
    tau, cur, it = c["tau"], 0, 0
    for _ in range(warmup):
        S.Step(it * tau, tau, cur, min(it + 1, 3))
        cur, it = (cur + 1) % 4, it + 1
    stream = torch.cuda.ExternalStream(S.stream())
    S.sync()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    S.phase_timing(True)
    e0.record(stream)
    for _ in range(steps):
        S.Step(it * tau, tau, cur, 3)
        cur, it = (cur + 1) % 4, it + 1
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / steps
    ph, nst = S.phase_times()
    S.phase_timing(False)
    ub = S.CalcIntegral(cur)[0] / p["area"]
    S.close()
    N = c["NX"] * c["NY"] * c["NZ"]
    w = 8 if precision == tb.FP64 else 4
    pk, kind = peak_gbs()
    return {"precision": "fp64" if precision == tb.FP64 else "mixed", "ms_per_step": ms,
            "cell_steps_per_s": N / (ms * 1e-3),
            "step_roofline_frac": STEP_WORDS * w * N / (ms * 1e-3) / 1e9 / pk, "peak_gbs": pk, "peak": kind,
            "phases_ms": {tb.PHASES[k]: round(ph[k] / max(1, nst), 5) for k in range(tb.NPHASE)},
            "bulk_velocity_after": ub}


def time_reference(c: dict, precision: str, steps: int, warmup: int) -> dict:
    script = os.path.join(ROOT, "oracle", "ref_gpu_time.py")
    try:
        r = subprocess.run([sys.executable, script, "--config", c["ref"], "--precision", precision, "--steps",
                            str(steps), "--warmup", str(warmup)], capture_output=True, text=True, timeout=900)
        lines = [x for x in r.stdout.splitlines() if x.startswith("{")]
        return json.loads(lines[-1]) if lines else {"unavailable": (r.stdout + r.stderr)[-300:]}
    except (subprocess.TimeoutExpired, OSError, ValueError) as e:
        return {"unavailable": f"{type(e).__name__}: {e}"[:300]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--configs", nargs="+", default=["c1", "c3"], choices=list(CONFIGS))
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--no-reference", action="store_true")
    a = ap.parse_args()
    for name in a.configs:
        c = CONFIGS[name]
        line = {"config": name, "workload": c["what"], "cells": c["NX"] * c["NY"] * c["NZ"],
                "fp64": time_ours(c, tb.FP64, a.steps, max(3, a.warmup)),
                "mixed": time_ours(c, tb.MIXED, a.steps, max(3, a.warmup))}
        if not a.no_reference:
            line["reference_gpu_f64"] = time_reference(c, "f64", a.steps, max(3, a.warmup))
            r = line["reference_gpu_f64"]
            if "ms_per_step" in r:
                line["reference_f64_ms_over_ours_fp64"] = r["ms_per_step"] / line["fp64"]["ms_per_step"]
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
