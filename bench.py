#!/usr/bin/env python
"""Throughput of the SBDF3 channel step on B200: cell-steps/s.

Workload (the configuration the metric is quoted on): staggered Verstappen-Veldman
4th-order DNS, Re_bulk 21900 (Re_tau ~ 590), 384 x 256 x 384 cells with the
wall-normal direction in the middle (library axes: NX=384 streamwise, NY=384
spanwise, NZ=256 wall-normal), domain 2pi x 2 x pi, tanh mesh (gamma 2.2),
dt = 0.0008, constant flow rate U_b = 1.  Seeded synthetic field: laminar
profile 1.5(1-y^2) plus MT19937-64(12345) uniform noise of amplitude 0.1,
projected divergence-free.

`value` is the mixed-precision form (float storage, stencils and FFTs; double
low-|k| banded solves, forcing and reductions); the plain FP64 form is measured
in the same run and reported under "fp64".  Every field level (450 MB float,
900 MB double) is far larger than the 126 MB L2, so no flush is needed between
steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-steps/s on 1 B200, mixed vs FP64, %HBM roofline; LES err vs filt. DNS"
WORKLOAD = dict(scheme=1, NX=384, NY=384, NZ=256, Lx=2 * math.pi, Ly=math.pi, Re_b=21900.0, gamma=2.2, tau=0.0008)
# Algorithmic words per cell moved by each phase of one step (the fixed model):
# flux+combine 21 (read v_n, v_{n-1}, v_{n-2}, F_{n-1}, F_{n-2}; write F_n, RHS),
# divergence+x-FFT 4, y-FFT 2, z-solve 2, inverse y-FFT 2, inverse x-FFT 2,
# gradient+correction 7 (read p, RHS; write v_{n+1}); total 40.
PHASE_WORDS = {"turb": 2, "flux": 21, "div_xfft": 4, "yfft": 2, "zsolve": 2, "iyfft": 2, "ixfft": 2, "correct": 7}
STEP_WORDS = 40
FALLBACK_HBM_GBS = 6650.0
# DRAM bytes per cell of one launch of a phase's kernels (dram__bytes_read.sum +
# dram__bytes_write.sum from one ncu capture with inputs larger than L2, divided by the
# captured grid's cells; traffic grows with the cell count, so it is scaled to the grid).
# The captures, their grids and commands are recorded in profiles/traffic_per_cell.json.
def traffic_per_cell() -> dict:
    path = os.path.join(ROOT, "profiles", "traffic_per_cell.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return {(e["phase"], int(e["word_bytes"])): float(e["bytes_per_cell"]) for e in d["captures"]}
    except (OSError, ValueError, KeyError):
        return {}


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


GRID = None  # (NX, NY, NZ) override for profiling runs (--grid); not a bench number
FLUX_STAGING = None  # --flux-staging: the float flux kernel's ring fill, None = the library default


def workload_params(precision: int, device: int, small: bool = False):
    import turbchannel_b200 as tb

    w = dict(WORKLOAD)
    if small:
        w.update(NX=96, NY=96, NZ=64)
    if GRID:
        w.update(NX=GRID[0], NY=GRID[1], NZ=GRID[2])
    p, zz = tb.channel_params(w["scheme"], w["NX"], w["NY"], w["NZ"], w["Lx"], w["Ly"], w["Re_b"], w["gamma"],
                              precision=precision, device=device)
    return p, zz, w


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.tmp = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=self.tmp, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        self.tmp.flush()
        rows = []
        with open(self.tmp.name) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.tmp.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower().startswith("active")})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


def time_arm(precision: int, steps: int, warmup: int, device: int, dist_ctx, small=False, clocks=True):
    """Device-timed K steps (CUDA events on the solver's stream), max over ranks."""
    import torch
    import turbchannel_b200 as tb

    p, zz, w = workload_params(precision, device, small)
    S = tb.Solver(p, zz)
    if FLUX_STAGING is not None:
        S.set_flux_staging(FLUX_STAGING)
    S.init_channel(0, seed=12345, amp=0.1, project=True)
    S.set_forcing(1, 1.0)
    tau = w["tau"]
    stream = torch.cuda.ExternalStream(S.stream(), device=device)
    cur, it = 0, 0
    for _ in range(warmup):
        S.Step(it * tau, tau, cur, min(it + 1, 3))
        cur, it = (cur + 1) % 4, it + 1
    S.sync()
    if dist_ctx:
        dist_ctx.barrier()
    torch.cuda.synchronize(device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sampler = ClockSampler(device) if clocks else None
    if sampler:
        sampler.start()
        time.sleep(0.3)
    S.phase_timing(True)
    n0 = S.launch_count()
    e0.record(stream)
    for _ in range(steps):
        S.Step(it * tau, tau, cur, min(it + 1, 3))
        cur, it = (cur + 1) % 4, it + 1
    e1.record(stream)
    e1.synchronize()
    n1 = S.launch_count()
    clk = sampler.stop() if sampler else None
    torch.cuda.synchronize(device)
    ms = e0.elapsed_time(e1)
    phase_ms, nst = S.phase_times()
    S.phase_timing(False)
    S.sync()
    ub = S.CalcIntegral(cur)[0] / p["area"]
    if dist_ctx:
        ms = dist_ctx.max(ms)
    return dict(solver=S, params=p, w=w, ms=ms, phase_ms=phase_ms, phase_steps=nst, launches=n1 - n0, clocks=clk,
                cur=cur, it=it, ub=ub)


def roofline_for(arm, peak_gbs, word_bytes):
    import turbchannel_b200 as tb

    N = arm["params"]["NX"] * arm["params"]["NY"] * arm["params"]["NZ"]
    per = {tb.PHASES[k]: arm["phase_ms"][k] / max(1, arm["phase_steps"]) for k in range(tb.NPHASE)}
    dom = max(per, key=lambda k: per[k])
    bytes_alg = PHASE_WORDS[dom] * word_bytes * N
    ach = bytes_alg / (per[dom] * 1e-3) / 1e9
    tpc = traffic_per_cell().get((dom, word_bytes))
    roof = {"kernel": dom, "bound": "hbm", "achieved": round(ach, 1), "peak": peak_gbs, "unit": "GB/s",
            "frac": round(ach / peak_gbs, 4), "traffic": None if tpc is None else round(tpc * N),
            "bytes_per_launch_alg": bytes_alg, "ms_per_launch": round(per[dom], 5)}
    step_ms = arm["ms"] / arm["steps"]
    step_ach = STEP_WORDS * word_bytes * N / (step_ms * 1e-3) / 1e9
    step_roof = {"bound": "hbm", "achieved": round(step_ach, 1), "peak": peak_gbs, "unit": "GB/s",
                 "frac": round(step_ach / peak_gbs, 4), "bytes_per_step_alg": STEP_WORDS * word_bytes * N}
    return roof, step_roof, {k: round(v, 5) for k, v in per.items()}


def e2e_arm(arm, steps, device):
    """End to end through the C ABI: upload the starting state from pinned host
    memory, K steps each followed by the reference driver's per-step diagnostics
    (CalcIntegral, CalcProfiles with its device->host copy, CalcCFL; one fused pass),
    and download of the final state -- all inside the timed region."""
    import torch

    S, p, w = arm["solver"], arm["params"], arm["w"]
    N = p["NX"] * p["NY"] * p["NZ"]
    vel_h = torch.empty((N, 3), dtype=torch.float64, pin_memory=True).numpy()
    p_h = torch.empty((N,), dtype=torch.float64, pin_memory=True).numpy()
    v, q = S.download_level(arm["cur"])
    vel_h[:] = v
    p_h[:] = q
    del v, q
    stream = torch.cuda.ExternalStream(S.stream(), device=device)
    tau = w["tau"]
    cur, it = arm["cur"], arm["it"]
    torch.cuda.synchronize(device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    S.upload_level(cur, vel_h, p_h)
    for _ in range(steps):
        S.Step(it * tau, tau, cur, 3)
        cur, it = (cur + 1) % 4, it + 1
        S.diagnostics(cur, tau)
    S.L.tc_download_level(S.h, cur, vel_h.ctypes.data, p_h.ctypes.data)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    # the per-step diagnostics alone (kernel, copy of the plane sums, host wait)
    nd = min(steps, 50)
    e0.record(stream)
    for _ in range(nd):
        S.diagnostics(cur, tau)
    e1.record(stream)
    e1.synchronize()
    diag_ms = e0.elapsed_time(e1) / nd
    diag_bytes = p["NZ"] * 19 * 8
    field_bytes = 4 * N * 8
    return dict(value=N * steps / (ms * 1e-3), unit="cell-steps/s", ms_per_step=ms / steps, steps=steps,
                amortised=f"one state upload and one download over the {steps} steps; per-step diagnostics copy",
                h2d_bytes_per_step=field_bytes // steps, d2h_bytes_per_step=diag_bytes + field_bytes // steps,
                diagnostics_ms=round(diag_ms, 4))


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


# The reference's own CPU path at the bench workload's size, compiled from its sources by
# `make -C oracle ref` (the 384 x 384 x 256 build uses the compile-time index-wrap
# generalisation of oracle/ref/index_wrap.h; nothing else of the reference changes).
REF_CPU_LIB = "stag_vv4_dns_c4_f64"


def cpu_baseline(small=False, budget_s=20.0, max_steps=3):
    """The reference's CPU path (oracle/_ref, OpenMP over all host threads) on a bounded
    sample of the same workload; the oracle (its CPU restatement, pinned to it) where that
    build is absent or for the --small grid.  Constant flow rate as the oracle's driver
    applies it after each step."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_py as op

    w = dict(WORKLOAD)
    if small:
        w.update(NX=96, NY=96, NZ=64)
    threads = os.cpu_count() or 1
    op.set_threads(threads)
    p, zz = op.channel_params(w["scheme"], w["NX"], w["NY"], w["NZ"], w["Lx"], w["Ly"], w["Re_b"], w["gamma"])
    kind = "reference" if (not small and op.ref_available(REF_CPU_LIB)) else "port"
    if kind == "reference":
        O = op.RefLib(REF_CPU_LIB)
        O.L.ref_set_threads(threads)
        O.setup(p, zz)
        import ref_gpu_time as rg

        v = rg.seeded_field(p, zz, w["scheme"])
        O.set_level(0, v, np.zeros(v.shape[0]))
        del v
        O.project(0)
        what = f"the reference's own CPU path (oracle/_ref/libref_{REF_CPU_LIB}.so)"
    else:
        O = op.Oracle(p, zz, "f64")
        O.init_channel(0, seed=12345, amp=0.1, project=True)
        what = "the oracle (CPU restatement of the reference's path)"
    tau = w["tau"]
    O.step(0.0, tau, 0, 1, cfr=1.0)  # untimed: first-touch of the solver's buffers
    cur, it, n = 1, 1, 0
    t0 = time.perf_counter()
    while n < max_steps:
        O.step(it * tau, tau, cur, min(it + 1, 3), cfr=1.0)
        cur, it, n = (cur + 1) % 4, it + 1, n + 1
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    N = w["NX"] * w["NY"] * w["NZ"]
    del O
    return {"value": N * n / dt, "unit": "cell-steps/s", "cores": threads, "kind": kind, "cpu": cpu_model(),
            "sample": f"{n} SBDF step(s) of the full {w['NX']}x{w['NZ']}x{w['NY']} VV4 grid after 1 untimed step, "
                      f"FP64, {what}, {threads} OpenMP threads, {dt:.1f} s"}


def workload_config(w: dict, world: int) -> dict:
    """The `config` object of both arms' lines (the same workload, whatever the precision)."""
    return {"workload": f"staggered VV4 DNS {w['NX']}x{w['NZ']}x{w['NY']} (x, wall-normal, span) cells, "
                        "Re_b 21900, 2pi x 2 x pi, tanh 2.2, dt 0.0008, constant flow rate",
            "grid": [w["NX"], w["NY"], w["NZ"]], "cells": w["NX"] * w["NY"] * w["NZ"],
            "parallelism": "replicas only" if world > 1 else "1 GPU",
            "l2": "inputs larger than L2 (one field level 450 MB f32 / 900 MB f64)"}


def reference_gpu(steps: int, warmup: int, device: int, precisions=("f64", "f32"), config="vv4_c4"):
    """The reference's own GPU path (its data_cuda solver: lambda kernels, cuFFT, Thrust),
    compiled from its sources into oracle/_ref, timed on this GPU by oracle/ref_gpu_time.py
    in a child process (its own CUDA context; the reference exits on a CUDA error)."""
    out = {}
    script = os.path.join(ROOT, "oracle", "ref_gpu_time.py")
    for prec in precisions:
        try:
            r = subprocess.run([sys.executable, script, "--config", config, "--precision", prec, "--steps",
                                str(steps), "--warmup", str(warmup), "--device", str(device)],
                               capture_output=True, text=True, timeout=600)
            lines = [x for x in r.stdout.splitlines() if x.startswith("{")]
            out[prec] = json.loads(lines[-1]) if lines else {"unavailable": f"no output (rc {r.returncode}): "
                                                                            f"{(r.stdout + r.stderr)[-300:]}"}
        except (subprocess.TimeoutExpired, OSError, ValueError) as e:
            out[prec] = {"unavailable": f"{type(e).__name__}: {e}"[:300]}
    return out


def aggregate_value(world: int, cells: int, steps: int, ms_max: float) -> float:
    """Whole-job cell-steps/s of `world` replicas, each of `cells` cells and `steps` steps,
    timed by the slowest rank (ms_max, the maximum over ranks)."""
    return world * cells * steps / (ms_max * 1e-3)


class Dist:
    """The ranks of a multi-GPU run (one process per GPU, replicas of the workload): a
    barrier before and after the timed region and the maximum over ranks of each time.
    backend "nccl" on the GPUs; "gloo" (CPU tensors) serves the CPU tests of this logic."""

    def __init__(self, backend: str = "nccl"):
        import datetime

        import torch
        import torch.distributed as dist

        self.dist = dist
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
        self.rank, self.world = dist.get_rank(), dist.get_world_size()
        self.torch = torch
        self.device = "cuda" if backend == "nccl" else "cpu"

    def barrier(self):
        self.dist.barrier()

    def max(self, x: float) -> float:
        t = self.torch.tensor([x], dtype=self.torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        self.dist.destroy_process_group()


def run_reference(args, world, rank):
    """Reference arm: the reference's own CPU path (its data_cpu solver, compiled from its
    sources into oracle/_ref at 384 x 384 x 256) timed on all host cores; the oracle port
    only where that build is absent."""
    if rank != 0:
        return
    w = dict(WORKLOAD)
    if args.small:
        w.update(NX=96, NY=96, NZ=64)
    base = cpu_baseline(small=args.small, budget_s=max(10.0, min(120.0, 2.0 * args.steps)), max_steps=max(1, args.steps))
    line = {"impl": "reference", "metric": METRIC, "value": base["value"], "unit": "cell-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(w, world),
            "cpu_baseline": base, "e2e": {"value": base["value"], "unit": "cell-steps/s", "h2d_bytes_per_step": 0,
                                         "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--small", action="store_true", help="96x64x96 grid (quick check, not a bench number)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip timing the reference's own GPU path on this GPU")
    ap.add_argument("--only", choices=["mixed", "fp64"], help="time one precision only (profiling)")
    ap.add_argument("--grid", type=int, nargs=3, metavar=("NX", "NY", "NZ"),
                    help="override the grid (profiling runs; not a bench number)")
    ap.add_argument("--flux-staging", type=int, choices=[0, 1], default=None,
                    help="float flux kernel ring fill: 0 cp.async, 1 TMA tensor boxes (tc_set_flux_staging)")
    args = ap.parse_args()
    global GRID, FLUX_STAGING
    if args.grid:
        GRID = tuple(args.grid)
    FLUX_STAGING = args.flux_staging
    if args.only == "mixed":
        args.no_fp64 = True
    args.warmup = max(3, args.warmup)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, world, rank)
        return

    import torch

    torch.cuda.set_device(local)
    dist_ctx = Dist() if world > 1 else None
    peak, peak_kind = peaks()
    import turbchannel_b200 as tb

    if args.only == "fp64":
        a = time_arm(tb.FP64, args.steps, args.warmup, local, dist_ctx, small=args.small, clocks=False)
        a["steps"] = args.steps
        r64, sr64, pp64 = roofline_for(a, peak, 8)
        if rank == 0:
            print(json.dumps({"fp64_only": True, "ms_per_step": a["ms"] / args.steps, "roofline": r64,
                              "step_roofline": sr64, "phases_ms": pp64}), flush=True)
        a["solver"].close()
        if dist_ctx:
            dist_ctx.close()
        return
    mixed = time_arm(tb.MIXED, args.steps, args.warmup, local, dist_ctx, small=args.small)
    mixed["steps"] = args.steps
    roof, step_roof, per_phase = roofline_for(mixed, peak, 4)
    e2e = e2e_arm(mixed, args.steps, local)
    launches = mixed["launches"]
    clocks = mixed["clocks"]
    N = mixed["params"]["NX"] * mixed["params"]["NY"] * mixed["params"]["NZ"]
    value = aggregate_value(world, N, args.steps, mixed["ms"])
    ub_mixed = mixed["ub"]
    mixed["solver"].close()
    del mixed["solver"]

    fp64 = None
    if not args.no_fp64:
        a = time_arm(tb.FP64, args.steps, args.warmup, local, dist_ctx, small=args.small, clocks=False)
        a["steps"] = args.steps
        r64, sr64, pp64 = roofline_for(a, peak, 8)
        fp64 = {"value": world * N * args.steps / (a["ms"] * 1e-3), "ms_per_step": a["ms"] / args.steps,
                "roofline": r64, "step_roofline": sr64, "phases_ms": pp64, "bulk_velocity": a["ub"]}
        a["solver"].close()

    base = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        base = cpu_baseline(small=args.small)
    ref_gpu = None
    if rank == 0 and world == 1 and not args.no_reference_gpu and not args.small and not GRID:
        ref_gpu = reference_gpu(args.steps, args.warmup, local)
        for prec, ours in (("f64", fp64["ms_per_step"] if fp64 else None), ("f32", mixed["ms"] / args.steps)):
            r = ref_gpu.get(prec, {})
            if ours and "ms_per_step" in r:
                # the reference's step time over ours (FP64 against FP64, its FP32 against our mixed form)
                r["reference_ms_over_ours"] = round(r["ms_per_step"] / ours, 3)

    if rank == 0:
        w = WORKLOAD if not args.small else dict(WORKLOAD, NX=96, NY=96, NZ=64)
        if GRID:
            w = dict(WORKLOAD, NX=GRID[0], NY=GRID[1], NZ=GRID[2])
        roof["peak_kind"] = f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind
        line = {
            "metric": METRIC, "value": value, "unit": "cell-steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": mixed["ms"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded MT19937-64 noise on the laminar profile, projected divergence-free)",
            "config": workload_config(w, world),
            "precision_form": "mixed: f32 storage/stencils/FFT, f64 low-k solves, forcing, reductions "
                              "(the plain FP64 form under \"fp64\")",
            "roofline": roof, "step_roofline": step_roof, "phases_ms": per_phase,
            "cpu_baseline": base, "e2e": e2e, "gpu_launches": launches, "clocks": clocks,
            "fp64": fp64, "mixed_vs_fp64": (value / fp64["value"]) if fp64 else None,
            "bulk_velocity_after": ub_mixed,
            "reference_gpu": ref_gpu,
        }
        print(json.dumps(line), flush=True)
    if dist_ctx:
        dist_ctx.close()


if __name__ == "__main__":
    main()
