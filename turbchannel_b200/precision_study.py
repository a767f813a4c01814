"""Mixed precision against FP64 on the flow configuration of the headline workload:
staggered VV4 DNS, 384 x 256 x 384 cells (x, wall-normal, span), Re_b 21900, 2pi x 2 x pi,
tanh 2.2, constant flow rate, from the seeded field plus large-scale vortices (the
transition trigger of les_experiment; the seeded noise alone decays).

    python -m turbchannel_b200.precision_study short --out short.json
    python -m turbchannel_b200.precision_study long --out long.json [--spinup-a 20000 ...]
    python -m turbchannel_b200.precision_study report short.json long.json > summary.md

short: both precisions from the same state, side by side, dt 0.0008; after 3, 100 and 1000
    steps the mixed form's error against FP64 per field (u, v, w, p: max and RMS relative
    to the FP64 field's max), and of the bulk velocity, kinetic energy, CFL number and the
    per-plane profiles.  Before transition the two trajectories have not separated, so this
    is the arithmetic's error, not chaos.
long: the turbulent statistics.  Each run: spin-up (dt 0.0006 through the transition,
    where the CFL number of the explicit convection peaks, then dt 0.0008), then
    statistics at dt 0.0008 accumulated on the device (tc_stats_accumulate every
    `--stat-every` steps) over the first W steps for each W of `--windows` and over all
    `--stat-steps`.
    Runs: FP64 and mixed from seed 12345, and FP64 and mixed from seed 12346.  Beyond a
    few thousand steps the trajectories of any two runs separate (the flow is chaotic), so
    their statistics differ by sampling error; FP64(12345) against FP64(12346) measures
    that spread, and the mixed-vs-FP64 difference is read against it.
    Statistics (staggered/main.cpp:316-333, staggered/io.cpp:71-96): mean U(z), the
    Reynolds stresses <u'u'>, <v'v'>, <w'w'>, <u'w'> (from the time means of the plane
    sums: <uu> - <u>^2, ...), p_rms, and Re_tau from the wall gradient of the mean u at the
    first cell of each wall (u_tau^2 = nu dU/dz).
"""
from __future__ import annotations

import argparse
import json
import sys
import time

import numpy as np

import turbchannel_b200 as tb

LX, LY, RE_B, GAMMA = 2 * np.pi, np.pi, 21900.0, 2.2
GRID = (384, 384, 256)  # library NX (x), NY (span), NZ (wall-normal)
STEP_POINTS = (3, 100, 1000)


def setup(precision: int, seed: int, vortex: float, grid=GRID):
    from turbchannel_b200.les_experiment import add_vortices

    p, zz = tb.channel_params(tb.VV4, grid[0], grid[1], grid[2], LX, LY, RE_B, GAMMA, precision=precision)
    S = tb.Solver(p, zz)
    S.init_channel(0, seed=seed, amp=0.1, project=True)
    if vortex > 0:
        add_vortices(S, p, zz, vortex, seed=(7 + seed - 12345) % 2**32)
    S.set_forcing(1, 1.0)
    return S, p, zz


def field_errors(a: np.ndarray, b: np.ndarray) -> dict:
    """Error of a against the reference b: max and RMS of a - b over max|b|."""
    d = a - b
    s = max(float(np.max(np.abs(b))), 1e-300)
    return {"max_rel": float(np.max(np.abs(d)) / s), "rms_rel": float(np.sqrt(np.mean(d * d)) / s)}


def short(args) -> dict:
    """Mixed against FP64 from one state over the first 1000 steps (before transition)."""
    S64, p, zz = setup(tb.FP64, args.seed, args.vortex, args.grid)
    S32, _, _ = setup(tb.MIXED, args.seed, args.vortex, args.grid)
    # both start from the FP64 solver's initial state (the float solver gets it rounded)
    v, q = S64.download_level(0)
    S32.upload_level(0, v, q)
    del v, q
    tau, cur, out = args.dt, 0, []
    for it in range(max(STEP_POINTS)):
        for S in (S64, S32):
            S.Step(it * tau, tau, cur, min(it + 1, 3))
        cur = (cur + 1) % 4
        if it + 1 in STEP_POINTS:
            rec = {"steps": it + 1}
            v64, p64 = S64.download_level(cur)
            v32, p32 = S32.download_level(cur)
            for c, name in enumerate("uvw"):
                rec[name] = field_errors(v32[:, c], v64[:, c])
            # pressure up to its arbitrary constant (both are normalised the same way)
            rec["p"] = field_errors(p32, p64)
            del v64, v32, p64, p32
            i64, c64, pr64 = S64.diagnostics(cur, tau)
            i32, c32, pr32 = S32.diagnostics(cur, tau)
            k64, k32 = S64.CalcKineticEnergy(cur), S32.CalcKineticEnergy(cur)
            rec["Ub"] = {"fp64": i64[0] / p["area"], "mixed": i32[0] / p["area"],
                         "rel": abs(i32[0] - i64[0]) / abs(i64[0])}
            rec["KE"] = {"fp64": k64, "mixed": k32, "rel": abs(k32 - k64) / abs(k64)}
            rec["CFL"] = {"fp64": c64, "mixed": c32, "rel": abs(c32 - c64) / abs(c64)}
            names = ["U", "V", "W", "uu", "vv", "ww", "uv", "uw", "vw", "nu_t", "P", "pp"]
            rec["profiles"] = {names[k]: field_errors(pr32[:, k], pr64[:, k])["max_rel"]
                               for k in range(12) if k != 9}
            rec["dpdx"] = {"fp64": S64.last_dpdx(), "mixed": S32.last_dpdx()}
            out.append(rec)
            print(json.dumps({"short": rec["steps"], "u": rec["u"], "p": rec["p"]}), flush=True)
    S64.close()
    S32.close()
    return {"kind": "short", "grid": list(args.grid), "dt": tau, "seed": args.seed, "vortex": args.vortex,
            "records": out}


def derived(prof: np.ndarray, zz: np.ndarray, visc: float) -> dict:
    """Turbulence statistics from time-averaged plane means (NZ, 12: <u>,<v>,<w>, <uu>,<vv>,
    <ww>,<uv>,<uw>,<vw>, <nu_t>, <p>,<pp>; w cell-centred)."""
    U, V, W = prof[:, 0], prof[:, 1], prof[:, 2]
    dz = np.diff(zz)
    H = 0.5 * (zz[-1] - zz[0])
    # u_tau^2 = nu dU/dz at each wall from the first cell (staggered/main.cpp:330-333)
    ut_lo = np.sqrt(max(visc * U[0] / (0.5 * dz[0]), 0.0))
    ut_hi = np.sqrt(max(visc * U[-1] / (0.5 * dz[-1]), 0.0))
    ut = 0.5 * (ut_lo + ut_hi)
    return {"U": U, "uu": prof[:, 3] - U * U, "vv": prof[:, 4] - V * V, "ww": prof[:, 5] - W * W,
            "uw": prof[:, 7] - U * W, "p_rms": np.sqrt(np.maximum(prof[:, 11] - prof[:, 10] ** 2, 0.0)),
            "u_tau": ut, "Re_tau": ut * H / visc, "Re_tau_walls": [ut_lo * H / visc, ut_hi * H / visc]}


def long_run(precision: int, seed: int, args, log) -> dict:
    S, p, zz = setup(precision, seed, args.vortex, args.grid)
    cur, it, t = 0, 0, 0.0
    t0 = time.time()
    name = f"{'fp64' if precision == tb.FP64 else 'mixed'}_seed{seed}"
    hist = []

    def advance(n, tau, first_order_restart):
        nonlocal cur, it, t
        for k in range(n):
            order = min(k + 1, 3) if first_order_restart else 3
            S.Step(t, tau, cur, order)
            t += tau
            cur = (cur + 1) % 4
            it += 1
            if it % 1000 == 0:
                integ, cfl, prof = S.diagnostics(cur, tau)  # raises on a non-finite level
                d = derived(prof, zz, p["visc"])
                hist.append({"step": it, "t": t, "Ub": integ[0] / p["area"], "cfl": cfl, "Re_tau": d["Re_tau"],
                             "dpdx": S.last_dpdx()})
                log(f"{name} step {it} t {t:.2f} Ub {hist[-1]['Ub']:.6f} CFL {cfl:.3f} Re_tau {d['Re_tau']:.1f} "
                    f"({time.time() - t0:.0f} s)")

    advance(args.spinup_a, args.dt_a, True)
    advance(args.spinup_b, args.dt, True)  # tau changed: the reference restarts the BDF order
    S.stats_reset()
    windows = {}
    done = 0
    for target in sorted({*args.windows, args.stat_steps}):
        while done < target:
            n = min(args.stat_every, target - done)
            advance(n, args.dt, False)
            done += n
            S.stats_accumulate(cur, n * args.dt)
        prof, wsum = S.stats_read()
        d = derived(prof, zz, p["visc"])
        windows[str(target)] = {"profiles": prof.tolist(), "time": wsum,
                                **{k: (v.tolist() if isinstance(v, np.ndarray) else v) for k, v in d.items()}}
    S.sync()
    ms = (time.time() - t0) * 1e3 / max(1, it)
    S.close()
    return {"name": name, "precision": "fp64" if precision == tb.FP64 else "mixed", "seed": seed, "steps": it,
            "wall_ms_per_step": ms, "history": hist, "windows": windows, "zz": list(zz), "visc": p["visc"]}


def long(args) -> dict:
    log = lambda s: print(s, file=sys.stderr, flush=True)  # noqa: E731
    runs = []
    for seed in args.seeds:
        for prec in (tb.FP64, tb.MIXED):
            try:
                runs.append(long_run(prec, seed, args, log))
            except tb.TcError as e:  # e.g. a non-finite level reported by the diagnostics
                runs.append({"name": f"{'fp64' if prec == tb.FP64 else 'mixed'}_seed{seed}", "seed": seed,
                             "failed": str(e)})
                log(f"run failed: {e}")
            with open(args.out + ".partial", "w") as f:
                json.dump({"kind": "long", "runs": runs}, f)
    return {"kind": "long", "grid": list(args.grid), "dt": args.dt, "dt_transition": args.dt_a,
            "spinup": [args.spinup_a, args.spinup_b], "stat_steps": args.stat_steps, "windows": args.windows,
            "stat_every": args.stat_every, "vortex": args.vortex, "runs": runs}


STATS = ("U", "uu", "vv", "ww", "uw", "p_rms")


def _sym(name: str, a: np.ndarray) -> np.ndarray:
    """Average of the two channel halves (uw is odd about the centre plane, the rest even)."""
    return 0.5 * (a - a[::-1]) if name == "uw" else 0.5 * (a + a[::-1])


def compare(a: dict, b: dict) -> dict:
    """Statistics of window a against window b: max over z of |a - b| over max|b| (halves
    averaged), relative L2, and the relative Re_tau difference."""
    out = {}
    for k in STATS:
        x, y = _sym(k, np.asarray(a[k])), _sym(k, np.asarray(b[k]))
        s = max(float(np.max(np.abs(y))), 1e-300)
        out[k] = {"max_rel": float(np.max(np.abs(x - y)) / s),
                  "l2_rel": float(np.linalg.norm(x - y) / max(np.linalg.norm(y), 1e-300))}
    out["Re_tau"] = abs(a["Re_tau"] - b["Re_tau"]) / b["Re_tau"]
    return out


def pooled(ws: list) -> dict:
    """Equal-weight mean of several runs' window statistics."""
    out = {k: np.mean([np.asarray(w[k]) for w in ws], axis=0) for k in STATS}
    out["Re_tau"] = float(np.mean([w["Re_tau"] for w in ws]))
    return out


def _pairs(long_res: dict) -> tuple[list, list]:
    """The compared pairs: mixed against FP64 per seed, seed against seed per precision, and
    the seeds' pooled statistics mixed against FP64."""
    seeds = sorted({r["seed"] for r in long_res["runs"]})
    pairs = [(f"mixed_seed{s}", f"fp64_seed{s}") for s in seeds]
    if len(seeds) > 1:
        pairs += [(f"fp64_seed{seeds[1]}", f"fp64_seed{seeds[0]}"),
                  (f"mixed_seed{seeds[1]}", f"mixed_seed{seeds[0]}"),
                  ("mixed_pooled", "fp64_pooled")]
    return seeds, pairs


def _window_stats(long_res: dict, w: str, seeds: list) -> dict:
    runs = {r["name"]: r for r in long_res["runs"] if "failed" not in r}
    wstats = {n: r["windows"][w] for n, r in runs.items()}
    if len(seeds) > 1 and all(f"{k}_seed{s}" in runs for k in ("fp64", "mixed") for s in seeds):
        for k in ("fp64", "mixed"):  # the seeds' statistics averaged: half the sampling variance
            wstats[f"{k}_pooled"] = pooled([wstats[f"{k}_seed{s}"] for s in seeds])
    return wstats


def _windows(long_res: dict) -> list:
    wins = long_res.get("windows", [long_res.get("window")])
    return sorted({*(str(x) for x in wins if x), str(long_res["stat_steps"])}, key=int)


def summary(short_res: dict | None, long_res: dict | None) -> dict:
    """The report's numbers as a compact dict (no profiles): per window and pair the relative
    differences of compare(), per run Re_tau and the centre velocity, and the short study's
    field errors."""
    out = {}
    if short_res:
        out["short"] = {"grid": short_res["grid"], "dt": short_res["dt"],
                        "records": [{**{k: r[k] for k in ("steps", "u", "v", "w", "p", "Ub", "KE", "CFL")},
                                     # V, W, uv, vw average to zero: a difference relative to them says nothing
                                     "profiles": {k: v for k, v in r["profiles"].items()
                                                  if k in ("U", "uu", "vv", "ww", "uw", "P", "pp")}}
                                    for r in short_res["records"]]}
    if long_res:
        seeds, pairs = _pairs(long_res)
        L = {k: long_res[k] for k in ("grid", "dt", "dt_transition", "spinup", "stat_steps", "stat_every")}
        L["windows"] = {}
        for w in _windows(long_res):
            ws = _window_stats(long_res, w, seeds)
            L["windows"][w] = {
                "pairs": {f"{a} vs {b}": compare(ws[a], ws[b]) for a, b in pairs if a in ws and b in ws},
                "runs": {r["name"]: {"Re_tau": r["windows"][w]["Re_tau"],
                                     "Re_tau_walls": r["windows"][w]["Re_tau_walls"],
                                     "U_centre": float(np.asarray(r["windows"][w]["U"])[len(r["windows"][w]["U"]) // 2]),
                                     "steps": r["steps"], "wall_ms_per_step": r["wall_ms_per_step"]}
                         for r in long_res["runs"] if "failed" not in r}}
        L["failed"] = {r["name"]: r["failed"] for r in long_res["runs"] if "failed" in r}
        out["long"] = L
    return out


def _round(x, digits: int = 4):
    """x with every float rounded to a few significant digits (the summary is read, not reused)."""
    if isinstance(x, float):
        return float(f"{x:.{digits}g}")
    if isinstance(x, dict):
        return {k: _round(v, digits) for k, v in x.items()}
    if isinstance(x, (list, tuple)):
        return [_round(v, digits) for v in x]
    return x


def report(short_res: dict | None, long_res: dict | None) -> str:
    L = []
    if short_res:
        L.append(f"### Mixed against FP64 from one state (grid {short_res['grid']}, dt {short_res['dt']})\n")
        L.append("| steps | u max / rms | v max / rms | w max / rms | p max / rms | Ub | KE | CFL | profiles U, uu, ww, P (max) |")
        L.append("|---:|---|---|---|---|---:|---:|---:|---|")
        for r in short_res["records"]:
            f = lambda e: f"{e['max_rel']:.1e} / {e['rms_rel']:.1e}"  # noqa: E731
            pr = r["profiles"]
            L.append(f"| {r['steps']} | {f(r['u'])} | {f(r['v'])} | {f(r['w'])} | {f(r['p'])} | {r['Ub']['rel']:.1e} | "
                     f"{r['KE']['rel']:.1e} | {r['CFL']['rel']:.1e} | {pr['U']:.1e}, {pr['uu']:.1e}, {pr['ww']:.1e}, "
                     f"{pr['P']:.1e} |")
        L.append("")
    if long_res:
        runs = {r["name"]: r for r in long_res["runs"] if "failed" not in r}
        for r in long_res["runs"]:
            if "failed" in r:
                L.append(f"Run {r['name']} failed: {r['failed']}\n")
        seeds, pairs = _pairs(long_res)
        for w in _windows(long_res):
            L.append(f"### Statistics over {w} steps at dt {long_res['dt']} (after {sum(long_res['spinup'])} "
                     f"spin-up steps)\n")
            L.append("| pair | mean U max (L2) | u'u' | v'v' | w'w' | u'w' | p_rms | Re_tau |")
            L.append("|---|---|---|---|---|---|---|---:|")
            wstats = _window_stats(long_res, w, seeds)
            for a, b in pairs:
                if a not in wstats or b not in wstats:
                    continue
                c = compare(wstats[a], wstats[b])
                cells = [f"{c['U']['max_rel']:.2%} ({c['U']['l2_rel']:.2%})"] + \
                        [f"{c[k]['max_rel']:.1%}" for k in STATS[1:]] + [f"{c['Re_tau']:.2%}"]
                L.append(f"| {a} vs {b} | " + " | ".join(cells) + " |")
            L.append("")
            L.append("| run | Re_tau (walls) | U centre | max u'u' | steps | wall ms/step |")
            L.append("|---|---|---:|---:|---:|---:|")
            for n, r in runs.items():
                d = r["windows"][w]
                U = np.asarray(d["U"])
                L.append(f"| {n} | {d['Re_tau']:.1f} ({d['Re_tau_walls'][0]:.1f}, {d['Re_tau_walls'][1]:.1f}) | "
                         f"{U[len(U) // 2]:.4f} | {max(d['uu']):.4f} | {r['steps']} | {r['wall_ms_per_step']:.2f} |")
            L.append("")
    return "\n".join(L)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("mode", choices=["short", "long", "report"])
    ap.add_argument("files", nargs="*", help="report: the short and/or long JSON results")
    ap.add_argument("--out", default="precision_study.json",
                    help="short/long: the results; report: also write the numbers as JSON here if given")
    ap.add_argument("--grid", type=int, nargs=3, default=list(GRID))
    ap.add_argument("--seed", type=int, default=12345)
    ap.add_argument("--seeds", type=int, nargs="+", default=[12345, 12346])
    ap.add_argument("--vortex", type=float, default=0.5)
    ap.add_argument("--dt", type=float, default=0.0008)
    ap.add_argument("--dt-a", type=float, default=0.0006, help="time step through the transition")
    ap.add_argument("--spinup-a", type=int, default=20000)
    ap.add_argument("--spinup-b", type=int, default=10000)
    ap.add_argument("--stat-steps", type=int, default=25000)
    ap.add_argument("--windows", type=int, nargs="+", default=[5000],
                    help="also report the statistics over the first W steps of the window")
    ap.add_argument("--stat-every", type=int, default=5)
    args = ap.parse_args()
    if args.mode == "report":
        res = [json.load(open(f)) for f in args.files]
        sr = next((r for r in res if r["kind"] == "short"), None)
        lr = next((r for r in res if r["kind"] == "long"), None)
        print(report(sr, lr))
        if "--out" in sys.argv:
            with open(args.out, "w") as f:
                json.dump(_round(summary(sr, lr)), f, separators=(",", ":"))
        return
    res = short(args) if args.mode == "short" else long(args)
    with open(args.out, "w") as f:
        json.dump(res, f)


if __name__ == "__main__":
    main()
