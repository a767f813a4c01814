"""Learned-closure LES experiment on one GPU: DNS -> filtered snapshots -> training ->
LES with the learned closure, the Smagorinsky-van Driest fallback and no model, each
compared with the filtered-DNS mean velocity profile.

    python -m turbchannel_b200.les_experiment [--coarsen 4x4 8x4 --dns-steps 50000 ...] --out res.json

1. DNS: staggered VV4, 384x256x384 cells (x, wall-normal, span), Re_b 21900, 2pi x 2 x pi,
   tanh 2.2, dt 0.0006, constant flow rate, mixed precision, from the seeded field plus
   large-scale vortices as a transition trigger (--vortex; the seeded noise alone decays
   and the flow stays laminar); spin-up,
   then statistics: the mean u profile every `--stat-every` steps and, every
   `--snap-every` steps, for each LES grid of `--coarsen` (R x RZ: every R-th DNS face in x
   and span, every RZ-th wall-normal), the snapshot box-filtered over the LES cells as
   closure training samples (features, targets nu*/nu, tc_les_samples).
2. Per LES grid, training of the MLP closure (tc_mlp_*, BF16 tensor cores, Adam) on the
   shuffled samples.
3. LES: staggered HW2 + NAIVE viscosity on that grid (4x4: 96x64x96 cells), started from
   the DNS's last field restricted by face averages (flux-conserving on the nested grids),
   run with each closure; mean u profile over the statistics window against the filtered
   DNS profile restricted to the LES cells.  Reported: relative L2 and max errors,
   bulk-normalised, and the profiles.
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

import turbchannel_b200 as tb

LX, LY, RE_B, GAMMA = 2 * np.pi, np.pi, 21900.0, 2.2


def restrict_to_les(vel, NX, NY, NZ, r, rz, dz_fine):
    """Face-average restriction of a staggered DNS field (N, 3) to the grid r times coarser
    in x and y and rz times in z (nested faces); dz_fine: the DNS cell heights."""
    u = vel[:, 0].reshape(NZ, NY, NX)
    v = vel[:, 1].reshape(NZ, NY, NX)
    w = vel[:, 2].reshape(NZ, NY, NX)
    nz, ny, nx = NZ // rz, NY // r, NX // r
    wz = dz_fine.reshape(nz, rz)
    wz = wz / wz.sum(axis=1, keepdims=True)
    # u on coarse x-face X = fine face r X, averaged over the coarse face (r fine y, rz fine z cells)
    uf = u[:, :, ::r].reshape(nz, rz, ny, r, nx)
    uc = np.einsum("zkyjx,zk->zyx", uf, wz) / r
    vf = v[:, ::r, :].reshape(nz, rz, ny, nx, r)
    vc = np.einsum("zkyxi,zk->zyx", vf, wz) / r
    wf = w[::rz, :, :].reshape(nz, ny, r, nx, r)
    wc = wf.mean(axis=(2, 4))
    out = np.zeros((nx * ny * nz, 3))
    out[:, 0], out[:, 1], out[:, 2] = uc.reshape(-1), vc.reshape(-1), wc.reshape(-1)
    return out


def add_vortices(S, p, zz, amp, seed=7):
    """Adds large-scale vortices to ring level 0 as a transition trigger: for (kx, ky) in
    {1, 2, 3}^2 with seeded random amplitudes and phases, u += -a cos(kx x' + f) sin(ky y' + g) G(z)
    and v += a (Ly/Lx)(kx/ky) sin(kx x' + f) cos(ky y' + g) G(z) (x' = 2 pi x/Lx, y' = 2 pi y/Ly),
    divergence-free mode by mode, G(z) = 1 - ((z - H)/H)^2; the total is scaled to a maximum
    of `amp` (units of the bulk velocity).  At staggered positions; the first step's
    projection removes the discretisation's residual divergence."""
    NX, NY, NZ = p["NX"], p["NY"], p["NZ"]
    v, q = S.download_level(0)
    zc = 0.5 * (zz[:-1] + zz[1:])
    H = 0.5 * (zz[-1] - zz[0])
    G = (1.0 - ((zc - zz[0] - H) / H) ** 2)[:, None, None]
    Lx, Ly = NX * p["hx"], NY * p["hy"]
    xf, xc = np.arange(NX) * p["hx"], (np.arange(NX) + 0.5) * p["hx"]
    yf, yc = np.arange(NY) * p["hy"], (np.arange(NY) + 0.5) * p["hy"]
    rng = np.random.default_rng(seed)
    du = np.zeros((NZ, NY, NX))
    dv = np.zeros((NZ, NY, NX))
    for kx in (1, 2, 3):
        for ky in (1, 2, 3):
            a, f, g = rng.uniform(0.5, 1.0), rng.uniform(0, 2 * np.pi), rng.uniform(0, 2 * np.pi)
            ax = 2 * np.pi * kx / Lx
            ay = 2 * np.pi * ky / Ly
            du += -a * (np.cos(ax * xf + f)[None, None, :] * np.sin(ay * yc + g)[None, :, None]) * G
            dv += a * (ax / ay) * (np.sin(ax * xc + f)[None, None, :] * np.cos(ay * yf + g)[None, :, None]) * G
    sc = amp / max(np.abs(du).max(), np.abs(dv).max())
    v[:, 0] += sc * du.reshape(-1)
    v[:, 1] += sc * dv.reshape(-1)
    S.upload_level(0, v, q)


def run_dns(args, log):
    p, zz = tb.channel_params(tb.VV4, args.nx, args.ny, args.nz, LX, LY, RE_B, GAMMA, precision=tb.MIXED)
    S = tb.Solver(p, zz)
    S.init_channel(0, seed=args.seed, amp=0.1, project=True)
    if args.vortex > 0:
        add_vortices(S, p, zz, args.vortex, seed=(7 + args.seed - 12345) % 2**32)
    S.set_forcing(1, 1.0)
    tau, cur = args.dt, 0
    prof, nprof = np.zeros(args.nz), 0
    samples = {cz: ([], []) for cz in args.coarsen}
    # resolved statistics of the filtered DNS on each LES grid, from the snapshots: per coarse
    # plane the sums of the filtered u, v, w and of their products (plane means, then time)
    fstat = {cz: np.zeros((args.nz // cz[1], 6)) for cz in args.coarsen}
    nfs = 0
    rng = np.random.default_rng(1)
    t0 = time.time()
    total = args.dns_steps + args.stat_steps
    for it in range(total):
        S.Step(it * tau, tau, cur, min(it + 1, 3))
        cur = (cur + 1) % 4
        if it >= args.dns_steps:
            k = it - args.dns_steps
            if k % args.stat_every == 0:
                prof += S.CalcProfiles(cur)[:, 0]
                nprof += 1
            if k % args.snap_every == 0:
                if args.snap_dir:  # the filtered snapshot of the first LES grid, 10 fields
                    r0, rz0 = args.coarsen[0]
                    np.save(os.path.join(args.snap_dir, f"snap_{k:07d}.npy"), S.les_filter(cur, r0, rz0))
                for (r, rz) in args.coarsen:
                    F = S.les_filter(cur, r, rz).astype(np.float64)
                    ub, vb, wb = F[0], F[1], F[2]
                    fstat[(r, rz)] += np.stack([ub.mean(axis=(1, 2)), vb.mean(axis=(1, 2)), wb.mean(axis=(1, 2)),
                                                (ub * ub).mean(axis=(1, 2)), (wb * wb).mean(axis=(1, 2)),
                                                (ub * wb).mean(axis=(1, 2))], axis=1)
                nfs += 1
                for (r, rz), (Xs, Ys) in samples.items():
                    X, Y = S.les_samples(cur, r, rz)
                    sel = rng.random(len(Y)) < args.sample_frac * r * r * rz / 64
                    Xs.append(X[sel])
                    Ys.append(Y[sel])
        if (it + 1) % 1000 == 0:
            ub = S.CalcIntegral(cur)[0] / p["area"]
            log(f"DNS step {it + 1}/{total}  Ub {ub:.5f}  dp/dx {S.last_dpdx():.5f}  {time.time() - t0:.0f} s")
    S.sync()
    vel, _ = S.download_level(cur)
    S.close()
    return dict(params=p, zz=zz, prof=prof / max(nprof, 1), vel=vel, wall_s=time.time() - t0, snapshots=nfs,
                fstat={cz: v / max(nfs, 1) for cz, v in fstat.items()},
                samples={cz: (np.concatenate(Xs), np.concatenate(Ys)) for cz, (Xs, Ys) in samples.items()})


def run_les(args, model, params, vel0, r, rz, log):
    p, zz = tb.channel_params(tb.HW2, args.nx // r, args.ny // r, args.nz // rz, LX, LY, RE_B, GAMMA,
                              precision=tb.FP64, visc_type=tb.VISC_NAIVE, turb=tb.TURB_SMAGORINSKY)
    S = tb.Solver(p, zz)
    if model == "mlp":
        S.set_turb_model(tb.TURB_MLP, params)
    elif model == "none":
        S.set_turb_model(tb.TURB_NONE)
    S.upload_level(0, vel0, np.zeros(len(vel0)))
    S.set_forcing(1, 1.0)
    tau, cur = args.les_dt, 0
    prof, wsum = np.zeros(p["NZ"]), 0.0
    full = np.zeros((p["NZ"], 12))
    total = args.les_steps + args.les_stat_steps
    import torch

    stream = torch.cuda.ExternalStream(S.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start, t, timed = 0, 0.0, False
    for it in range(total):
        if it == args.les_steps:
            e0.record(stream)
            timed = True
        S.Step(t, tau, cur, min(it - start + 1, 3))
        cur = (cur + 1) % 4
        t += tau
        if it >= args.les_steps and (it - args.les_steps) % args.stat_every == 0:
            pf = S.CalcProfiles(cur)
            prof += tau * pf[:, 0]
            full += tau * pf
            wsum += tau
        if it % 10 == 9:  # the reference driver's CFL control (staggered/main.cpp:361-370)
            cfl = S.CalcCFL(cur, tau, 3)
            if not np.isfinite(cfl):
                break
            while cfl > args.cfl_max:
                cfl *= 0.5
                tau *= 0.5
                start = it + 1
            if cfl < args.cfl_min:
                tau *= 1.5
                start = it + 1
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / max(1, args.les_stat_steps) if timed else float("nan")
    ub = S.CalcIntegral(cur)[0] / p["area"]
    ok = bool(np.all(np.isfinite(prof)))
    S.close()
    log(f"LES {args.nx // r}x{args.nz // rz}x{args.ny // r} {model}: Ub {ub:.5f}, {ms:.4f} ms/step "
        f"(with the per-sample profile calls)")
    full = full / max(wsum, 1e-300)
    stress = {"uu": full[:, 3] - full[:, 0] ** 2, "ww": full[:, 5] - full[:, 2] ** 2,
              "uw": full[:, 7] - full[:, 0] * full[:, 2]}
    return dict(prof=prof / max(wsum, 1e-300), ms_per_step=ms, ub=ub, finite=ok, zz=zz, final_tau=tau,
                cells=p["NX"] * p["NY"] * p["NZ"], stress=stress)


def summarize(paths: list) -> str:
    """Markdown table of experiment results (one JSON per run): per LES grid and model the
    mean-u error and the resolved-stress errors against the filtered DNS, and the cost."""
    rows = ["| run | LES grid | model | mean u rel. L2 | <u'u'> | <w'w'> | <u'w'> | ms/step | ns/cell-step |",
            "|---|---|---|---:|---:|---:|---:|---:|---:|"]
    agg = {}
    for path in paths:
        with open(path) as f:
            res = json.load(f)
        run = os.path.basename(path).rsplit(".", 1)[0]
        for case in res["cases"]:
            g = "x".join(str(v) for v in case["les_grid"])
            for model, r in case["les"].items():
                st = r.get("stress_rel_l2_err", {})
                rows.append(f"| {run} | {g} | {model} | {r['rel_l2_err_mean_u']:.2%} | {st.get('uu', float('nan')):.1%} "
                            f"| {st.get('ww', float('nan')):.1%} | {st.get('uw', float('nan')):.1%} | "
                            f"{r['ms_per_step']:.3f} | {r.get('ns_per_cell_step', float('nan')):.3f} |")
                agg.setdefault((g, model), []).append(r["rel_l2_err_mean_u"])
    rows += ["", "| LES grid | model | mean u rel. L2: mean over runs | min | max | runs |", "|---|---|---:|---:|---:|---:|"]
    for (g, model), v in sorted(agg.items()):
        rows.append(f"| {g} | {model} | {np.mean(v):.2%} | {np.min(v):.2%} | {np.max(v):.2%} | {len(v)} |")
    return "\n".join(rows)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--nx", type=int, default=384)
    ap.add_argument("--ny", type=int, default=384)
    ap.add_argument("--nz", type=int, default=256)
    ap.add_argument("--dt", type=float, default=0.0006,
                    help="DNS time step; during transition the CFL number at 0.0008 reaches 0.8-1.0, the edge of "
                         "the explicit SBDF3 convection's stability")
    ap.add_argument("--vortex", type=float, default=0.5,
                    help="maximum amplitude (units of the bulk velocity) of large-scale vortices added to the "
                         "seeded field as a transition trigger; the seeded noise alone decays without transition")
    ap.add_argument("--seed", type=int, default=12345,
                    help="seed of the DNS initial noise (the vortex trigger uses (seed - 12338) mod 2^32: 7 by default)")
    ap.add_argument("--dns-steps", type=int, default=50000)
    ap.add_argument("--stat-steps", type=int, default=25000)
    ap.add_argument("--stat-every", type=int, default=10)
    ap.add_argument("--snap-every", type=int, default=500)
    ap.add_argument("--sample-frac", type=float, default=0.2)
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--les-dt", type=float, default=0.002)
    ap.add_argument("--cfl-min", type=float, default=0.1)
    ap.add_argument("--cfl-max", type=float, default=0.4)
    ap.add_argument("--les-steps", type=int, default=10000)
    ap.add_argument("--les-stat-steps", type=int, default=20000)
    ap.add_argument("--coarsen", type=lambda t: tuple(int(v) for v in t.split("x")), nargs="+", default=[(4, 4)],
                    help="LES grids as coarsening factors RxRZ (x and span R, wall-normal RZ), e.g. 4x4 8x4")
    ap.add_argument("--dissipation-weighted", action="store_true",
                    help="train on samples drawn with probability proportional to (S:S)^2 (the squared "
                         "sub-filter dissipation error per unit viscosity error)")
    ap.add_argument("--snap-dir", default="",
                    help="directory for the box-filtered snapshots (float32 .npy, fields u, v, w, p, uu, vv, ww, uv, "
                         "uw, vw on the first LES grid of --coarsen)")
    ap.add_argument("--out", default="les_experiment.json")
    ap.add_argument("--summary", nargs="+", metavar="JSON", help="print the markdown summary of finished runs")
    args = ap.parse_args()
    if args.summary:
        print(summarize(args.summary))
        return
    if args.snap_dir:
        os.makedirs(args.snap_dir, exist_ok=True)
    t_start = time.time()

    def log(msg):
        print(f"[{time.time() - t_start:7.1f} s] {msg}", flush=True)

    dns = run_dns(args, log)
    dz = np.diff(dns["zz"])
    res = {"dns": {"grid": [args.nx, args.nz, args.ny], "steps": args.dns_steps + args.stat_steps, "dt": args.dt,
                   "wall_s": dns["wall_s"]}, "cases": []}
    for r, rz in args.coarsen:
        X, Y = dns["samples"][(r, rz)]
        log(f"coarsening {r} x {rz} x {r}: samples {len(Y)}  target mean {Y.mean():.4g}  max {Y.max():.4g}")
        perm = np.random.default_rng(2).permutation(len(Y))
        X, Y = X[perm], Y[perm]
        nval = max(1, len(Y) // 10)
        m = tb.Mlp(seed=12345)
        Xt, Yt = X[nval:], Y[nval:]
        if args.dissipation_weighted:
            # weighted least squares by resampling: the sub-filter dissipation error of a
            # prediction is 2 (nu - nu*) S:S, so each sample counts with (S:S)^2, S:S =
            # sinh of the first feature (wall units)
            wgt = np.sinh(Xt[:, 0].astype(np.float64)) ** 2
            idx = np.random.default_rng(3).choice(len(Yt), size=len(Yt), p=wgt / wgt.sum())
            Xt, Yt = Xt[idx], Yt[idx]
        m.set_data(Xt, Yt)
        losses = m.train(args.epochs, args.batch, args.lr)
        pred = m.forward(X[:nval])
        params = m.params
        m.close()
        val_mse = float(np.mean((pred - Y[:nval]) ** 2))
        zero_mse = float(np.mean(Y[:nval] ** 2))
        log(f"training: loss {losses[0]:.4g} -> {losses[-1]:.4g}; held-out MSE {val_mse:.4g} (nu_t = 0: {zero_mse:.4g})")
        vel0 = restrict_to_les(dns["vel"], args.nx, args.ny, args.nz, r, rz, dz)
        # filtered-DNS mean u profile on the LES cells (dz-weighted average of rz DNS cells)
        wz = dz.reshape(-1, rz)
        ref = (dns["prof"].reshape(-1, rz) * wz).sum(axis=1) / wz.sum(axis=1)
        fs = dns["fstat"][(r, rz)]  # filtered DNS: resolved <u'u'>, <w'w'>, <u'w'> per LES plane
        fref = {"uu": fs[:, 3] - fs[:, 0] ** 2, "ww": fs[:, 4] - fs[:, 2] ** 2, "uw": fs[:, 5] - fs[:, 0] * fs[:, 2]}
        case = {"les_grid": [args.nx // r, args.nz // rz, args.ny // r], "filter": [r, rz, r],
                "snapshots": dns["snapshots"],
                "filtered_dns_stress": {k: v.tolist() for k, v in fref.items()},
                "training": {"samples": int(len(Y)), "epochs": args.epochs, "loss_first": float(losses[0]),
                             "loss_last": float(losses[-1]), "heldout_mse": val_mse, "heldout_mse_no_model": zero_mse},
                "filtered_dns_mean_u": ref.tolist(), "les": {}}
        for model in ("mlp", "smagorinsky", "none"):
            out = run_les(args, model, params, vel0, r, rz, log)
            err = out["prof"] - ref
            case["les"][model] = {"rel_l2_err_mean_u": float(np.linalg.norm(err) / np.linalg.norm(ref)),
                                  "max_err_mean_u": float(np.max(np.abs(err))), "ms_per_step": out["ms_per_step"],
                                  "bulk_velocity": out["ub"], "finite": out["finite"], "mean_u": out["prof"].tolist(),
                                  "ns_per_cell_step": out["ms_per_step"] * 1e6 / out["cells"],
                                  "stress_rel_l2_err": {k: float(np.linalg.norm(out["stress"][k] - fref[k]) /
                                                                 max(np.linalg.norm(fref[k]), 1e-300))
                                                        for k in fref}}
            log(f"  {model}: rel L2 error of the mean u profile {case['les'][model]['rel_l2_err_mean_u']:.4f}")
        res["cases"].append(case)
    with open(args.out, "w") as f:
        json.dump(res, f, indent=1)
    log(f"wrote {args.out}")


if __name__ == "__main__":
    main()
