"""Trains and judges the learned SGS closure on the perturbed-ellipsoid case.

  python -m aerosim_b200.sgs_training [--fine-steps 24000] [--out results.json]
                                      [--weights aerosim_b200/data/sgs_mlp_ellipsoid.npz]

1. Fine plain run: 512x256x256, Smagorinsky (Cs = 0.1), FP32 -- the reference
   solution.  Its Cd is averaged over the second half of the run (a sample every 200
   steps); from the second half on, every `--snapshot-every` steps its macro fields are
   box-filtered onto the
   256x128x128 lattice into training samples (aerosim_sgs_samples).
   The eddy-viscosity target is the least-squares fit of the subgrid stress per coarse
   cell, or over each cell's (2r+1)^3 neighbourhood (--average-radius r), clipped below at
   --min-ratio x nu_0 (0: no backscatter; a negative bound keeps it in the targets).
2. Training on the GPU (aerosim_mlp_train, Adam) on all snapshots but the last; the
   last one is held out: the closure's eddy viscosity and Smagorinsky's are both scored
   against the filtered subgrid stress (mean squared error of nu_t / nu_0).
3. Coarse runs at 256x128x128 over the same physical time (half the steps): plain
   Smagorinsky, the learned closure and no eddy viscosity at all.  Cd over the second half of each run against the
   fine run's (with the standard error of each mean from 10 block means), and device time
   of each run.

The weights are written to `--weights` (FP32 parameter vector, aerosim_b200.sgs
layout) and the metrics to `--out`.
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import LBMEngine, cases, frontal_area, sgs


def _engine(case, precision: str = "f32", cs: float | None = None) -> LBMEngine:
    pos = case.mesh[0]
    e = LBMEngine(0)
    e.voxelize(case.mesh, None, case.tunnel, {"nx": case.nx, "ny": case.ny, "nz": case.nz},
               {"uInletLattice": case.u_inlet, "nuLattice": case.nu,
                "smagorinskyCs": case.cs if cs is None else cs,
                "precision": precision, "frontalAreaM2": frontal_area(case.mesh),
                "characteristicLengthM": float(pos[:, 0].max() - pos[:, 0].min())})
    return e


def _run(e: LBMEngine, steps: int, every: int, on_sample=None):
    """Steps `steps`, reading Cd every `every` steps over the second half; returns
    (Cd samples, device milliseconds of the steps)."""
    cd, ms, done = [], 0.0, 0
    half = steps // 2
    while done < steps:
        k = min(every, steps - done) if done >= half else min(half - done, steps - done)
        e.step(k)
        ms += e.last_step_timing()[0]
        done += k
        if done > half or done == steps:
            cd.append(e.read_forces().cd)
            if on_sample:
                on_sample(done)
    return np.array(cd), ms


def block_se(x: np.ndarray, blocks: int = 10) -> float:
    """Standard error of the mean of a correlated series from the means of `blocks`
    consecutive blocks (batch means); 0 for fewer samples than blocks."""
    n = (len(x) // blocks) * blocks
    if n < blocks or blocks < 2:
        return 0.0
    m = x[:n].reshape(blocks, -1).mean(axis=1)
    return float(m.std(ddof=1) / np.sqrt(blocks))


def main(argv=None) -> dict:
    ap = argparse.ArgumentParser()
    ap.add_argument("--fine-steps", type=int, default=24000)
    ap.add_argument("--snapshot-every", type=int, default=2000)
    ap.add_argument("--samples-per-snapshot", type=int, default=600000)
    ap.add_argument("--iters", type=int, default=4000)
    ap.add_argument("--batch", type=int, default=16384)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--average-radius", type=int, default=0,
                    help="least-squares eddy viscosity over (2r+1)^3 coarse cells (0: per cell)")
    ap.add_argument("--min-ratio", type=float, default=0.0,
                    help="lower clip of the targets in units of nu_0 (negative: keep backscatter)")
    ap.add_argument("--scale", type=int, default=1, help="1: 512x256x256 / 256x128x128; 2: half of each")
    ap.add_argument("--out", default="")
    ap.add_argument("--weights", default="")
    a = ap.parse_args(argv)
    rng = np.random.default_rng(a.seed)
    nx, ny, nz = 256 // a.scale, 128 // a.scale, 128 // a.scale
    fine_case = cases.scaled_ellipsoid(2 * nx, 2 * ny, 2 * nz)
    coarse_case = cases.scaled_ellipsoid(nx, ny, nz)
    res: dict = {"fine": f"{2 * nx}x{2 * ny}x{2 * nz}", "coarse": f"{nx}x{ny}x{nz}", "fine_steps": a.fine_steps,
                 "min_ratio": a.min_ratio, "average_radius": a.average_radius}

    # ---- 1. fine plain run and training samples ----
    t0 = time.perf_counter()
    fine = _engine(fine_case)
    coarse_geo = _engine(coarse_case)  # coarse voxel grid: wall distances of the samples
    snaps: list[tuple[np.ndarray, np.ndarray]] = []

    def take(step):
        if step > a.fine_steps // 2 and step % a.snapshot_every == 0:
            X, Y = sgs.samples(fine, coarse_geo, average_radius=a.average_radius, min_ratio=a.min_ratio)
            k = min(a.samples_per_snapshot, X.shape[0])
            sel = rng.choice(X.shape[0], k, replace=False)
            snaps.append((X[sel], Y[sel]))

    cd_f, ms_f = _run(fine, a.fine_steps, 200, take)
    res["fine_cd_mean"] = float(cd_f.mean())
    res["fine_cd_std"] = float(cd_f.std())
    res["fine_cd_se"] = block_se(cd_f)
    res["fine_device_ms"] = ms_f
    res["snapshots"] = len(snaps)
    fine.close()

    # ---- 2. training and held-out scoring ----
    Xt = np.concatenate([s[0] for s in snaps[:-1]])
    Yt = np.concatenate([s[1] for s in snaps[:-1]])
    Xv, Yv = snaps[-1]
    p, curve = sgs.train(sgs.init_params(a.seed), Xt, Yt, iters=a.iters, batch=a.batch, lr=a.lr, seed=a.seed)
    nu0 = (max(3.0 * coarse_case.nu + 0.5, 0.5015) - 0.5) / 3.0
    pred = sgs.forward(p, Xv)
    smag = sgs.smagorinsky_ratio(Xv, nu0, coarse_case.cs)
    res["train_samples"] = int(Xt.shape[0])
    res["heldout_samples"] = int(Xv.shape[0])
    res["loss_first_last"] = [float(curve[:20].mean()), float(curve[-100:].mean())]
    res["heldout_mse_mlp"] = float(np.mean((pred - Yv) ** 2))
    res["heldout_mse_smagorinsky"] = float(np.mean((smag - Yv) ** 2))
    res["heldout_mse_zero"] = float(np.mean(Yv ** 2))
    res["heldout_target_mean"] = float(Yv.mean())
    coarse_geo.close()

    # ---- 3. coarse runs: plain and learned closure ----
    steps_c = a.fine_steps // 2
    # coarse_no_model: no eddy viscosity at all (Cs = 0, the molecular tau with the
    # reference's clamp): how much of the coarse Cd error any viscosity model can act on
    for name, params, cs in (("coarse_smagorinsky", None, None), ("coarse_mlp", p, None),
                             ("coarse_no_model", None, 0.0)):
        e = _engine(coarse_case, cs=cs)
        if params is not None:
            e.set_sgs_mlp(params)
        cd, ms = _run(e, steps_c, 100)
        m = e.mass_stats()
        se = block_se(cd)
        res[name] = {"cd_mean": float(cd.mean()), "cd_std": float(cd.std()), "cd_se": se, "device_ms": ms,
                     "cd_err_vs_fine": float(abs(cd.mean() - res["fine_cd_mean"]) / abs(res["fine_cd_mean"])),
                     # standard error of the relative difference (both means' block errors)
                     "cd_err_se": float(np.hypot(se, res["fine_cd_se"]) / abs(res["fine_cd_mean"])),
                     "speedup_vs_fine": ms_f / ms, "nan": bool(m["hasNaN"])}
        e.close()
    res["wall_s"] = time.perf_counter() - t0
    if a.weights:
        os.makedirs(os.path.dirname(os.path.abspath(a.weights)), exist_ok=True)
        np.savez(a.weights, params=p, nu0=nu0, meta=json.dumps({k: res[k] for k in ("fine", "coarse", "fine_steps")}))
    if a.out:
        with open(a.out, "w") as f:
            json.dump(res, f, indent=1)
    print(json.dumps(res), flush=True)
    return res


if __name__ == "__main__":
    main()
