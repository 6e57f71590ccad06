"""Train the learned closure for one basin recipe and write its weights.

    python -m sailfish_b200.train_closure --config basin4 --out sailfish_b200/weights/closure_basin4.npz

Training data (--source columns, closure.generate) are plain-GLS runs on a sub-basin of the
recipe (same N, dx, dt, depth profile): peak wind stress from U[0, 0.3] N/m2 in a random direction, varying
across the basin as the basins' wind does (cos(pi y / Ly)), the stratification scale varying
across the basin over [200, 1000] m, wind-driven currents in half of the runs and an ocean at
rest under the wind in the other half.  Training is on the GPU with the library's own tensor-core kernels.  A
held-out set of runs with other seeds gives the stated error: log10 RMS of Akv/Akt against
plain GLS, next to the reference's constant AKv = 1e-3 m2/s (modules/mod_ocean.py:91).
With --source roms (closure.generate_roms) the snapshots come from ROMS-form model runs from
rest with plain GLS instead: the flow and the turbulence evolve together as in a simulation;
--source both trains on the two sets together.
"""
import argparse
import json
import os

import torch

from . import closure, configs

RECIPES = {
    # sub-basins of the recipes: same N, dx, dt and depth recipe
    "basin4": lambda: configs.basin(256, 128, 50, 1.0e3, [(1.0 / 3.0, 0.6), (2.0 / 3.0, 0.6)],
                                    dt=120.0, ndtfast=40),
    "basin1": lambda: configs.basin(256, 128, 32, 2.0e3, [(0.5, 0.6)], dt=240.0, ndtfast=30),
    # config 1's own basin (512 x 256 x 32): 131,072 columns per snapshot
    "basin1-full": configs.basin1,
}


def train(config, out, runs=16, rest_runs=8, spin=300, every=25, keep=4, steps=6000, batch=4096,
          lr=1e-3, seed=1, act="relu", gls_model="k-epsilon", source="columns", hours=48.0,
          spin_hours=4.0):
    """source "columns": GLS is spun up `spin` steps at fixed forcing and analytic currents
    (10 h at dt = 120 s: the turbulence fields settle to their forced state), then `keep`
    snapshots `every` steps apart are kept (closure.generate).  source "roms": snapshots every
    `every` steps along `runs` ROMS-form model runs of `hours` from rest with plain GLS, after
    `spin_hours` (closure.generate_roms)."""
    cfg = RECIPES[config]()
    N = cfg["grid"].N
    if source in ("roms", "both"):
        X, T = closure.generate_roms(cfg, runs=runs, hours=hours, spin_hours=spin_hours,
                                     every=every, seed=seed, gls_model=gls_model)
        Xv, Tv = closure.generate_roms(cfg, runs=max(1, runs // 8), hours=hours,
                                       spin_hours=spin_hours, every=4 * every, seed=seed + 1000,
                                       gls_model=gls_model)
        if source == "both":   # and the forced columns at fixed flow, including an ocean at rest
            X2, T2 = closure.generate(cfg, runs=runs, spin=spin, keep=keep, every=25,
                                      seed=seed + 500, rest_runs=rest_runs, pattern=True,
                                      spread=True, gls_model=gls_model)
            X, T = torch.cat([X, X2]), torch.cat([T, T2])
            del X2, T2
        spin = int(round(spin_hours * 3600.0 / cfg["dt"]))
    else:
        X, T = closure.generate(cfg, runs=runs, spin=spin, keep=keep, every=every, seed=seed,
                                rest_runs=rest_runs, pattern=True, spread=True,
                                gls_model=gls_model)
        Xv, Tv = closure.generate(cfg, runs=4, spin=spin, keep=2, every=every, seed=seed + 1000,
                                  rest_runs=2, pattern=True, spread=True, gls_model=gls_model)
    net = closure.Network(N, seed=seed, act=act, gls_model=gls_model)
    net.fit_normalisation(X)
    hist = net.train(X, T, steps=steps, batch=batch, lr=lr, seed=seed, log_every=500)
    e = closure.log_rms(net.infer(Xv), Tv, N)
    const = torch.zeros_like(Tv)
    const[:, :N - 1] = -3.0
    const[:, N - 1:2 * (N - 1)] = -6.0
    ec = closure.log_rms(const, Tv, N)
    report = {"config": config, "source": source, "N": N, "act": act, "gls_model": gls_model,
              "rows": int(X.shape[0]),
              "heldout_rows": int(Xv.shape[0]),
              "gls_spinup": spin, "steps": steps, "batch": batch, "loss": hist,
              "heldout_log10_rms_akv": e[0], "heldout_log10_rms_akt": e[1],
              "constant_log10_rms_akv": ec[0], "constant_log10_rms_akt": ec[1]}
    os.makedirs(os.path.dirname(os.path.abspath(out)), exist_ok=True)
    net.save(out, heldout_log10_rms=list(e), constant_log10_rms=list(ec), seed=seed)
    return report


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", default="basin4", choices=sorted(RECIPES))
    ap.add_argument("--out", required=True)
    ap.add_argument("--steps", type=int, default=6000)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--act", default="relu", choices=["relu", "gelu"])
    ap.add_argument("--gls-model", default="k-epsilon", choices=sorted(closure.GLS_PRESETS))
    ap.add_argument("--runs", type=int, default=16)
    ap.add_argument("--rest-runs", type=int, default=8)
    ap.add_argument("--keep", type=int, default=4)
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--source", default="columns", choices=["columns", "roms", "both"])
    ap.add_argument("--every", type=int, default=None)
    ap.add_argument("--hours", type=float, default=48.0)
    ap.add_argument("--spin-hours", type=float, default=4.0)
    a = ap.parse_args()
    every = a.every if a.every is not None else (25 if a.source == "columns" else 10)
    print(json.dumps(train(a.config, a.out, runs=a.runs, rest_runs=a.rest_runs, keep=a.keep,
                           every=every, steps=a.steps, batch=a.batch, seed=a.seed, act=a.act,
                           gls_model=a.gls_model, source=a.source, hours=a.hours,
                           spin_hours=a.spin_hours)))


if __name__ == "__main__":
    main()
