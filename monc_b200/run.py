"""Run the GPU dynamical core on a dry convective-boundary-layer case from the command line.

    python -m monc_b200.run --nx 256 --ny 256 --nz 128 --dx 25 --dz 15 --dt 0.5 --ug 5 \\
        --fcoriol 1e-4 --noise-levels 10 --steps 500 --precision fp64

The case is MONC's dry CBL set-up (theta' = 0 up to 800 m, +0.003 K/m above, seeded uniform
theta noise near the surface, surface sensible heat flux 0.1 K m/s, Cs = 0.23, FFT solver).
The first step is MONC's forward step, the rest are centred.  One JSON line is printed: the
wall time, the number of kernel launches and the final domain-mean theta and w'^2 profiles
(a few levels).
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import api, config as cf, init as ini


def build_case(a) -> tuple:
    prec = cf.FP32_MIXED if a.precision == "fp32_mixed" else cf.FP64
    solver = cf.SOLVER_ITERATIVE if a.solver == "iterative" else cf.SOLVER_FFT
    cfg = cf.dry_cbl_config(a.nx, a.ny, a.nz, a.dx, a.dz, a.dt, ug=a.ug, fcoriol=a.fcoriol, precision=prec,
                            solver=solver)
    cfg.reproducible = int(a.reproducible)
    zn = api.reference_profile(cfg, "zn")
    state = ini.dry_cbl_state(a.nx, a.ny, a.nz, zn, seed=a.seed, noise_levels=a.noise_levels, ug=a.ug)
    return cfg, state


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--nx", type=int, default=64)
    ap.add_argument("--ny", type=int, default=64)
    ap.add_argument("--nz", type=int, default=65)
    ap.add_argument("--dx", type=float, default=50.0)
    ap.add_argument("--dz", type=float, default=25.0)
    ap.add_argument("--dt", type=float, default=1.0)
    ap.add_argument("--ug", type=float, default=0.0)
    ap.add_argument("--fcoriol", type=float, default=0.0)
    ap.add_argument("--noise-levels", type=int, default=8)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--precision", choices=["fp64", "fp32_mixed"], default="fp64")
    ap.add_argument("--solver", choices=["fft", "iterative"], default="fft")
    ap.add_argument("--reproducible", action="store_true", help="unfused multiply-adds (MONC's rounding)")
    a = ap.parse_args(argv)
    cfg, state = build_case(a)
    with api.Model(cfg) as m:
        m.set_state(state)
        t0 = time.perf_counter()
        m.step(a.steps)
        th, w2 = m.diagnostics()
        wall = time.perf_counter() - t0
        launches = m.launches
    pick = sorted({1, a.nz // 4, a.nz // 2, a.nz - 2})
    print(json.dumps({"steps": a.steps, "grid": [a.nx, a.ny, a.nz], "precision": a.precision, "wall_s": round(wall, 4),
                      "launches": launches, "finite": bool(np.isfinite(th).all() and np.isfinite(w2).all()),
                      "mean_theta": {int(k): float(th[k]) for k in pick},
                      "mean_w2": {int(k): float(w2[k]) for k in pick}}))


if __name__ == "__main__":
    main()
