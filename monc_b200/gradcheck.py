"""Gradient check and adjoint timing on the dry convective boundary layer.

    python -m monc_b200.gradcheck --nx 128 --ny 128 --nz 96 --dx 50 --dz 20 --dt 1 \\
        --steps 300 --interval 25 --directions 64 --eps 1e-6

Objective: the horizontally averaged resolved TKE integrated over 0-1 km at the final step.  The
gradient with respect to the seeded initial theta noise (lowest 10 levels) and to Cs comes from
torch.autograd through monc_b200.autodiff.MoncWindow (the library's adjoint).  It is checked
against central finite differences along random directions in the theta-noise space, and against
the tangent-linear model along the same directions.  The forward window and its adjoint are timed
with CUDA events on the model's stream; one JSON line reports the agreement and the
adjoint/forward time ratio.

    python -m monc_b200.gradcheck ... --directions 8 --sweep 1e-4 1e-5 1e-6 1e-7 1e-8 1e-9

runs the finite differences at each eps instead, the two runs of each difference stepped side by
side: for every step it counts the branch decisions (TVD limiter and upwind choices of theta, the
Smagorinsky regime) in which the two runs differ (mgpu_branch_flips).  A difference whose runs
differ in no decision measures a smooth function and must converge to the adjoint as eps shrinks,
until the rounding of J dominates; one that straddles kinks measures a secant.  The derivative
with respect to rmlmax (= Cs dx) is checked the same way with relative steps.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np
import torch

from . import api, autodiff, config as cf, init as ini


def setup(a):
    cfg = cf.dry_cbl_config(a.nx, a.ny, a.nz, a.dx, a.dz, a.dt, ug=a.ug, fcoriol=a.fcoriol)
    cfg.reproducible = 1
    zn = api.reference_profile(cfg, "zn")
    dz = api.reference_profile(cfg, "dz")
    base = ini.dry_cbl_state(a.nx, a.ny, a.nz, zn, seed=a.seed, noise_levels=10, ug=a.ug)
    base = {k: base[k] for k in api.STATE_FIELDS}
    return cfg, zn, dz, base


def objective_np(state, zn, dz, ztop):
    u, v, w = (torch.from_numpy(state[f]) for f in ("u", "v", "w"))
    mask = torch.from_numpy(((zn <= ztop) & (np.arange(len(zn)) >= 1)).astype(np.float64))
    return float(autodiff.resolved_tke(u, v, w, torch.from_numpy(dz), mask))


def timed_window(cfg, state, nsteps, adjoint_seed=None, interval=25, warm=True):
    """Forward window (and optionally its adjoint) timed with CUDA events on the model's stream.

    With warm, each is timed on its second run from the same state: the first, untimed, allocates
    the model's work buffers (for the adjoint, its checkpoints and the segment being reversed)."""
    m = api.Model(cfg)
    stream = torch.cuda.ExternalStream(m.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(2 if warm else 1):
        m.set_state(state)
        m.set_timestep(1)
        torch.cuda.synchronize()
        e0.record(stream)
        m.step(nsteps)
        e1.record(stream)
        e1.synchronize()
    fwd_ms = e0.elapsed_time(e1)
    adj_ms = None
    if adjoint_seed is not None:
        m2 = api.Model(cfg)
        s2 = torch.cuda.ExternalStream(m2.stream)
        for _ in range(2 if warm else 1):
            m2.set_state(state)
            m2.set_timestep(1)
            for f in api.STATE_FIELDS:
                m2.upload("adj:" + f, adjoint_seed[f])
            torch.cuda.synchronize()
            e0.record(s2)
            m2.adjoint_run(nsteps, interval)
            e1.record(s2)
            e1.synchronize()
        adj_ms = e0.elapsed_time(e1)
        m2.close()
    final = {f: m.download(f) for f in api.STATE_FIELDS}
    m.close()
    return final, fwd_ms, adj_ms


def state_objective(m, zn, dz, ztop):
    return objective_np({f: m.download(f) for f in ("u", "v", "w")}, zn, dz, ztop)


def central_difference(plus, minus, nsteps, zn, dz, ztop):
    """(J(plus) - J(minus)) / 2 after nsteps steps of two models, each given as (config, state),
    stepped side by side, and the branch decisions in which their steps differed, summed over the
    steps."""
    mp, mm = api.Model(plus[0]), api.Model(minus[0])
    mp.set_state(plus[1])
    mm.set_state(minus[1])
    mp.set_timestep(1)
    mm.set_timestep(1)
    flips = 0
    for _ in range(nsteps):
        flips += mp.branch_flips(mm)
        mp.step(1)
        mm.step(1)
    half = 0.5 * (state_objective(mp, zn, dz, ztop) - state_objective(mm, zn, dz, ztop))
    mp.close()
    mm.close()
    return half, flips


def sweep(a, cfg, zn, dz, base):
    """Finite differences against the adjoint over a range of eps on one set of directions, with
    the branch decisions each pair of runs straddles; and the Cs derivative the same way."""
    dev = torch.device("cuda")
    mask = torch.from_numpy(((zn <= a.ztop) & (np.arange(a.nz) >= 1)).astype(np.float64)).to(dev)
    window = autodiff.Window(cfg, base, a.steps, a.interval)
    th0 = torch.from_numpy(base["th"]).to(dev).requires_grad_(True)
    rml = torch.tensor(cfg.rmlmax, dtype=torch.float64, device=dev, requires_grad=True)
    u, v, w, _ = autodiff.MoncWindow.apply(th0, rml, window)
    J = autodiff.resolved_tke(u, v, w, torch.from_numpy(dz).to(dev), mask)
    J.backward()
    g_th = th0.grad.cpu().numpy()
    g_rml = float(rml.grad)
    rng = np.random.default_rng(a.seed)
    dirs = []
    for _ in range(a.directions):
        dth = np.zeros_like(base["th"])
        dth[1:11] = rng.uniform(-1.0, 1.0, size=dth[1:11].shape)
        dirs.append(dth)
    table = []
    for eps in a.eps_list:
        rows = []
        for dth in dirs:
            sp, sm = dict(base), dict(base)
            sp["th"] = base["th"] + eps * dth
            sm["th"] = base["th"] - eps * dth
            half, flips = central_difference((cfg, sp), (cfg, sm), a.steps, zn, dz, a.ztop)
            fd = half / eps
            ad = float(np.vdot(g_th, dth))
            rows.append((abs(ad - fd) / max(abs(fd), 1e-300), flips))
        err = np.array([r[0] for r in rows])
        fl = np.array([r[1] for r in rows])
        smooth = err[fl == 0]
        table.append({"eps": eps, "median_rel_err": float(np.median(err)), "max_rel_err": float(err.max()),
                      "directions_with_flips": int((fl > 0).sum()), "median_flips": float(np.median(fl)),
                      "max_rel_err_without_flips": float(smooth.max()) if smooth.size else None,
                      "per_direction": [{"rel_err": float(e), "flips": int(f)} for e, f in rows]})
    cs_rows = []
    for eps in a.eps_list:
        cp, cm = setup(a)[0], setup(a)[0]
        cp.rmlmax = cfg.rmlmax * (1.0 + eps)
        cm.rmlmax = cfg.rmlmax * (1.0 - eps)
        half, flips = central_difference((cp, base), (cm, base), a.steps, zn, dz, a.ztop)
        fd = half / (eps * cfg.rmlmax)
        cs_rows.append({"eps_relative": eps, "fd_dJ_drmlmax": fd, "flips": flips,
                        "rel_err": abs(g_rml - fd) / max(abs(fd), 1e-300)})
    return {"grid": [a.nx, a.ny, a.nz], "steps": a.steps, "J": float(J.detach()), "directions": a.directions,
            "adjoint_dJ_drmlmax": g_rml, "adjoint_dJ_dCs": g_rml * cfg.dxx, "theta": table, "cs": cs_rows}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--nx", type=int, default=128)
    ap.add_argument("--ny", type=int, default=128)
    ap.add_argument("--nz", type=int, default=96)
    ap.add_argument("--dx", type=float, default=50.0)
    ap.add_argument("--dz", type=float, default=20.0)
    ap.add_argument("--dt", type=float, default=1.0)
    ap.add_argument("--ug", type=float, default=0.0)
    ap.add_argument("--fcoriol", type=float, default=0.0)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--interval", type=int, default=25)
    ap.add_argument("--directions", type=int, default=64)
    ap.add_argument("--eps", type=float, default=1e-6)
    ap.add_argument("--ztop", type=float, default=1000.0)
    ap.add_argument("--sweep", type=float, nargs="*", dest="eps_list",
                    help="finite differences at each of these eps on --directions directions, with the branch "
                         "decisions each pair of runs straddles, and the Cs derivative (one JSON line)")
    a = ap.parse_args(argv)
    cfg, zn, dz, base = setup(a)
    if a.eps_list:
        print(json.dumps(sweep(a, cfg, zn, dz, base)))
        return
    dev = torch.device("cuda")
    mask = torch.from_numpy(((zn <= a.ztop) & (np.arange(a.nz) >= 1)).astype(np.float64)).to(dev)
    dzt = torch.from_numpy(dz).to(dev)
    window = autodiff.Window(cfg, base, a.steps, a.interval)
    th0 = torch.from_numpy(base["th"]).to(dev).requires_grad_(True)
    rml = torch.tensor(cfg.rmlmax, dtype=torch.float64, device=dev, requires_grad=True)
    t0 = time.perf_counter()
    u, v, w, th = autodiff.MoncWindow.apply(th0, rml, window)
    J = autodiff.resolved_tke(u, v, w, dzt, mask)
    J.backward()
    wall = time.perf_counter() - t0
    g_th = th0.grad.cpu().numpy()
    g_cs = float(rml.grad) * cfg.dxx  # rmlmax = Cs * dx
    # finite differences and tangent-linear derivatives along random theta-noise directions
    rng = np.random.default_rng(a.seed)
    rows = []
    for d in range(a.directions):
        dth = np.zeros_like(base["th"])
        dth[1:11] = rng.uniform(-1.0, 1.0, size=dth[1:11].shape)
        ad = float(np.vdot(g_th, dth))
        Js = []
        for sgn in (1.0, -1.0):
            st = dict(base)
            st["th"] = base["th"] + sgn * a.eps * dth
            fin, _, _ = timed_window(cfg, st, a.steps, warm=False)
            Js.append(objective_np(fin, zn, dz, a.ztop))
        fd = (Js[0] - Js[1]) / (2 * a.eps)
        # tangent-linear along the same direction: dJ = <dJ/dstate_final, tangent_final>
        m = api.Model(cfg)
        m.set_state(base)
        for f in api.STATE_FIELDS:
            m.upload("tl:" + f, dth if f == "th" else np.zeros_like(dth))
        m.tl_step(a.steps)
        fin = {f: m.download(f) for f in ("u", "v", "w")}
        tan = {f: m.download("tl:" + f) for f in ("u", "v", "w")}
        m.close()
        tl = 0.0
        lev = (zn <= a.ztop) & (np.arange(a.nz) >= 1)
        for f in ("u", "v", "w"):
            pert = fin[f] - fin[f].mean(axis=(1, 2), keepdims=True)
            tl += float(np.sum(pert * tan[f] / (a.nx * a.ny) * (dz * lev)[:, None, None]))
        rows.append((ad, fd, tl))
    rows = np.array(rows)
    rel_fd = np.abs(rows[:, 0] - rows[:, 1]) / np.maximum(np.abs(rows[:, 1]), 1e-300)
    rel_tl = np.abs(rows[:, 0] - rows[:, 2]) / np.maximum(np.abs(rows[:, 2]), 1e-300)
    # timing: forward window and its adjoint (objective seeds)
    seed = {f: np.zeros_like(base["th"]) for f in api.STATE_FIELDS}
    fin, _, _ = timed_window(cfg, base, a.steps)
    lev = (zn <= a.ztop) & (np.arange(a.nz) >= 1)
    for f in ("u", "v", "w"):
        pert = fin[f] - fin[f].mean(axis=(1, 2), keepdims=True)
        seed[f] = pert / (a.nx * a.ny) * (dz * lev)[:, None, None]
    _, fwd_ms, adj_ms = timed_window(cfg, base, a.steps, seed, a.interval)
    print(json.dumps({
        "grid": [a.nx, a.ny, a.nz], "steps": a.steps, "checkpoint_interval": a.interval, "J": float(J.detach()),
        "dJ_dCs": g_cs, "directions": a.directions, "eps": a.eps,
        "adjoint_vs_fd_rel_err": {"median": float(np.median(rel_fd)), "max": float(rel_fd.max())},
        "adjoint_vs_tl_rel_err": {"median": float(np.median(rel_tl)), "max": float(rel_tl.max())},
        "forward_ms": round(fwd_ms, 3), "adjoint_ms": round(adj_ms, 3),
        "adjoint_forward_ratio": round(adj_ms / fwd_ms, 3), "autograd_wall_s": round(wall, 3)}))


if __name__ == "__main__":
    main()
