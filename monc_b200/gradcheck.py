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
    a = ap.parse_args(argv)
    cfg, zn, dz, base = setup(a)
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
