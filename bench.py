#!/usr/bin/env python
"""Headline benchmark: MONC dynamical-core timestep throughput (Mpoint-steps/s) on B200.

Workload (the GPU configuration of the reference's benchmark set): dry convective boundary
layer, 256 x 256 x 128 points, dx = dy = 25 m, dz = 15 m, geostrophic wind 5 m/s with
f = 1e-4 s^-1, seeded +-0.1 K theta noise on the lowest 10 levels, dt = 0.5 s, FFT pressure
solver.  `value` is the FP64 path (fields double precision throughout); the FP32-mixed path on
the same grid is reported beside it.  A "step" is one full MONC timestep; the first (forward)
step is part of the warm-up, timed steps are centred leapfrog steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 (one process per GPU under torchrun) decomposes a 256 x (256*N) x 128 domain into N
y-slabs of the single-GPU grid (weak scaling): each step exchanges 4 halo rows of the state and
1 of the pressure with the neighbouring slabs and transposes the pressure spectrum with two
all-to-alls, all over NCCL (monc_b200/decomposition.py).  The initial state is the single-GPU
one repeated in y.  Every rank's steps are timed on its model's stream with CUDA events between
barriers and the slowest rank is reported.  --replicas runs N independent single-GPU models
instead.
`--impl reference` times the CPU restatement of MONC's Fortran (oracle/), the only runnable
form of the reference here (no Fortran compiler on this machine or the GPU machine).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NX, NY, NZ = 256, 256, 128
DX, DZ, DT, UG, FCOR = 25.0, 15.0, 0.5, 5.0, 1e-4
WORKLOAD = "dry CBL 256x256x128, dx=dy=25 m, dz=15 m, u_g=5 m/s, f=1e-4, dt=0.5 s, FFT solver"
METRIC = "Mpoint-steps/s (MONC dynamical-core timestep, 1 B200)"
# array passes (full 3-D arrays read + written, each counted once per kernel) per point and step, by
# kernel, for the dry centred step.  The horizontal transforms are counted as what they must move:
# the field in and the half spectrum out (forward), and back (inverse), whether one fused kernel per
# level or an x and a y kernel does it.
# When the forward x transform forms the pressure source itself ("source_fft_fwd"), it reads zu,
# zv, zw and writes the half spectrum.
KERNEL_PASSES = {"subgrid": 6, "dynamics_scalars": 8, "dynamics_momentum": 11, "pressure_source": 4,
                 "fft_fwd": 2, "source_fft_fwd": 4, "tridiag": 2, "fft_inv": 2, "pstep_swap": 16}


def kernel_times(stages: dict) -> dict:
    """Per-kernel ms from the library's stage times (the dynamics stage holds two kernels; the x and
    y transform stages of a direction are one fused kernel on grids that allow it)."""
    out = {k: v for k, v in stages.items() if k in KERNEL_PASSES}
    if "dynamics" in stages and "dynamics_momentum" in stages:
        out["dynamics_scalars"] = stages["dynamics"] - stages["dynamics_momentum"]
        out["dynamics_momentum"] = stages["dynamics_momentum"]
    if "fft_x_fwd" in stages:
        out["fft_fwd"] = stages["fft_x_fwd"] + stages.get("fft_y_fwd", 0.0)
    if "fft_x_inv" in stages:
        out["fft_inv"] = stages["fft_x_inv"] + stages.get("fft_y_inv", 0.0)
    if "fft_fwd" in out and stages.get("pressure_source", 1.0) < 0.01:
        # no source kernel (the stage's events enclose nothing): the forward transform formed it
        out["source_fft_fwd"] = out.pop("fft_fwd") + out.pop("pressure_source", 0.0)
    return out


def make_config(precision):
    from monc_b200 import config as cf

    return cf.dry_cbl_config(NX, NY, NZ, DX, DZ, DT, ug=UG, fcoriol=FCOR, precision=precision)


def initial_state(cfg):
    from monc_b200 import api, init as ini

    zn = api.reference_profile(cfg, "zn")
    return ini.dry_cbl_state(NX, NY, NZ, zn, seed=20261203, noise_levels=10, ug=UG)


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int, rank: int):
        import torch

        # nvidia-smi numbers GPUs independently of CUDA_VISIBLE_DEVICES: address the device by UUID
        try:
            self.gpu = "GPU-" + str(torch.cuda.get_device_properties(device).uuid)
        except Exception:
            self.gpu = str(device)
        self.proc = None
        # the raw samples; BENCH_OUT_DIR names a folder to keep them in
        out_dir = os.environ.get("BENCH_OUT_DIR") or os.path.join(ROOT, "_bench_out")
        self.path = os.path.join(out_dir, f"clocks_rank{rank}.csv")

    def start(self, wait_s: float = 10.0):
        """Start sampling every 100 ms and return once the first sample has been written."""
        os.makedirs(os.path.dirname(self.path), exist_ok=True)
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", self.gpu, f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return
        t0 = time.time()
        while time.time() - t0 < wait_s and self.proc.poll() is None:
            if os.path.getsize(self.path) > 0:
                break
            time.sleep(0.05)

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax = float(parts[2])
                except ValueError:
                    continue
                for nm, val in zip(names, parts[5:9]):
                    if val.lower() == "active":
                        reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def slab_state(cfg, geo, rank):
    """Rows of a slab (halo rows included) of the single-GPU initial state repeated in y."""
    st = initial_state(cfg)
    rows = geo.rows(rank) % NY
    return {k: np.ascontiguousarray(v[:, rows, :]) for k, v in st.items()}


def decomposed_domain(prec, world, rank, pinned_torch=None):
    """The 256 x (256*world) x 128 domain split into one y-slab per rank over NCCL."""
    from monc_b200 import decomposition as dc

    cfg = make_config(prec)
    cfg.ny = NY * world
    d = dc.SlabDomain(cfg, dc.TorchComm(), halo=4)
    st = slab_state(make_config(prec), d.geo, rank)
    if pinned_torch is not None:
        pinned = {}
        for k, v in st.items():
            t = pinned_torch.empty(v.shape, dtype=pinned_torch.float64, pin_memory=True)
            t.numpy()[...] = v
            pinned[k] = t.numpy()
        st = pinned
    for k, v in st.items():
        d.upload_local(k, [v])
    return d, st


def time_steps(model, steps, torch):
    stream = torch.cuda.ExternalStream(model.stream)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    model.step(steps)
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1)


def run_ours(args):
    import torch
    import torch.distributed as dist

    from monc_b200 import api, config as cf

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if not torch.cuda.is_available():
        raise SystemExit("bench.py: no CUDA device")
    torch.cuda.set_device(local)
    decomposed = (world > 1 and not args.replicas) or args.decomposed
    if world > 1 or decomposed:
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        os.environ.setdefault("MASTER_PORT", "29533")
        dist.init_process_group("nccl", rank=rank, world_size=world,
                                timeout=__import__("datetime").timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    npts = NX * NY * NZ

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    results = {}
    for prec_name, prec in (("fp64", cf.FP64), ("fp32_mixed", cf.FP32_MIXED)):
        cfg = make_config(prec)
        model = api.Model(cfg)
        model.set_state(initial_state(cfg))
        model.step(args.warmup)  # step 1 (forward) and the first centred steps
        # per-stage device times, outside the timed region
        model.set_profiling(True)
        model.step(3)
        stages = {k: v[0] / max(v[1], 1) for k, v in model.stage_times().items() if v[1] > 0}
        model.set_profiling(False)
        if decomposed:
            # the timed run is the decomposed domain; the single-domain model only gave the stages
            model.close()
            model, _ = decomposed_domain(prec, world, rank)
            model.step(args.warmup)
        clocks = ClockSampler(local, rank)
        barrier()
        if prec_name == "fp64":
            clocks.start()
        if decomposed:
            s0 = model.slabs[0].m
            l0 = s0.launches
            stream = torch.cuda.ExternalStream(s0.stream)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            model.step(args.steps)
            e1.record(stream)
            e1.synchronize()
            ms = e0.elapsed_time(e1)
            launches = s0.launches - l0
        else:
            l0 = model.launches
            ms = time_steps(model, args.steps, torch)
            launches = model.launches - l0
        barrier()
        ck = clocks.stop() if prec_name == "fp64" else None
        ms = max_over_ranks(ms)
        per_step = ms / args.steps
        th, w2 = (model.slabs[0].m if decomposed else model).diagnostics()
        finite = bool(np.isfinite(th).all() and np.isfinite(w2).all())
        results[prec_name] = {"ms_per_step": per_step, "value": world * npts / (per_step * 1e-3) / 1e6,
                              "stages": stages, "launches": launches, "clocks": ck, "finite": finite}
        model.close()

    # end to end through the C ABI: host-resident initial state (pinned) uploaded inside the timed
    # region, K steps, each followed by a device->host read of the mean theta and w'^2 profiles
    cfg = make_config(cf.FP64)
    if decomposed:
        model, pinned = decomposed_domain(cf.FP64, world, rank, pinned_torch=torch)
        upload = lambda st: [model.upload_local(k, [v]) for k, v in st.items()]  # noqa: E731
        local_model = model.slabs[0].m
    else:
        state = initial_state(cfg)
        pinned = {}
        for k, v in state.items():
            t = torch.empty(v.shape, dtype=torch.float64, pin_memory=True)
            t.numpy()[...] = v
            pinned[k] = t.numpy()
        model = api.Model(cfg)
        model.set_state(pinned)
        upload = model.set_state
        local_model = model
    model.step(args.warmup)
    th = np.empty(NZ)
    w2 = np.empty(NZ)
    barrier()
    t0 = time.perf_counter()
    upload(pinned)
    for _ in range(args.steps):
        model.step(1)
        local_model.diagnostics(th, w2)
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    model.close()
    h2d = sum(v.nbytes for v in pinned.values()) / args.steps
    e2e = {"value": world * npts * args.steps / e2e_s / 1e6, "unit": "Mpoint-steps/s",
           "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": 2 * NZ * 8,
           "note": "initial state (8 FP64 fields, pinned host; each rank its slab) uploaded in the timed "
                   "region and amortised over the steps; per-step read-back of the mean theta and w'^2 "
                   "profiles"}

    # the metric's second part: adjoint/forward time ratio on the differentiation window (dry CBL
    # 128x128x96, 300 steps, checkpoint every 25), and FP32-mixed vs FP64 on the moist layer;
    # single-GPU runs only (every rank would repeat the same work)
    extra = {}
    if world == 1 and not args.skip_extra:
        extra["adjoint"] = adjoint_ratio()
        extra["tvd_flow_fields"] = tvd_flow_fields()
        extra["precision_moist"] = precision_moist()
        if args.large:
            extra["large_fp32_mixed"] = large_fp32_mixed()

    if dist.is_initialized():
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return

    r64 = results["fp64"]
    peak, peak_kind = measured_peaks()
    kt = kernel_times(r64["stages"])
    step_passes = sum(KERNEL_PASSES[k] for k in kt)
    dom = max(kt, key=lambda k: kt[k])
    dom_ms = kt[dom]
    dom_bytes = KERNEL_PASSES[dom] * 8 * npts
    achieved = dom_bytes / (dom_ms * 1e-3) / 1e9
    per_kernel = {k: {"ms": round(v, 4), "GB/s": round(KERNEL_PASSES[k] * 8 * npts / (v * 1e-3) / 1e9, 1),
                      "frac": round(KERNEL_PASSES[k] * 8 * npts / (v * 1e-3) / 1e9 / peak, 4)}
                  for k, v in kt.items() if v > 0}
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tfile):
        try:
            traffic = json.load(open(tfile)).get("fp64", {}).get(dom)
        except Exception:
            traffic = None
    cpu = cpu_baseline(args)
    out = {
        "metric": METRIC,
        "value": round(r64["value"], 2),
        "unit": "Mpoint-steps/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(r64["ms_per_step"], 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded initial state; no dataset involved)",
        "config": {"workload": WORKLOAD if not decomposed else
                   f"dry CBL {NX}x{NY * world}x{NZ} in {world} y-slabs of {NX}x{NY}x{NZ} (halo 4 rows, "
                   "NCCL halo exchange + all-to-all FFT transposes), dx=dy=25 m, dz=15 m, u_g=5 m/s, f=1e-4, "
                   "dt=0.5 s, FFT solver",
                   "nx": NX, "ny": NY * world if decomposed else NY, "nz": NZ, "precision": "fp64",
                   "solver": "fft",
                   "parallelism": f"y-slabs x{world}" if decomposed else ("replicas" if world > 1 else "single"),
                   "l2": "working set (~1.1 GB of fields per GPU) larger than the 126 MB L2; no flush needed"},
        "fp32_mixed": {"value": round(results["fp32_mixed"]["value"], 2),
                       "ms_per_step": round(results["fp32_mixed"]["ms_per_step"], 4),
                       "stages_ms": {k: round(v, 4) for k, v in results["fp32_mixed"]["stages"].items()},
                       "speedup_vs_fp64": round(r64["ms_per_step"] / results["fp32_mixed"]["ms_per_step"], 3)},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
                     "traffic": traffic,
                     "algorithmic_bytes_per_launch": dom_bytes},
        "step_roofline": {"algorithmic_bytes_per_point": step_passes * 8,
                          "frac": round(step_passes * 8 * npts / (r64["ms_per_step"] * 1e-3) / 1e9 / peak, 4)},
        "kernels": per_kernel,
        "stages_ms": {k: round(v, 4) for k, v in r64["stages"].items()},
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": r64["launches"],
        "clocks": r64["clocks"],
        "finite": r64["finite"],
    }
    out.update(extra)
    print(json.dumps(out), flush=True)


def tvd_flow_fields():
    """The benchmarked grid with MONC's TVD advection of u, v, w (advection_flow_fields = tvd)
    instead of Piacsek-Williams, FP64: device time per step (CUDA events on the model's stream)."""
    import torch

    from monc_b200 import api, config as cf

    out = {"case": WORKLOAD + ", TVD flow advection"}
    for name, adv in (("pw", cf.ADVECT_PW), ("tvd", cf.ADVECT_TVD)):
        c = make_config(cf.FP64)
        c.advection_flow_fields = adv
        m = api.Model(c)
        m.set_state(initial_state(c))
        m.step(5)
        ms = time_steps(m, 20, torch) / 20
        m.close()
        out[f"{name}_ms_per_step"] = round(ms, 4)
        out[f"{name}_mpoint_steps_per_s"] = round(NX * NY * NZ / (ms * 1e-3) / 1e6, 1)
    out["tvd_over_pw_time"] = round(out["tvd_ms_per_step"] / out["pw_ms_per_step"], 3)
    return out


def adjoint_ratio():
    """Forward window and its adjoint (objective: resolved TKE below 1 km at the last step), CUDA
    events on the model's stream."""
    import argparse as _ap

    from monc_b200 import api, gradcheck as gc

    a = _ap.Namespace(nx=128, ny=128, nz=96, dx=50.0, dz=20.0, dt=1.0, ug=0.0, fcoriol=0.0, seed=1)
    cfg, zn, dz, base = gc.setup(a)
    steps, interval = 300, 25
    fin, _, _ = gc.timed_window(cfg, base, steps)
    lev = (zn <= 1000.0) & (np.arange(a.nz) >= 1)
    seed = {f: np.zeros_like(base["th"]) for f in api.STATE_FIELDS}
    for f in ("u", "v", "w"):
        pert = fin[f] - fin[f].mean(axis=(1, 2), keepdims=True)
        seed[f] = pert / (a.nx * a.ny) * (dz * lev)[:, None, None]
    _, fwd_ms, adj_ms = gc.timed_window(cfg, base, steps, seed, interval)
    return {"window": "dry CBL 128x128x96, dx=50 m, dz=20 m, dt=1 s, 300 steps, FP64, checkpoint every 25 steps",
            "timing": "second run of each from the same state; the first allocates the work buffers",
            "forward_ms": round(fwd_ms, 3), "adjoint_ms": round(adj_ms, 3),
            "adjoint_forward_ratio": round(adj_ms / fwd_ms, 2)}


def precision_moist():
    """FP32-mixed vs FP64 on the moist stratocumulus-like layer (512x512x160, 500 steps)."""
    import argparse as _ap

    from monc_b200 import config as cf, precision as pr

    a = _ap.Namespace(nx=512, ny=512, nz=160, dx=35.0, dz_bottom=5.0, dz_top=20.0, dt=0.3, steps=500, seed=1,
                      noise_levels=10, solver="fft", tolerance=1e-4)
    f64, f32 = {}, {}
    ms64, th64, w64, qv64, _ = pr.run(a, cf.FP64, fields=f64)
    ms32, th32, w32, qv32, _ = pr.run(a, cf.FP32_MIXED, fields=f32)
    per_field = pr.field_errors(f32, f64)
    del f64, f32
    out = {"case": "moist layer 512x512x160, dx=35 m, dz 5->20 m, dt=0.3 s, simplecloud, 500 steps",
           "fp64_ms_per_step": round(ms64, 4), "fp32_mixed_ms_per_step": round(ms32, 4),
           "speedup": round(ms64 / ms32, 3), "rel_err_mean_theta": pr.rel(th32, th64),
           "rel_err_mean_w2": pr.rel(w32, w64), "rel_err_mean_qv": pr.rel(qv32, qv64),
           "fields_fp32_vs_fp64": per_field}
    # the same layer with the iterative solver over its first ITER_STEPS steps (BiCGStab, FP64
    # refinement around FP32 corrections in the FP32-mixed run): at MONC's default tolerance and at
    # a strict one
    runs = []
    for tol in ITER_TOLERANCES:
        ai = _ap.Namespace(**{**vars(a), "solver": "iterative", "steps": ITER_STEPS, "tolerance": tol})
        g64, g32 = {}, {}
        mi64, ti64, wi64, _, _ = pr.run(ai, cf.FP64, fields=g64)
        it64 = ai.iterations_per_step
        mi32, ti32, wi32, _, _ = pr.run(ai, cf.FP32_MIXED, fields=g32)
        it32 = ai.iterations_per_step
        runs.append({"tolerance": tol, "fp64_ms_per_step": round(mi64, 4), "fp32_mixed_ms_per_step": round(mi32, 4),
                     "speedup": round(mi64 / mi32, 3),
                     "iterations_per_step": {"fp64": round(it64, 2), "fp32_mixed": round(it32, 2)},
                     "rel_err_mean_theta": pr.rel(ti32, ti64), "rel_err_mean_w2": pr.rel(wi32, wi64),
                     "fields_fp32_vs_fp64": pr.field_errors(g32, g64)})
    out["iterative"] = {"steps": ITER_STEPS, "solver": "BiCGStab", "max_iterations": 500, "by_tolerance": runs}
    return out


# steps of the iterative-solver runs on the moist layer, and their tolerances: 1e-4 is MONC's
# default (global_config), 1e-8 a strict one.  Tighter tolerances are below what the FP64 solve
# reaches here (like MONC's it has no compatibility shift; it stalls near a relative residual of
# 5e-8 on this layer and ends most solves at the iteration cap), so a run there times the cap.
ITER_STEPS = 20
ITER_TOLERANCES = (1e-4, 1e-8)


def _large_run(precision, fields=None):
    """One run of the largest configuration in the given precision: ms per step over steps 2..200
    (CUDA events on the model's stream), the mean theta and w'^2 profiles, and (when `fields` is a
    dict) the final u, v, w, theta, vapour and liquid fields."""
    import torch

    from monc_b200 import api, config as cf, init as ini

    nx = ny = 1024
    nz, steps = 200, 200
    z = cf.stretched_levels(nz, 10.0, 50.0, ztop=6000.0)
    c = cf.moist_config(nx, ny, z, 25.0, 0.5, shf_wm2=150.0, lhf_wm2=200.0, max_height_cloud=5000.0, n_tracers=3,
                        precision=precision)
    m = api.Model(c)
    # the state of init.moist_layer_state, built and uploaded one field at a time (each 1.7 GB on
    # the host): theta with +-0.2 K noise on the lowest levels, vapour, no liquid, three tracers
    zn = api.reference_profile(c, "zn")
    shape = (nz, ny, nx)
    th_prof = np.where(zn > 840.0, 297.5 + 0.00365 * (zn - 840.0), 289.0) - 289.0
    f = np.broadcast_to(th_prof[:, None, None], shape).copy()
    f[1:9] += ini.uniform_noise((8, ny, nx), 5, 3, 0.2)
    f[0] = f[1]
    m.upload("th", f)
    m.upload("zth", f)
    f[:] = np.where(zn > 840.0, 1.5e-3, 9e-3)[:, None, None]
    m.upload("q0", f)
    m.upload("zq0", f)
    # a uniform 2 m/s wind: with u = v = 0 the convective surface formula of lowerbc.F90:601-633
    # takes u* from its free-convection limit and cancels to a condition number of ~1e10, which
    # FP32 cannot carry
    f[:] = 2.0
    m.upload("u", f)
    m.upload("zu", f)
    f[:] = 0.0
    for name in ("v", "w", "zv", "zw", "q1", "zq1"):
        m.upload(name, f)
    for t in range(3):
        for k in range(nz):
            f[k] = np.exp(0.5 * ini.uniform_noise((1, ny, nx), 5 + k, 40 + t, 1.0)[0]) * np.exp(-zn[k] / 200.0)
        m.upload(f"q{2 + t}", f)
        m.upload(f"zq{2 + t}", f)
    del f
    m.step(1)
    stream = torch.cuda.ExternalStream(m.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    m.step(steps - 1)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / (steps - 1)
    th, w2 = m.diagnostics()
    if fields is not None:
        for name in ("u", "v", "w", "th", "q0", "q1"):
            fields[name] = m.download(name)
    m.close()
    return ms, th, w2, nx * ny * nz


def large_fp32_mixed():
    """The largest configuration: 1024x1024x200 FP32-mixed, dz 10->50 m to 6 km, vapour, liquid and
    three passive tracers with log-normal surface sources, 150 / 200 W m-2 surface fluxes, +-0.2 K
    noise, dt = 0.5 s, 200 steps; CUDA events on the model's stream over steps 2..200.  The same
    run in FP64 (about 80 GB of fields, inside the 180 GB of one B200) gives the reference for the
    FP32-mixed run's per-field and mean-profile differences."""
    from monc_b200 import config as cf, precision as pr

    f32, f64 = {}, {}
    ms32, th32, w32, npts = _large_run(cf.FP32_MIXED, f32)
    ms64, th64, w64, _ = _large_run(cf.FP64, f64)
    finite = bool(np.isfinite(th32).all() and np.isfinite(w32).all())
    per_field = pr.field_errors(f32, f64)
    del f32, f64
    return {"case": "1024x1024x200 FP32-mixed, dx=25 m, dz 10->50 m to 6 km, u = 2 m/s, vapour + liquid + "
                    "3 tracers, shf 150 / lhf 200 W m-2, dt=0.5 s, 200 steps",
            "ms_per_step": round(ms32, 3), "mpoint_steps_per_s": round(npts / (ms32 * 1e-3) / 1e6, 1),
            "fp64_ms_per_step": round(ms64, 3), "fp64_mpoint_steps_per_s": round(npts / (ms64 * 1e-3) / 1e6, 1),
            "speedup_vs_fp64": round(ms64 / ms32, 3), "finite": finite,
            "rel_err_mean_theta": pr.rel(th32, th64), "rel_err_mean_w2": pr.rel(w32, w64),
            "fields_fp32_vs_fp64": per_field}


def _oracle_run(steps, warmup=1):
    """One oracle instance on the benchmark grid: `warmup` untimed steps (the forward step first),
    then `steps` timed centred steps."""
    sys.path.insert(0, ROOT)
    from monc_b200 import config as cf, init as ini
    from oracle import pyoracle as po

    cfg = make_config(cf.FP64)
    o = po.Oracle(cfg)
    st = ini.dry_cbl_state(NX, NY, NZ, o.profile("zn"), seed=20261203, noise_levels=10, ug=UG)
    for name, fid in (("u", 0), ("v", 1), ("w", 2), ("th", 3), ("zu", 4), ("zv", 5), ("zw", 6), ("zth", 7)):
        o.set(fid, st[name])
    o.step(max(1, warmup))
    t0 = time.perf_counter()
    o.step(steps)
    dt = time.perf_counter() - t0
    o.close()
    return dt


def cpu_baseline(args):
    """The oracle (C++ restatement of MONC's Fortran, single thread, the -O3 -march=native build)
    on a bounded sample of the benchmark workload: the full grid for 2 centred steps after the
    forward step."""
    os.environ["MONC_ORACLE_LIB"] = "native"
    steps = 2
    dt = _oracle_run(steps)
    return {"value": round(NX * NY * NZ * steps / dt / 1e6, 3), "unit": "Mpoint-steps/s", "cores": 1,
            "kind": "port", "sample": f"{NX}x{NY}x{NZ} grid, {steps} centred steps after the forward step, "
                                       f"{dt:.1f} s, single-threaded oracle built -O3 -march=native"}


def run_reference(args):
    """Reference arm: the oracle port, built -O3 -march=native on this machine, on every host core:
    one single-threaded replica of the full grid per core (MONC parallelises by domain
    decomposition over MPI ranks; independent replicas bound that from above, with no exchange
    cost), each stepping as many centred steps as the GPU arm times (at most 20)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import multiprocessing as mp

    from oracle import pyoracle as po

    po.build(native=True)
    os.environ["MONC_ORACLE_LIB"] = "native"  # the spawned replicas load the native build
    cores = os.cpu_count() or 1
    steps = max(1, min(args.steps, 20))
    warmup = max(1, min(args.warmup, 3))  # bounded: each oracle step of the full grid takes seconds
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(cores) as pool:
        times = pool.starmap(_oracle_run, [(steps, warmup)] * cores)
    wall = time.perf_counter() - t0
    slowest = max(times)
    value = cores * NX * NY * NZ * steps / slowest / 1e6
    out = {
        "impl": "reference",
        "metric": METRIC,
        "value": round(value, 3),
        "unit": "Mpoint-steps/s",
        "n_gpus": int(os.environ.get("WORLD_SIZE", "1")),
        "steps": steps,
        "warmup": warmup,
        "ms_per_step": round(slowest / steps * 1e3, 2),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded initial state; no dataset involved)",
        "config": {"workload": WORKLOAD, "nx": NX, "ny": NY, "nz": NZ, "precision": "fp64", "solver": "fft"},
        "cpu_baseline": {"value": round(value, 3), "unit": "Mpoint-steps/s", "cores": cores, "kind": "port",
                         "sample": f"{cores} single-threaded oracle replicas (built -O3 -march=native), each the "
                                   f"full {NX}x{NY}x{NZ} grid, {warmup} untimed steps (the forward step first) + "
                                   f"{steps} timed centred steps ({wall:.0f} s wall); MONC itself "
                                   "cannot be built (no Fortran/MPI/NetCDF toolchain)"},
        "e2e": {"value": round(value, 3), "unit": "Mpoint-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def launch_plan(gpus: int, env) -> str:
    """How `--gpus N` is honoured: "run" when this process is one of N ranks (or N = 1 without a
    launcher), "spawn" when N > 1 was asked for without a launcher (bench.py then starts N ranks
    under torch.distributed.run itself).  A launcher whose world size differs from N is an error,
    so that a run never reports a GPU count other than the one requested."""
    if gpus < 1:
        raise SystemExit(f"bench.py: --gpus must be >= 1 (got {gpus})")
    world = env.get("WORLD_SIZE")
    if world is None:
        return "spawn" if gpus > 1 else "run"
    if int(world) != gpus:
        raise SystemExit(f"bench.py: --gpus {gpus} but the launcher started WORLD_SIZE={world} ranks")
    return "run"


def spawn_ranks(gpus: int, argv: list) -> int:
    """Re-run this command as `gpus` ranks under torch.distributed.run on 127.0.0.1."""
    import socket

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={gpus}",
           "--master-addr", "127.0.0.1", f"--master-port={port}", os.path.abspath(__file__), *argv]
    return subprocess.call(cmd)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--replicas", action="store_true",
                    help="N > 1: independent single-GPU models instead of the decomposed domain")
    ap.add_argument("--decomposed", action="store_true",
                    help="run the decomposed domain even on one GPU (one slab; exercises the NCCL path)")
    ap.add_argument("--large", action="store_true",
                    help="also run the 1024x1024x200 FP32-mixed case with three tracers (about a minute)")
    ap.add_argument("--skip-extra", action="store_true",
                    help="skip the adjoint-ratio and moist-precision measurements (single-GPU runs)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if launch_plan(args.gpus, os.environ) == "spawn":
        raise SystemExit(spawn_ranks(args.gpus, sys.argv[1:]))
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
