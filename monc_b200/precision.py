"""FP32-mixed against FP64 on the moist stratocumulus-like layer: speed and accuracy.

    python -m monc_b200.precision --nx 512 --ny 512 --nz 160 --steps 500

The case: dx = dy = 35 m, stretched dz from 5 m at the surface to 20 m at the top, theta 289 K
below an 840 m inversion and 297.5 K above it with a 0.00365 K/m lapse, total water 9 g/kg below
and 1.5 g/kg above (as vapour; simplecloud forms the cloud), seeded +-0.1 K noise, dt = 0.3 s.
Both precisions start from the same state.  Reported: ms per step of each (CUDA events on the
model's stream, after the first step), the speed-up, and after the last step the maximum
relative difference of the domain-mean theta and w'^2 profiles (max |a-b| / max |b| over
levels), plus the same for the mean vapour, and for every prognostic field (u, v, w, theta,
vapour, liquid) its maximum and RMS relative difference from the FP64 run: max |a-b| / max |b|
and rms(a-b) / rms(b) over the grid, theta as its departure from the reference state thref0.
With --solver iterative both runs solve for the pressure with BiCGStab to --tolerance (FP64, and
FP32 corrections inside FP64 iterative refinement for FP32-mixed); the iterations per step are
reported (each step is then queued on its own, to read its solve's iteration count).
"""
from __future__ import annotations

import argparse
import json

import numpy as np
import torch

from . import api, config as cf, init as ini


def build(a, precision):
    z = cf.stretched_levels(a.nz, a.dz_bottom, a.dz_top)
    c = cf.moist_config(a.nx, a.ny, z, a.dx, a.dt, precision=precision,
                        solver=cf.SOLVER_ITERATIVE if a.solver == "iterative" else cf.SOLVER_FFT)
    if a.solver == "iterative":
        c.tolerance = a.tolerance
    zn = api.reference_profile(c, "zn")
    st = ini.moist_layer_state(a.nx, a.ny, a.nz, zn, seed=a.seed, noise_levels=a.noise_levels)
    return c, st


FIELDS = ("u", "v", "w", "th", "q0", "q1")


def run(a, precision, reproducible=0, round_state=False, fields=None):
    """ms per step, the mean theta, w'^2, vapour and liquid profiles after a.steps steps, and
    (when `fields` is a dict) the final prognostic fields in it; iterations per step of an
    iterative solve in a.iterations_per_step."""
    c, st = build(a, precision)
    c.reproducible = reproducible
    if round_state:  # the initial state as the FP32-mixed model holds it
        st = {k: v.astype(np.float32).astype(np.float64) for k, v in st.items()}
    m = api.Model(c)
    m.set_state(st)
    m.step(1)  # the forward step
    stream = torch.cuda.ExternalStream(m.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    if a.solver == "iterative":
        its = 0
        for _ in range(a.steps - 1):
            m.step(1)
            its += m.reductions().solver_iterations
        a.iterations_per_step = its / max(a.steps - 1, 1)
    else:
        m.step(a.steps - 1)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / max(a.steps - 1, 1)
    th, w2 = m.diagnostics()
    qv = m.mean_profile("q0")
    ql = m.mean_profile("q1")
    if fields is not None:
        for f in FIELDS:
            fields[f] = m.download(f)
    m.close()
    return ms, th, w2, qv, ql


def field_errors(test: dict, ref: dict) -> dict:
    """Per field: max |a-b| / max |b| and rms(a-b) / rms(b) over the grid (theta as the departure
    from the reference state, which is what the model holds)."""
    out = {}
    for f in FIELDS:
        a, b = test[f], ref[f]
        d = a - b
        out[f] = {"max_rel": float(np.abs(d).max() / max(np.abs(b).max(), 1e-300)),
                  "rms_rel": float(np.sqrt(np.mean(d * d)) / max(np.sqrt(np.mean(b * b)), 1e-300))}
    return out


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--nx", type=int, default=512)
    ap.add_argument("--ny", type=int, default=512)
    ap.add_argument("--nz", type=int, default=160)
    ap.add_argument("--dx", type=float, default=35.0)
    ap.add_argument("--dz-bottom", type=float, default=5.0)
    ap.add_argument("--dz-top", type=float, default=20.0)
    ap.add_argument("--dt", type=float, default=0.3)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--noise-levels", type=int, default=10)
    ap.add_argument("--solver", choices=["fft", "iterative"], default="fft")
    ap.add_argument("--tolerance", type=float, default=1e-4)
    ap.add_argument("--no-control", dest="control", action="store_false",
                    help="skip the FP64 run with separately rounded multiply-adds")
    a = ap.parse_args(argv)
    f64, f32 = {}, {}
    ms64, th64, w64, qv64, ql64 = run(a, cf.FP64, fields=f64)
    its64 = getattr(a, "iterations_per_step", None)
    ms32, th32, w32, qv32, ql32 = run(a, cf.FP32_MIXED, fields=f32)
    its32 = getattr(a, "iterations_per_step", None)
    per_field = field_errors(f32, f64)
    del f64, f32
    # control: the same FP64 model with separately rounded multiply-adds; the difference shows how
    # far rounding-level changes alone grow in this developing convection
    _, thr, wr, qvr, _ = run(a, cf.FP64, reproducible=1) if a.control else (None, th64, w64, qv64, None)
    # second control: FP64 throughout, from the initial state rounded to FP32 -- how far the
    # rounding of the initial fields alone carries the flow, whatever the arithmetic
    _, thi, wi, qvi, _ = run(a, cf.FP64, round_state=True) if a.control else (None, th64, w64, qv64, None)
    zmax = float(cf.stretched_levels(a.nz, a.dz_bottom, a.dz_top)[-1])
    print(json.dumps({
        "case": f"moist layer {a.nx}x{a.ny}x{a.nz}, dx={a.dx} m, dz {a.dz_bottom}->{a.dz_top} m (top {zmax:.0f} m), "
                f"dt={a.dt} s, simplecloud, {a.solver} solver",
        "steps": a.steps,
        "fp64_ms_per_step": round(ms64, 4), "fp32_mixed_ms_per_step": round(ms32, 4),
        "speedup": round(ms64 / ms32, 3),
        "fp64_mpoint_steps_per_s": round(a.nx * a.ny * a.nz / (ms64 * 1e-3) / 1e6, 1),
        "fp32_mixed_mpoint_steps_per_s": round(a.nx * a.ny * a.nz / (ms32 * 1e-3) / 1e6, 1),
        "rel_err_mean_theta": rel(th32, th64),
        "rel_err_mean_theta_deviation": rel(th32 - th64[1], th64 - th64[1]),
        "rel_err_mean_w2": rel(w32, w64),
        "rel_err_mean_qv": rel(qv32, qv64),
        "max_mean_ql_fp64": float(ql64.max()),
        "rel_err_mean_ql": rel(ql32, ql64),
        "fields_fp32_vs_fp64": per_field,
        "iterations_per_step": {"fp64": its64, "fp32_mixed": its32} if a.solver == "iterative" else None,
        "fp64_fma_vs_separate_rounding": {"rel_err_mean_theta": rel(thr, th64), "rel_err_mean_w2": rel(wr, w64),
                                           "rel_err_mean_qv": rel(qvr, qv64)},
        "fp64_from_fp32_rounded_initial_state": {"rel_err_mean_theta": rel(thi, th64), "rel_err_mean_w2": rel(wi, w64),
                                                 "rel_err_mean_qv": rel(qvi, qv64)},
    }))


if __name__ == "__main__":
    main()
