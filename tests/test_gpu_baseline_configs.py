"""GPU FP64 against the oracle at the benchmark configurations' own sizes and settings.

* Dry CBL 64x64x65 (dx = 50 m, dz = 25 m, dt = 1 s, u = v = w = 0, noise on the lowest 8 levels):
  200 steps.  The domain-mean theta' and w'^2 profiles after 200 steps agree to MEAN_TOL, and
  every field to FIELD_TOL_200 (max |a-b| / max |b|).  The tolerances are set from what moves
  the two apart: the GPU solves the pressure with another FFT algorithm (1e-11 per solve, see
  the fftsolver component test) and the bench build contracts multiply-adds; in this flow a
  rounding-level change of the initial state (theta * (1 + 1e-15)) moves the oracle's own mean
  profiles by ~1e-15 after 200 steps, so the flow does not amplify those differences, and the
  accumulated difference stays orders of magnitude below the tolerance.
* Dry CBL 256x256x128 (the benchmarked grid: dx = 25 m, dz = 15 m, u_g = 5 m/s, f = 1e-4,
  dt = 0.5 s, noise on the lowest 10 levels): every field <= 1e-10 after 1 and 2 steps.
* Moist layer 512x512x160 (dx = 35 m, stretched dz 5 -> 20 m, dt = 0.3 s, simplecloud), FP64:
  every field, vapour and liquid included, <= 1e-10 after 1 step.
* Dry CBL 128x128x96 (dx = 50 m, dz = 20 m, dt = 1 s, windless): every field <= 1e-10 after the
  first step above level 1; at level 1 the windless surface scheme's conditioning sets the bound
  (see LEVEL1_WINDLESS_TOL).

The oracle runs MONC's column order in FP64 on one host core; these sizes take it from about a
second (128x128x96) to about 15 s per step (512x512x160, with ~12 GB of host memory).
"""
import numpy as np
import pytest

from monc_b200 import api, config as cf, init as ini
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

STEP_TOL = 1e-10          # per field, after 1-2 steps
MEAN_TOL = 1e-9           # domain-mean theta' and w'^2 profiles after 200 steps
FIELD_TOL_200 = 1e-8      # every field after 200 steps
FIELDS = ["u", "v", "w", "th", "zu", "zv", "zw", "zth", "p", "vis", "diff"]


def rel_err(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def mean_profiles(th, w):
    """Domain-mean theta' and w'^2 per level."""
    thm = th.mean(axis=(1, 2))
    w2 = ((w - w.mean(axis=(1, 2), keepdims=True)) ** 2).mean(axis=(1, 2))
    return thm, w2


def pair(cfg, state, reproducible=0):
    cfg.reproducible = reproducible
    o = po.Oracle(cfg)
    m = api.Model(cfg)
    for name, arr in state.items():
        o.set(api.field_id(name), arr)
        m.upload(name, arr)
    return o, m


def check_fields(o, m, fields, tol, what):
    worst = {}
    for f in fields:
        worst[f] = rel_err(m.download(f), o.get(api.field_id(f)))
    bad = {f: e for f, e in worst.items() if not e <= tol}
    assert not bad, f"{what}: fields beyond {tol:g}: {bad}"
    return worst


@pytest.mark.parametrize("reproducible", [0, 1], ids=["fma", "exact"])
def test_dry_cbl_64x64x65_200_steps_mean_profiles(gpu_lib, reproducible):
    cfg = cf.dry_cbl_config(64, 64, 65, 50.0, 25.0, 1.0)
    zn = api.reference_profile(cfg, "zn")
    st = ini.dry_cbl_state(64, 64, 65, zn, seed=1, noise_levels=8)
    o, m = pair(cfg, st, reproducible)
    o.step(200)
    m.step(200)
    th_g, w2_g = mean_profiles(m.download("th"), m.download("w"))
    th_o, w2_o = mean_profiles(o.get(api.field_id("th")), o.get(api.field_id("w")))
    assert np.isfinite(th_g).all() and np.isfinite(w2_g).all()
    assert w2_o.max() > 1e-4, "no resolved convection developed; the comparison would be empty"
    e_th, e_w2 = rel_err(th_g, th_o), rel_err(w2_g, w2_o)
    assert e_th <= MEAN_TOL, f"mean theta' after 200 steps: rel err {e_th:.3e}"
    assert e_w2 <= MEAN_TOL, f"mean w'^2 after 200 steps: rel err {e_w2:.3e}"
    check_fields(o, m, FIELDS, FIELD_TOL_200, "200 steps")
    m.close()
    o.close()


def test_dry_cbl_256x256x128_benchmark_grid(gpu_lib):
    cfg = cf.dry_cbl_config(256, 256, 128, 25.0, 15.0, 0.5, ug=5.0, fcoriol=1e-4)
    zn = api.reference_profile(cfg, "zn")
    st = ini.dry_cbl_state(256, 256, 128, zn, seed=20261203, noise_levels=10, ug=5.0)
    o, m = pair(cfg, st)
    for n in (1, 2):
        o.step(1)
        m.step(1)
        check_fields(o, m, FIELDS, STEP_TOL, f"step {n}")
    m.close()
    o.close()


# In a windless start the surface scheme is ill-conditioned at level 1: with u = v = 0 the
# convective branch of lowerbc.F90:601-633 takes u* from the free-convection limit (~1e-8 m/s),
# and its denominator zlogth - 2 log((1 + sqrt(1 + X1)) / (1 + sqrt(1 + X2))) (X ~ 1e23) cancels to
# ~6e-11 out of ~4.6, a condition number of ~8e10.  One unit in the last place of log moves the
# level-1 diffusivity by ~1e-5 relative, and the ghost value theta(1) with it, so the GPU's log and
# the host's differ there by that much although both are correctly computed.  The surface flux
# diff(1) (theta(1) - theta(2)) that the interior sees in the same step is well-conditioned, so
# every field above level 1 is held to STEP_TOL after the first step.  From the second step on,
# the diffusion at level 2 pairs the new diff(1) with the last step's theta(1), which no longer
# cancels, and the level-1 difference reaches theta at level 2 (1e-6 after two steps), so the
# windless start is compared over one step.
LEVEL1_WINDLESS_TOL = 1e-4


def test_dry_cbl_128x128x96_differentiation_grid(gpu_lib):
    cfg = cf.dry_cbl_config(128, 128, 96, 50.0, 20.0, 1.0)
    zn = api.reference_profile(cfg, "zn")
    st = ini.dry_cbl_state(128, 128, 96, zn, seed=1, noise_levels=10)
    o, m = pair(cfg, st)
    for n in (1,):
        o.step(1)
        m.step(1)
        bad = {}
        for f in FIELDS:
            a, b = m.download(f), o.get(api.field_id(f))
            e = rel_err(a[1:], b[1:])
            if not e <= STEP_TOL:
                bad[f] = e
            tol1 = LEVEL1_WINDLESS_TOL if f in ("diff", "th", "zth") else STEP_TOL
            e1 = rel_err(a[0], b[0]) if np.abs(b[0]).max() > 0 else float(np.abs(a[0]).max())
            if not e1 <= tol1:
                bad[f + "(level 1)"] = e1
        assert not bad, f"step {n}: {bad}"
    m.close()
    o.close()


def test_moist_layer_512x512x160_fp64(gpu_lib):
    z = cf.stretched_levels(160, 5.0, 20.0)
    cfg = cf.moist_config(512, 512, z, 35.0, 0.3)
    zn = api.reference_profile(cfg, "zn")
    st = ini.moist_layer_state(512, 512, 160, zn, seed=1, noise_levels=10)
    o, m = pair(cfg, st)
    o.step(1)
    m.step(1)
    check_fields(o, m, FIELDS + ["q0", "q1", "zq0", "zq1"], STEP_TOL, "step 1")
    m.close()
    o.close()
