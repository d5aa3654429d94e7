"""Seeded initial states for the synthetic workloads.

MONC seeds its initial noise through the Fortran compiler's intrinsic generator
(randomnoise.F90:81-141), which no other toolchain reproduces.  This module uses a documented
counter-based generator instead -- SplitMix64 applied to (seed, field id, global point index) --
so that every implementation (the CPU oracle, the GPU library, any future MONC checkpoint) can
be fed the identical arrays.  Arrays are C order [nz][ny][nx] (x fastest), interior points only.
"""
from __future__ import annotations

import numpy as np

_MASK = np.uint64(0xFFFFFFFFFFFFFFFF)


def _splitmix64(x: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        z = x + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def uniform_noise(shape, seed: int, field: int, amplitude: float) -> np.ndarray:
    """Uniform values in [-amplitude, amplitude) keyed on (seed, field, flat index)."""
    n = int(np.prod(shape))
    idx = np.arange(n, dtype=np.uint64)
    key = np.uint64((seed & 0xFFFFFFFF) << 24) ^ np.uint64((field & 0xFF) << 56)
    bits = _splitmix64(idx ^ key) >> np.uint64(11)
    u01 = bits.astype(np.float64) * (1.0 / 9007199254740992.0)  # 2**53
    return ((2.0 * u01 - 1.0) * amplitude).reshape(shape)


def zn_levels(z: np.ndarray) -> np.ndarray:
    """Pressure-level heights from w-level heights (gridmanager.F90:2483-2487)."""
    kkp = len(z)
    zn = np.zeros(kkp)
    for k in range(3, kkp):  # 1-based k=3..kkp-1
        zn[k - 1] = 0.0625 * (9.0 * (z[k - 2] + z[k - 1]) - z[k] - z[k - 3])
    zn[1] = 0.5 * (z[0] + z[1])
    zn[0] = -zn[1]
    zn[kkp - 1] = 0.5 * (z[kkp - 2] + z[kkp - 1])
    return zn


def dry_cbl_state(nx, ny, nz, zn, seed=1, noise_levels=8, noise_amp=0.1, inversion=800.0,
                  lapse=0.003, ug=0.0, zfields_from_prognostics=False):
    """Dry CBL: theta' = 0 below `inversion`, +lapse*(z-inversion) above, uniform noise on the
    lowest `noise_levels` levels above the surface (k=2..noise_levels+1), u = ug, v = w = 0.

    With zfields_from_prognostics=False the z-fields are zero, as in a MONC cold start.
    """
    shape = (nz, ny, nx)
    th = np.zeros(shape)
    prof = np.where(zn > inversion, lapse * (zn - inversion), 0.0)
    th += prof[:, None, None]
    noise = uniform_noise(shape, seed, 3, noise_amp)
    th[1:1 + noise_levels] += noise[1:1 + noise_levels]
    th[0] = 0.0
    u = np.full(shape, float(ug))
    v = np.zeros(shape)
    w = np.zeros(shape)
    st = {"u": u, "v": v, "w": w, "th": th}
    if zfields_from_prognostics:
        st.update({"zu": u.copy(), "zv": v.copy(), "zw": w.copy(), "zth": th.copy()})
    else:
        st.update({"zu": np.zeros(shape), "zv": np.zeros(shape), "zw": np.zeros(shape), "zth": np.zeros(shape)})
    return st


def random_flow_state(nx, ny, nz, seed=7, amp_uv=2.0, amp_w=0.5, amp_th=0.5, ug=0.0):
    """A state with resolved motion everywhere (for stencil parity tests): noise in every field,
    w = 0 on level 1 and the top level, z-fields a perturbed copy of the prognostics."""
    shape = (nz, ny, nx)
    u = ug + uniform_noise(shape, seed, 0, amp_uv)
    v = uniform_noise(shape, seed, 1, amp_uv)
    w = uniform_noise(shape, seed, 2, amp_w)
    w[0] = 0.0
    w[-1] = 0.0
    th = uniform_noise(shape, seed, 3, amp_th)
    st = {"u": u, "v": v, "w": w, "th": th}
    st["zu"] = u + uniform_noise(shape, seed, 4, 0.1 * amp_uv)
    st["zv"] = v + uniform_noise(shape, seed, 5, 0.1 * amp_uv)
    zw = w + uniform_noise(shape, seed, 6, 0.1 * amp_w)
    zw[0] = 0.0
    zw[-1] = 0.0
    st["zw"] = zw
    st["zth"] = th + uniform_noise(shape, seed, 7, 0.1 * amp_th)
    return st


def moist_layer_state(nx, ny, nz, zn, seed=1, theta_below=289.0, theta_above=297.5, inversion=840.0,
                      lapse=0.00365, qt_below=9e-3, qt_above=1.5e-3, thref0=289.0, noise_levels=8,
                      noise_amp=0.1, ug=0.0, n_tracers=0):
    """Stratocumulus-like layer: theta (as theta' = theta - thref0) well mixed below `inversion`
    and `theta_above` + lapse*(z - inversion) above it; total water as vapour (q0) with no
    liquid (q1) -- the saturation adjustment forms the cloud in the first steps; uniform theta
    noise on the lowest levels; passive tracers (q2...) log-normal near the surface."""
    shape = (nz, ny, nx)
    th_prof = np.where(zn > inversion, theta_above + lapse * (zn - inversion), theta_below) - thref0
    th = np.broadcast_to(th_prof[:, None, None], shape).copy()
    noise = uniform_noise(shape, seed, 3, noise_amp)
    th[1:1 + noise_levels] += noise[1:1 + noise_levels]
    th[0] = th[1]
    qv = np.broadcast_to(np.where(zn > inversion, qt_above, qt_below)[:, None, None], shape).copy()
    st = {"u": np.full(shape, float(ug)), "v": np.zeros(shape), "w": np.zeros(shape), "th": th,
          "q0": qv, "q1": np.zeros(shape)}
    for t in range(n_tracers):
        g = uniform_noise(shape, seed, 40 + t, 1.0)
        src = np.exp(0.5 * g) * np.exp(-zn / 200.0)[:, None, None]
        st[f"q{2 + t}"] = src
    for name in list(st):
        st["z" + name] = st[name].copy()
    return st
