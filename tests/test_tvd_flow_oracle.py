"""TVD advection of the flow fields in the CPU oracle (advection_flow_fields = tvd,
tvdadvection.F90:603-908 with interpolate_to_dual, stencil.F90:87-169), pinned by properties:

* the flux form conserves u and v momentum in a periodic domain closed at the bottom and top
  (sum over levels of dz(k) times the horizontal sum of the source vanishes);
* on a smooth, well-resolved flow the TVD and Piacsek-Williams sources are two discretisations of
  the same advection and agree closely;
* a step in v carried by a uniform, non-divergent flow stays within its initial range (TVD
  property).
"""
import numpy as np

from monc_b200 import api, config as cf, init as ini
from oracle import pyoracle as po

F = api.FIELDS
C = api.COMPONENTS


def oracle(nx, ny, nz, adv=cf.ADVECT_TVD, dz=25.0):
    c = cf.dry_cbl_config(nx, ny, nz, 50.0, dz, 1.0)
    c.advection_flow_fields = adv
    return c, po.Oracle(c)


def sources(o, st, comp, shape):
    for name, arr in st.items():
        o.set(F[name], arr)
    for f in ("su", "sv", "sw"):
        o.set(F[f], np.zeros(shape))
    o.set_timestep(2)
    o.component(C[comp])
    return {f: o.get(F[f]) for f in ("su", "sv", "sw")}


def test_tvd_flow_conserves_horizontal_momentum():
    n, nz = 32, 20
    c, o = oracle(n, n, nz)
    st = ini.random_flow_state(n, n, nz, seed=8, amp_uv=2.0, amp_w=0.5, amp_th=1.0)
    for f in ("w", "zw"):
        st[f][0] = 0.0
        st[f][-1] = 0.0
    s = sources(o, st, "tvd_advection", (nz, n, n))
    dz = o.profile("dz")
    for f in ("su", "sv"):
        weighted = s[f][1:] * dz[1:, None, None]
        assert abs(weighted.sum()) <= 1e-12 * np.abs(weighted).sum(), f


def test_tvd_and_pw_agree_on_a_smooth_flow():
    """A smooth, divergence-free flow: u(y, z) and v(x, z) shear plus an x-z overturning cell from
    a streamfunction on the staggered grid.  The flux form (TVD) and PW's form of the advection
    are equal for a divergence-free flow, so the two sources differ by discretisation only.  (On a
    divergent flow they differ by construction: for u = u(x) alone the flux form gives -2 u u' and
    PW -1.5 u u'.)"""
    n, nz = 32, 24
    shape = (nz, n, n)
    kk, jj, ii = np.meshgrid(np.arange(nz), np.arange(n), np.arange(n), indexing="ij")
    ph, H, dx, dz = 2 * np.pi / n, nz - 1, 50.0, 25.0
    zf = np.sin(np.pi * kk / H)
    amp = 0.05 * dz
    u = 3.0 + 0.5 * np.sin(ph * jj) * zf + amp * np.pi / (H * dz) * np.sin(ph * (ii + 0.5)) * np.cos(np.pi * (kk - 0.5) / H)
    v = -1.0 + 0.5 * np.sin(ph * ii) * zf
    w = -amp * ph / dx * np.cos(ph * ii) * np.sin(np.pi * kk / H)
    w[0] = w[-1] = 0.0
    st = {"u": u, "v": v, "w": w, "zu": u, "zv": v, "zw": w, "th": np.zeros(shape), "zth": np.zeros(shape)}
    out = {}
    for adv, comp in ((cf.ADVECT_TVD, "tvd_advection"), (cf.ADVECT_PW, "pw_advection")):
        c, o = oracle(n, n, nz, adv, dz)
        out[adv] = sources(o, st, comp, shape)
    for f in ("su", "sv", "sw"):
        a, b = out[cf.ADVECT_TVD][f][1:-1], out[cf.ADVECT_PW][f][1:-1]
        assert np.linalg.norm(a - b) <= 0.03 * np.linalg.norm(b), f


def test_tvd_flow_step_stays_bounded():
    """A step in v (varying in x only) carried by a uniform u, w = 0: the flow advecting v is then
    non-divergent, and zv + 2 dt sv stays within the initial [min, max] (TVD property).  (A step in
    u carried by u itself compresses the flow and is not bounded by any flux form.)"""
    n, nz = 32, 12
    c, o = oracle(n, n, nz)
    shape = (nz, n, n)
    step = np.where((np.arange(n) >= 8) & (np.arange(n) < 20), 1.0, 0.0)[None, None, :] * np.ones(shape)
    v = -3.0 + 0.8 * step
    u = np.full(shape, 4.0)
    z = np.zeros(shape)
    st = {"u": u, "zu": u, "v": v, "zv": v, "w": z, "zw": z, "th": z, "zth": z}
    s = sources(o, st, "tvd_advection", shape)
    new = v + 2.0 * c.dtm * s["sv"]
    assert new[1:].min() >= v.min() - 1e-12
    assert new[1:].max() <= v.max() + 1e-12
    assert np.abs(s["sv"]).max() > 0  # the step moved
