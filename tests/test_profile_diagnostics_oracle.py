"""profile_diagnostics (profile_diagnostics.F90:311-636) in the CPU oracle, pinned by numpy sums of
the oracle's own fields and mean profiles: the winds, w moments, theta and its variance about
olthbar, the w-theta and u-w, v-w fluxes (with the mean-profile wind removed), and the moist
totals, fluxes and relative humidity; and olthbar itself, the mean of theta after stepfields'
time smoothing.
"""
import numpy as np

from monc_b200 import api, config as cf, init as ini
from oracle import pyoracle as po

F = api.FIELDS
NX, NY, NZ = 16, 16, 20


def run(c, st, steps):
    o = po.Oracle(c)
    for k, v in st.items():
        o.set(api.field_id(k), v)
    o.step(steps)
    return o


def test_dry_sums():
    c = cf.dry_cbl_config(NX, NY, NZ, 50.0, 25.0, 1.0, ug=3.0, fcoriol=1e-4)
    c.profile_diagnostics_enabled = 1
    st = ini.random_flow_state(NX, NY, NZ, seed=3, amp_uv=1.0, amp_w=0.3, amp_th=0.5, ug=3.0)
    o = run(c, st, 3)
    pd = o.profile_diagnostics()
    mp = o.mean_profiles()
    u, v, w, th = (o.get(F[f]) for f in ("u", "v", "w", "th"))
    thref = o.profile("thref")
    tol = dict(rtol=1e-12, atol=1e-10)
    np.testing.assert_allclose(pd["u_wind_total_local"], u.sum(axis=(1, 2)), **tol)
    np.testing.assert_allclose(pd["ww_total_local"], (w * w).sum(axis=(1, 2)), **tol)
    np.testing.assert_allclose(pd["www_total_local"][1:], (w ** 3).sum(axis=(1, 2))[1:], **tol)
    assert pd["w_wind_total_local"][0] == 0.0
    np.testing.assert_allclose(pd["theta_total_local"], (th + thref[:, None, None]).sum(axis=(1, 2)), **tol)
    np.testing.assert_allclose(pd["th2_total_local"],
                               ((th - mp["olthbar"][:, None, None]) ** 2).sum(axis=(1, 2)), **tol)
    wth = w[1:-1] * 0.5 * (th[1:-1] + th[2:])
    np.testing.assert_allclose(pd["wtheta_cn_total_local"][1:-1], wth.sum(axis=(1, 2)), **tol)
    ubar = mp["olubar"]
    uw = 0.25 * (u[:-1] + np.roll(u[:-1], 1, axis=2) + u[1:] + np.roll(u[1:], 1, axis=2)) - \
        0.5 * (ubar[:-1] + ubar[1:])[:, None, None]
    np.testing.assert_allclose(pd["uw_total_local"][:-1], (uw * w[:-1]).sum(axis=(1, 2)), **tol)
    vbar = mp["olvbar"]
    vw = 0.25 * (v[:-1] + np.roll(v[:-1], 1, axis=1) + v[1:] + np.roll(v[1:], 1, axis=1)) - \
        0.5 * (vbar[:-1] + vbar[1:])[:, None, None]
    np.testing.assert_allclose(pd["vw_total_local"][:-1], (vw * w[:-1]).sum(axis=(1, 2)), **tol)
    assert "vapour_mmr_total_local" not in pd


def test_olthbar_is_the_time_smoothed_theta():
    """One more centred step: olthbar is the mean of c1 th + c2 zth of the state before it."""
    c = cf.dry_cbl_config(NX, NY, NZ, 50.0, 25.0, 1.0, ug=3.0)
    c.profile_diagnostics_enabled = 1
    st = ini.random_flow_state(NX, NY, NZ, seed=4, amp_uv=1.0, amp_w=0.3, amp_th=0.5, ug=3.0)
    o = run(c, st, 2)
    th, zth, u = o.get(F["th"]), o.get(F["zth"]), o.get(F["u"])
    o.step(1)
    mp = o.mean_profiles()
    c1, c2 = 1.0 - 2.0 * 1e-2, 1e-2
    # level 1 is lower_bc's ghost value, rewritten in the subgrid group before stepfields
    np.testing.assert_allclose(mp["olthbar"][1:], (c1 * th + c2 * zth).mean(axis=(1, 2))[1:], rtol=1e-13,
                               atol=1e-14)
    np.testing.assert_allclose(mp["olubar"], u.mean(axis=(1, 2)), rtol=1e-13, atol=1e-14)


def test_moist_sums():
    z = cf.stretched_levels(NZ, 20.0, 60.0, ztop=1000.0)
    c = cf.moist_config(NX, NY, z, 35.0, 0.3, shf_wm2=10.0, lhf_wm2=50.0, max_height_cloud=700.0)
    c.profile_diagnostics_enabled = 1
    st = ini.moist_layer_state(NX, NY, NZ, api.reference_profile(c, "zn"), seed=2)
    flow = ini.random_flow_state(NX, NY, NZ, seed=5, amp_uv=0.5, amp_w=0.2)
    for k in ("u", "v", "w", "zu", "zv", "zw"):
        st[k] = flow[k]
    o = run(c, st, 3)
    pd = o.profile_diagnostics()
    qv, ql, w = o.get(api.field_id("q0")), o.get(api.field_id("q1")), o.get(F["w"])
    tol = dict(rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(pd["vapour_mmr_total_local"], qv.sum(axis=(1, 2)), **tol)
    np.testing.assert_allclose(pd["liquid_mmr_total_local"], ql.sum(axis=(1, 2)), **tol)
    np.testing.assert_allclose(pd["wqv_cn_total_local"][1:-1],
                               (0.5 * (qv[1:-1] + qv[2:]) * w[1:-1]).sum(axis=(1, 2)), **tol)
    assert np.all(pd["rh_total_local"] > 0.0)
    assert np.all(pd["rh_total_local"] < 2.0 * NX * NY)  # relative humidity near or below 1
