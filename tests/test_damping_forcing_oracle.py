"""Damping, mean profiles and subsidence forcing in the CPU oracle (damping.F90:124-409,
meanprofiles.F90:95-216, forcing.F90:447-1166, interpolation.F90:15-58), pinned by their
definitions, and the library's reference-state profiles (dmpco, dmpcoz, w_subs, which need no
GPU) against the oracle's:

* dmpco = dmptim (exp((zn - zdmp)/hdmp) - 1) on the levels at or above zdmp, dmpcoz the same on
  the w levels, and nothing below the first level under zdmp;
* w_subs is the piecewise-linear interpolation of the nodes (numpy.interp inside their range) or,
  for a divergence input, -div z;
* the mean profiles are numpy means of zu, zv, zth, zq;
* one damping call subtracts dmpco (zf - mean) from the sources;
* the mean-profile subsidence of a linear theta profile is w_subs dtheta/dz;
* damping and forcing wait for timestep 3, as MONC's do.
"""
import numpy as np
import pytest

from monc_b200 import api, config as cf, init as ini
from oracle import pyoracle as po

F = api.FIELDS
C = api.COMPONENTS
NX, NY, NZ = 16, 16, 20


def damped_config(**kw):
    c = cf.dry_cbl_config(NX, NY, NZ, 50.0, 25.0, 1.0, ug=3.0, fcoriol=1e-4)
    cf.enable_damping(c, kw.get("dmptim", 0.01), kw.get("zdmp", 300.0), kw.get("hdmp", 100.0))
    return c


def test_damping_coefficients():
    c = damped_config()
    o = po.Oracle(c)
    zn, z = o.profile("zn"), o.profile("z")
    dmpco, dmpcoz = o.profile("dmpco"), o.profile("dmpcoz")
    above = zn >= 300.0
    np.testing.assert_allclose(dmpco[above], 0.01 * (np.exp((zn[above] - 300.0) / 100.0) - 1.0), rtol=1e-14)
    assert np.all(dmpco[~above] == 0.0)
    kmin = int(np.argmax(above))  # first level at or above zdmp (0-based); kdmpmin is the one below
    zabove = z >= 300.0
    zabove[: kmin - 1] = False
    np.testing.assert_allclose(dmpcoz[zabove], 0.01 * (np.exp((z[zabove] - 300.0) / 100.0) - 1.0), rtol=1e-14)
    assert np.all(dmpcoz[~zabove] == 0.0)
    for name in ("dmpco", "dmpcoz"):
        np.testing.assert_array_equal(api.reference_profile(c, name), o.profile(name))


@pytest.mark.parametrize("input_type", [cf.SUBS_VELOCITY, cf.SUBS_DIVERGENCE], ids=["velocity", "divergence"])
def test_subsidence_profile(input_type):
    c = cf.dry_cbl_config(NX, NY, NZ, 50.0, 25.0, 1.0)
    zn_nodes = [0.0, 150.0, 320.0, 600.0]
    f_nodes = [0.0, -0.004, -0.006, -0.002] if input_type == cf.SUBS_VELOCITY else [3e-6, 3e-6, 2e-6, 1e-6]
    cf.enable_subsidence(c, zn_nodes, f_nodes, input_type=input_type)
    o = po.Oracle(c)
    z = o.profile("z")
    w = o.profile("w_subs")
    inside = z <= 600.0
    ref = np.interp(z[inside], zn_nodes, f_nodes)
    if input_type == cf.SUBS_DIVERGENCE:
        ref = -ref * z[inside]
    np.testing.assert_allclose(w[inside], ref, rtol=1e-13, atol=1e-18)
    assert np.all(w[~inside] == 0.0)  # above the last node (MONC leaves these unset)
    np.testing.assert_array_equal(api.reference_profile(c, "w_subs"), w)


def flow_state(seed=3):
    st = ini.random_flow_state(NX, NY, NZ, seed=seed, amp_uv=1.0, amp_w=0.3, amp_th=0.5, ug=3.0)
    return st


def load(o, st):
    for k, v in st.items():
        o.set(F[k], v)


def test_mean_profiles_and_damping_step():
    c = damped_config()
    o = po.Oracle(c)
    st = flow_state()
    load(o, st)
    o.component(C["mean_profiles"])
    mp = o.mean_profiles()
    np.testing.assert_allclose(mp["olzubar"], st["zu"].mean(axis=(1, 2)), rtol=1e-14, atol=1e-15)
    np.testing.assert_allclose(mp["olzthbar"], st["zth"].mean(axis=(1, 2)), rtol=1e-14, atol=1e-15)
    z = np.zeros((NZ, NY, NX))
    for f in ("su", "sv", "sw", "sth"):
        o.set(F[f], z)
    o.set_timestep(2)
    o.component(C["damping"])  # timestep < 3: nothing
    assert all(np.abs(o.get(F[f])).max() == 0.0 for f in ("su", "sv", "sw", "sth"))
    o.set_timestep(5)
    o.component(C["damping"])
    dmpco = o.profile("dmpco")[:, None, None]
    dmpcoz = o.profile("dmpcoz")[:, None, None]
    ubar = mp["olzubar"][:, None, None]
    np.testing.assert_allclose(o.get(F["su"]), -dmpco * (st["zu"] - ubar), rtol=1e-13, atol=1e-16)
    thbar = mp["olzthbar"][:, None, None]
    np.testing.assert_allclose(o.get(F["sth"]), -dmpco * (st["zth"] - thbar), rtol=1e-13, atol=1e-16)
    sw = o.get(F["sw"])
    np.testing.assert_allclose(sw[:-1], (-dmpcoz * st["zw"])[:-1], rtol=1e-13, atol=1e-16)
    assert np.abs(sw[-1]).max() == 0.0


def test_mean_profile_subsidence_of_linear_theta():
    c = cf.dry_cbl_config(NX, NY, NZ, 50.0, 25.0, 1.0)
    cf.enable_subsidence(c, [0.0, 500.0], [-0.002, -0.005], theta=True)
    o = po.Oracle(c)
    zn = o.profile("zn")
    shape = (NZ, NY, NX)
    st = {f: np.zeros(shape) for f in ("u", "v", "w", "zu", "zv", "zw")}
    lapse = 0.004
    th = np.broadcast_to((lapse * zn)[:, None, None], shape).copy()
    st["th"] = th
    st["zth"] = th.copy()
    load(o, st)
    o.component(C["mean_profiles"])
    for f in ("su", "sv", "sth"):
        o.set(F[f], np.zeros(shape))
    o.set_timestep(3)
    o.component(C["forcing"])
    w = o.profile("w_subs")
    rdzn = o.profile("rdzn")
    sth = o.get(F["sth"])[:, 0, 0]
    k = np.arange(1, NZ - 1)  # 0-based levels 2..nz-1
    expect = -w[k] * (lapse * (zn[k + 1] - zn[k])) * rdzn[k + 1]
    np.testing.assert_allclose(sth[k], expect, rtol=1e-12)
    assert np.all(sth[1:] > 0.0)  # subsiding air warms a stable layer
    assert np.abs(o.get(F["su"])).max() == 0.0  # uniform (zero) wind


def test_damped_steps_relax_upper_levels():
    """Five steps with a damping layer above 300 m leave less upper-level variance than without."""
    var = []
    for damp in (False, True):
        c = cf.dry_cbl_config(NX, NY, NZ, 50.0, 25.0, 1.0, ug=3.0, fcoriol=1e-4)
        if damp:
            cf.enable_damping(c, 0.05, 300.0, 100.0)
        o = po.Oracle(c)
        load(o, flow_state())
        o.step(5)
        zn = o.profile("zn")
        up = zn > 350.0
        u = o.get(F["u"])[up]
        var.append(float(((u - u.mean(axis=(1, 2), keepdims=True)) ** 2).sum()))
    assert var[1] < var[0]
