"""cfltest in the CPU oracle (cfltest.F90:62-191 with the gathers of stepfields.F90:372-393 and
smagorinsky.F90:143-173): the evaluation schedule, the Courant numbers recomputed in numpy from
the fields the gathers read, the ratchet towards the target dtm, the immediate cut when the CFL
number is too high, l_constant_dtm, the stop below cfl_dtmmin, and the Galilean transformation
(the frame at the middle of the zu, zv range; a frame at rest changes nothing)."""
import numpy as np
import pytest

from monc_b200 import api, config as cf, init as ini
from oracle import pyoracle as po

F = api.FIELDS
NX, NY, NZ = 16, 16, 12


def setup(dtm=1.0, amp=2.0, **cfl):
    c = cf.dry_cbl_config(NX, NY, NZ, 50.0, 25.0, dtm, ug=5.0, fcoriol=1e-4)
    cf.enable_cfl(c, **cfl)
    o = po.Oracle(c)
    st = ini.random_flow_state(NX, NY, NZ, seed=3, amp_uv=amp, amp_w=0.5, ug=5.0)
    for k, v in st.items():
        o.set(F[k], v)
    return c, o, st


def test_evaluation_schedule():
    """Every step up to cfl_frequency + 1, then every cfl_frequency steps (timestep mod f == 1)."""
    c, o, _ = setup(frequency=3)
    evaluated = []
    for n in range(1, 15):
        before = o.cfl_state()["cfl_evaluations"]
        o.step(1)
        if o.cfl_state()["cfl_evaluations"] > before:
            evaluated.append(n)
    assert evaluated == [1, 2, 3, 4, 7, 10, 13]


def test_first_evaluation_matches_numpy():
    c, o, st = setup(frequency=5)
    o.step(1)
    s = o.cfl_state()
    zu, zv, zw = st["zu"], st["zv"], st["zw"]
    rdzn = o.profile("rdzn")  # level k at index k-1
    vis, diff = o.get(F["vis"]), o.get(F["diff"])
    cvel_x = max(abs(zu[1:].max()), abs(zu[1:].min()))
    cvel_y = max(abs(zv[1:].max()), abs(zv[1:].min()))
    cvel_z = max(0.0, max((np.abs(zw[k - 1]).max() * rdzn[k]) for k in range(2, NZ)))
    cx = cy = 1.0 / 50.0
    fac = [(rdzn[k] * rdzn[k] + cx * cx) + cy * cy for k in range(2, NZ)]
    cvis = max(0.0, max((np.maximum(vis[k - 1], diff[k - 1]) * fac[k - 2]).max() for k in range(2, NZ)))
    dtm = c.dtm
    assert s["cvel_x"] == cvel_x and s["cvel_y"] == cvel_y and s["cvel_z"] == cvel_z
    cvel = (cvel_x * cx + cvel_y * cy + cvel_z) * dtm
    assert s["cvel"] == cvel
    assert s["cvis"] == cvis * (dtm * 4)
    cfl = s["cvis"] / c.cfl_cvismax + cvel / c.cfl_cvelmax
    assert s["cfl_number"] == cfl
    assert cfl > 1.0 + c.cfl_tollerance  # this flow is too fast for dtm = 1 s
    assert s["absolute_new_dtm"] == dtm / cfl
    assert s["dtm_new"] == min(dtm * (1 + c.cfl_rincmax), dtm / cfl, c.cfl_dtmmax)


def test_ratchet_then_hold():
    """A slow flow: the target is far above dtm, which grows by rincmax per step (also between
    evaluations) until it reaches cfl_dtmmax."""
    c, o, _ = setup(dtm=0.05, amp=0.2, frequency=4, dtmmax=0.06, rincmax=0.05)
    dtms = []
    for _ in range(8):
        o.step(1)
        dtms.append(o.cfl_state()["dtm"])
    expect = [0.05]
    for _ in range(7):
        expect.append(min(expect[-1] * 1.05, 0.06))
    np.testing.assert_allclose(dtms, expect, rtol=1e-15)
    assert dtms[-1] == 0.06


def test_constant_dtm_holds_the_timestep():
    c, o, _ = setup(frequency=2, constant_dtm=True)
    for _ in range(4):
        o.step(1)
        s = o.cfl_state()
        assert s["dtm"] == c.dtm and s["dtm_new"] == c.dtm
    assert s["cfl_number"] > 1.1  # it would have cut the timestep


def test_stop_below_dtmmin():
    c, o, _ = setup(frequency=2, dtmmin=0.9)
    with pytest.raises(po.CflError):
        o.step(1)


def test_disabled_cfl_keeps_dtm():
    c = cf.dry_cbl_config(NX, NY, NZ, 50.0, 25.0, 1.0, ug=5.0, fcoriol=1e-4)
    assert c.cfl_enabled == 0
    o = po.Oracle(c)
    st = ini.random_flow_state(NX, NY, NZ, seed=3, amp_uv=2.0, amp_w=0.5, ug=5.0)
    for k, v in st.items():
        o.set(F[k], v)
    o.step(3)
    s = o.cfl_state()
    assert s["cfl_evaluations"] == 0 and s["dtm"] == 1.0


def galilean_setup(ugal=None, vgal=None, **cfl):
    c = cf.dry_cbl_config(NX, NY, NZ, 50.0, 25.0, 1.0, ug=5.0, fcoriol=1e-4)
    cf.enable_cfl(c, **cfl)
    cf.enable_galilean(c, ugal, vgal)
    o = po.Oracle(c)
    st = ini.random_flow_state(NX, NY, NZ, seed=3, amp_uv=2.0, amp_w=0.5, ug=5.0)
    for k, v in st.items():
        o.set(F[k], v)
    return c, o, st


def test_galilean_frame_is_the_middle_of_the_range():
    """cfltest.F90:184-230: an evaluation puts the frame at the middle of the (undone) zu, zv range,
    and the advective Courant numbers are the half ranges; the forward step's pressure terms then
    move u, zu into that frame (pstep.F90:453-469), so the old-time field zu holds u - ugal."""
    c, o, st = galilean_setup(frequency=3, dtmmax=2.0)
    o.step(1)
    s = o.cfl_state()
    zu, zv = st["zu"][1:], st["zv"][1:]
    ugal, vgal = 0.5 * (zu.min() + zu.max()), 0.5 * (zv.min() + zv.max())
    assert s["ugal"] == ugal and s["vgal"] == vgal
    assert ugal > 3.0  # the flow has a mean wind of 5 m/s to follow
    assert s["cvel_x"] == max(abs(zu.max() - ugal), abs(zu.min() - ugal))
    assert s["cvel_y"] == max(abs(zv.max() - vgal), abs(zv.min() - vgal))
    np.testing.assert_allclose(o.get(F["zu"]), st["u"] - ugal, rtol=0, atol=1e-13)
    np.testing.assert_allclose(o.get(F["zv"]), st["v"] - vgal, rtol=0, atol=1e-13)


def test_galilean_frame_at_rest_changes_nothing():
    """A frame fixed at zero velocity is the untransformed model, bit for bit."""
    out = []
    for gal in (False, True):
        c, o, st = setup(frequency=3, dtmmax=2.0)
        if gal:
            cf.enable_galilean(c, 0.0, 0.0)
            o = po.Oracle(c)
            for k, v in st.items():
                o.set(F[k], v)
        o.step(6)
        out.append({f: o.get(F[f]) for f in ("u", "v", "w", "th", "zu", "zv")})
    for f in out[0]:
        np.testing.assert_array_equal(out[1][f], out[0][f], err_msg=f)

