"""Damping, mean profiles and subsidence forcing on the GPU against the oracle: the
mean_profiles, damping and forcing components, fused steps (dry and moist, subsidence from the
mean profiles and from the column), the tiled kernels against the point kernel, FP32-mixed
against FP64.  The GPU sums each level in a tree, the oracle in sequence, so the mean profiles
agree to rounding (1e-14) rather than bit for bit, and the components that read them to 1e-12.
"""
import numpy as np
import pytest

from monc_b200 import api, config as cf, init as ini
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

NX, NY, NZ = 32, 32, 24
STATE = ["u", "v", "w", "th", "zu", "zv", "zw", "zth"]


def rel_err(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def dry(precision=cf.FP64, local=False, damp=True, subs=True):
    c = cf.dry_cbl_config(NX, NY, NZ, 50.0, 25.0, 0.5, ug=5.0, fcoriol=1e-4, precision=precision)
    c.reproducible = 1
    if damp:
        cf.enable_damping(c, 0.02, 300.0, 150.0)
    if subs:
        cf.enable_subsidence(c, [0.0, 200.0, 450.0, 700.0], [0.0, -0.003, -0.005, -0.004], theta=True,
                             local_theta=local)
    st = ini.random_flow_state(NX, NY, NZ, seed=6, amp_uv=1.0, amp_w=0.3, amp_th=0.5, ug=5.0)
    zn = api.reference_profile(c, "zn")
    for f in ("th", "zth"):
        st[f] = st[f] + 0.004 * zn[:, None, None]  # a stable layer for the subsidence to act on
    return c, st


def moist(precision=cf.FP64, local=False):
    z = cf.stretched_levels(NZ, 20.0, 60.0, ztop=1000.0)
    c = cf.moist_config(NX, NY, z, 35.0, 0.3, shf_wm2=10.0, lhf_wm2=50.0, max_height_cloud=700.0,
                        precision=precision)
    c.reproducible = 1
    cf.enable_damping(c, 0.01, 600.0, 200.0)
    cf.enable_subsidence(c, [0.0, 1000.0], [0.0, -0.005], theta=True, q=True, local_theta=local, local_q=local)
    st = ini.moist_layer_state(NX, NY, NZ, api.reference_profile(c, "zn"), seed=2)
    flow = ini.random_flow_state(NX, NY, NZ, seed=5, amp_uv=0.5, amp_w=0.2)
    for k in ("u", "v", "w", "zu", "zv", "zw"):
        st[k] = flow[k]
    return c, st


def pair(c, st):
    o, m = po.Oracle(c), api.Model(c)
    for k, v in st.items():
        o.set(api.field_id(k), v)
        m.upload(k, v)
    return o, m


@pytest.mark.parametrize("local", [False, True], ids=["mean-profile", "local"])
def test_components_match_oracle(gpu_lib, local):
    c, st = dry(local=local)
    o, m = pair(c, st)
    o.component(api.COMPONENTS["mean_profiles"])
    m.component("mean_profiles")
    mo, mg = o.mean_profiles(), m.mean_profiles()
    for n in ("olzubar", "olzvbar", "olzthbar"):
        assert rel_err(mg[n], mo[n]) <= 1e-14, n
    z = np.zeros((NZ, NY, NX))
    for f in ("su", "sv", "sw", "sth"):
        o.set(api.field_id(f), z)
        m.upload(f, z)
    o.set_timestep(4)
    m.set_timestep(4)
    for comp in ("damping", "forcing"):
        o.component(api.COMPONENTS[comp])
        m.component(comp)
        for f in ("su", "sv", "sw", "sth"):
            a, b = m.download(f), o.get(api.field_id(f))
            assert rel_err(a, b) <= 1e-12, (comp, f)
    assert np.abs(m.download("sth")).max() > 0


@pytest.mark.parametrize("local", [False, True], ids=["mean-profile", "local"])
def test_fused_dry_steps_match_oracle(gpu_lib, local):
    c, st = dry(local=local)
    o, m = pair(c, st)
    o.step(5)
    m.step(5)
    for f in STATE + ["p"]:
        assert rel_err(m.download(f), o.get(api.field_id(f))) <= 1e-10, f
    mo, mg = o.mean_profiles(), m.mean_profiles()
    for n in mo:
        assert rel_err(mg[n], mo[n]) <= 1e-10, n
    m.close()


@pytest.mark.parametrize("local", [False, True], ids=["mean-profile", "local"])
def test_fused_moist_steps_match_oracle(gpu_lib, local):
    c, st = moist(local=local)
    o, m = pair(c, st)
    o.step(5)
    m.step(5)
    for f in STATE + ["q0", "q1", "zq0", "zq1", "p"]:
        assert rel_err(m.download(f), o.get(api.field_id(f))) <= 1e-10, f
    m.close()


def test_damping_and_subsidence_change_the_steps(gpu_lib):
    """The same five steps without damping and subsidence end elsewhere (the terms are live)."""
    out = []
    for on in (True, False):
        c, st = dry(damp=on, subs=on)
        m = api.Model(c)
        m.set_state(st)
        m.step(5)
        out.append(m.download("th"))
        m.close()
    assert rel_err(out[0], out[1]) > 1e-8


@pytest.mark.parametrize("precision", [cf.FP64, cf.FP32_MIXED], ids=["fp64", "fp32"])
def test_tiled_bit_identical_to_point_kernel(gpu_lib, monkeypatch, precision):
    outs = []
    for point in ("1", "0"):
        monkeypatch.setenv("MGPU_POINT_DYNAMICS", point)
        c, st = dry(precision=precision, local=True)
        m = api.Model(c)
        m.set_state(st)
        m.step(5)
        outs.append({f: m.download(f) for f in STATE})
        m.close()
    for f in STATE:
        np.testing.assert_array_equal(outs[0][f], outs[1][f], err_msg=f)


@pytest.mark.parametrize("local", [False, True], ids=["mean-profile", "local"])
def test_fp32_mixed_tracks_fp64(gpu_lib, local):
    out = []
    for prec in (cf.FP64, cf.FP32_MIXED):
        c, st = dry(precision=prec, local=local)
        m = api.Model(c)
        m.set_state(st)
        m.step(5)
        out.append({f: m.download(f) for f in ("u", "v", "w", "th")})
        m.close()
    for f in out[0]:
        assert rel_err(out[1][f], out[0][f]) <= 1e-4, f


def test_component_groups_match_fused_step(gpu_lib):
    """One MONC timestep through the per-component entry points equals mgpu_step."""
    c, st = dry()
    res = []
    for fused in (True, False):
        m = api.Model(c)
        m.set_state(st)
        m.step(3)  # reach the steps where damping and forcing act
        if fused:
            m.step(1)
        else:
            api.run_groups(m)
        res.append({f: m.download(f) for f in STATE})
        m.close()
    for f in STATE:
        assert rel_err(res[1][f], res[0][f]) <= 1e-10, f


def test_tangent_linear_refuses_damping(gpu_lib):
    c, st = dry()
    m = api.Model(c)
    m.set_state(st)
    with pytest.raises(api.MgpuError):
        m.tl_step(1)
    m.close()
