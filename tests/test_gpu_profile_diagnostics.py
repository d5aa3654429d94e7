"""profile_diagnostics on the GPU (mgpu_profile_diagnostics) against the oracle: the sums after
fused steps (dry and moist, FP64), the mean profiles they read (olubar, olvbar, olthbar from the
fused step against those of the per-component path), FP32-mixed against FP64, and the
field_value_retrieval of the component descriptor.  Sums over different orders agree to
rounding: 1e-10 relative, with an absolute floor for the rows that cancel (sum of w, fluxes).
"""
import numpy as np
import pytest

from monc_b200 import api, config as cf, init as ini
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

NX, NY, NZ = 32, 32, 24


def dry(precision=cf.FP64):
    c = cf.dry_cbl_config(NX, NY, NZ, 50.0, 25.0, 0.5, ug=5.0, fcoriol=1e-4, precision=precision)
    c.reproducible = 1
    c.profile_diagnostics_enabled = 1
    st = ini.random_flow_state(NX, NY, NZ, seed=6, amp_uv=1.0, amp_w=0.3, amp_th=0.5, ug=5.0)
    return c, st


def moist():
    z = cf.stretched_levels(NZ, 20.0, 60.0, ztop=1000.0)
    c = cf.moist_config(NX, NY, z, 35.0, 0.3, shf_wm2=10.0, lhf_wm2=50.0, max_height_cloud=700.0)
    c.reproducible = 1
    c.profile_diagnostics_enabled = 1
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


def close(a, b, rtol):
    floor = 1e-12 * NX * NY
    assert np.all(np.abs(a - b) <= rtol * np.abs(b).max() + floor)


@pytest.mark.parametrize("case", ["dry", "moist"])
def test_sums_match_oracle(gpu_lib, case):
    c, st = dry() if case == "dry" else moist()
    o, m = pair(c, st)
    for steps in (1, 3):  # after the forward step, then after centred steps
        o.step(steps)
        m.step(steps)
        po_, pg = o.profile_diagnostics(), m.profile_diagnostics()
        assert list(pg) == list(po_) and len(pg) == (16 if case == "moist" else 11)
        for name in po_:
            close(pg[name], po_[name], 1e-10)
        mo, mg = o.mean_profiles(), m.mean_profiles()
        for name in ("olubar", "olvbar", "olthbar"):
            close(mg[name], mo[name], 1e-12)
    m.close()


def test_fused_means_match_component_path(gpu_lib):
    """The fused step takes olubar, olvbar, olthbar from u + ugal and the time-smoothed old theta;
    the per-component path from MONC's own fields at solver time."""
    c, st = dry()
    res = []
    for fused in (True, False):
        m = api.Model(c)
        m.set_state(st)
        m.step(3)
        if fused:
            m.step(1)
        else:
            api.run_groups(m)
        res.append((m.mean_profiles(), m.profile_diagnostics()))
        m.close()
    for name in ("olubar", "olvbar", "olthbar", "olzubar", "olzthbar"):
        close(res[1][0][name], res[0][0][name], 1e-12)
    for name in res[0][1]:
        close(res[1][1][name], res[0][1][name], 1e-10)


def test_fp32_mixed_tracks_fp64(gpu_lib):
    out = []
    for prec in (cf.FP64, cf.FP32_MIXED):
        c, st = dry(prec)
        m = api.Model(c)
        m.set_state(st)
        m.step(4)
        out.append(m.profile_diagnostics())
        m.close()
    for name in ("u_wind_total_local", "theta_total_local", "ww_total_local", "th2_total_local"):
        close(out[1][name], out[0][name], 1e-4)


def test_field_value_retrieval_and_refusals(gpu_lib):
    c, st = dry()
    m = api.Model(c)
    m.set_state(st)
    m.step(2)
    desc = api.component_descriptor("profile_diagnostics")
    assert "theta_total_local" in desc.published_fields
    np.testing.assert_array_equal(desc.field_value_retrieval(m, "theta_total_local"),
                                  m.profile_diagnostics()["theta_total_local"])
    with pytest.raises(KeyError):
        desc.field_value_retrieval(m, "rh_total_local")  # a dry model publishes no moist sums
    m.close()
    c.profile_diagnostics_enabled = 0
    m = api.Model(c)
    with pytest.raises(api.MgpuError):
        m.profile_diagnostics()
    m.close()
