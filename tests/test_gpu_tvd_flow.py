"""TVD advection of the flow fields on the GPU (advection_flow_fields = tvd) against the oracle:
the tvd_advection component's u, v, w and theta sources, and fused steps (forward and centred,
dry and moist), FP64 with unfused multiply-adds; FP32-mixed within FP32 rounding."""
import numpy as np
import pytest

from monc_b200 import api, config as cf, init as ini
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

NX, NY, NZ = 32, 32, 24
STATE = ["u", "v", "w", "th", "zu", "zv", "zw", "zth"]


def rel_err(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def dry(precision=cf.FP64):
    c = cf.dry_cbl_config(NX, NY, NZ, 50.0, 25.0, 0.5, ug=5.0, fcoriol=1e-4, precision=precision)
    c.advection_flow_fields = cf.ADVECT_TVD
    c.reproducible = 1
    st = ini.random_flow_state(NX, NY, NZ, seed=6, amp_uv=1.0, amp_w=0.3, amp_th=0.5, ug=5.0)
    return c, st


def pair(c, st):
    o, m = po.Oracle(c), api.Model(c)
    for k, v in st.items():
        o.set(api.field_id(k), v)
        m.upload(k, v)
    return o, m


@pytest.mark.parametrize("timestep", [1, 2], ids=["forward", "centred"])
def test_tvd_component_with_flow_matches_oracle(gpu_lib, timestep):
    c, st = dry()
    o, m = pair(c, st)
    z = np.zeros((NZ, NY, NX))
    for f in ("su", "sv", "sw", "sth"):
        o.set(api.field_id(f), z)
        m.upload(f, z)
    o.set_timestep(timestep)
    m.set_timestep(timestep)
    o.component(api.COMPONENTS["tvd_advection"])
    m.component("tvd_advection")
    for f in ("su", "sv", "sw", "sth"):
        a, b = m.download(f), o.get(api.field_id(f))
        assert rel_err(a, b) <= 1e-12, f
    assert np.abs(m.download("sw")).max() > 0
    # with TVD carrying the flow, pw_advection leaves the flow sources alone
    m.upload("su", z)
    m.component("pw_advection")
    assert np.abs(m.download("su")).max() == 0.0
    m.close()


@pytest.mark.parametrize("nsteps", [1, 3])
def test_fused_steps_with_tvd_flow_match_oracle(gpu_lib, nsteps):
    c, st = dry()
    o, m = pair(c, st)
    o.step(nsteps)
    m.step(nsteps)
    for f in STATE + ["p"]:
        assert rel_err(m.download(f), o.get(api.field_id(f))) <= 1e-10, f
    m.close()


def test_moist_steps_with_tvd_flow_match_oracle(gpu_lib):
    z = cf.stretched_levels(NZ, 20.0, 60.0, ztop=1000.0)
    c = cf.moist_config(NX, NY, z, 35.0, 0.3, shf_wm2=10.0, lhf_wm2=50.0, max_height_cloud=700.0)
    c.advection_flow_fields = cf.ADVECT_TVD
    c.reproducible = 1
    st = ini.moist_layer_state(NX, NY, NZ, api.reference_profile(c, "zn"), seed=2)
    flow = ini.random_flow_state(NX, NY, NZ, seed=5, amp_uv=0.5, amp_w=0.2)
    for k in ("u", "v", "w", "zu", "zv", "zw"):
        st[k] = flow[k]
    o, m = pair(c, st)
    o.step(3)
    m.step(3)
    for f in STATE + ["q0", "q1", "p"]:
        assert rel_err(m.download(f), o.get(api.field_id(f))) <= 1e-10, f
    m.close()


@pytest.mark.parametrize("precision", [cf.FP64, cf.FP32_MIXED], ids=["fp64", "fp32"])
def test_tiled_tvd_flow_bit_identical_to_point_kernel(gpu_lib, monkeypatch, precision):
    """Centred steps advect u, v, w in three tiled kernels (one per component, faces shared through
    shared memory, the z face carried up the column) and the momentum kernel takes their sources;
    the point kernel evaluates tvd_flow_point per point.  Same expressions, so the same bits, for
    any split of the levels into chunks."""
    c = cf.dry_cbl_config(64, 64, 40, 50.0, 25.0, 0.5, ug=5.0, fcoriol=1e-4, precision=precision)
    c.advection_flow_fields = cf.ADVECT_TVD
    c.reproducible = 1
    st = ini.random_flow_state(64, 64, 40, seed=9, amp_uv=1.0, amp_w=0.3, amp_th=0.5, ug=5.0)
    outs = []
    for point, chunks in (("1", "0"), ("0", "0"), ("0", "1"), ("0", "4"), ("0", "19")):
        monkeypatch.setenv("MGPU_POINT_DYNAMICS", point)
        monkeypatch.setenv("MGPU_LEVEL_CHUNKS", chunks)
        m = api.Model(c)
        m.set_state(st)
        m.step(3)
        outs.append({f: m.download(f) for f in STATE})
        m.close()
    for n, res in enumerate(outs[1:], 1):
        for f in STATE:
            np.testing.assert_array_equal(outs[0][f], res[f], err_msg=f"{f} (setting {n})")


def test_fp32_mixed_tvd_flow_tracks_fp64(gpu_lib):
    out = []
    for prec in (cf.FP64, cf.FP32_MIXED):
        c, st = dry(prec)
        m = api.Model(c)
        m.set_state(st)
        m.step(3)
        out.append({f: m.download(f) for f in ("u", "v", "w", "th")})
        m.close()
    for f in out[0]:
        assert rel_err(out[1][f], out[0][f]) <= 1e-4, f


def test_adjoint_refuses_tvd_flow(gpu_lib):
    c, st = dry()
    m = api.Model(c)
    m.set_state(st)
    with pytest.raises(api.MgpuError):
        m.tl_step(1)
    m.close()
