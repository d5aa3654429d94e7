"""th_advection (thadvection.F90:129-219) and the geostrophic shear of coriolis on the GPU against
the oracle: the component bit for bit, fused steps to 1e-10, the tiled dynamics kernels bit for
bit against the point kernel, and the component groups against the fused step."""
import numpy as np
import pytest

from monc_b200 import api, config as cf, init as ini
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

STATE = ["u", "v", "w", "th", "zu", "zv", "zw", "zth"]


def rel_err(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def config(n=32, nz=24, precision=cf.FP64, reproducible=0):
    c = cf.dry_cbl_config(n, n, nz, 50.0, 25.0, 1.0, ug=4.0, fcoriol=1e-4, precision=precision)
    c.surface_geostrophic_wind_y = -1.5
    cf.enable_baroclinicity(c, 2e-3, -1e-3)
    c.reproducible = reproducible
    return c


def state(c, seed=7):
    zn = api.reference_profile(c, "zn")
    st = ini.dry_cbl_state(c.nx, c.ny, c.nz, zn, seed=seed, ug=4.0)
    flow = ini.random_flow_state(c.nx, c.ny, c.nz, seed=seed + 1, amp_uv=0.5, amp_w=0.2, amp_th=0.0, ug=4.0)
    for k in ("u", "v", "w"):
        st[k] = flow[k]
    return st


@pytest.mark.parametrize("timestep", [1, 2], ids=["forward", "centred"])
def test_th_advection_component_bit_exact(gpu_lib, timestep):
    c = config(reproducible=1)
    o, m = po.Oracle(c), api.Model(c)
    st = state(c)
    st["sth"] = ini.uniform_noise((c.nz, c.ny, c.nx), 9, 2, 1e-3)
    for name, arr in st.items():
        o.set(api.field_id(name), arr)
        m.upload(name, arr)
    o.set_timestep(timestep)
    m.set_timestep(timestep)
    o.component(api.COMPONENTS["th_advection"])
    m.component("th_advection")
    a, b = m.download("sth"), o.get(api.field_id("sth"))
    assert not np.array_equal(b, st["sth"]), "the term is zero: nothing was tested"
    np.testing.assert_array_equal(a, b)
    m.close()
    o.close()


@pytest.mark.parametrize("reproducible", [0, 1], ids=["fma", "exact"])
def test_fused_steps_with_baroclinicity_match_oracle(gpu_lib, reproducible):
    c = config(n=64, nz=40, reproducible=reproducible)
    o, m = po.Oracle(c), api.Model(c)
    for name, arr in state(c).items():
        o.set(api.field_id(name), arr)
        m.upload(name, arr)
    o.step(4)
    m.step(4)
    for f in STATE + ["p"]:
        e = rel_err(m.download(f), o.get(api.field_id(f)))
        assert e <= 1e-10, f"{f}: rel err {e:.3e}"
    m.close()
    o.close()


def test_tiled_kernels_bit_identical_to_point_kernel_with_baroclinicity(gpu_lib, monkeypatch):
    outs = []
    for point in ("1", "0"):
        monkeypatch.setenv("MGPU_POINT_DYNAMICS", point)
        c = config(n=64, nz=40, reproducible=1)
        m = api.Model(c)
        m.set_state(state(c))
        m.step(3)
        outs.append({f: m.download(f) for f in STATE})
        m.close()
    for f in STATE:
        np.testing.assert_array_equal(outs[0][f], outs[1][f], err_msg=f)


def test_component_groups_match_fused_step_with_baroclinicity(gpu_lib):
    c = config(reproducible=1)
    st = state(c)
    m_fused, m_comp = api.Model(c), api.Model(config(reproducible=1))
    m_fused.set_state(st)
    m_comp.set_state(st)
    for _ in range(3):
        m_fused.step(1)
        api.run_groups(m_comp)
    for f in STATE:
        e = rel_err(m_comp.download(f), m_fused.download(f))
        assert e <= 1e-11, f"{f}: component chain vs fused rel err {e:.3e}"


def test_th_advection_fp32_close_to_fp64(gpu_lib):
    res = []
    for prec in (cf.FP64, cf.FP32_MIXED):
        c = config(n=64, nz=40, precision=prec)
        m = api.Model(c)
        m.set_state(state(c))
        m.step(4)
        res.append({f: m.download(f) for f in ("u", "v", "th")})
        m.close()
    for f in ("u", "v", "th"):
        assert rel_err(res[1][f], res[0][f]) <= 1e-4, f


def test_adjoint_refuses_th_advection(gpu_lib):
    c = config()
    m = api.Model(c)
    m.set_state(state(c))
    with pytest.raises(api.MgpuError):
        m.tl_step(1)
    m.close()
