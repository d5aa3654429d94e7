"""cfltest on the GPU (adaptive dtm inside mgpu_step) against the oracle: the same evaluation
schedule and Courant numbers, the same dtm sequence, and the fields after steps of varying dtm;
the device gather against numpy; the stop below cfl_dtmmin; FP32-mixed runs."""
import numpy as np
import pytest

from monc_b200 import api, config as cf, init as ini
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

NX, NY, NZ = 32, 32, 24
KEYS = ["dtm", "dtm_new", "absolute_new_dtm", "cvel", "cvis", "cfl_number", "cvel_x", "cvel_y", "cvel_z"]


def setup(precision=cf.FP64, dtm=1.0, amp=2.0, **cfl):
    c = cf.dry_cbl_config(NX, NY, NZ, 50.0, 25.0, dtm, ug=5.0, fcoriol=1e-4, precision=precision)
    cf.enable_cfl(c, **cfl)
    c.reproducible = 1
    st = ini.random_flow_state(NX, NY, NZ, seed=3, amp_uv=amp, amp_w=0.5, ug=5.0)
    return c, st


def test_cfl_sequence_matches_oracle(gpu_lib):
    c, st = setup(frequency=3, dtmmax=2.0)
    o = po.Oracle(c)
    m = api.Model(c)
    for k, v in st.items():
        o.set(api.FIELDS[k], v)
        m.upload(k, v)
    changed = 0
    for n in range(1, 13):
        o.step(1)
        m.step(1)
        so, r = o.cfl_state(), m.reductions()
        assert r.cfl_evaluations == so["cfl_evaluations"] and r.last_cfl_timestep == so["last_cfl_timestep"], n
        for k in KEYS:
            a, b = getattr(r, k), so[k]
            assert abs(a - b) <= 1e-12 * max(abs(b), 1e-30), (n, k, a, b)
        changed += r.dtm != c.dtm
    assert changed > 0  # the timestep did change
    for f in ("u", "v", "w", "th", "zu", "zv", "zw", "zth", "p"):
        a, b = m.download(f), o.get(api.FIELDS[f])
        assert np.abs(a - b).max() <= 1e-10 * np.abs(b).max(), f
    m.close()


def test_device_gather_matches_numpy(gpu_lib):
    c, st = setup(frequency=3)
    m = api.Model(c)
    m.set_state(st)
    m.step(2)
    g = m.cfl_gather()
    zu, zv, zw = (m.download(f) for f in ("zu", "zv", "zw"))
    vis, diff = m.download("vis"), m.download("diff")
    rdzn = m.profile("rdzn")
    cx2 = cy2 = (1.0 / 50.0) ** 2
    expect = [zu[1:].min(), zu[1:].max(), zv[1:].min(), zv[1:].max(),
              max(0.0, max((np.abs(zw[k - 1]) * rdzn[k]).max() for k in range(2, NZ))),
              max(0.0, max((np.maximum(vis[k - 1], diff[k - 1]) * ((rdzn[k] * rdzn[k] + cx2) + cy2)).max()
                           for k in range(2, NZ)))]
    np.testing.assert_array_equal(g, np.array(expect))
    m.close()


def test_cfl_stop_below_dtmmin(gpu_lib):
    c, st = setup(frequency=2, dtmmin=0.9)
    m = api.Model(c)
    m.set_state(st)
    with pytest.raises(api.MgpuError) as e:
        m.step(1)
    assert e.value.code == api.ERR_CFL
    m.close()


def test_fp32_mixed_cfl_follows_fp64(gpu_lib):
    out = []
    for prec in (cf.FP64, cf.FP32_MIXED):
        c, st = setup(precision=prec, frequency=3, dtmmax=2.0)
        m = api.Model(c)
        m.set_state(st)
        dtms = []
        for _ in range(8):
            m.step(1)
            dtms.append(m.reductions().dtm)
        out.append(np.array(dtms))
        m.close()
    np.testing.assert_allclose(out[1], out[0], rtol=1e-5)


def test_adjoint_refuses_adaptive_dtm(gpu_lib):
    c, st = setup(frequency=3)
    m = api.Model(c)
    m.set_state(st)
    with pytest.raises(api.MgpuError):
        m.tl_step(1)
    m.close()


def galilean_pair(precision=cf.FP64, ugal=None, vgal=None, cfl=True):
    c, st = setup(precision=precision, frequency=3, dtmmax=2.0)
    if not cfl:
        c.cfl_enabled = 0
    cf.enable_galilean(c, ugal, vgal)
    return c, st


def test_galilean_sequence_matches_oracle(gpu_lib):
    """The frame follows the middle of the zu, zv range at each evaluation; the pressure terms move
    the flow into it; the dtm and frame sequences and the fields after 12 steps match the oracle."""
    c, st = galilean_pair()
    o = po.Oracle(c)
    m = api.Model(c)
    for k, v in st.items():
        o.set(api.FIELDS[k], v)
        m.upload(k, v)
    for n in range(1, 13):
        o.step(1)
        m.step(1)
        so, r = o.cfl_state(), m.reductions()
        for k in KEYS + ["ugal", "vgal"]:
            a, b = getattr(r, k), so[k]
            assert abs(a - b) <= 1e-12 * max(abs(b), 1e-30), (n, k, a, b)
    assert abs(m.reductions().ugal) > 3.0  # the frame took up the mean wind
    for f in ("u", "v", "w", "th", "zu", "zv", "zw", "zth", "p"):
        a, b = m.download(f), o.get(api.FIELDS[f])
        assert np.abs(a - b).max() <= 1e-10 * np.abs(b).max(), f
    m.close()


def test_fixed_galilean_frame_matches_oracle(gpu_lib):
    """fix_ugal, fix_vgal without cfltest: a constant moving frame."""
    c, st = galilean_pair(ugal=3.0, vgal=-1.5, cfl=False)
    o = po.Oracle(c)
    m = api.Model(c)
    for k, v in st.items():
        o.set(api.FIELDS[k], v)
        m.upload(k, v)
    o.step(6)
    m.step(6)
    assert (m.reductions().ugal, m.reductions().vgal) == (3.0, -1.5)
    for f in ("u", "v", "w", "th", "zu", "zv", "zw", "zth", "p"):
        a, b = m.download(f), o.get(api.FIELDS[f])
        assert np.abs(a - b).max() <= 1e-10 * np.abs(b).max(), f
    m.close()


def test_galilean_component_groups_match_fused_step(gpu_lib):
    """The per-component entry points, with the frame set through mgpu_set_galilean_velocity, step
    as mgpu_step does."""
    c, st = galilean_pair(ugal=3.0, vgal=-1.5, cfl=False)
    res = []
    for fused in (True, False):
        m = api.Model(c)
        m.set_state(st)
        m.step(2)
        if fused:
            m.step(1)
        else:
            m.set_galilean_velocity(3.0, -1.5)
            api.run_groups(m)
        res.append({f: m.download(f) for f in ("u", "v", "w", "th", "zu", "zv", "zw", "zth")})
        m.close()
    for f in res[0]:
        b = res[0][f]
        assert np.abs(res[1][f] - b).max() <= 1e-10 * np.abs(b).max(), f


def test_fp32_mixed_galilean_follows_fp64(gpu_lib):
    out = []
    for prec in (cf.FP64, cf.FP32_MIXED):
        c, st = galilean_pair(precision=prec)
        m = api.Model(c)
        m.set_state(st)
        seq = []
        for _ in range(8):
            m.step(1)
            r = m.reductions()
            seq.append((r.dtm, r.ugal, r.vgal))
        out.append(np.array(seq))
        m.close()
    np.testing.assert_allclose(out[1], out[0], rtol=1e-5, atol=1e-5)


def test_adjoint_refuses_moving_frame(gpu_lib):
    c, st = galilean_pair(ugal=3.0, cfl=False)
    m = api.Model(c)
    m.set_state(st)
    with pytest.raises(api.MgpuError):
        m.tl_step(1)
    m.close()
