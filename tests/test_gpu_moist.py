"""Moist path on the GPU against the oracle: simplecloud saturation adjustment, vapour and liquid
advected by TVD, moist Richardson number in the Smagorinsky closure, liquid loading in the
buoyancy, and negative-q clipping in stepfields.

simplecloud calls exp and pow, whose CUDA and C-library results can differ in the last bit, so
the component is held to 1e-12 relative; full steps to 1e-10 relative per field.
"""
import numpy as np
import pytest

from monc_b200 import api, config as cf, init as ini
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

NX, NY, NZ = 32, 32, 24
FIELDS = ["u", "v", "w", "th", "zu", "zv", "zw", "zth", "q0", "q1", "zq0", "zq1", "p"]


def rel_err(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def moist_pair(precision=cf.FP64, n_tracers=0, max_height_cloud=700.0, reproducible=0):
    z = cf.stretched_levels(NZ, 20.0, 60.0, ztop=1000.0)
    c = cf.moist_config(NX, NY, z, 35.0, 0.3, shf_wm2=10.0, lhf_wm2=50.0, max_height_cloud=max_height_cloud,
                        n_tracers=n_tracers, precision=precision)
    c.reproducible = reproducible
    o = po.Oracle(c)
    m = api.Model(c)
    st = ini.moist_layer_state(NX, NY, NZ, o.profile("zn"), seed=2, n_tracers=n_tracers)
    flow = ini.random_flow_state(NX, NY, NZ, seed=5, amp_uv=0.5, amp_w=0.2)
    for k in ("u", "v", "w", "zu", "zv", "zw"):
        st[k] = flow[k]
    for name, arr in st.items():
        o.set(api.field_id(name), arr)
        m.upload(name, arr)
    return o, m


@pytest.mark.parametrize("timestep", [1, 2], ids=["forward", "centred"])
def test_simplecloud_component_matches_oracle(gpu_lib, timestep):
    o, m = moist_pair()
    shape = (NZ, NY, NX)
    # sources that push some points over saturation and evaporate cloud above max_height_cloud
    ql = np.where(ini.uniform_noise(shape, 8, 1, 1.0) > 0, 2e-4, 0.0)
    src = {"sth": ini.uniform_noise(shape, 9, 2, 1e-3), "sq0": 1e-5 + ini.uniform_noise(shape, 9, 3, 1e-5),
           "sq1": ini.uniform_noise(shape, 9, 4, 1e-6), "q1": ql, "zq1": ql}
    for name, arr in src.items():
        o.set(api.field_id(name), arr)
        m.upload(name, arr)
    o.set_timestep(timestep)
    m.set_timestep(timestep)
    o.component(api.COMPONENTS["simplecloud"])
    m.component("simplecloud")
    for f in ("sth", "sq0", "sq1"):
        a, b = m.download(f), o.get(api.field_id(f))
        assert rel_err(a, b) <= 1e-12, f
    # the adjustment did something on both sides of max_height_cloud
    assert np.abs(m.download("sq1") - src["sq1"]).max() > 0
    m.close()


@pytest.mark.parametrize("n_tracers", [0, 1], ids=["vapour-liquid", "with-tracer"])
@pytest.mark.parametrize("nsteps", [1, 3])
def test_moist_fused_step_matches_oracle(gpu_lib, nsteps, n_tracers):
    """Full steps of the contracted (FMA) build: with vapour and liquid only the centred steps run
    the one-kernel moist step, with a tracer the per-scalar kernels and the cloud step."""
    o, m = moist_pair(n_tracers=n_tracers)
    o.step(nsteps)
    m.step(nsteps)
    for f in FIELDS + (["q2", "zq2"] if n_tracers else []):
        assert rel_err(m.download(f), o.get(api.field_id(f))) <= 1e-10, f
    assert m.download("q1").max() > 0  # cloud has formed
    m.close()


def test_moist_fp32_mixed_tracks_fp64(gpu_lib):
    """Ten steps of the FP32-mixed path stay within 1e-4 of FP64 in the mean theta and vapour
    profiles."""
    res = []
    for prec in (cf.FP64, cf.FP32_MIXED):
        o, m = moist_pair(precision=prec)
        m.step(10)
        res.append((m.mean_profile("th"), m.mean_profile("q0")))
        m.close()
    for a, b in zip(res[1], res[0]):
        assert np.abs(a - b).max() <= 1e-4 * max(np.abs(b).max(), 1e-3)


@pytest.mark.parametrize("timestep", [1, 2], ids=["forward", "centred"])
def test_fp32_surface_ghost_theta_keeps_the_perturbation(gpu_lib, timestep):
    """lower_bc's ghost value theta(1) = theta(2) + flux dzn / diff + thref(2) - thref(1) in FP32
    carries theta(2) and the flux term (up to 1.4 K here) at FP32 precision, within 2e-6 K, not at
    the spacing of thref = 289 K (3e-5 K) that MONC's order of the sum would round theta(2) to."""
    out = []
    for prec in (cf.FP64, cf.FP32_MIXED):
        _, m = moist_pair(precision=prec)
        m.set_timestep(timestep)
        m.component("lower_bc")
        out.append(m.download("th" if timestep == 1 else "zth")[0])
        m.close()
    assert np.abs(out[0]).max() > 1e-3  # the perturbation and the surface flux term are there
    assert np.abs(out[1] - out[0]).max() <= 2e-6


@pytest.mark.parametrize("n_tracers", [0, 1], ids=["vapour-liquid", "with-tracer"])
@pytest.mark.parametrize("precision", [cf.FP64, cf.FP32_MIXED], ids=["fp64", "fp32"])
def test_moist_tiled_bit_identical_to_point_kernel(gpu_lib, monkeypatch, precision, n_tracers):
    """The tiled moist step reproduces the point kernel bit for bit, for any split of the levels:
    with vapour and liquid only, one kernel for theta and both q fields (sources, cloud and
    stepping included); with a tracer as well, one kernel per scalar and the cloud step."""
    outs = []
    extra = ["q2", "zq2"] if n_tracers else []
    for point, chunks in (("1", "0"), ("0", "0"), ("0", "1"), ("0", "3"), ("0", "7")):
        monkeypatch.setenv("MGPU_POINT_DYNAMICS", point)
        monkeypatch.setenv("MGPU_LEVEL_CHUNKS", chunks)
        o, m = moist_pair(precision=precision, n_tracers=n_tracers, reproducible=1)
        m.step(4)
        outs.append({f: m.download(f) for f in FIELDS + extra})
        m.close()
    for res in outs[1:]:
        for f in outs[0]:
            np.testing.assert_array_equal(outs[0][f], res[f], err_msg=f)
