"""Restart from a checkpoint on the GPU: a run interrupted by a checkpoint write, and continued by a
new model that reads it, ends bit for bit where the uninterrupted run does -- with damping (its
mean profiles are in the file), cfltest's adaptive dtm (its state is in the file), moist fields,
the FP32-mixed path (whose FP32 fields survive the FP64 file exactly), and the Galilean frame
(ugal, vgal in the file)."""
import numpy as np
import pytest

from monc_b200 import api, config as cf, init as ini

pytestmark = pytest.mark.gpu

NX, NY, NZ = 32, 32, 24
FIELDS = ["u", "v", "w", "th", "zu", "zv", "zw", "zth", "p"]


def dry(precision=cf.FP64):
    c = cf.dry_cbl_config(NX, NY, NZ, 50.0, 25.0, 1.0, ug=5.0, fcoriol=1e-4, precision=precision)
    cf.enable_damping(c, 0.02, 300.0, 150.0)
    cf.enable_cfl(c, frequency=2, dtmmax=2.0)
    st = ini.random_flow_state(NX, NY, NZ, seed=4, amp_uv=2.0, amp_w=0.5, amp_th=0.5, ug=5.0)
    return c, st


def moist():
    z = cf.stretched_levels(NZ, 20.0, 60.0, ztop=1000.0)
    c = cf.moist_config(NX, NY, z, 35.0, 0.3, shf_wm2=10.0, lhf_wm2=50.0, max_height_cloud=700.0)
    cf.enable_subsidence(c, [0.0, 1000.0], [0.0, -0.005], theta=True, q=True)
    st = ini.moist_layer_state(NX, NY, NZ, api.reference_profile(c, "zn"), seed=2)
    flow = ini.random_flow_state(NX, NY, NZ, seed=5, amp_uv=0.5, amp_w=0.2)
    for k in ("u", "v", "w", "zu", "zv", "zw"):
        st[k] = flow[k]
    return c, st


def restart_matches(c, st, n1, n2, path, extra=()):
    names = FIELDS + list(extra)
    a = api.Model(c)
    a.set_state(st)
    a.step(n1 + n2)
    ref = {f: a.download(f) for f in names}
    ref_ts, ref_dtm = a.reductions().timestep, a.reductions().dtm
    ref_gal = (a.reductions().ugal, a.reductions().vgal)
    a.close()
    b = api.Model(c)
    b.set_state(st)
    b.step(n1)
    b.checkpoint_write(path)
    keep = bool(c.damping_enabled or c.l_subs_pl_theta or c.l_subs_pl_q)
    mp = b.mean_profiles() if keep else {}
    b.close()
    d = api.Model(c)
    d.checkpoint_read(path)
    assert d.reductions().timestep == n1 + 1
    # every mean profile comes back: olz*bar and olubar, olvbar, olthbar, olqbar(n)
    for n, prof in (d.mean_profiles() if keep else {}).items():
        np.testing.assert_array_equal(prof, mp[n], err_msg=n)
    d.step(n2)
    for f in names:
        np.testing.assert_array_equal(d.download(f), ref[f], err_msg=f)
    assert d.reductions().timestep == ref_ts and d.reductions().dtm == ref_dtm
    assert (d.reductions().ugal, d.reductions().vgal) == ref_gal
    d.close()


def test_dry_restart_with_damping_and_adaptive_dtm(gpu_lib, tmp_path):
    c, st = dry()
    restart_matches(c, st, 4, 5, str(tmp_path / "dry.nc"))


def test_moist_restart_with_subsidence(gpu_lib, tmp_path):
    c, st = moist()
    restart_matches(c, st, 3, 4, str(tmp_path / "moist.nc"), extra=("q0", "q1", "zq0", "zq1"))


def test_fp32_mixed_restart(gpu_lib, tmp_path):
    c, st = dry(cf.FP32_MIXED)
    restart_matches(c, st, 4, 3, str(tmp_path / "fp32.nc"))


def test_galilean_restart(gpu_lib, tmp_path):
    """The frame velocity travels in the file (ugal, vgal), so a restarted run stays in it."""
    c, st = dry()
    cf.enable_galilean(c)
    restart_matches(c, st, 4, 5, str(tmp_path / "gal.nc"))
