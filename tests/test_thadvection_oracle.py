"""th_advection and the geostrophic shear (thadvection.F90:129-219, coriolis.F90:155-163) without a
GPU: the oracle's restatement against the formulas, and the library's host-built geostrophic
profile against the oracle's.

With baroclinicity_use_geostrophic_shear the geostrophic wind grows with height, ug(k) = ug0 +
rate_x zn(k), and th_advection adds ((v + vgal) mfx - (u + ugal) mfy), mfx = rate_x thref0 fcoriol
/ G, to sth at levels 2..nz.  MONC advects the mean baroclinicity only with passive q.
"""
import numpy as np

from monc_b200 import api, config as cf, init as ini
from oracle import pyoracle as po

N, NZ = 16, 12


def cfg_baroclinic(rate_x=2e-3, rate_y=-1e-3):
    c = cf.dry_cbl_config(N, N, NZ, 50.0, 25.0, 1.0, ug=4.0, fcoriol=1e-4)
    c.surface_geostrophic_wind_y = -1.5
    return cf.enable_baroclinicity(c, rate_x, rate_y)


def test_oracle_th_advection_is_the_baroclinicity_term():
    c = cfg_baroclinic()
    o = po.Oracle(c)
    st = ini.random_flow_state(N, N, NZ, seed=3, ug=4.0)
    sth0 = ini.uniform_noise((NZ, N, N), 5, 1, 1e-2)
    for name, arr in st.items():
        o.set(api.field_id(name), arr)
    o.set(api.field_id("sth"), sth0)
    o.set_timestep(2)
    o.component(api.COMPONENTS["th_advection"])
    got = o.get(api.field_id("sth"))
    fcg = c.fcoriol / c.G
    mfx = c.rate_change_geostrophic_wind_x * c.thref0 * fcg
    mfy = c.rate_change_geostrophic_wind_y * c.thref0 * fcg
    want = sth0.copy()
    want[1:] = sth0[1:] + ((st["v"][1:] + 0.0) * mfx - (st["u"][1:] + 0.0) * mfy)
    np.testing.assert_array_equal(got, want)


def test_oracle_th_advection_needs_passive_q_and_the_switch():
    st = ini.random_flow_state(N, N, NZ, seed=4)
    sth0 = ini.uniform_noise((NZ, N, N), 6, 1, 1e-2)
    for tweak in ("disabled", "no_shear", "active_q"):
        c = cfg_baroclinic()
        if tweak == "disabled":
            c.th_advection_enabled = 0
        elif tweak == "no_shear":
            c.baroclinicity_use_geostrophic_shear = 0
        else:
            c.passive_q = 0
            c.number_q_fields = 2
        o = po.Oracle(c)
        for name, arr in st.items():
            o.set(api.field_id(name), arr)
        o.set(api.field_id("sth"), sth0)
        o.set_timestep(2)
        o.component(api.COMPONENTS["th_advection"])
        np.testing.assert_array_equal(o.get(api.field_id("sth")), sth0, err_msg=tweak)


def test_geostrophic_shear_profile_library_equals_oracle():
    c = cfg_baroclinic()
    o = po.Oracle(c)
    zn = o.profile("zn")
    for axis, surface, rate in (("x", 4.0, c.geostrophic_wind_rate_of_change_in_x),
                                ("y", -1.5, c.geostrophic_wind_rate_of_change_in_y)):
        lib = api.reference_profile(c, f"geostrophic_wind_{axis}")
        orc = o.profile(f"geostrophic_wind_{axis}")
        np.testing.assert_array_equal(lib, orc)
        np.testing.assert_array_equal(orc, surface + rate * zn)
