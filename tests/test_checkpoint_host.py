"""Checkpoint files in MONC's layout (writecheckpoint.F90, checkpointcommon.F90), written and read
by the library's host codec without a GPU, and checked against an independent NetCDF reader and
writer (scipy.io.netcdf_file):

* a write / read round trip returns every field, the mean profiles and the step state exactly;
* the file is NetCDF classic (64-bit offsets) with MONC's dimensions, variable names, dimension
  order (x, y, zn with z fastest), attributes, options database and q indices;
* a classic-format file written by scipy in MONC's layout (what a serial MONC run writes) is read
  back by the library;
* a file whose grid differs from the model's is refused.
"""
import os

import numpy as np
import pytest
from scipy.io import netcdf_file

from monc_b200 import api, config as cf, init as ini

NX, NY, NZ = 16, 8, 12


def dry_case():
    c = cf.dry_cbl_config(NX, NY, NZ, 50.0, 25.0, 1.0, ug=3.0)
    cf.enable_damping(c, 0.01, 150.0, 80.0)
    st = ini.random_flow_state(NX, NY, NZ, seed=3, amp_uv=1.0, amp_w=0.3, amp_th=0.5, ug=3.0)
    st["p"] = np.random.default_rng(1).normal(size=(NZ, NY, NX))
    # mgpu_mean_profiles' rows: olzubar, olzvbar, olzthbar, then olubar, olvbar, olthbar
    mean = np.random.default_rng(2).normal(size=(6, NZ))
    return c, st, mean


def moist_case():
    z = cf.stretched_levels(NZ, 20.0, 60.0, ztop=500.0)
    c = cf.moist_config(NX, NY, z, 35.0, 0.3)
    st = ini.moist_layer_state(NX, NY, NZ, api.reference_profile(c, "zn"), seed=2, inversion=300.0)
    st["p"] = np.zeros((NZ, NY, NX))
    return c, st


def meta(**kw):
    m = api.CheckpointMeta(timestep=7, last_cfl_timestep=5, time=7.25, dtm=1.0, dtm_new=1.05,
                           absolute_new_dtm=1.1, ugal=0.0, vgal=0.0)
    for k, v in kw.items():
        setattr(m, k, v)
    return m


def test_round_trip(tmp_path):
    c, st, mean = dry_case()
    path = str(tmp_path / "ck.nc")
    api.checkpoint_write_host(c, path, st, meta(), mean)
    f, m, md = api.checkpoint_read_host(c, path)
    for k in api.CHECKPOINT_FIELDS:
        np.testing.assert_array_equal(f[k], st[k], err_msg=k)
    np.testing.assert_array_equal(m, mean)
    assert (md.timestep, md.last_cfl_timestep) == (7, 5)
    assert (md.time, md.dtm, md.dtm_new, md.absolute_new_dtm) == (7.25, 1.0, 1.05, 1.1)


def test_layout_read_by_scipy(tmp_path):
    c, st, mean = dry_case()
    path = str(tmp_path / "ck.nc")
    api.checkpoint_write_host(c, path, st, meta(), mean)
    nc = netcdf_file(path, "r", mmap=False)
    try:
        assert nc.version_byte == 2
        assert nc.title == b"MONC checkpoint file" and len(nc.created) > 0
        dims = nc.dimensions
        assert (dims["x"], dims["y"], dims["z"], dims["zn"], dims["string"], dims["kvp"]) == (NX, NY, NZ, NZ, 150, 2)
        v = nc.variables
        for name, src in (("u_nogal", "u"), ("v_nogal", "v"), ("w", "w"), ("th", "th"), ("zu", "zu"),
                          ("zv", "zv"), ("zw", "zw"), ("zth", "zth"), ("p", "p")):
            assert v[name].dimensions == ("x", "y", "zn"), name
            np.testing.assert_array_equal(v[name].data, st[src].transpose(2, 1, 0), err_msg=name)
        for name, row in (("olzubar", 0), ("olzvbar", 1), ("olzthbar", 2), ("olubar", 3), ("olvbar", 4),
                          ("olthbar", 5)):
            assert v[name].dimensions == ("z",), name
            np.testing.assert_array_equal(v[name].data, mean[row])
        np.testing.assert_array_equal(v["z"].data, api.reference_profile(c, "z"))
        np.testing.assert_array_equal(v["zn"].data, api.reference_profile(c, "zn"))
        assert v["z"].units == b"m" and v["x_resolution"].units == b"m"
        assert float(v["x_resolution"].data) == 50.0 and float(v["x_top"].data) == NX * 50.0
        assert int(v["timestep"].data) == 7 and v["timestep"].data.dtype.kind == "i"
        assert int(v["nqfields"].data) == 0
        opts = v["options_database"].data
        kv = {b"".join(opts[q, 0]).rstrip(b"\0").decode(): b"".join(opts[q, 1]).rstrip(b"\0").decode()
              for q in range(opts.shape[0])}
        assert kv["x_size"] == str(NX) and kv["z_size"] == str(NZ)
        assert float(kv["dxx"]) == 50.0 and kv["damping_enabled"] == ".true."
        assert kv["advection_flow_fields"] == "pw"
        order = list(v.keys())
        assert order.index("options_database") < order.index("z") < order.index("u_nogal") < order.index("timestep")
    finally:
        nc.close()


def test_moist_q_fields_and_indices(tmp_path):
    c, st = moist_case()
    path = str(tmp_path / "ck.nc")
    mean = np.random.default_rng(4).normal(size=(10, NZ))  # olz*bar (3 + 2 q), ol*bar (3 + 2 q)
    api.checkpoint_write_host(c, path, st, meta(), mean)
    nc = netcdf_file(path, "r", mmap=False)
    try:
        v = nc.variables
        assert v["q"].dimensions == ("q", "x", "y", "zn") and nc.dimensions["q"] == 2
        np.testing.assert_array_equal(v["q"].data[0], st["q0"].transpose(2, 1, 0))
        np.testing.assert_array_equal(v["zq"].data[1], st["zq1"].transpose(2, 1, 0))
        qi = v["q_indicies"].data
        names = [b"".join(qi[q, 0]).rstrip(b"\0").decode() for q in range(qi.shape[0])]
        assert names == ["vapour", "cloud_liquid_mass"]
        assert int(v["nqfields"].data) == 2
        for name, rows in (("olzqbar", mean[3:5]), ("olqbar", mean[8:10])):
            assert v[name].dimensions == ("q", "z"), name
            np.testing.assert_array_equal(v[name].data, rows, err_msg=name)
    finally:
        nc.close()
    f, m, _ = api.checkpoint_read_host(c, path)
    for k in ("q0", "q1", "zq0", "zq1"):
        np.testing.assert_array_equal(f[k], st[k], err_msg=k)
    np.testing.assert_array_equal(m, mean)


def test_reads_a_classic_file_in_monc_layout(tmp_path):
    """A CDF-1 file as a serial MONC run writes it (NF90_CLOBBER), made with scipy."""
    c, st, _ = dry_case()
    path = str(tmp_path / "monc.nc")
    nc = netcdf_file(path, "w", version=1)
    for name, n in (("empty_dim", 1), ("z", NZ), ("zn", NZ), ("y", NY), ("x", NX)):
        nc.createDimension(name, n)
    for name, src in (("u_nogal", "u"), ("zu", "zu"), ("v_nogal", "v"), ("zv", "zv"), ("w", "w"), ("zw", "zw"),
                      ("th", "th"), ("zth", "zth"), ("p", "p")):
        var = nc.createVariable(name, "d", ("x", "y", "zn"))
        var[:] = st[src].transpose(2, 1, 0)
    for name, val, typ in (("timestep", 11, "i"), ("time", 11.5, "d"), ("dtm", 1.0, "d"), ("dtm_new", 1.0, "d"),
                           ("absolute_new_dtm", 1.0, "d"), ("ugal", 0.0, "d"), ("vgal", 0.0, "d"),
                           ("nqfields", 0, "i"), ("last_cfl_timestep", 10, "i")):
        var = nc.createVariable(name, typ, ())
        var[...] = val
    nc.close()
    f, mean, md = api.checkpoint_read_host(c, path)
    for k in api.CHECKPOINT_FIELDS:
        np.testing.assert_array_equal(f[k], st[k], err_msg=k)
    assert mean is None and md.timestep == 11 and md.time == 11.5 and md.last_cfl_timestep == 10


def test_reads_the_olz_profiles_alone(tmp_path):
    """MONC reads each mean profile only if the file has it: a file with olzubar, olzvbar and
    olzthbar but no olubar, olvbar, olthbar gives those rows, the others zero."""
    c, st, mean = dry_case()
    path = str(tmp_path / "ck.nc")
    api.checkpoint_write_host(c, path, st, meta(), mean)
    src = netcdf_file(path, "r", mmap=False)
    dst_path = str(tmp_path / "olz_only.nc")
    dst = netcdf_file(dst_path, "w", version=2)
    try:
        for name, n in src.dimensions.items():
            dst.createDimension(name, n)
        for name, var in src.variables.items():
            if name in ("olubar", "olvbar", "olthbar"):
                continue
            out = dst.createVariable(name, var.data.dtype, var.dimensions)
            out[...] = var.data
    finally:
        src.close()
        dst.close()
    _, m, _ = api.checkpoint_read_host(c, dst_path)
    np.testing.assert_array_equal(m[:3], mean[:3])
    assert not m[3:].any()


def test_refuses_a_different_grid(tmp_path):
    c, st, mean = dry_case()
    path = str(tmp_path / "ck.nc")
    api.checkpoint_write_host(c, path, st, meta(), mean)
    other = cf.dry_cbl_config(NX, NY + 8, NZ, 50.0, 25.0, 1.0)
    with pytest.raises(api.MgpuError):
        api.checkpoint_read_host(other, path)
    assert os.path.getsize(path) > NX * NY * NZ * 8 * 9
