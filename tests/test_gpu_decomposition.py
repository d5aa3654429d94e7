"""The y-slab decomposed step on one GPU: every slab a separate model with an external pressure
solve, exchanged through the loopback communicator (device copies between the slabs' buffers
after all queued work has finished; no kernel waits on another slab).

* FP64 with reproducible arithmetic: 2 and 4 slabs reproduce the single-domain model bit for
  bit, dry and moist, on the forward and centred steps; and both agree with the CPU oracle.
* Default (contracted) FP64 arithmetic and FP32-mixed: the decomposed run tracks the
  single-domain run (FP32-mixed differs by the order in which the level means are summed).
* Damping, mean-profile subsidence and profile_diagnostics on the slabs: the mean profiles
  averaged over the slabs and the diagnostics sums added over them match the single domain.
* cfltest on the slabs: the extrema combined by a maximum give the single domain's dtm sequence,
  and the fields of the adaptive-dtm run bit for bit.
* iterativesolver on the slabs, BiCGStab and conjugate gradients: the inner products summed over
  the slabs, the iterates match the single domain's to rounding; the FP32-mixed refinement
  reaches the same residual.
* Checkpoints of a decomposed run: one whole-domain file, restarts bit for bit.
* The slab entry points themselves: halo rows, the transposed column solve, argument checks.
"""
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest
import torch

from monc_b200 import api, config as cf, decomposition as dc, init as ini
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

NX, NY, NZ = 64, 64, 24
STATE = ["u", "v", "w", "th", "zu", "zv", "zw", "zth"]


def dry_config(precision=cf.FP64, reproducible=1):
    c = cf.dry_cbl_config(NX, NY, NZ, 50.0, 25.0, 0.5, ug=5.0, fcoriol=1e-4, precision=precision)
    c.reproducible = reproducible
    return c


def dry_state(seed=4):
    return ini.random_flow_state(NX, NY, NZ, seed=seed, amp_uv=1.0, amp_w=0.3, amp_th=0.5, ug=5.0)


def run_single(cfg, state, nsteps, fields):
    m = api.Model(cfg)
    m.set_state(state)
    m.step(nsteps)
    out = {f: m.download(f) for f in fields}
    m.close()
    return out


def run_slabs(cfg, state, nsteps, nranks, fields, halo=4):
    d = dc.SlabDomain(cfg, dc.LoopbackComm(nranks), halo=halo)
    d.set_state(state)
    d.step(nsteps)
    out = {f: d.download(f) for f in fields}
    d.close()
    return out


@pytest.mark.parametrize("nranks", [2, 4])
@pytest.mark.parametrize("nsteps", [1, 3])
def test_dry_fp64_slabs_bit_identical(gpu_lib, nranks, nsteps):
    cfg, st = dry_config(), dry_state()
    ref = run_single(cfg, st, nsteps, STATE + ["p"])
    got = run_slabs(cfg, st, nsteps, nranks, STATE + ["p"])
    for f in STATE + ["p"]:
        np.testing.assert_array_equal(got[f], ref[f], err_msg=f)


@pytest.mark.parametrize("nranks", [2, 4])
def test_slab_mean_diagnostics(gpu_lib, nranks):
    """mgpu_diagnostics on a slab averages its interior rows only; the slabs' means averaged over
    the slabs are the domain's mean theta and w'^2 profiles (to the order of the sums)."""
    cfg, st = dry_config(), dry_state()
    m = api.Model(cfg)
    m.set_state(st)
    m.step(3)
    th_ref, w2_ref = m.diagnostics()
    m.close()
    d = dc.SlabDomain(cfg, dc.LoopbackComm(nranks))
    d.set_state(st)
    d.step(3)
    th, w2 = d.diagnostics()
    d.close()
    np.testing.assert_allclose(th, th_ref, rtol=1e-14)
    np.testing.assert_allclose(w2, w2_ref, rtol=1e-12, atol=1e-14 * np.abs(w2_ref).max())


def test_dry_fp64_slabs_match_oracle(gpu_lib):
    cfg, st = dry_config(), dry_state(seed=7)
    o = po.Oracle(cfg)
    for name, arr in st.items():
        o.set(api.FIELDS[name], arr)
    o.step(2)
    got = run_slabs(cfg, st, 2, 4, STATE)
    for f in STATE:
        ref = o.get(api.FIELDS[f])
        assert np.abs(got[f] - ref).max() <= 1e-10 * np.abs(ref).max(), f


def moist_setup(precision=cf.FP64):
    z = cf.stretched_levels(NZ, 20.0, 60.0, ztop=1000.0)
    c = cf.moist_config(NX, NY, z, 35.0, 0.3, shf_wm2=10.0, lhf_wm2=50.0, max_height_cloud=700.0, n_tracers=1,
                        precision=precision)
    c.reproducible = 1
    zn = api.reference_profile(c, "zn")
    st = ini.moist_layer_state(NX, NY, NZ, zn, seed=2, n_tracers=1)
    flow = ini.random_flow_state(NX, NY, NZ, seed=5, amp_uv=0.5, amp_w=0.2)
    for k in ("u", "v", "w", "zu", "zv", "zw"):
        st[k] = flow[k]
    return c, st


def test_moist_fp64_slabs_bit_identical(gpu_lib):
    cfg, st = moist_setup()
    fields = STATE + ["q0", "q1", "q2", "zq0", "zq1", "zq2", "p"]
    ref = run_single(cfg, st, 3, fields)
    got = run_slabs(cfg, st, 3, 2, fields)
    for f in fields:
        np.testing.assert_array_equal(got[f], ref[f], err_msg=f)
    assert ref["q1"].max() > 0


def test_contracted_fp64_slabs_match(gpu_lib):
    cfg, st = dry_config(reproducible=0), dry_state()
    ref = run_single(cfg, st, 3, STATE)
    got = run_slabs(cfg, st, 3, 4, STATE)
    for f in STATE:
        assert np.abs(got[f] - ref[f]).max() <= 1e-12 * np.abs(ref[f]).max(), f


def test_fp32_mixed_slabs_track_single_domain(gpu_lib):
    cfg, st = moist_setup(precision=cf.FP32_MIXED)
    fields = ["th", "w", "q0", "q1"]
    ref = run_single(cfg, st, 5, fields)
    got = run_slabs(cfg, st, 5, 4, fields)
    for f in fields:
        scale = np.abs(ref[f]).max()
        assert np.abs(got[f] - ref[f]).max() <= 1e-5 * scale, f
        assert np.abs(got[f].mean(axis=(1, 2)) - ref[f].mean(axis=(1, 2))).max() <= 1e-6 * scale, f


def forced_setup(precision=cf.FP64, moist=False):
    """Damping above 300 m, subsidence from the mean profiles and profile_diagnostics on."""
    if moist:
        c, st = moist_setup(precision)
        cf.enable_subsidence(c, [0.0, 1000.0], [0.0, -0.005], theta=True, q=True)
    else:
        c, st = dry_config(precision), dry_state()
        cf.enable_subsidence(c, [0.0, 200.0, 450.0, 700.0], [0.0, -0.003, -0.005, -0.004], theta=True)
        zn = api.reference_profile(c, "zn")
        for f in ("th", "zth"):
            st[f] = st[f] + 0.004 * zn[:, None, None]
    cf.enable_damping(c, 0.02, 300.0, 150.0)
    c.profile_diagnostics_enabled = 1
    return c, st


@pytest.mark.parametrize("nranks", [2, 4])
@pytest.mark.parametrize("moist", [False, True], ids=["dry", "moist"])
def test_damping_subsidence_and_diagnostics_on_slabs(gpu_lib, nranks, moist):
    """Damping and mean-profile subsidence read the domain mean profiles (the slabs' means
    averaged by the driver), and the profile_diagnostics sums add up over the slabs: five steps
    (damping and forcing act from the third) match the single domain to rounding, the order of
    the level sums being the only difference."""
    c, st = forced_setup(moist=moist)
    fields = STATE + (["q0", "q1", "zq0", "zq1"] if moist else [])
    m = api.Model(c)
    m.set_state(st)
    m.step(5)
    ref = {f: m.download(f) for f in fields}
    ref_pd, ref_mp = m.profile_diagnostics(), m.mean_profiles()
    m.close()
    d = dc.SlabDomain(c, dc.LoopbackComm(nranks))
    d.set_state(st)
    d.step(5)
    for f in fields:
        assert np.abs(d.download(f) - ref[f]).max() <= 1e-11 * np.abs(ref[f]).max(), f
    got_mp = d.slabs[0].m.mean_profiles()
    for n in ref_mp:
        assert np.abs(got_mp[n] - ref_mp[n]).max() <= 1e-12 * max(np.abs(ref_mp[n]).max(), 1e-30), n
    got_pd = d.profile_diagnostics()
    assert set(got_pd) == set(ref_pd)
    for n in ref_pd:
        scale = np.abs(ref_pd[n]).max()
        if n == "w_wind_total_local":  # sums to zero by continuity: scale by the sum of |w|
            scale = NX * NY * np.abs(ref["w"]).max()
        assert np.abs(got_pd[n] - ref_pd[n]).max() <= 1e-11 * max(scale, 1e-30), n
    d.close()


def test_slab_forcing_is_live(gpu_lib):
    """The slab run with damping and subsidence ends elsewhere than the one without."""
    c, st = forced_setup()
    out = []
    for cfg in (c, dry_config()):
        d = dc.SlabDomain(cfg, dc.LoopbackComm(2))
        d.set_state(st)
        d.step(5)
        out.append(d.download("th"))
        d.close()
    assert np.abs(out[0] - out[1]).max() > 1e-8 * np.abs(out[1]).max()


def test_fp32_mixed_forced_slabs_track_single_domain(gpu_lib):
    c, st = forced_setup(cf.FP32_MIXED, moist=True)
    fields = ["th", "w", "q0", "q1"]
    ref = run_single(c, st, 5, fields)
    got = run_slabs(c, st, 5, 4, fields)
    for f in fields:
        assert np.abs(got[f] - ref[f]).max() <= 1e-5 * np.abs(ref[f]).max(), f


CFL_KEYS = ["dtm", "dtm_new", "absolute_new_dtm", "cvel", "cvis", "cfl_number", "cvel_x", "cvel_y", "cvel_z",
            "cfl_evaluations", "last_cfl_timestep", "timestep", "ugal", "vgal"]


def cfl_setup(precision=cf.FP64, **kw):
    c = dry_config(precision)
    c.dtm = 1.0
    cf.enable_cfl(c, **kw)
    st = ini.random_flow_state(NX, NY, NZ, seed=3, amp_uv=2.0, amp_w=0.5, ug=5.0)
    return c, st


@pytest.mark.parametrize("galilean", [False, True], ids=["rest", "galilean"])
@pytest.mark.parametrize("nranks", [2, 4])
def test_cfl_on_slabs_bit_identical(gpu_lib, nranks, galilean):
    """cfltest on slabs: each slab's extrema over its interior rows, combined by a maximum across
    the slabs (exact in any order), give the single domain's Courant numbers, dtm sequence and
    Galilean frame, and the steps of varying dtm end bit for bit where the single domain's do."""
    c, st = cfl_setup(frequency=3, dtmmax=2.0)
    if galilean:
        cf.enable_galilean(c)
    m = api.Model(c)
    m.set_state(st)
    d = dc.SlabDomain(c, dc.LoopbackComm(nranks))
    d.set_state(st)
    changed = 0
    for n in range(10):
        m.step(1)
        d.step(1)
        ref = m.reductions()
        for s in d.slabs:
            got = s.m.reductions()
            for k in CFL_KEYS:
                assert getattr(got, k) == getattr(ref, k), (n, k)
        changed += ref.dtm != c.dtm
    assert changed > 0  # the timestep did change
    for f in STATE + ["p"]:
        np.testing.assert_array_equal(d.download(f), m.download(f), err_msg=f)
    d.close()
    m.close()


def test_cfl_on_slabs_stops_below_dtmmin(gpu_lib):
    c, st = cfl_setup(frequency=2, dtmmin=0.9)
    d = dc.SlabDomain(c, dc.LoopbackComm(2))
    d.set_state(st)
    with pytest.raises(api.MgpuError) as e:
        d.step(1)
    assert e.value.code == api.ERR_CFL
    d.close()


def test_fp32_mixed_cfl_on_slabs_follows_single_domain(gpu_lib):
    c, st = cfl_setup(cf.FP32_MIXED, frequency=3, dtmmax=2.0)
    m = api.Model(c)
    m.set_state(st)
    d = dc.SlabDomain(c, dc.LoopbackComm(4))
    d.set_state(st)
    for n in range(8):
        m.step(1)
        d.step(1)
        assert abs(d.slabs[0].m.reductions().dtm - m.reductions().dtm) <= 1e-5 * c.dtm, n
    d.close()
    m.close()


def iterative_config(tol, max_it, stype=cf.ITER_BICGSTAB):
    c = dry_config()
    c.solver = cf.SOLVER_ITERATIVE
    c.solver_type = stype
    c.tolerance = tol
    c.max_iterations = max_it
    return c


ITER_TYPES = pytest.mark.parametrize("stype", [cf.ITER_BICGSTAB, cf.ITER_CG], ids=["bicgstab", "cg"])


@ITER_TYPES
@pytest.mark.parametrize("nranks", [2, 4])
def test_iterative_solve_on_slabs_fixed_iterations(gpu_lib, nranks, stype):
    """BiCGStab (halo rows of x, pp, cs) and conjugate gradients (x, then z and the old direction)
    over the slabs, every inner product summed over the slabs, with the tolerance out of reach:
    the same 8 iterations per step as the single domain, whose iterates differ only by the order
    of the dot-product sums (1e-10 after 3 steps)."""
    c = iterative_config(1e-30, 8, stype)
    st = dry_state()
    m = api.Model(c)
    m.set_state(st)
    m.step(3)
    ref = {f: m.download(f) for f in STATE + ["p"]}
    assert m.reductions().solver_iterations == 8
    m.close()
    d = dc.SlabDomain(c, dc.LoopbackComm(nranks))
    d.set_state(st)
    d.step(3)
    for s in d.slabs:
        assert s.m.reductions().solver_iterations == 8
    for f in STATE + ["p"]:
        assert np.abs(d.download(f) - ref[f]).max() <= 1e-10 * np.abs(ref[f]).max(), f
    d.close()


@ITER_TYPES
def test_iterative_solve_on_slabs_to_tolerance(gpu_lib, stype):
    """Solved to a tolerance: every slab stops at the same iteration with the residual met, and
    within three of the single domain's.  The slabs sum their inner products in another order
    (per slab, then across slabs), and near the tolerance BiCGStab's stopping iteration moves by
    a few with the rounding of those sums."""
    c = iterative_config(1e-10, 500, stype)
    st = dry_state()
    m = api.Model(c)
    m.set_state(st)
    m.step(3)
    ref = {f: m.download(f) for f in STATE}
    its = m.reductions().solver_iterations
    m.close()
    d = dc.SlabDomain(c, dc.LoopbackComm(4))
    d.set_state(st)
    d.step(3)
    got = [(s.m.reductions().solver_iterations, s.m.reductions().solver_residual) for s in d.slabs]
    assert len(set(got)) == 1 and abs(got[0][0] - its) <= 3 and got[0][1] < 1e-10, (got, its)
    for f in STATE:
        assert np.abs(d.download(f) - ref[f]).max() <= 1e-8 * np.abs(ref[f]).max(), f
    d.close()


@pytest.mark.parametrize("nranks", [2, 4])
def test_slab_checkpoint_restart(gpu_lib, tmp_path, nranks):
    """A decomposed run checkpointed into one whole-domain file (damping, cfltest and the Galilean
    frame on, so the mean profiles and step state travel too) and continued by a new decomposed
    domain that reads it ends bit for bit where the uninterrupted run does; the single-domain
    model reads the same file and agrees with both to rounding."""
    c, st = forced_setup()
    cf.enable_cfl(c, frequency=2, dtmmax=1.0)
    cf.enable_galilean(c)
    path = str(tmp_path / "slabs.nc")
    a = dc.SlabDomain(c, dc.LoopbackComm(nranks))
    a.set_state(st)
    a.step(7)
    ref = {f: a.download(f) for f in STATE}
    ref_state = a.slabs[0].m.reductions()
    a.close()
    b = dc.SlabDomain(c, dc.LoopbackComm(nranks))
    b.set_state(st)
    b.step(4)
    b.checkpoint_write(path)
    b.close()
    d = dc.SlabDomain(c, dc.LoopbackComm(nranks))
    d.checkpoint_read(path)
    d.step(3)
    for f in STATE:
        np.testing.assert_array_equal(d.download(f), ref[f], err_msg=f)
    r = d.slabs[0].m.reductions()
    assert (r.timestep, r.dtm, r.ugal) == (ref_state.timestep, ref_state.dtm, ref_state.ugal)
    d.close()
    m = api.Model(c)
    m.checkpoint_read(path)
    m.step(3)
    for f in STATE:
        assert np.abs(m.download(f) - ref[f]).max() <= 1e-10 * np.abs(ref[f]).max(), f
    m.close()


@ITER_TYPES
def test_fp32_mixed_iterative_solve_on_slabs(gpu_lib, stype):
    """The FP32-mixed solve on slabs (the compatible right-hand side, FP64 residuals over the
    slabs' interior rows, FP32 corrections, each with its sums over the slabs) reaches the
    single domain's residual and tracks its fields."""
    c = iterative_config(1e-8, 500, stype)
    c.precision = cf.FP32_MIXED
    st = dry_state()
    m = api.Model(c)
    m.set_state(st)
    m.step(3)
    ref = {f: m.download(f) for f in STATE}
    res_ref = m.reductions().solver_residual
    m.close()
    d = dc.SlabDomain(c, dc.LoopbackComm(2))
    d.set_state(st)
    d.step(3)
    res = [s.m.reductions().solver_residual for s in d.slabs]
    assert len(set(res)) == 1 and res[0] < 1e-8 and res_ref < 1e-8
    for f in STATE:
        assert np.abs(d.download(f) - ref[f]).max() <= 1e-5 * np.abs(ref[f]).max(), f
    d.close()


def test_halo_rows_pack_and_unpack(gpu_lib):
    """Pack takes the first and last `depth` interior rows, unpack writes the rows just outside."""
    halo, nyl = 4, 16
    c = dry_config()
    c.ny = nyl + 2 * halo
    c.solver = cf.SOLVER_EXTERNAL
    m = api.Model(c)
    m.slab_init(NY, halo, NX // 2 + 1)
    fields = {f: ini.uniform_noise((NZ, c.ny, NX), 3, n, 1.0) for n, f in enumerate(STATE)}
    for f, a in fields.items():
        m.upload(f, a)
    nf = m.halo_fields(cf.HALO_STATE)
    assert nf == 8
    for depth in (1, 3, halo):
        lo = torch.zeros(nf * NZ * depth * NX, dtype=torch.float64, device="cuda")
        hi = torch.zeros_like(lo)
        m.halo_pack(cf.HALO_STATE, depth, lo.data_ptr(), hi.data_ptr())
        torch.cuda.synchronize()
        for n, f in enumerate(STATE):
            blo = lo.view(nf, NZ, depth, NX)[n].cpu().numpy()
            bhi = hi.view(nf, NZ, depth, NX)[n].cpu().numpy()
            np.testing.assert_array_equal(blo, fields[f][:, halo:halo + depth])
            np.testing.assert_array_equal(bhi, fields[f][:, c.ny - halo - depth:c.ny - halo])
        # unpack marked buffers and check the rows they land in, and that nothing else moved
        lo.fill_(7.0)
        hi.fill_(-7.0)
        m.halo_unpack(cf.HALO_STATE, depth, lo.data_ptr(), hi.data_ptr())
        torch.cuda.synchronize()
        for f in STATE:
            a = m.download(f)
            expect = fields[f].copy()
            expect[:, halo - depth:halo] = 7.0
            expect[:, c.ny - halo:c.ny - halo + depth] = -7.0
            np.testing.assert_array_equal(a, expect)
            m.upload(f, fields[f])
    m.close()


@pytest.mark.parametrize("nranks", [1, 2, 4])
def test_slab_solve_and_its_transpose_match_fftsolver(gpu_lib, nranks):
    """x-FFT + all-to-all + column solve + all-to-all + inverse x-FFT over the slabs equals the
    fftsolver component on the whole domain, bit for bit, for the solve and for its transpose."""
    rhs = ini.uniform_noise((NZ, NY, NX), 11, 1, 1e-3)
    rhs[0] = 0.0
    for transpose in (False, True):
        ref_m = api.Model(dry_config())
        ref_m.upload("p", rhs)
        if transpose:
            ref_m.fftsolver_adjoint()
        else:
            ref_m.component("fftsolver")
        ref = ref_m.download("p")
        ref_m.close()
        d = dc.SlabDomain(dry_config(), dc.LoopbackComm(nranks))
        d.upload("p", rhs)
        g = d.geo
        for s in d.slabs:
            s.m.slab_fft_x(s.spec_x.data_ptr(), g.nranks, False)
        d.comm.all_to_all([s.x_blocks for s in d.slabs], [s.t_blocks for s in d.slabs])
        for s in d.slabs:
            k0, w = g.blocks[s.rank]
            s.m.slab_solve_columns(s.spec_t.data_ptr(), k0, w, g.nyl, transpose)
        d.comm.all_to_all([s.t_blocks for s in d.slabs], [s.x_blocks for s in d.slabs])
        for s in d.slabs:
            s.m.slab_fft_x(s.spec_x.data_ptr(), g.nranks, True)
        torch.cuda.synchronize()
        got = d.download("p")
        d.close()
        np.testing.assert_array_equal(got, ref)


def test_slab_entry_points_check_arguments(gpu_lib):
    c = dry_config()
    c.ny = 24
    c.solver = cf.SOLVER_EXTERNAL
    m = api.Model(c)
    with pytest.raises(api.MgpuError):
        m.step(1)  # the pressure solve is external
    with pytest.raises(api.MgpuError):
        m.halo_pack(cf.HALO_STATE, 1, 1, 1)  # before slab_init
    with pytest.raises(api.MgpuError):
        m.slab_init(64, 12, 8)  # no interior rows left
    with pytest.raises(api.MgpuError):
        m.slab_init(56, 4, 8)  # ny_global with a prime factor above 5
    m.slab_init(64, 4, 9)
    buf = torch.zeros(8 * NZ * 4 * NX, dtype=torch.float64, device="cuda")
    with pytest.raises(api.MgpuError):
        m.halo_pack(cf.HALO_STATE, 5, buf.data_ptr(), buf.data_ptr())  # deeper than the halo
    with pytest.raises(api.MgpuError):
        m.halo_pack(7, 1, buf.data_ptr(), buf.data_ptr())  # unknown set
    with pytest.raises(api.MgpuError):
        m.slab_solve_columns(buf.data_ptr(), 0, 10, 16)  # more columns than slab_init allowed
    with pytest.raises(api.MgpuError):
        m.slab_solve_columns(buf.data_ptr(), 30, 5, 16)  # past nx/2+1
    with pytest.raises(api.MgpuError):
        m.slab_fft_x(buf.data_ptr(), NX // 2 + 2, False)  # more blocks than wavenumbers
    m.close()
    c32 = dry_config(precision=cf.FP32_MIXED)
    c32.ny = 24
    c32.solver = cf.SOLVER_EXTERNAL
    m = api.Model(c32)
    m.slab_init(64, 4, 9)
    m.step_phase(cf.PHASE_SUBGRID)
    with pytest.raises(api.MgpuError):
        m.step_phase(cf.PHASE_DYNAMICS)  # FP32-mixed needs the domain level means first
    m.close()
    c = dry_config()
    c.ny = 24
    c.solver = cf.SOLVER_EXTERNAL
    m = api.Model(c)
    m.slab_init(64, 4, 9)
    with pytest.raises(api.MgpuError):
        m.slab_mean_profiles(buf.data_ptr(), False)  # no damping, subsidence or diagnostics: no profiles
    with pytest.raises(api.MgpuError):
        m.slab_cfl_extrema(buf.data_ptr(), False)  # cfltest off
    m.close()
    plain = api.Model(dry_config())
    with pytest.raises(api.MgpuError):
        plain.step_phase(cf.PHASE_SUBGRID)
    with pytest.raises(api.MgpuError):
        plain.slab_init(64, 4, 9)
    plain.close()


NCCL_ONE_RANK = textwrap.dedent("""
    import datetime, os, sys
    import numpy as np, torch, torch.distributed as dist
    sys.path.insert(0, os.getcwd())
    from monc_b200 import api, config as cf, decomposition as dc, init as ini
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60),
                            device_id=torch.device("cuda", 0))
    mode = sys.argv[2]
    c = cf.dry_cbl_config(64, 64, 24, 50.0, 25.0, 0.5, ug=5.0, fcoriol=1e-4, precision=int(sys.argv[1]))
    c.reproducible = 1
    tol = 0.0 if c.precision == cf.FP64 else 1e-5
    if mode == "forced":
        # damping and subsidence (mean-profile all-reduce), profile diagnostics (sum), cfltest
        # with the Galilean frame (max all-reduce)
        cf.enable_damping(c, 0.02, 300.0, 150.0)
        cf.enable_subsidence(c, [0.0, 700.0], [0.0, -0.004], theta=True)
        c.profile_diagnostics_enabled = 1
        cf.enable_cfl(c, frequency=2, dtmmax=1.0)
        cf.enable_galilean(c)
        tol = max(tol, 1e-11)
    elif mode == "iterative":
        # conjugate gradients: halo sets of the solver vectors and the sum all-reduce
        c.solver, c.solver_type, c.tolerance, c.max_iterations = cf.SOLVER_ITERATIVE, cf.ITER_CG, 1e-30, 6
        tol = 1e-10
    st = ini.random_flow_state(64, 64, 24, seed=4, amp_uv=1.0, amp_w=0.3, amp_th=0.5, ug=5.0)
    m = api.Model(c)
    m.set_state(st)
    m.step(5)
    d = dc.SlabDomain(c, dc.TorchComm(), halo=4)
    d.set_state(st)
    d.step(5)
    for f in ("u", "v", "w", "th", "zu", "zv", "zw", "zth"):
        a, b = d.download(f), m.download(f)
        err = np.abs(a - b).max() / np.abs(b).max()
        assert err <= tol, (f, err)
    if mode == "forced":
        rd, rm = d.slabs[0].m.reductions(), m.reductions()
        assert abs(rd.dtm - rm.dtm) <= 1e-12 * rm.dtm and abs(rd.ugal - rm.ugal) <= 1e-12 * abs(rm.ugal)
        assert rm.ugal != 0.0 and rd.cfl_evaluations == rm.cfl_evaluations
        pd, ref = d.profile_diagnostics(), m.profile_diagnostics()
        for n in ref:
            scale = max(np.abs(ref[n]).max(), 64 * 64 * np.abs(m.download("w")).max())
            assert np.abs(pd[n] - ref[n]).max() <= 1e-11 * scale, n
    d.close()
    m.close()
    dist.destroy_process_group()
    print("SLAB-NCCL-OK")
""")


@pytest.mark.parametrize("precision,mode", [(cf.FP64, "plain"), (cf.FP32_MIXED, "plain"), (cf.FP64, "forced"),
                                            (cf.FP64, "iterative")],
                         ids=["fp64", "fp32_mixed", "forced", "iterative"])
def test_torch_comm_over_nccl_single_rank(gpu_lib, precision, mode):
    """The torch.distributed communicator on NCCL with one rank (the model's stream as the
    collectives' stream, all-to-all and halo exchange as local copies, the FP32 level-mean,
    mean-profile, extrema and inner-product all-reduces through NCCL) reproduces the
    single-domain model; run in a child process so the process group does not outlive the test."""
    port = 29600 + 10 * precision + ["plain", "forced", "iterative"].index(mode)
    env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", NCCL_ONE_RANK, str(precision), mode], cwd=root, env=env,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "SLAB-NCCL-OK" in r.stdout, r.stdout[-2000:] + r.stderr[-2000:]
