"""GPU iterative pressure solves (iterativesolver: BiCGStab, and cg_solver on the symmetric form
of the operator) against the CPU oracle and the FFT solve.

The GPU solver accumulates its inner products in a different order (block partials) and
contracts multiply-adds, so its iterates differ from the oracle's at rounding level.  With a
fixed number of iterations the solutions agree to 1e-10 relative; solved to a tolerance, the
iteration counts agree within one and both residuals meet the tolerance.  The same right-hand
side solved with the FFT solver must give the same pressure, to the iterative tolerance.
"""
import numpy as np
import pytest

from monc_b200 import api, config as cf, init as ini
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

NX, NY, NZ = 32, 32, 24


def rel_err(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


TYPES = pytest.mark.parametrize("stype", [cf.ITER_BICGSTAB, cf.ITER_CG], ids=["bicgstab", "cg"])


def config(solver=cf.SOLVER_ITERATIVE, precision=cf.FP64, tol=1e-4, max_it=500, stype=cf.ITER_BICGSTAB):
    c = cf.dry_cbl_config(NX, NY, NZ, 50.0, 25.0, 0.5, ug=5.0, fcoriol=1e-4, precision=precision, solver=solver)
    c.tolerance = tol
    c.max_iterations = max_it
    c.solver_type = stype
    return c


def rhs(seed=3):
    """Zero horizontal mean on every level, as the divergence of a periodic flow has (the
    horizontal-mean problem is singular otherwise)."""
    b = ini.uniform_noise((NZ, NY, NX), seed, 9, 1e-3)
    b -= b.mean(axis=(1, 2), keepdims=True)
    b[0] = 0.0
    return b


@TYPES
@pytest.mark.parametrize("iterations", [1, 2, 5, 12])
def test_iterates_match_oracle(gpu_lib, iterations, stype):
    """With the tolerance out of reach, both solvers run exactly `iterations` iterations; the
    iterates then agree to rounding (different dot-product order, contracted multiply-adds)."""
    c = config(tol=1e-30, max_it=iterations, stype=stype)
    o = po.Oracle(c)
    m = api.Model(c)
    b = rhs()
    o.set(api.FIELDS["p"], b)
    m.upload("p", b)
    o.component(api.COMPONENTS["iterativesolver"])
    m.component("iterativesolver")
    it_o, res_o = o.solver_stats()
    red = m.reductions()
    assert red.solver_iterations == it_o == iterations
    assert abs(red.solver_residual - res_o) <= 1e-9 * res_o
    assert rel_err(m.download("p"), o.get(api.FIELDS["p"])) <= 1e-10
    m.close()


@TYPES
@pytest.mark.parametrize("tol", [1e-4, 1e-10])
def test_converges_like_oracle(gpu_lib, tol, stype):
    """To a tolerance, the iteration counts agree within one (the stopping test sits on a
    rounding-level residual) and both solutions meet it."""
    c = config(tol=tol, stype=stype)
    o = po.Oracle(c)
    m = api.Model(c)
    b = rhs()
    o.set(api.FIELDS["p"], b)
    m.upload("p", b)
    o.component(api.COMPONENTS["iterativesolver"])
    m.component("iterativesolver")
    it_o, res_o = o.solver_stats()
    red = m.reductions()
    assert abs(red.solver_iterations - it_o) <= 1
    assert res_o < tol and red.solver_residual < tol
    assert rel_err(m.download("p"), o.get(api.FIELDS["p"])) <= max(1e-8, 10 * tol)
    m.close()


@TYPES
def test_warm_start_matches_oracle(gpu_lib, stype):
    """The second solve starts from the first solution (MONC keeps prev_p)."""
    c = config(tol=1e-30, max_it=6, stype=stype)
    o = po.Oracle(c)
    m = api.Model(c)
    for seed in (3, 4):
        b = rhs(seed)
        o.set(api.FIELDS["p"], b)
        m.upload("p", b)
        o.component(api.COMPONENTS["iterativesolver"])
        m.component("iterativesolver")
    assert rel_err(m.download("p"), o.get(api.FIELDS["p"])) <= 1e-10
    m.close()


@TYPES
@pytest.mark.parametrize("precision", [cf.FP64, cf.FP32_MIXED], ids=["fp64", "fp32_mixed_refined"])
def test_agrees_with_fft_solve(gpu_lib, precision, stype):
    b = rhs(5)
    out = {}
    for solver in (cf.SOLVER_FFT, cf.SOLVER_ITERATIVE):
        m = api.Model(config(solver=solver, precision=precision, tol=1e-11, stype=stype))
        m.upload("p", b)
        m.component("fftsolver" if solver == cf.SOLVER_FFT else "iterativesolver")
        out[solver] = m.download("p")[1:]
        if solver == cf.SOLVER_ITERATIVE:
            assert m.reductions().solver_residual < 1e-11
        m.close()
    d = out[cf.SOLVER_FFT] - out[cf.SOLVER_ITERATIVE]
    d -= d.mean()
    # the FP32-mixed FFT solve transforms in FP32, which limits that comparison to FP32 rounding
    tol = 1e-7 if precision == cf.FP64 else 1e-5
    assert np.abs(d).max() <= tol * np.abs(out[cf.SOLVER_FFT]).max()


@TYPES
def test_fused_step_matches_oracle(gpu_lib, stype):
    """Three fused steps with a fixed number of solver iterations per step."""
    c = config(tol=1e-30, max_it=8, stype=stype)
    o = po.Oracle(c)
    m = api.Model(c)
    st = ini.random_flow_state(NX, NY, NZ, seed=6, ug=5.0)
    for name, arr in st.items():
        o.set(api.FIELDS[name], arr)
        m.upload(name, arr)
    o.step(3)
    m.step(3)
    for f in ("u", "v", "w", "th", "zu", "zv", "zw", "zth", "p"):
        assert rel_err(m.download(f), o.get(api.FIELDS[f])) <= 1e-8, f
    m.close()


@TYPES
def test_reports_non_convergence(gpu_lib, stype):
    """At max_iterations the solve stops, the step still succeeds (MONC only warns) and the
    residual reported is above the tolerance."""
    c = config(tol=1e-14, max_it=2, stype=stype)
    m = api.Model(c)
    m.upload("p", rhs())
    m.component("iterativesolver")
    red = m.reductions()
    assert red.solver_iterations == 2
    assert red.solver_residual > 1e-14
    m.close()


def test_step_reports_divergence_error(gpu_lib):
    """With the iterative solver, mgpu_step reports diverr's divergence error of the velocities
    each step starts from (global_divmax: max |p| over levels 2..nz, diverr.F90:69-82, 120-175),
    checked against numpy on the downloaded fields."""
    c = config(tol=1e-8)
    st = ini.random_flow_state(NX, NY, NZ, seed=3, amp_uv=1.0, amp_w=0.3, amp_th=0.5, ug=5.0)
    m = api.Model(c)
    m.set_state(st)
    m.step(2)
    zu, zv, zw = (m.download(f) for f in ("zu", "zv", "zw"))
    m.step(1)  # centred: diverr reads zu, zv, zw
    got = m.reductions().global_divmax
    tzc1, tzc2 = m.profile("tzc1"), m.profile("tzc2")
    cx = cy = 1.0 / 50.0
    div = (cx * (zu - np.roll(zu, 1, axis=2)) + cy * (zv - np.roll(zv, 1, axis=1)))[1:]
    div = div + 4.0 * (tzc2[1:, None, None] * zw[1:] - tzc1[1:, None, None] * zw[:-1])
    expect = np.abs(div / (2.0 * c.dtm)).max()
    assert expect > 0 and abs(got - expect) <= 1e-12 * expect
    m.close()


@pytest.mark.parametrize("tol", [1e-4, 1e-8])
def test_fp32_mixed_refinement_meets_tolerance_on_a_large_layer(gpu_lib, tol):
    """The FP32-mixed refinement on the moist layer at 512 x 512 x 160: every step's FP64 residual
    meets the tolerance, each FP32 correction solve asked only for the reduction the FP64
    residual needs (at most 1e-3).  Asking each correction for a fixed 1e-5 ran most of them into
    the FP32 iteration's attainable accuracy and the iteration cap here, and left the FP64
    residual near 4e-7."""
    import argparse

    from monc_b200 import precision as pr

    a = argparse.Namespace(nx=512, ny=512, nz=160, dx=35.0, dz_bottom=5.0, dz_top=20.0, dt=0.3, seed=1,
                           noise_levels=10, solver="iterative", tolerance=tol)
    c, st = pr.build(a, cf.FP32_MIXED)
    m = api.Model(c)
    m.set_state(st)
    m.step(1)
    for _ in range(4):
        m.step(1)
        red = m.reductions()
        assert red.solver_residual < tol
        assert red.solver_iterations < 150
    m.close()
