"""Known-answer tests of the CPU oracle (no GPU needed).

MONC ships no golden vectors for the dynamical core and cannot be compiled here, so the oracle is
pinned by properties with known answers: the FFTPACK restatement against a direct DFT, the
reference-state coefficients against closed forms, a divergence-free velocity after the pressure
step, discrete conservation and boundedness of the TVD scheme, and the Smagorinsky closure on an
analytic shear.
"""
import numpy as np
import pytest

from monc_b200 import api, config as cf, init as ini
from oracle import pyoracle as po

F = api.FIELDS


def direct_dft(x, sign):
    n = len(x)
    k = np.arange(n)
    return np.exp(sign * 2j * np.pi * np.outer(k, k) / n) @ x


@pytest.mark.parametrize("n", [4, 8, 16, 32, 64, 128, 256, 512, 1024, 3, 5, 6, 10, 12, 15, 24, 30, 45, 60, 96, 100,
                               360, 384, 750])
def test_fftpack_matches_direct_dft(n):
    rng = np.random.RandomState(n)
    x = rng.randn(n) + 1j * rng.randn(n)
    fwd = po.fft_c2c(x, -1)
    bwd = po.fft_c2c(x, +1)
    scale = np.abs(x).sum()
    assert np.abs(fwd - direct_dft(x, -1)).max() <= 1e-13 * scale
    assert np.abs(bwd - direct_dft(x, +1)).max() <= 1e-13 * scale
    rt = po.fft_c2c(fwd, +1) / n
    assert np.abs(rt - x).max() <= 1e-14 * np.abs(x).max() * np.log2(n)


@pytest.mark.parametrize("n", [7, 14, 22, 26, 49])
def test_fftpack_rejects_factors_beyond_five(n):
    """FFTPACK's general passf.f90 (prime factors above 5) is not restated."""
    with pytest.raises(ValueError):
        po.fft_c2c(np.ones(n, dtype=complex), -1)


def test_uniform_grid_coefficients():
    dz = 25.0
    c = cf.dry_cbl_config(16, 16, 33, 50.0, dz, 1.0)
    o = po.Oracle(c)
    z, zn = o.profile("z"), o.profile("zn")
    np.testing.assert_allclose(z, dz * np.arange(33), rtol=0, atol=1e-9)
    np.testing.assert_allclose(zn[1:], dz * (np.arange(1, 33) - 0.5), rtol=0, atol=1e-9)
    np.testing.assert_allclose(o.profile("tzc1")[1:-1], 0.25 / dz, rtol=1e-12)
    np.testing.assert_allclose(o.profile("czb")[1:], 1.0 / dz ** 2, rtol=1e-9)
    np.testing.assert_allclose(o.profile("cza")[1:-1], 1.0 / dz ** 2, rtol=1e-9)
    assert o.profile("cza")[-1] == 0.0
    np.testing.assert_allclose(o.profile("buoy_co")[:-1], 9.81 / 300.0, rtol=1e-15)
    # neutral mixing length sqrt(1/(1/(k(z+z0))^2 + 1/rmlmax^2)), rmlmax = Cs*dx with Cs=0.23
    rml = 0.23 * 50.0
    k = np.arange(1, 32)
    expect = 1.0 / (1.0 / (0.4 * (z[k] + 0.1)) ** 2 + 1.0 / rml ** 2)
    np.testing.assert_allclose(o.profile("rneutml_sq")[k], expect, rtol=1e-12)


def test_product_reference_state_equals_oracle():
    """The library's host-side grid builder and the oracle agree bit for bit."""
    cfgs = [cf.dry_cbl_config(64, 64, 65, 50.0, 25.0, 1.0),
            cf.dry_cbl_config(32, 32, 40, 35.0, 15.0, 0.3)]
    c3 = cf.dry_cbl_config(32, 32, 41, 35.0, 10.0, 0.3)
    cf.set_explicit_levels(c3, cf.stretched_levels(41, 5.0, 20.0))
    cfgs.append(c3)
    names = ["z", "zn", "dz", "dzn", "rdz", "rdzn", "czb", "cza", "czg", "czh", "tzc1", "tzc2", "tzd1", "tzd2",
             "rneutml_sq", "buoy_co", "prefn", "prefrcp", "tref", "qsat", "dqsatdt", "qsatfac"]
    for c in cfgs:
        o = po.Oracle(c)
        for nm in names:
            np.testing.assert_array_equal(api.reference_profile(c, nm), o.profile(nm), err_msg=nm)


def divergence(u, v, w, tzc1, tzc2, cx, cy):
    d = cx * (u - np.roll(u, 1, axis=2)) + cy * (v - np.roll(v, 1, axis=1))
    d[1:] += 4.0 * (tzc2[1:, None, None] * w[1:] - tzc1[1:, None, None] * w[:-1])
    return d[1:]


@pytest.mark.parametrize("nsteps", [1, 2])
def test_pressure_step_leaves_divergence_free_flow(nsteps):
    n, nz = 32, 24
    c = cf.dry_cbl_config(n, n, nz, 50.0, 25.0, 1.0, ug=5.0, fcoriol=1e-4)
    o = po.Oracle(c)
    st = ini.random_flow_state(n, n, nz, seed=4, amp_uv=1.0, amp_w=0.3, ug=5.0)
    for name, arr in st.items():
        o.set(F[name], arr)
    o.step(nsteps)
    u, v, w = o.get(F["u"]), o.get(F["v"]), o.get(F["w"])
    tzc1, tzc2 = o.profile("tzc1"), o.profile("tzc2")
    d = divergence(u, v, w, tzc1, tzc2, 1 / 50.0, 1 / 50.0)
    scale = max(np.abs(u).max(), np.abs(v).max(), np.abs(w).max()) / 25.0
    assert np.abs(d).max() <= 1e-12 * scale


def test_tvd_conserves_theta():
    n, nz = 32, 20
    c = cf.dry_cbl_config(n, n, nz, 50.0, 25.0, 1.0)
    o = po.Oracle(c)
    st = ini.random_flow_state(n, n, nz, seed=8, amp_uv=2.0, amp_w=0.5, amp_th=1.0)
    for name, arr in st.items():
        o.set(F[name], arr)
    o.set(F["sth"], np.zeros((nz, n, n)))
    o.set_timestep(2)
    o.component(api.COMPONENTS["tvd_advection"])
    s = o.get(F["sth"])
    dz = o.profile("dz")
    weighted = s[1:] * dz[1:, None, None]
    assert abs(weighted.sum()) <= 1e-12 * np.abs(weighted).sum()


def test_tvd_step_stays_bounded():
    """A theta step advected by a uniform wind stays within its initial range (TVD property)."""
    n, nz = 32, 12
    c = cf.dry_cbl_config(n, n, nz, 50.0, 25.0, 1.0)
    o = po.Oracle(c)
    shape = (nz, n, n)
    zth = np.where((np.arange(n) >= 8) & (np.arange(n) < 20), 1.0, 0.0)[None, None, :] * np.ones(shape)
    zth += 0.3 * np.where(np.arange(n) < 16, 1.0, -1.0)[None, :, None]
    u = np.full(shape, 5.0)
    v = np.full(shape, -3.0)
    w = np.zeros(shape)
    for name, arr in (("u", u), ("v", v), ("w", w), ("zu", u), ("zv", v), ("zw", w), ("th", zth), ("zth", zth)):
        o.set(F[name], arr)
    o.set(F["sth"], np.zeros(shape))
    o.set_timestep(2)
    o.component(api.COMPONENTS["tvd_advection"])
    new = zth + 2.0 * c.dtm * o.get(F["sth"])
    assert new[1:].min() >= zth.min() - 1e-12
    assert new[1:].max() <= zth.max() + 1e-12


def test_smagorinsky_on_linear_shear():
    """u = alpha*z, theta' = gamma*z: ssq = alpha^2, Ri = g*gamma/(theta0*alpha^2), stable branch."""
    n, nz = 8, 16
    alpha, gamma = 0.02, 0.001
    c = cf.dry_cbl_config(n, n, nz, 50.0, 25.0, 1.0)
    o = po.Oracle(c)
    zn = o.profile("zn")
    shape = (nz, n, n)
    u = alpha * zn[:, None, None] * np.ones(shape)
    th = gamma * zn[:, None, None] * np.ones(shape)
    z0 = np.zeros(shape)
    for name, arr in (("u", u), ("zu", u), ("v", z0), ("zv", z0), ("w", z0), ("zw", z0), ("th", th), ("zth", th)):
        o.set(F[name], arr)
    o.set_timestep(2)
    o.component(api.COMPONENTS["smagorinsky"])
    vis = o.get(F["vis"])[1:-1, 0, 0]
    diff = o.get(F["diff"])[1:-1, 0, 0]
    ssq = alpha ** 2 + float(np.float32(1e-14))
    ri = 9.81 / 300.0 * gamma / ssq
    rifac = (1.0 - ri / 0.25) ** 4
    rml2 = o.profile("rneutml_sq")[1:-1]
    np.testing.assert_allclose(vis, rifac * rml2 * np.sqrt(ssq), rtol=1e-10)
    np.testing.assert_allclose(diff, rifac * (1 / 0.7) * (1 - 1.2 * ri) * rml2 * np.sqrt(ssq), rtol=1e-10)


def test_oracle_is_deterministic():
    n, nz = 16, 12
    c = cf.dry_cbl_config(n, n, nz, 50.0, 25.0, 1.0, ug=2.0, fcoriol=1e-4)
    outs = []
    for _ in range(2):
        o = po.Oracle(c)
        st = ini.random_flow_state(n, n, nz, seed=1, ug=2.0)
        for name, arr in st.items():
            o.set(F[name], arr)
        o.step(3)
        outs.append(o.get(F["th"]))
    np.testing.assert_array_equal(outs[0], outs[1])


@pytest.mark.parametrize("stype", [cf.ITER_BICGSTAB, cf.ITER_CG], ids=["bicgstab", "cg"])
def test_iterative_solvers_agree_with_fft_solve(stype):
    """The oracle's BiCGStab / conjugate-gradient and FFT solves of one right-hand side agree (the
    discrete operators are the same; CG solves the symmetric form, rows scaled by dz).  The
    right-hand side has zero horizontal mean on every level, as the divergence of a periodic flow
    has; the horizontal-mean problem is singular otherwise."""
    n, nz = 16, 12
    b = ini.uniform_noise((nz, n, n), 3, 9, 1e-3)
    b -= b.mean(axis=(1, 2), keepdims=True)
    b[0] = 0.0
    out = []
    for solver in (cf.SOLVER_FFT, cf.SOLVER_ITERATIVE):
        c = cf.dry_cbl_config(n, n, nz, 50.0, 25.0, 1.0, solver=solver)
        c.solver_type = stype
        c.tolerance = 1e-12
        o = po.Oracle(c)
        o.set(F["p"], b)
        o.component(api.COMPONENTS["fftsolver" if solver == cf.SOLVER_FFT else "iterativesolver"])
        out.append(o.get(F["p"])[1:])
        if solver == cf.SOLVER_ITERATIVE:
            its, res = o.solver_stats()
            assert res < 1e-12 and its > 0
    d = out[0] - out[1]
    d -= d.mean()
    assert np.abs(d).max() <= 1e-8 * np.abs(out[0]).max()
