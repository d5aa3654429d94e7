"""Tangent-linear and adjoint runs of the dry FP64 step on the GPU.

* The tangent-linear model (dual numbers through the step's device functions) matches central
  finite differences of the forward model.
* The adjoint (per-thread tapes, transposed pressure solve, checkpointed reverse sweep) satisfies
  the dot-product identity <ybar, L dx> = <L^T ybar, dx> against the tangent-linear model,
  including the Smagorinsky mixing-length parameter rmlmax.
* The gradient of a resolved-TKE objective with respect to the initial theta and to Cs matches
  central finite differences.
"""
import numpy as np
import pytest

from monc_b200 import api, config as cf, init as ini

pytestmark = pytest.mark.gpu

NX, NY, NZ = 32, 32, 24
DX, DZ = 50.0, 25.0
STATE = api.STATE_FIELDS


def config():
    c = cf.dry_cbl_config(NX, NY, NZ, DX, DZ, 1.0, ug=5.0, fcoriol=1e-4)
    c.reproducible = 1
    return c


def base_state(seed=4):
    st = ini.random_flow_state(NX, NY, NZ, seed=seed, amp_uv=1.0, amp_w=0.3, amp_th=0.5, ug=5.0)
    return {k: st[k] for k in STATE}


def direction(seed, scale=1.0):
    d = {}
    for n, f in enumerate(STATE):
        a = ini.uniform_noise((NZ, NY, NX), seed, 50 + n, scale)
        if f in ("w", "zw"):
            a[0] = 0.0
            a[-1] = 0.0
        d[f] = a
    return d


def run(state, nsteps, timestep=1, cfg=None):
    m = api.Model(cfg or config())
    m.set_state(state)
    m.set_timestep(timestep)
    m.step(nsteps)
    out = {f: m.download(f) for f in STATE}
    m.close()
    return out


def dot(a, b):
    return sum(float(np.vdot(a[f], b[f])) for f in STATE)


@pytest.mark.parametrize("timestep,nsteps", [(1, 1), (1, 3), (3, 2)], ids=["forward", "fwd+2", "centred"])
def test_tangent_linear_matches_finite_differences(gpu_lib, timestep, nsteps):
    x0 = base_state()
    dx = direction(7)
    # at 1e-6 a few faces of this strongly limited random state cross a limiter branch
    eps = 1e-7
    m = api.Model(config())
    m.set_state(x0)
    for f in STATE:
        m.upload("tl:" + f, dx[f])
    m.set_timestep(timestep)
    m.tl_step(nsteps)
    tl = {f: m.download("tl:" + f) for f in STATE}
    m.close()
    xp = run({f: x0[f] + eps * dx[f] for f in STATE}, nsteps, timestep)
    xm = run({f: x0[f] - eps * dx[f] for f in STATE}, nsteps, timestep)
    # A perturbation can move a few TVD faces across a limiter branch, where the step is not
    # differentiable; those points are allowed to differ (at most 0.1% of them), everything else
    # and a weighted sum over all points must agree.
    c = direction(13)
    for f in STATE:
        fd = (xp[f] - xm[f]) / (2 * eps)
        scale = max(np.abs(fd).max(), 1e-300)
        bad = np.abs(tl[f] - fd) > 1e-5 * scale
        assert bad.mean() <= 1e-3, (f, int(bad.sum()))
        jt, jf = float(np.vdot(c[f], tl[f])), float(np.vdot(c[f], fd))
        assert abs(jt - jf) <= 1e-4 * max(abs(jf), 1e-3 * scale * np.abs(c[f]).sum()), (f, jt, jf)


@pytest.mark.parametrize("timestep,nsteps,interval", [(1, 1, 1), (1, 3, 2), (2, 4, 3)])
def test_adjoint_dot_product_identity(gpu_lib, timestep, nsteps, interval):
    x0 = base_state()
    dx = direction(9)
    ybar = direction(11)
    dr = 0.7
    m = api.Model(config())
    m.set_state(x0)
    for f in STATE:
        m.upload("tl:" + f, dx[f])
    m.set_timestep(timestep)
    m.tl_step(nsteps, dr)
    lhs = dot(ybar, {f: m.download("tl:" + f) for f in STATE})
    m.close()
    m = api.Model(config())
    m.set_state(x0)
    m.set_timestep(timestep)
    for f in STATE:
        m.upload("adj:" + f, ybar[f])
    rbar = m.adjoint_run(nsteps, interval)
    xbar = {f: m.download("adj:" + f) for f in STATE}
    m.close()
    rhs = dot(xbar, dx) + rbar * dr
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs), (lhs, rhs)


@pytest.mark.parametrize("timestep,nsteps,rhobous", [(1, 2, 1.0), (3, 3, 1.0), (2, 2, 1.17)],
                         ids=["forward", "centred", "anelastic-rho"])
def test_hand_written_adjoint_matches_tape(gpu_lib, timestep, nsteps, rhobous):
    """The hand-written adjoint kernels and the operator-overloading tape transpose the same
    passes: the adjoints of the initial state and of rmlmax agree to rounding."""
    x0 = base_state()
    ybar = direction(11)
    res = []
    for taped in (1, 0):
        c = config()
        c.rhobous = rhobous
        c.adjoint_taped = taped
        m = api.Model(c)
        m.set_state(x0)
        m.set_timestep(timestep)
        for f in STATE:
            m.upload("adj:" + f, ybar[f])
        rbar = m.adjoint_run(nsteps, 2)
        res.append(({f: m.download("adj:" + f) for f in STATE}, rbar))
        m.close()
    for f in STATE:
        a, b = res[1][0][f], res[0][0][f]
        assert np.abs(a - b).max() <= 1e-11 * np.abs(b).max(), f
    assert abs(res[1][1] - res[0][1]) <= 1e-11 * abs(res[0][1])


def tke_objective(state, zn, dz, ztop=500.0):
    """J = sum over levels with zn <= ztop of <0.5 (u'^2 + v'^2 + w'^2)>_xy dz, and dJ/d(u, v, w)."""
    lev = (zn <= ztop) & (np.arange(NZ) >= 1)
    J = 0.0
    grad = {f: np.zeros((NZ, NY, NX)) for f in STATE}
    for f in ("u", "v", "w"):
        a = state[f]
        pert = a - a.mean(axis=(1, 2), keepdims=True)
        J += float((0.5 * (pert ** 2).mean(axis=(1, 2)) * dz * lev).sum())
        grad[f] = pert / (NX * NY) * (dz * lev)[:, None, None]
    return J, grad


def test_objective_gradient_matches_finite_differences(gpu_lib):
    nsteps = 4
    c = config()
    zn = api.reference_profile(c, "zn")
    dz = api.reference_profile(c, "dz")
    x0 = base_state(seed=6)
    m = api.Model(c)
    m.set_state(x0)
    m.step(nsteps)
    J0, g = tke_objective({f: m.download(f) for f in STATE}, zn, dz)
    m.close()
    m = api.Model(c)
    m.set_state(x0)
    for f in STATE:
        m.upload("adj:" + f, g[f])
    rbar = m.adjoint_run(nsteps, 2)
    th_bar = m.download("adj:th")
    m.close()
    # theta direction: noise on the lowest 10 levels
    dth = np.zeros((NZ, NY, NX))
    dth[1:11] = ini.uniform_noise((10, NY, NX), 21, 1, 1.0)
    eps = 1e-7

    def J_of(th_shift=0.0, rml=None):
        cc = config()
        if rml is not None:
            cc.rmlmax = rml
        st = dict(x0)
        st["th"] = x0["th"] + th_shift * dth
        out = run(st, nsteps, 1, cc)
        return tke_objective(out, zn, dz)[0]

    fd_th = (J_of(eps) - J_of(-eps)) / (2 * eps)
    ad_th = float(np.vdot(th_bar, dth))
    assert abs(fd_th - ad_th) <= 1e-4 * abs(fd_th), (fd_th, ad_th)
    rml0 = c.rmlmax
    h = 1e-6 * rml0
    fd_r = (J_of(rml=rml0 + h) - J_of(rml=rml0 - h)) / (2 * h)
    assert abs(fd_r - rbar) <= 1e-4 * abs(fd_r), (fd_r, rbar)


def test_autograd_function_gradient(gpu_lib):
    """torch.autograd through MoncWindow gives the adjoint gradient; it matches central finite
    differences of the same objective computed in torch."""
    import torch

    from monc_b200 import autodiff

    c = config()
    zn = api.reference_profile(c, "zn")
    dz = torch.from_numpy(api.reference_profile(c, "dz"))
    mask = torch.from_numpy(((zn <= 500.0) & (np.arange(NZ) >= 1)).astype(np.float64))
    base = base_state(seed=6)
    window = autodiff.Window(c, base, nsteps=3, checkpoint_interval=2)

    def J(th, r):
        u, v, w, _ = autodiff.MoncWindow.apply(th, r, window)
        return autodiff.resolved_tke(u, v, w, dz, mask)

    th0 = torch.from_numpy(base["th"]).requires_grad_(True)
    r0 = torch.tensor(c.rmlmax, dtype=torch.float64, requires_grad=True)
    J(th0, r0).backward()
    dth = torch.from_numpy(ini.uniform_noise((NZ, NY, NX), 33, 1, 1.0))
    eps = 1e-7
    with torch.no_grad():
        fd = (J(th0 + eps * dth, r0) - J(th0 - eps * dth, r0)) / (2 * eps)
        fd_r = (J(th0, r0 * (1 + 1e-6)) - J(th0, r0 * (1 - 1e-6))) / (2e-6 * r0)
    ad = float((th0.grad * dth).sum())
    assert abs(ad - float(fd)) <= 1e-4 * abs(float(fd)), (ad, float(fd))
    assert abs(float(r0.grad) - float(fd_r)) <= 1e-4 * abs(float(fd_r)), (float(r0.grad), float(fd_r))


def test_autograd_function_keeps_cuda_tensors_on_the_device(gpu_lib):
    """CUDA tensors cross the MoncWindow boundary device to device (MGPU_LAYOUT_DEVICE); outputs
    and gradients are those of the host-array path, to the bit, and live on the GPU."""
    import torch

    from monc_b200 import autodiff

    c = config()
    zn = api.reference_profile(c, "zn")
    dz = torch.from_numpy(api.reference_profile(c, "dz"))
    mask = torch.from_numpy(((zn <= 500.0) & (np.arange(NZ) >= 1)).astype(np.float64))
    base = base_state(seed=7)
    window = autodiff.Window(c, base, nsteps=3, checkpoint_interval=2)
    grads = {}
    for dev in ("cpu", "cuda"):
        th0 = torch.from_numpy(base["th"]).to(dev).requires_grad_(True)
        r0 = torch.tensor(c.rmlmax, dtype=torch.float64, device=dev, requires_grad=True)
        u, v, w, th = autodiff.MoncWindow.apply(th0, r0, window)
        assert u.device.type == dev and th.device.type == dev
        autodiff.resolved_tke(u, v, w, dz.to(dev), mask.to(dev)).backward()
        assert th0.grad.device.type == dev
        grads[dev] = (th.detach().cpu().numpy(), th0.grad.cpu().numpy(), float(r0.grad))
    assert np.array_equal(grads["cpu"][0], grads["cuda"][0])
    # the objective's own seeds come from torch on each device, so they may differ in the last bit
    g0, g1 = grads["cpu"][1], grads["cuda"][1]
    assert np.abs(g0 - g1).max() <= 1e-12 * np.abs(g0).max()
    assert abs(grads["cpu"][2] - grads["cuda"][2]) <= 1e-12 * abs(grads["cpu"][2])


def test_device_layout_round_trip(gpu_lib):
    """upload_tensor / download_tensor copy in HBM, for FP64 and FP32-mixed models."""
    import torch

    for prec in (cf.FP64, cf.FP32_MIXED):
        c = cf.dry_cbl_config(NX, NY, NZ, DX, DZ, 1.0, precision=prec)
        m = api.Model(c)
        a = torch.from_numpy(ini.uniform_noise((NZ, NY, NX), 8, 3, 300.0)).cuda()
        m.upload_tensor("th", a)
        host = m.download("th")
        dev = m.download_tensor("th", a.device)
        m.close()
        want = a.cpu().numpy() if prec == cf.FP64 else a.cpu().numpy().astype(np.float32).astype(np.float64)
        assert np.array_equal(host, want)
        assert np.array_equal(dev.cpu().numpy(), want)


def test_branch_flips_counts_differing_decisions(gpu_lib):
    """Two models on one state take the same branches; a perturbation of order one changes some
    limiter, upwind or Richardson-regime decisions; the count is symmetric."""
    c = config()
    st = base_state()
    a, b = api.Model(c), api.Model(config())
    a.set_state(st)
    b.set_state(st)
    for m in (a, b):
        m.set_timestep(2)
    assert a.branch_flips(b) == 0
    pert = dict(st)
    pert["u"] = st["u"] + ini.uniform_noise((NZ, NY, NX), 77, 1, 1.0)
    pert["zth"] = st["zth"] + ini.uniform_noise((NZ, NY, NX), 78, 1, 0.5)
    b.set_state(pert)
    b.set_timestep(2)
    n_ab = a.branch_flips(b)
    assert n_ab > 0
    assert b.branch_flips(a) == n_ab
    a.step(1)
    b.step(1)
    assert a.branch_flips(b) > 0
    a.close()
    b.close()
