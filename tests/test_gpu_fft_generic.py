"""Horizontal sizes that are not powers of two (MONC's FFTPACK factorises 2, 3, 4 and 5; for
example 96 = 2^5 3, 100 = 2^2 5^2, 384 = 2^7 3): the mixed-radix FFT kernels in the pressure
solve against the oracle's FFTPACK restatement, the component alone and whole fused steps."""
import numpy as np
import pytest

from monc_b200 import api, config as cf, init as ini
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


def rel_err(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("precision", [cf.FP64, cf.FP32_MIXED], ids=["fp64", "fp32"])
@pytest.mark.parametrize("nx,ny,nz", [(96, 96, 24), (100, 60, 16), (90, 150, 12), (384, 48, 10), (30, 64, 12)])
def test_fftsolver_component_matches_oracle(gpu_lib, nx, ny, nz, precision):
    cfg = cf.dry_cbl_config(nx, ny, nz, 50.0, 20.0, 1.0, precision=precision)
    o, m = po.Oracle(cfg), api.Model(cfg)
    rhs = ini.uniform_noise((nz, ny, nx), 3, 9, 1e-2)
    rhs[0] = 0.0
    o.set(api.FIELDS["p"], rhs)
    m.upload("p", rhs)
    o.set_timestep(2)
    m.set_timestep(2)
    o.component(api.COMPONENTS["fftsolver"])
    m.component("fftsolver")
    e = rel_err(m.download("p"), o.get(api.FIELDS["p"]))
    assert e <= (1e-11 if precision == cf.FP64 else 2e-4), f"rel err {e:.3e}"
    m.close()
    o.close()


@pytest.mark.parametrize("n,nz", [(96, 40), (60, 24)])
def test_fused_steps_on_generic_grid_match_oracle(gpu_lib, n, nz):
    cfg = cf.dry_cbl_config(n, n, nz, 50.0, 25.0, 1.0, ug=5.0, fcoriol=1e-4)
    o, m = po.Oracle(cfg), api.Model(cfg)
    zn = o.profile("zn")
    st = ini.dry_cbl_state(n, n, nz, zn, seed=5, ug=5.0)
    flow = ini.random_flow_state(n, n, nz, seed=6, amp_uv=0.5, amp_w=0.2, amp_th=0.0, ug=5.0)
    for k in ("u", "v", "w"):
        st[k] = flow[k]
    for name, arr in st.items():
        o.set(api.field_id(name), arr)
        m.upload(name, arr)
    o.step(4)
    m.step(4)
    for f in ("u", "v", "w", "th", "zu", "zv", "zw", "zth", "p"):
        e = rel_err(m.download(f), o.get(api.field_id(f)))
        assert e <= 1e-10, f"{f}: rel err {e:.3e}"
    m.close()
    o.close()


def test_transposed_solve_on_generic_grid_is_the_adjoint(gpu_lib):
    """<A^-1 x, y> = <x, A^-T y> for the mixed-radix solve and its transpose."""
    cfg = cf.dry_cbl_config(96, 60, 20, 50.0, 20.0, 1.0)
    shape = (cfg.nz, cfg.ny, cfg.nx)
    x = ini.uniform_noise(shape, 1, 1, 1.0)
    y = ini.uniform_noise(shape, 2, 1, 1.0)
    x[0] = 0.0
    y[0] = 0.0
    m = api.Model(cfg)
    m.upload("p", x)
    m.set_timestep(2)
    m.component("fftsolver")
    ax = m.download("p")
    m.upload("p", y)
    m.fftsolver_adjoint()
    aty = m.download("p")
    m.close()
    lhs, rhs = float(np.vdot(ax, y)), float(np.vdot(x, aty))
    assert abs(lhs - rhs) <= 1e-10 * max(abs(lhs), 1e-300)
