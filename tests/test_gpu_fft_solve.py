"""The FFT pressure solve on deep columns, where the tridiagonal solve stages many chunks of levels
through shared memory: FP64 against the oracle, FP32-mixed against FP64, and repeated solves of
one right-hand side bit for bit identical (a race between threads' staging slots would show up as
run-to-run differences).
"""
import numpy as np
import pytest

from monc_b200 import api, config as cf, init as ini
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


def setup(nx, ny, nz, precision):
    c = cf.dry_cbl_config(nx, ny, nz, 50.0, 20.0, 0.5, precision=precision)
    rhs = ini.uniform_noise((nz, ny, nx), 17, 3, 1e-3)
    rhs[0] = 0.0
    return c, rhs


def solve(c, rhs, repeats=1, adjoint=False):
    m = api.Model(c)
    outs = []
    for _ in range(repeats):
        m.upload("p", rhs)
        if adjoint:
            m.fftsolver_adjoint()
        else:
            m.component("fftsolver")
        outs.append(m.download("p"))
    m.close()
    return outs


@pytest.mark.parametrize("nx,ny,nz", [(64, 64, 160), (128, 32, 67)])
def test_deep_fp64_solve_matches_oracle(gpu_lib, nx, ny, nz):
    c, rhs = setup(nx, ny, nz, cf.FP64)
    o = po.Oracle(c)
    o.set(api.FIELDS["p"], rhs)
    o.component(api.COMPONENTS["fftsolver"])
    ref = o.get(api.FIELDS["p"])
    got = solve(c, rhs)[0]
    assert np.abs(got - ref).max() <= 1e-11 * np.abs(ref).max()


@pytest.mark.parametrize("adjoint", [False, True], ids=["solve", "transpose"])
def test_deep_fp32_solve_tracks_fp64_and_repeats_exactly(gpu_lib, adjoint):
    c64, rhs = setup(64, 64, 160, cf.FP64)
    c32, _ = setup(64, 64, 160, cf.FP32_MIXED)
    ref = solve(c64, rhs, adjoint=adjoint)[0]
    outs = solve(c32, rhs, repeats=8, adjoint=adjoint)
    for o in outs[1:]:
        np.testing.assert_array_equal(o, outs[0])
    assert np.abs(outs[0] - ref).max() <= 2e-5 * np.abs(ref).max()
    outs64 = solve(c64, rhs, repeats=4, adjoint=adjoint)
    for o in outs64:
        np.testing.assert_array_equal(o, ref)
