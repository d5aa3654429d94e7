"""The allocation-free pressure solve (mgpu_poisson_fft_noalloc) against the fftsolver component.

mgpu_poisson_fft_noalloc serves callers that may not allocate device memory (for instance code
running under CUDA graph capture): the caller owns the pressure array, the library keeps its
working storage in a fixed device array.  These tests call it through the C ABI on a device
buffer the test owns and compare it with the handle-based fftsolver component on the same
right-hand side, within the FFT-solve tolerance the other parity tests use, on two calls in a
row (the second call sees the scratch the first call left behind).  The file sorts last so that
a run stopping at the first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from monc_b200 import api, config as cf, init as ini

pytestmark = pytest.mark.gpu

FFT_TOL = 1e-11  # the fftsolver tolerance of tests/test_gpu_parity.py


def rel_err(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def _coeffs(cfg):
    return [np.ascontiguousarray(api.reference_profile(cfg, n)) for n in ("czb", "cza", "czg", "czh")]


def _noalloc(cfg, rhs, torch):
    p_dev = torch.tensor(rhs, dtype=torch.float64, device="cuda")
    czb, cza, czg, czh = _coeffs(cfg)
    rc = api.lib().mgpu_poisson_fft_noalloc(
        C.c_void_p(p_dev.data_ptr()), cfg.nx, cfg.ny, cfg.nz, cfg.dxx, cfg.dyy,
        czb.ctypes.data, cza.ctypes.data, czg.ctypes.data, czh.ctypes.data, None)
    torch.cuda.synchronize()
    return rc, p_dev.cpu().numpy()


def test_noalloc_poisson_matches_fftsolver_component(gpu_lib):
    import torch

    cfg = cf.dry_cbl_config(64, 32, 40, 50.0, 20.0, 1.0)
    shape = (cfg.nz, cfg.ny, cfg.nx)
    for call, seed in enumerate((3, 4)):
        rhs = ini.uniform_noise(shape, seed, 9, 1e-2)
        rhs[0] = 0.0  # level 1 carries p = 0, as diverr leaves it
        m = api.Model(cfg)
        m.upload("p", rhs)
        m.component("fftsolver")
        ref = m.download("p")
        m.close()
        rc, got = _noalloc(cfg, rhs, torch)
        assert rc == api.OK, f"call {call + 1}: status {rc}"
        err = rel_err(got, ref)
        assert err <= FFT_TOL, f"call {call + 1}: rel err {err:.3e}"


def test_noalloc_poisson_rejects_grids_beyond_its_scratch(gpu_lib):
    import torch

    cfg = cf.dry_cbl_config(256, 256, 64, 50.0, 20.0, 1.0)
    rhs = np.zeros((cfg.nz, cfg.ny, cfg.nx))
    rc, _ = _noalloc(cfg, rhs, torch)
    assert rc == api.ERR_ARGUMENT
