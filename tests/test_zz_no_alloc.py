"""The allocation-free pressure solve (mgpu_poisson_fft_noalloc) against the fftsolver component.

mgpu_poisson_fft_noalloc serves host models that cannot call cudaMalloc, because their device
memory belongs to another allocator and may not grow during a run: the caller owns the pressure
array and the vertical coefficients on the device, the library keeps its working storage in a
fixed device array.  These tests call it through the C ABI on device buffers the test owns and
compare it with the handle-based fftsolver component on the same right-hand side, within the
FFT-solve tolerance the other parity tests use, on two calls in a row (the second call sees the
scratch the first call left behind).  The free device memory is the same before and after a
call.  The file sorts last so that a run stopping at the first failure has already run every
other test.
"""
import ctypes as C

import numpy as np
import pytest

from monc_b200 import api, config as cf, init as ini

pytestmark = pytest.mark.gpu

FFT_TOL = 1e-11  # the fftsolver tolerance of tests/test_gpu_parity.py


def rel_err(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def _coeffs_on_device(cfg, torch):
    return [torch.tensor(np.ascontiguousarray(api.reference_profile(cfg, n)), dtype=torch.float64, device="cuda")
            for n in ("czb", "cza", "czg", "czh")]


def _noalloc(cfg, p_dev, coeffs):
    czb, cza, czg, czh = (C.c_void_p(t.data_ptr()) for t in coeffs)
    return api.lib().mgpu_poisson_fft_noalloc(C.c_void_p(p_dev.data_ptr()), cfg.nx, cfg.ny, cfg.nz, cfg.dxx,
                                              cfg.dyy, czb, cza, czg, czh, None)


def test_noalloc_poisson_matches_fftsolver_component(gpu_lib):
    import torch

    cfg = cf.dry_cbl_config(64, 32, 40, 50.0, 20.0, 1.0)
    shape = (cfg.nz, cfg.ny, cfg.nx)
    coeffs = _coeffs_on_device(cfg, torch)
    for call, seed in enumerate((3, 4)):
        rhs = ini.uniform_noise(shape, seed, 9, 1e-2)
        rhs[0] = 0.0  # level 1 carries p = 0, as diverr leaves it
        m = api.Model(cfg)
        m.upload("p", rhs)
        m.component("fftsolver")
        ref = m.download("p")
        m.close()
        p_dev = torch.tensor(rhs, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        rc = _noalloc(cfg, p_dev, coeffs)
        torch.cuda.synchronize()
        free_after = torch.cuda.mem_get_info()[0]
        assert rc == api.OK, f"call {call + 1}: status {rc}"
        if call > 0:  # the first call on the device may load the library's module image
            assert free_after == free_before, f"call {call + 1}: free device memory {free_before} -> {free_after}"
        err = rel_err(p_dev.cpu().numpy(), ref)
        assert err <= FFT_TOL, f"call {call + 1}: rel err {err:.3e}"


def test_noalloc_poisson_rejects_grids_beyond_its_scratch(gpu_lib):
    import torch

    cfg = cf.dry_cbl_config(256, 256, 64, 50.0, 20.0, 1.0)
    p_dev = torch.zeros((cfg.nz, cfg.ny, cfg.nx), dtype=torch.float64, device="cuda")
    rc = _noalloc(cfg, p_dev, _coeffs_on_device(cfg, torch))
    torch.cuda.synchronize()
    assert rc == api.ERR_ARGUMENT
