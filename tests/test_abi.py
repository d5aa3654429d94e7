"""The C ABI without a GPU: the library loads, exports every entry include/monc_gpu.h declares,
its structs match the ctypes mirror byte for byte, and the host-only entries behave."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest
import torch

from monc_b200 import api, config as cf, init as ini

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "monc_gpu.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"//[^\n]*", "", text)
    return sorted(set(re.findall(r"\b(mgpu_\w+)\s*\(", text)) - {"mgpu_config", "mgpu_handle"})


def test_header_declares_the_path_entries():
    names = declared_functions()
    for must in ("mgpu_create", "mgpu_destroy", "mgpu_step", "mgpu_component_timestep", "mgpu_upload_field",
                 "mgpu_download_field", "mgpu_poisson_fft_noalloc", "mgpu_last_error"):
        assert must in names


def test_library_exports_every_declared_symbol():
    L = api.lib()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing


def _compile_layout_probe(tmp_path, struct, fields):
    src = tmp_path / "probe.c"
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "monc_gpu.h"', "int main(void){",
             f'printf("size %zu\\n", sizeof({struct}));']
    for f in fields:
        lines.append(f'printf("{f} %zu\\n", offsetof({struct}, {f}));')
    lines += ["return 0;}"]
    src.write_text("\n".join(lines))
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    return {k: int(v) for k, v in (ln.split() for ln in out.strip().splitlines())}


def test_config_struct_layout_matches_ctypes(tmp_path):
    fields = [f for f, _ in cf.MgpuConfig._fields_]
    got = _compile_layout_probe(tmp_path, "mgpu_config", fields)
    assert got["size"] == C.sizeof(cf.MgpuConfig)
    for f in fields:
        assert got[f] == getattr(cf.MgpuConfig, f).offset, f


def test_reductions_struct_layout_matches_ctypes(tmp_path):
    fields = [f for f, _ in api.Reductions._fields_]
    got = _compile_layout_probe(tmp_path, "mgpu_reductions", fields)
    assert got["size"] == C.sizeof(api.Reductions)
    for f in fields:
        assert got[f] == getattr(api.Reductions, f).offset, f


def test_config_defaults_match_python_mirror():
    c_side = cf.MgpuConfig()
    api.lib().mgpu_config_defaults(C.byref(c_side))
    py_side = cf.default_config()
    for f, t in cf.MgpuConfig._fields_:
        a, b = getattr(c_side, f), getattr(py_side, f)
        if hasattr(a, "__len__"):
            assert list(a) == list(b), f
        else:
            assert a == b, f


def test_reference_profile_rejects_unknown_name():
    cfg = cf.dry_cbl_config(16, 16, 10, 50.0, 25.0, 1.0)
    with pytest.raises(api.MgpuError):
        api.reference_profile(cfg, "no_such_profile")


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the no-device path")
def test_create_without_device_fails_loudly():
    cfg = cf.dry_cbl_config(16, 16, 10, 50.0, 25.0, 1.0)
    h = C.c_void_p()
    rc = api.lib().mgpu_create(C.byref(cfg), C.byref(h))
    assert rc == api.ERR_NO_DEVICE
    assert not h.value
    with pytest.raises(api.MgpuError):
        api.Model(cfg)


@pytest.mark.parametrize("nx,ny,nz", [(28, 32, 10), (32, 22, 10), (32, 27, 10), (32, 32, 2), (2, 32, 10),
                                      (8192, 32, 10)])
def test_create_rejects_unsupported_grids(nx, ny, nz):
    """Horizontal sizes with a prime factor above 5 or beyond 4096 points (FFT), odd sizes and
    fewer than 3 levels are argument errors, checked on the host before any device work."""
    cfg = cf.dry_cbl_config(nx, ny, nz, 50.0, 25.0, 1.0)
    h = C.c_void_p()
    rc = api.lib().mgpu_create(C.byref(cfg), C.byref(h))
    assert rc == api.ERR_ARGUMENT
    assert not h.value


def test_null_handle_is_an_argument_error():
    L = api.lib()
    assert L.mgpu_step(None, 1) == api.ERR_ARGUMENT
    assert L.mgpu_destroy(None) == api.ERR_ARGUMENT
    assert L.mgpu_last_error(None)


def test_noalloc_rejects_bad_arguments_on_host():
    L = api.lib()
    prof = np.zeros(64)
    p = prof.ctypes.data
    # nx not a power of two, then a grid whose spectrum exceeds the static scratch
    assert L.mgpu_poisson_fft_noalloc(p, 48, 32, 8, 1.0, 1.0, p, p, p, p, None) == api.ERR_ARGUMENT
    assert L.mgpu_poisson_fft_noalloc(p, 512, 512, 128, 1.0, 1.0, p, p, p, p, None) == api.ERR_ARGUMENT
    assert L.mgpu_poisson_fft_noalloc(None, 32, 32, 8, 1.0, 1.0, p, p, p, p, None) == api.ERR_ARGUMENT


def test_splitmix_generator_matches_scalar_definition():
    """uniform_noise is SplitMix64 of index ^ (seed << 24) ^ (field << 56), top 53 bits mapped to
    [-amp, amp)."""
    M = (1 << 64) - 1

    def splitmix(x):
        x = (x + 0x9E3779B97F4A7C15) & M
        z = x
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M
        return z ^ (z >> 31)

    a = ini.uniform_noise((2, 3, 4), seed=7, field=3, amplitude=0.5)
    flat = a.reshape(-1)
    for idx in (0, 5, 23):
        r = splitmix(idx ^ (7 << 24) ^ (3 << 56)) >> 11
        expect = 0.5 * (2.0 * (r * 2.0 ** -53) - 1.0)
        assert flat[idx] == expect
