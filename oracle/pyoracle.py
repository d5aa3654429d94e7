"""ctypes wrapper of the CPU oracle (test infrastructure only).

The oracle is a C++ restatement of MONC's Fortran dynamical-core timestep (monc_oracle.cpp).
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this module, as the
checker; the GPU library never calls it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libmonc_oracle.so")
# MONC_ORACLE_LIB=native loads the -O3 -march=native build that bench.py times as the CPU
# baseline; the checker (tests, smoke) always uses the default build
_NATIVE_PATH = os.path.join(_HERE, "_build", "libmonc_oracle_native.so")
_lib = None


def build(native: bool = False) -> str:
    subprocess.run(["make", "-s", "-C", _HERE] + (["native"] if native else []), check=True)
    return _NATIVE_PATH if native else _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        native = os.environ.get("MONC_ORACLE_LIB") == "native"
        L = C.CDLL(build(native))  # make is a no-op when the library is newer than its sources
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.c_void_p]
        L.orc_destroy.argtypes = [C.c_void_p]
        for name in ("orc_set_field", "orc_get_field", "orc_get_field_monc"):
            f = getattr(L, name)
            f.restype = C.c_int
            f.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        L.orc_get_profile.restype = C.c_int
        L.orc_get_profile.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p]
        L.orc_step.restype = C.c_int
        L.orc_step.argtypes = [C.c_void_p, C.c_int]
        L.orc_set_timestep.restype = C.c_int
        L.orc_set_timestep.argtypes = [C.c_void_p, C.c_int]
        L.orc_component.restype = C.c_int
        L.orc_component.argtypes = [C.c_void_p, C.c_int]
        L.orc_divmax.restype = C.c_double
        L.orc_divmax.argtypes = [C.c_void_p]
        L.orc_solver_iterations.restype = C.c_int
        L.orc_solver_iterations.argtypes = [C.c_void_p]
        L.orc_solver_residual.restype = C.c_double
        L.orc_solver_residual.argtypes = [C.c_void_p]
        L.orc_fft_c2c.restype = C.c_int
        L.orc_fft_c2c.argtypes = [C.c_int, C.c_void_p, C.c_int]
        L.orc_lookup_ustr.restype = C.c_double
        L.orc_lookup_ustr.argtypes = [C.c_void_p, C.c_double]
        L.orc_mean_q_profile.restype = C.c_int
        L.orc_mean_q_profile.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        L.orc_profile_diagnostics.restype = C.c_int
        L.orc_profile_diagnostics.argtypes = [C.c_void_p, C.c_void_p]
        L.orc_cfl_state.restype = C.c_int
        L.orc_cfl_state.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        _lib = L
    return _lib


CFL_TOO_SMALL = -7  # MGPU_ERR_CFL


class CflError(RuntimeError):
    pass


class Oracle:
    """One CPU model instance (MONC layout internally, [nz][ny][nx] arrays at the boundary)."""

    def __init__(self, cfg):
        self.cfg = cfg
        self.nx, self.ny, self.nz = cfg.nx, cfg.ny, cfg.nz
        self.h = lib().orc_create(C.byref(cfg))
        if not self.h:
            raise RuntimeError("oracle creation failed")

    def close(self):
        if self.h:
            lib().orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set(self, fid: int, arr: np.ndarray):
        a = np.ascontiguousarray(arr, dtype=np.float64).reshape(self.nz, self.ny, self.nx)
        if lib().orc_set_field(self.h, fid, a.ctypes.data) != 0:
            raise KeyError(fid)

    def get(self, fid: int) -> np.ndarray:
        a = np.empty((self.nz, self.ny, self.nx), dtype=np.float64)
        if lib().orc_get_field(self.h, fid, a.ctypes.data) != 0:
            raise KeyError(fid)
        return a

    def get_monc(self, fid: int) -> np.ndarray:
        a = np.empty((self.nx + 4, self.ny + 4, self.nz), dtype=np.float64)
        if lib().orc_get_field_monc(self.h, fid, a.ctypes.data) != 0:
            raise KeyError(fid)
        return a

    def mean_profiles(self) -> dict:
        """olzubar, olzvbar, olzthbar and olzqbar(n) as the last mean_profiles left them."""
        out = {n: self.profile(n) for n in ("olzubar", "olzvbar", "olzthbar", "olubar", "olvbar", "olthbar")}
        for n in range(self.cfg.number_q_fields):
            a = np.empty(self.nz, dtype=np.float64)
            if lib().orc_mean_q_profile(self.h, n, a.ctypes.data) != 0:
                raise RuntimeError("orc_mean_q_profile")
            out[f"olzqbar{n}"] = a
        return out

    def profile_diagnostics(self) -> dict:
        """profile_diagnostics sums from the current state (MGPU_PD_* rows), by MONC's names."""
        from monc_b200.api import PROFILE_DIAGNOSTICS
        out = np.empty((len(PROFILE_DIAGNOSTICS), self.nz), dtype=np.float64)
        rows = lib().orc_profile_diagnostics(self.h, out.ctypes.data)
        return dict(zip(PROFILE_DIAGNOSTICS[:rows], out[:rows]))

    def profile(self, name: str) -> np.ndarray:
        a = np.empty(self.nz, dtype=np.float64)
        if lib().orc_get_profile(self.h, name.encode(), a.ctypes.data) != 0:
            raise KeyError(name)
        return a

    def step(self, n: int = 1):
        rc = lib().orc_step(self.h, n)
        if rc == CFL_TOO_SMALL:
            raise CflError("cfltest: the new timestep fell below cfl_dtmmin")
        if rc != 0:
            raise RuntimeError("oracle step failed")

    def cfl_state(self) -> dict:
        """cfltest's state after the last step (the mgpu_reductions fields of the same names)."""
        v = np.zeros(11)
        i = np.zeros(2, dtype=np.int32)
        lib().orc_cfl_state(self.h, v.ctypes.data, i.ctypes.data)
        keys = ["dtm", "dtm_new", "absolute_new_dtm", "cvel", "cvis", "cfl_number", "cvel_x", "cvel_y", "cvel_z",
                "ugal", "vgal"]
        out = dict(zip(keys, (float(x) for x in v)))
        out["cfl_evaluations"], out["last_cfl_timestep"] = int(i[0]), int(i[1])
        return out

    def set_timestep(self, ts: int):
        lib().orc_set_timestep(self.h, ts)

    def component(self, cid: int):
        rc = lib().orc_component(self.h, cid)
        if rc != 0:
            raise RuntimeError(f"oracle component {cid} failed ({rc})")

    def divmax(self) -> float:
        return lib().orc_divmax(self.h)

    def solver_stats(self):
        return lib().orc_solver_iterations(self.h), lib().orc_solver_residual(self.h)

    def lookup_ustr(self, vel: float) -> float:
        return lib().orc_lookup_ustr(self.h, vel)


def fft_c2c(x: np.ndarray, sign: int) -> np.ndarray:
    """FFTPACK zfftf (sign=-1) / zfftb (sign=+1) of a complex vector, unnormalised."""
    n = len(x)
    buf = np.empty(2 * n, dtype=np.float64)
    buf[0::2] = x.real
    buf[1::2] = x.imag
    if lib().orc_fft_c2c(n, buf.ctypes.data, sign) != 0:
        raise ValueError("length must have no prime factor above 5")
    return buf[0::2] + 1j * buf[1::2]
