"""Python binding of libmoncgpu.so and a host-side mirror of MONC's component API.

`Model` owns one device-resident model (mgpu_create ... mgpu_destroy).  `component_descriptor`
returns, for each dynamical-core component MONC registers (monc_component.F90:62-71), a
descriptor with the same name and initialisation / timestep / finalisation callbacks, whose
timestep callback runs the GPU kernel of that component over the whole domain -- the form a
MONC `entire` group expects.

The CUDA library is required: every entry point raises if libmoncgpu.so cannot be loaded or
no CUDA device is visible; nothing falls back to the CPU.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass
from typing import Callable, Optional

import numpy as np

from . import config as cf

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmoncgpu.so")

OK = 0
ERR_ARGUMENT = -1
ERR_CUDA = -2
ERR_NOT_CONVERGED = -3
ERR_TIMEOUT = -4
ERR_UNSUPPORTED = -5
ERR_NO_DEVICE = -6
ERR_CFL = -7

LAYOUT_XFAST = 0
LAYOUT_MONC = 1
LAYOUT_DEVICE = 2

FIELDS = {
    "u": 0, "v": 1, "w": 2, "th": 3, "zu": 4, "zv": 5, "zw": 6, "zth": 7, "p": 8,
    "su": 9, "sv": 10, "sw": 11, "sth": 12, "vis": 13, "diff": 14,
    "savu": 15, "savv": 16, "savw": 17,
}
Q0, ZQ0, SQ0 = 32, 48, 64
TANGENT0, ADJOINT0 = 1024, 2048  # + id of a state field (u v w th zu zv zw zth = 0..7)
STATE_FIELDS = ["u", "v", "w", "th", "zu", "zv", "zw", "zth"]

STAGES = ["subgrid", "dynamics", "pressure_source", "fft_x_fwd", "fft_y_fwd", "tridiag", "fft_y_inv",
          "fft_x_inv", "pstep_swap", "iterative", "dynamics_momentum"]

# registered MONC component names -> mgpu_component_id
COMPONENTS = {
    "clearsourceterms": 0,
    "stepping_direction": 1,
    "halo_swapper": 2,
    "lower_bc": 3,
    "smagorinsky": 4,
    "pw_advection": 5,
    "tvd_advection": 6,
    "diffusion": 7,
    "viscosity": 8,
    "coriolis": 9,
    "buoyancy": 10,
    "set_consistent_lowbc": 11,
    "simplecloud": 12,
    "diverr": 13,
    "psrce": 14,
    "stepfields": 15,
    "fftsolver": 16,
    "iterativesolver": 17,
    "pstep": 18,
    "swap_smooth": 19,
    "mean_profiles": 20,
    "damping": 21,
    "forcing": 22,
    "th_advection": 23,
}

# the profile_diagnostics sums mgpu_profile_diagnostics returns, under the names MONC's component
# publishes them (profile_diagnostics.F90:74-118), in the MGPU_PD_* row order
PROFILE_DIAGNOSTICS = ["u_wind_total_local", "v_wind_total_local", "w_wind_total_local", "ww_total_local",
                       "www_total_local", "wwww_total_local", "theta_total_local", "th2_total_local",
                       "wtheta_cn_total_local", "uw_total_local", "vw_total_local", "vapour_mmr_total_local",
                       "liquid_mmr_total_local", "wqv_cn_total_local", "wql_cn_total_local", "rh_total_local"]

# MONC's default group layout of these components (global_config:77-92)
GROUPS = {
    "start": ["clearsourceterms", "stepping_direction", "halo_swapper"],
    "subgrid": ["lower_bc", "smagorinsky"],
    "dynamics": ["pw_advection", "tvd_advection", "th_advection", "diffusion", "viscosity", "coriolis", "buoyancy",
                 "damping", "forcing", "set_consistent_lowbc", "simplecloud", "diverr", "psrce", "stepfields"],
    "solver": ["mean_profiles", "fftsolver", "iterativesolver"],
    "pressure-terms": ["pstep", "swap_smooth"],
}


class CheckpointMeta(C.Structure):
    """mgpu_checkpoint_meta: the step count, time and dtm state a MONC checkpoint carries."""
    _fields_ = [("timestep", C.c_int32), ("last_cfl_timestep", C.c_int32), ("time", C.c_double),
                ("dtm", C.c_double), ("dtm_new", C.c_double), ("absolute_new_dtm", C.c_double),
                ("ugal", C.c_double), ("vgal", C.c_double)]


class MgpuError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"libmoncgpu error {code}: {msg}")
        self.code = code


class Reductions(C.Structure):
    _fields_ = [("global_divmax", C.c_double), ("solver_iterations", C.c_int32),
                ("solver_residual", C.c_double), ("timestep", C.c_int32),
                ("dtm", C.c_double), ("dtm_new", C.c_double), ("absolute_new_dtm", C.c_double),
                ("cvel", C.c_double), ("cvis", C.c_double), ("cfl_number", C.c_double),
                ("cvel_x", C.c_double), ("cvel_y", C.c_double), ("cvel_z", C.c_double),
                ("cfl_evaluations", C.c_int32), ("last_cfl_timestep", C.c_int32),
                ("ugal", C.c_double), ("vgal", C.c_double)]


_lib = None


def lib():
    """Load libmoncgpu.so (building it first if it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        from .build import build
        build()
    L = C.CDLL(LIB_PATH)
    L.mgpu_config_defaults.argtypes = [C.c_void_p]
    L.mgpu_config_defaults.restype = None
    L.mgpu_create.argtypes = [C.c_void_p, C.POINTER(C.c_void_p)]
    L.mgpu_create.restype = C.c_int
    L.mgpu_destroy.argtypes = [C.c_void_p]
    L.mgpu_destroy.restype = C.c_int
    for name in ("mgpu_upload_field", "mgpu_download_field"):
        f = getattr(L, name)
        f.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32]
        f.restype = C.c_int
    L.mgpu_get_profile.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p, C.POINTER(C.c_int32)]
    L.mgpu_get_profile.restype = C.c_int
    L.mgpu_step.argtypes = [C.c_void_p, C.c_int32]
    L.mgpu_step.restype = C.c_int
    L.mgpu_component_timestep.argtypes = [C.c_void_p, C.c_int32]
    L.mgpu_component_timestep.restype = C.c_int
    L.mgpu_set_timestep.argtypes = [C.c_void_p, C.c_int32]
    L.mgpu_set_timestep.restype = C.c_int
    L.mgpu_get_reductions.argtypes = [C.c_void_p, C.c_void_p]
    L.mgpu_get_reductions.restype = C.c_int
    L.mgpu_cfl_gather.argtypes = [C.c_void_p, C.c_void_p]
    L.mgpu_cfl_gather.restype = C.c_int
    L.mgpu_mean_profile.argtypes = [C.c_void_p, C.c_int32, C.c_void_p]
    L.mgpu_mean_profile.restype = C.c_int
    L.mgpu_stream.argtypes = [C.c_void_p]
    L.mgpu_stream.restype = C.c_void_p
    L.mgpu_launch_count.argtypes = [C.c_void_p]
    L.mgpu_launch_count.restype = C.c_int64
    L.mgpu_diagnostics.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    L.mgpu_diagnostics.restype = C.c_int
    L.mgpu_mean_profiles.argtypes = [C.c_void_p, C.c_void_p]
    L.mgpu_mean_profiles.restype = C.c_int
    L.mgpu_profile_diagnostics.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_int32)]
    L.mgpu_profile_diagnostics.restype = C.c_int
    for name in ("mgpu_checkpoint_write", "mgpu_checkpoint_read"):
        f = getattr(L, name)
        f.argtypes = [C.c_void_p, C.c_char_p]
        f.restype = C.c_int
    L.mgpu_checkpoint_write_host.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.mgpu_checkpoint_write_host.restype = C.c_int
    L.mgpu_checkpoint_read_host.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                            C.c_void_p]
    L.mgpu_checkpoint_read_host.restype = C.c_int
    L.mgpu_set_profiling.argtypes = [C.c_void_p, C.c_int32]
    L.mgpu_set_profiling.restype = C.c_int
    L.mgpu_stage_times.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    L.mgpu_stage_times.restype = C.c_int
    L.mgpu_reference_profile.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p]
    L.mgpu_reference_profile.restype = C.c_int
    L.mgpu_poisson_fft_noalloc.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_double, C.c_double,
                                           C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.mgpu_poisson_fft_noalloc.restype = C.c_int
    L.mgpu_branch_flips.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_int64)]
    L.mgpu_branch_flips.restype = C.c_int
    L.mgpu_fftsolver_adjoint.argtypes = [C.c_void_p]
    L.mgpu_fftsolver_adjoint.restype = C.c_int
    L.mgpu_tl_step.argtypes = [C.c_void_p, C.c_int32, C.c_double]
    L.mgpu_tl_step.restype = C.c_int
    L.mgpu_adjoint_run.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.POINTER(C.c_double)]
    L.mgpu_adjoint_run.restype = C.c_int
    L.mgpu_last_error.argtypes = [C.c_void_p]
    L.mgpu_last_error.restype = C.c_char_p
    L.mgpu_slab_init.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_int32]
    L.mgpu_slab_init.restype = C.c_int
    L.mgpu_step_phase.argtypes = [C.c_void_p, C.c_int32]
    L.mgpu_step_phase.restype = C.c_int
    L.mgpu_halo_fields.argtypes = [C.c_void_p, C.c_int32]
    L.mgpu_halo_fields.restype = C.c_int
    for name in ("mgpu_halo_pack", "mgpu_halo_unpack"):
        f = getattr(L, name)
        f.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p]
        f.restype = C.c_int
    L.mgpu_slab_level_means.argtypes = [C.c_void_p, C.c_void_p]
    L.mgpu_slab_level_means.restype = C.c_int
    L.mgpu_slab_iter.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.POINTER(C.c_int32)]
    L.mgpu_slab_iter.restype = C.c_int
    L.mgpu_checkpoint_state.argtypes = [C.c_void_p, C.c_void_p]
    L.mgpu_checkpoint_state.restype = C.c_int
    L.mgpu_restore_state.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    L.mgpu_restore_state.restype = C.c_int
    L.mgpu_set_galilean_velocity.argtypes = [C.c_void_p, C.c_double, C.c_double]
    L.mgpu_set_galilean_velocity.restype = C.c_int
    L.mgpu_slab_mean_profiles.argtypes = [C.c_void_p, C.c_void_p, C.c_int32]
    L.mgpu_slab_mean_profiles.restype = C.c_int
    L.mgpu_slab_cfl_extrema.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.POINTER(C.c_int32)]
    L.mgpu_slab_cfl_extrema.restype = C.c_int
    L.mgpu_slab_fft_x.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_int32]
    L.mgpu_slab_fft_x.restype = C.c_int
    L.mgpu_slab_solve_columns.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32]
    L.mgpu_slab_solve_columns.restype = C.c_int
    _lib = L
    return _lib


def field_id(name_or_id) -> int:
    if isinstance(name_or_id, (int, np.integer)):
        return int(name_or_id)
    name = str(name_or_id)
    if name in FIELDS:
        return FIELDS[name]
    for prefix, base in (("tl:", TANGENT0), ("adj:", ADJOINT0)):
        if name.startswith(prefix) and name[len(prefix):] in STATE_FIELDS:
            return base + FIELDS[name[len(prefix):]]
    for prefix, base in (("zq", ZQ0), ("sq", SQ0), ("q", Q0)):
        if name.startswith(prefix) and name[len(prefix):].isdigit():
            return base + int(name[len(prefix):])
    raise KeyError(name)


def reference_profile(cfg: cf.MgpuConfig, name: str) -> np.ndarray:
    """Host-only reference-state profile of a configuration (no device needed)."""
    out = np.empty(cfg.nz, dtype=np.float64)
    rc = lib().mgpu_reference_profile(C.byref(cfg), name.encode(), out.ctypes.data)
    if rc != OK:
        raise MgpuError(rc, f"reference profile {name}")
    return out


class Model:
    """A device-resident MONC dynamical core on the current CUDA device."""

    def __init__(self, cfg: cf.MgpuConfig):
        self.cfg = cfg
        self.nx, self.ny, self.nz = cfg.nx, cfg.ny, cfg.nz
        h = C.c_void_p()
        rc = lib().mgpu_create(C.byref(cfg), C.byref(h))
        if rc != OK:
            raise MgpuError(rc, "mgpu_create failed (no CUDA device, bad configuration or out of memory)")
        self.h = h

    # -- lifecycle
    def close(self):
        if getattr(self, "h", None):
            lib().mgpu_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int, what: str):
        if rc != OK:
            msg = lib().mgpu_last_error(self.h)
            raise MgpuError(rc, f"{what}: {msg.decode() if msg else ''}")

    # -- data
    def upload(self, name, arr: np.ndarray, layout: int = LAYOUT_XFAST):
        a = np.ascontiguousarray(arr, dtype=np.float64)
        if layout == LAYOUT_XFAST:
            a = a.reshape(self.nz, self.ny, self.nx)
        self._check(lib().mgpu_upload_field(self.h, field_id(name), a.ctypes.data, layout), f"upload {name}")

    def download(self, name, layout: int = LAYOUT_XFAST) -> np.ndarray:
        if layout == LAYOUT_XFAST:
            a = np.empty((self.nz, self.ny, self.nx), dtype=np.float64)
        else:
            a = np.empty((self.nx + 4, self.ny + 4, self.nz), dtype=np.float64)
        self._check(lib().mgpu_download_field(self.h, field_id(name), a.ctypes.data, layout), f"download {name}")
        return a

    def upload_tensor(self, name, t):
        """Copy a contiguous FP64 CUDA tensor [nz][ny][nx] into the model; it stays in HBM."""
        import torch

        if not (t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()
                and tuple(t.shape) == (self.nz, self.ny, self.nx)):
            raise ValueError(f"upload {name}: needs a contiguous float64 CUDA tensor of shape "
                             f"{(self.nz, self.ny, self.nx)}")
        torch.cuda.current_stream(t.device).synchronize()  # the tensor's producers have finished
        self._check(lib().mgpu_upload_field(self.h, field_id(name), t.data_ptr(), LAYOUT_DEVICE), f"upload {name}")

    def download_tensor(self, name, device):
        """A new FP64 CUDA tensor [nz][ny][nx] on `device` holding the field, copied in HBM."""
        import torch

        out = torch.empty((self.nz, self.ny, self.nx), dtype=torch.float64, device=device)
        torch.cuda.current_stream(out.device).synchronize()  # the memory's earlier users are done with it
        self._check(lib().mgpu_download_field(self.h, field_id(name), out.data_ptr(), LAYOUT_DEVICE),
                    f"download {name}")
        return out

    def set_state(self, state: dict):
        for k, v in state.items():
            self.upload(k, v)

    def profile(self, name: str) -> np.ndarray:
        out = np.empty(self.nz, dtype=np.float64)
        n = C.c_int32()
        self._check(lib().mgpu_get_profile(self.h, name.encode(), out.ctypes.data, C.byref(n)), f"profile {name}")
        return out

    # -- stepping
    def step(self, n: int = 1):
        self._check(lib().mgpu_step(self.h, n), "step")

    def component(self, name: str):
        self._check(lib().mgpu_component_timestep(self.h, COMPONENTS[name]), f"component {name}")

    def set_timestep(self, ts: int):
        self._check(lib().mgpu_set_timestep(self.h, ts), "set_timestep")

    def branch_flips(self, other: "Model") -> int:
        """Branch decisions (theta TVD faces, Smagorinsky regime) in which this model's next step
        and `other`'s differ (dry FP64 models of one grid)."""
        n = C.c_int64(0)
        self._check(lib().mgpu_branch_flips(self.h, other.h, C.byref(n)), "branch_flips")
        return int(n.value)

    def fftsolver_adjoint(self):
        """Apply the transpose of the FFT pressure solve to p in place."""
        self._check(lib().mgpu_fftsolver_adjoint(self.h), "fftsolver_adjoint")

    def tl_step(self, n: int = 1, d_rmlmax: float = 0.0):
        """Advance the state and its tangent (fields "tl:u" ...) n steps (dry FP64 models)."""
        self._check(lib().mgpu_tl_step(self.h, n, d_rmlmax), "tl_step")

    def adjoint_run(self, n: int, checkpoint_interval: int = 25) -> float:
        """Adjoint of n steps from the current state: fields "adj:u" ... hold dJ/d(state after n
        steps) on entry and dJ/d(current state) on return; the state ends n steps on.  Returns
        dJ/d rmlmax."""
        out = C.c_double(0.0)
        self._check(lib().mgpu_adjoint_run(self.h, n, checkpoint_interval, C.byref(out)), "adjoint_run")
        return out.value

    def reductions(self) -> Reductions:
        r = Reductions()
        self._check(lib().mgpu_get_reductions(self.h, C.byref(r)), "reductions")
        return r

    def set_galilean_velocity(self, ugal: float, vgal: float):
        self._check(lib().mgpu_set_galilean_velocity(self.h, ugal, vgal), "set_galilean_velocity")

    def cfl_gather(self) -> np.ndarray:
        """cfltest's extrema from the current fields: min zu, max zu, min zv, max zv,
        max |zw| rdzn(k+1), max max(vis, diff) (rdzn(k+1)^2 + cx2 + cy2)."""
        out = np.zeros(6, dtype=np.float64)
        self._check(lib().mgpu_cfl_gather(self.h, out.ctypes.data), "cfl_gather")
        return out

    def mean_profile(self, name) -> np.ndarray:
        out = np.empty(self.nz, dtype=np.float64)
        self._check(lib().mgpu_mean_profile(self.h, field_id(name), out.ctypes.data), "mean_profile")
        return out

    def mean_profiles(self) -> dict:
        """The mean profiles (meanprofiles.F90): olzubar, olzvbar, olzthbar, olzqbar(n), olubar,
        olvbar, olthbar, olqbar(n), as refreshed by the last step or mean_profiles component."""
        out = self.mean_profile_rows()
        return dict(zip(mean_profile_names(self.cfg.number_q_fields), out))

    def mean_profile_rows(self) -> np.ndarray:
        """mgpu_mean_profiles' rows, (2 (3 + number_q_fields), nz): the checkpoints' `mean`."""
        out = np.empty((2 * (3 + self.cfg.number_q_fields), self.nz), dtype=np.float64)
        self._check(lib().mgpu_mean_profiles(self.h, out.ctypes.data), "mean_profiles")
        return out

    def profile_diagnostics(self) -> dict:
        """MONC's profile_diagnostics sums (<name>_total_local, per level) from the current state,
        as the component would accumulate them in the next step (needs profile_diagnostics_enabled)."""
        out = np.empty((len(PROFILE_DIAGNOSTICS), self.nz), dtype=np.float64)
        rows = C.c_int32(0)
        self._check(lib().mgpu_profile_diagnostics(self.h, out.ctypes.data, C.byref(rows)), "profile_diagnostics")
        return dict(zip(PROFILE_DIAGNOSTICS[:rows.value], out[:rows.value]))

    def checkpoint_write(self, path: str):
        """Write a MONC-layout checkpoint (NetCDF classic) of the model's state."""
        self._check(lib().mgpu_checkpoint_write(self.h, os.fsencode(path)), "checkpoint_write")

    def checkpoint_state(self) -> "CheckpointMeta":
        """The step count, time, dtm state and Galilean frame a checkpoint of the model carries."""
        meta = CheckpointMeta()
        self._check(lib().mgpu_checkpoint_state(self.h, C.byref(meta)), "checkpoint_state")
        return meta

    def restore_state(self, meta: "CheckpointMeta", mean: np.ndarray | None = None):
        """Continue after the step `meta` describes; mean: mgpu_mean_profiles' rows,
        (2 (3 + number_q_fields), nz)."""
        m = None if mean is None else np.ascontiguousarray(mean, dtype=np.float64)
        self._check(lib().mgpu_restore_state(self.h, C.byref(meta), None if m is None else m.ctypes.data),
                    "restore_state")

    def checkpoint_read(self, path: str):
        """Restart from a MONC-layout checkpoint: state, mean profiles, step count, time, dtm."""
        self._check(lib().mgpu_checkpoint_read(self.h, os.fsencode(path)), "checkpoint_read")

    def diagnostics(self, out_th: np.ndarray | None = None, out_w2: np.ndarray | None = None):
        """Device-computed horizontal means: theta (incl. thref) and w**2 per level."""
        th = out_th if out_th is not None else np.empty(self.nz, dtype=np.float64)
        w2 = out_w2 if out_w2 is not None else np.empty(self.nz, dtype=np.float64)
        self._check(lib().mgpu_diagnostics(self.h, th.ctypes.data, w2.ctypes.data), "diagnostics")
        return th, w2

    def set_profiling(self, on: bool):
        self._check(lib().mgpu_set_profiling(self.h, 1 if on else 0), "set_profiling")

    def stage_times(self) -> dict:
        ms = np.zeros(len(STAGES), dtype=np.float64)
        n = np.zeros(len(STAGES), dtype=np.int64)
        self._check(lib().mgpu_stage_times(self.h, ms.ctypes.data, n.ctypes.data), "stage_times")
        return {name: (float(ms[i]), int(n[i])) for i, name in enumerate(STAGES)}

    # -- one y-slab of a decomposed domain (solver SOLVER_EXTERNAL); buffers are device addresses
    def slab_init(self, ny_global: int, halo: int, max_cols: int):
        self._check(lib().mgpu_slab_init(self.h, ny_global, halo, max_cols), "slab_init")

    def step_phase(self, phase: int):
        self._check(lib().mgpu_step_phase(self.h, phase), f"step_phase {phase}")

    def halo_fields(self, halo_set: int) -> int:
        n = lib().mgpu_halo_fields(self.h, halo_set)
        if n < 0:
            self._check(n, "halo_fields")
        return n

    def halo_pack(self, halo_set: int, depth: int, lo: int, hi: int):
        self._check(lib().mgpu_halo_pack(self.h, halo_set, depth, lo, hi), "halo_pack")

    def halo_unpack(self, halo_set: int, depth: int, lo: int, hi: int):
        self._check(lib().mgpu_halo_unpack(self.h, halo_set, depth, lo, hi), "halo_unpack")

    def slab_level_means(self, means: int):
        self._check(lib().mgpu_slab_level_means(self.h, means), "slab_level_means")

    def slab_mean_profiles(self, buf: int, put: bool):
        self._check(lib().mgpu_slab_mean_profiles(self.h, buf, 1 if put else 0), "slab_mean_profiles")

    def slab_iter(self, step: int, sums: int = 0) -> bool:
        """One step of the slab BiCGStab (mgpu_slab_iter); returns the done flag of a FINISH."""
        done = C.c_int32(0)
        self._check(lib().mgpu_slab_iter(self.h, step, sums or None, C.byref(done)), f"slab_iter {step}")
        return bool(done.value)

    def slab_cfl_extrema(self, buf: int, put: bool) -> bool:
        """Fetch (put=False) or hand back (put=True) this slab's cfltest extrema in max form;
        returns whether this step gathered them."""
        g = C.c_int32(0)
        self._check(lib().mgpu_slab_cfl_extrema(self.h, buf, 1 if put else 0, C.byref(g)), "slab_cfl_extrema")
        return bool(g.value)

    def slab_fft_x(self, spec: int, nblocks: int, inverse: bool):
        self._check(lib().mgpu_slab_fft_x(self.h, spec, nblocks, 1 if inverse else 0), "slab_fft_x")

    def slab_solve_columns(self, spec: int, kx0: int, nkx: int, row_block: int, transpose: bool = False):
        self._check(lib().mgpu_slab_solve_columns(self.h, spec, kx0, nkx, row_block, 1 if transpose else 0),
                    "slab_solve_columns")

    @property
    def stream(self) -> int:
        return lib().mgpu_stream(self.h) or 0

    @property
    def launches(self) -> int:
        return int(lib().mgpu_launch_count(self.h))


@dataclass
class ComponentDescriptor:
    """Mirror of component_descriptor_type (monc_component.F90:62-71)."""

    name: str
    version: float
    initialisation: Optional[Callable] = None
    timestep: Optional[Callable] = None
    finalisation: Optional[Callable] = None
    published_fields: Optional[list] = None
    field_value_retrieval: Optional[Callable] = None


def component_descriptor(name: str) -> ComponentDescriptor:
    """The descriptor a MONC registry would receive for a GPU drop-in of `name`.

    The callbacks take the `Model` that stands for `current_state`.  `profile_diagnostics` has
    no timestep work here: its field_value_retrieval(model, field_name) computes the named sums
    on the device when the IO server asks for them."""
    if name == "profile_diagnostics":
        def retrieve(model: Model, field_name: str) -> np.ndarray:
            values = model.profile_diagnostics()
            if field_name not in values:
                raise KeyError(f"profile_diagnostics publishes no {field_name} for this model")
            return values[field_name]

        return ComponentDescriptor(name=name, version=0.1, published_fields=list(PROFILE_DIAGNOSTICS),
                                   field_value_retrieval=retrieve)
    if name not in COMPONENTS:
        raise KeyError(f"no GPU drop-in for component {name}")

    def timestep(model: Model):
        model.component(name)

    return ComponentDescriptor(name=name, version=0.1, timestep=timestep)


def run_groups(model: Model, groups=("start", "subgrid", "dynamics", "solver", "pressure-terms")):
    """One MONC timestep through the per-component entry points, in the configured group order
    (timestepper.F90:40-54).  mgpu_step runs the same sequence with the fused kernels."""
    solver = "fftsolver" if model.cfg.solver == cf.SOLVER_FFT else "iterativesolver"
    for g in groups:
        for name in GROUPS[g]:
            if name in ("fftsolver", "iterativesolver") and name != solver:
                continue
            if name == "simplecloud" and not model.cfg.simplecloud_enabled:
                continue
            if name == "coriolis" and not model.cfg.coriolis_enabled:
                continue
            if name == "th_advection" and not model.cfg.th_advection_enabled:
                continue
            if name == "damping" and not model.cfg.damping_enabled:
                continue
            if name == "forcing" and not (model.cfg.l_subs_pl_theta or model.cfg.l_subs_pl_q):
                continue
            if name == "mean_profiles" and not (model.cfg.damping_enabled or model.cfg.l_subs_pl_theta
                                                or model.cfg.l_subs_pl_q or model.cfg.profile_diagnostics_enabled):
                continue
            model.component(name)
    ts = model.reductions().timestep
    model.set_timestep(ts + 1)


CHECKPOINT_FIELDS = ["u", "v", "w", "th", "zu", "zv", "zw", "zth", "p"]


def _checkpoint_names(cfg) -> list:
    nq = cfg.number_q_fields
    return CHECKPOINT_FIELDS + [f"q{n}" for n in range(nq)] + [f"zq{n}" for n in range(nq)]


def mean_profile_names(nq: int) -> list:
    """Names of mgpu_mean_profiles' rows."""
    return (["olzubar", "olzvbar", "olzthbar"] + [f"olzqbar{n}" for n in range(nq)]
            + ["olubar", "olvbar", "olthbar"] + [f"olqbar{n}" for n in range(nq)])


def checkpoint_write_host(cfg, path: str, fields: dict, meta: CheckpointMeta, mean: np.ndarray | None = None):
    """Write a MONC-layout checkpoint from host arrays (no GPU): fields by name, each (nz, ny, nx);
    mean, when given, mgpu_mean_profiles' rows (2 (3 + number_q_fields), nz): olz*bar, then
    olubar, olvbar, olthbar, olqbar(n)."""
    names = _checkpoint_names(cfg)
    arrs = [np.ascontiguousarray(fields[n], dtype=np.float64) for n in names]
    ptrs = (C.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])
    m = None if mean is None else np.ascontiguousarray(mean, dtype=np.float64)
    rc = lib().mgpu_checkpoint_write_host(C.byref(cfg), os.fsencode(path), ptrs,
                                          None if m is None else m.ctypes.data, C.byref(meta))
    if rc != OK:
        raise MgpuError(rc, "mgpu_checkpoint_write_host")


def checkpoint_read_host(cfg, path: str):
    """Read a MONC-layout checkpoint into host arrays: (fields, mean or None, meta).  mean has
    mgpu_mean_profiles' rows; those of olubar .. olqbar are zero when the file lacks them."""
    names = _checkpoint_names(cfg)
    shape = (cfg.nz, cfg.ny, cfg.nx)
    arrs = [np.empty(shape, dtype=np.float64) for _ in names]
    ptrs = (C.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])
    mean = np.empty((2 * (3 + cfg.number_q_fields), cfg.nz), dtype=np.float64)
    has_mean = C.c_int32(0)
    meta = CheckpointMeta()
    rc = lib().mgpu_checkpoint_read_host(C.byref(cfg), os.fsencode(path), ptrs, mean.ctypes.data,
                                         C.byref(has_mean), C.byref(meta))
    if rc != OK:
        raise MgpuError(rc, "mgpu_checkpoint_read_host")
    return dict(zip(names, arrs)), (mean if has_mean.value else None), meta
