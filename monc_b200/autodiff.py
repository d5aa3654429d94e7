"""torch.autograd interface to the GPU model: a window of timesteps as a differentiable function.

`MoncWindow.apply(th0, rmlmax, window)` runs `window.nsteps` timesteps of the dry FP64 model from
`window.base` with theta replaced by `th0` and the Smagorinsky mixing length `rmlmax` (= Cs*dx),
and returns the final (u, v, w, th).  Its backward pass is the library's adjoint
(`mgpu_adjoint_run`): a checkpointed reverse sweep of hand-differentiated step kernels, which
returns the gradients with respect to th0 and rmlmax.  CUDA tensors stay in HBM: they are copied
device to device into and out of the model (MGPU_LAYOUT_DEVICE); CPU tensors go through float64
host arrays.  The model state itself stays on the GPU throughout.
"""
from __future__ import annotations

from dataclasses import dataclass

import torch

from . import api, config as cf


@dataclass
class Window:
    cfg: cf.MgpuConfig
    base: dict  # initial state (u v w th zu zv zw zth), [nz][ny][nx] float64
    nsteps: int
    checkpoint_interval: int = 25
    timestep: int = 1


def _put(m: api.Model, name: str, a):
    """A CUDA tensor device to device, anything else through a host array."""
    if isinstance(a, torch.Tensor) and a.is_cuda:
        m.upload_tensor(name, a.detach().to(torch.float64).contiguous())
    elif isinstance(a, torch.Tensor):
        m.upload(name, a.detach().to(torch.float64).numpy())
    else:
        m.upload(name, a)


def _get(m: api.Model, name: str, device: torch.device) -> torch.Tensor:
    if device.type == "cuda":
        return m.download_tensor(name, device)
    return torch.from_numpy(m.download(name))


def _model(window: Window, th0, rmlmax: float) -> api.Model:
    c = cf.MgpuConfig.from_buffer_copy(window.cfg)
    c.rmlmax = float(rmlmax)
    m = api.Model(c)
    m.set_state({k: v for k, v in window.base.items() if k != "th"})
    _put(m, "th", th0)
    m.set_timestep(window.timestep)
    return m


class MoncWindow(torch.autograd.Function):
    @staticmethod
    def forward(ctx, th0: torch.Tensor, rmlmax: torch.Tensor, window: Window):
        th_in = th0.detach().to(torch.float64)
        r = float(rmlmax.detach().cpu())
        m = _model(window, th_in, r)
        m.step(window.nsteps)
        outs = [_get(m, f, th0.device) for f in ("u", "v", "w", "th")]
        m.close()
        ctx.window = window
        ctx.th0 = th_in
        ctx.r = r
        ctx.device = th0.device
        return tuple(outs)

    @staticmethod
    def backward(ctx, gu, gv, gw, gth):
        window = ctx.window
        m = _model(window, ctx.th0, ctx.r)
        seeds = {"u": gu, "v": gv, "w": gw, "th": gth}
        for f in api.STATE_FIELDS:
            g = seeds.get(f)
            _put(m, "adj:" + f, torch.zeros_like(ctx.th0) if g is None else g)
        rbar = m.adjoint_run(window.nsteps, window.checkpoint_interval)
        th_bar = _get(m, "adj:th", ctx.device)
        m.close()
        return th_bar, torch.tensor(rbar, dtype=torch.float64, device=ctx.device), None


def resolved_tke(u: torch.Tensor, v: torch.Tensor, w: torch.Tensor, dz: torch.Tensor, mask: torch.Tensor):
    """sum_k mask_k dz_k <0.5 (u'^2 + v'^2 + w'^2)>_xy, primes = deviations from the level mean."""
    tke = 0.0
    for a in (u, v, w):
        pert = a - a.mean(dim=(1, 2), keepdim=True)
        tke = tke + 0.5 * (pert * pert).mean(dim=(1, 2))
    return (tke * dz * mask).sum()
