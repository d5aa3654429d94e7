"""torch.autograd interface to the GPU model: a window of timesteps as a differentiable function.

`MoncWindow.apply(th0, rmlmax, window)` runs `window.nsteps` timesteps of the dry FP64 model from
`window.base` with theta replaced by `th0` and the Smagorinsky mixing length `rmlmax` (= Cs*dx),
and returns the final (u, v, w, th).  Its backward pass is the library's adjoint
(`mgpu_adjoint_run`): a checkpointed reverse sweep of hand-differentiated step kernels, which
returns the gradients with respect to th0 and rmlmax.  Tensors cross the boundary as float64
host arrays; the model state itself stays on the GPU throughout.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from . import api, config as cf


@dataclass
class Window:
    cfg: cf.MgpuConfig
    base: dict  # initial state (u v w th zu zv zw zth), [nz][ny][nx] float64
    nsteps: int
    checkpoint_interval: int = 25
    timestep: int = 1


def _model(window: Window, th0: np.ndarray, rmlmax: float) -> api.Model:
    c = cf.MgpuConfig.from_buffer_copy(window.cfg)
    c.rmlmax = float(rmlmax)
    m = api.Model(c)
    st = dict(window.base)
    st["th"] = th0
    m.set_state(st)
    m.set_timestep(window.timestep)
    return m


class MoncWindow(torch.autograd.Function):
    @staticmethod
    def forward(ctx, th0: torch.Tensor, rmlmax: torch.Tensor, window: Window):
        th0_np = th0.detach().to("cpu", torch.float64).numpy()
        r = float(rmlmax.detach().cpu())
        m = _model(window, th0_np, r)
        m.step(window.nsteps)
        outs = [torch.from_numpy(m.download(f)) for f in ("u", "v", "w", "th")]
        m.close()
        ctx.window = window
        ctx.th0 = th0_np
        ctx.r = r
        ctx.device = th0.device
        return tuple(o.to(th0.device) for o in outs)

    @staticmethod
    def backward(ctx, gu, gv, gw, gth):
        window = ctx.window
        m = _model(window, ctx.th0, ctx.r)
        shape = ctx.th0.shape
        seeds = {"u": gu, "v": gv, "w": gw, "th": gth}
        for f in api.STATE_FIELDS:
            g = seeds.get(f)
            arr = np.zeros(shape) if g is None else g.detach().to("cpu", torch.float64).numpy()
            m.upload("adj:" + f, arr)
        rbar = m.adjoint_run(window.nsteps, window.checkpoint_interval)
        th_bar = torch.from_numpy(m.download("adj:th")).to(ctx.device)
        m.close()
        return th_bar, torch.tensor(rbar, dtype=torch.float64, device=ctx.device), None


def resolved_tke(u: torch.Tensor, v: torch.Tensor, w: torch.Tensor, dz: torch.Tensor, mask: torch.Tensor):
    """sum_k mask_k dz_k <0.5 (u'^2 + v'^2 + w'^2)>_xy, primes = deviations from the level mean."""
    tke = 0.0
    for a in (u, v, w):
        pert = a - a.mean(dim=(1, 2), keepdim=True)
        tke = tke + 0.5 * (pert * pert).mean(dim=(1, 2))
    return (tke * dz * mask).sum()
