"""Y-slab domain decomposition of the dynamical core: one slab of the horizontal domain per GPU.

MONC decomposes the horizontal domain into 2-D blocks of whole columns (decomposition.F90:57-123),
swaps halos of depth 2 with its neighbours before the dynamics (haloswapper.F90:62-71 over
halocommunication.F90:109-163) and solves the pressure on pencils reached by all-to-all
transposes (pencilfft.F90:126-159).  Here the domain is split along y only, so every slab keeps
whole x rows (x stays periodic inside each model) and the FFT solve needs one transpose each way:

    per step, on every slab
      halo exchange of the state (u v w th zu zv zw zth q zq), `halo` rows each side
      subgrid phase
      cfltest evaluation steps: the six extrema, max-reduced over all slabs
      FP32-mixed: level means of th and q over the slab, averaged over all slabs
      dynamics phase (dynamics, scalar swap, pressure source)
      damping, mean-profile subsidence or profile diagnostics: the mean profiles, averaged
      FFT solve:
        x-FFT of the interior rows, written straight into per-destination kx blocks
        all-to-all: rank q receives kx block q of every slab (all rows of its wavenumbers)
        y-FFT, tridiagonal solve, inverse y-FFT on those columns
        all-to-all back, inverse x-FFT into the interior rows of p
      or iterative solve (BiCGStab or conjugate gradients, FP32-mixed refinement around them):
        depth-1 halo rows of each vector before A is applied to it, every inner product summed
      halo exchange of p (1 row each side: the pressure gradient reaches row j+1)
      pstep phase (cfltest and the Galilean frame, pressure step, swap_smooth)

`halo` = 4 rows covers the step's stencil reach: 2 rows for TVD advection and the viscous and
diffusive fluxes, 1 more for the pressure source, which reads the stepped velocities at j-1.
Halo rows are recomputed by every phase (with the slab's own periodic wrap) and hold stale
values until the next exchange; the interior rows never read them beyond that reach.

The exchanges go through a communicator object: `TorchComm` (one slab per process over
torch.distributed, NCCL between GPUs) or `LoopbackComm` (every slab in this process on one
device, each exchange a set of device copies made after all queued work has finished; the
slabs never wait on each other inside a kernel).  With `reproducible` set, an FP64 decomposed
run reproduces the single-domain run bit for bit: each interior point is computed by the same
operations on the same values, the x-FFT pairs the same rows (slab heights are even) and the y
transforms and tridiagonal solves see the same columns.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch
import torch.distributed as dist

from . import api
from . import config as cf


def kx_blocks(nxh: int, nranks: int) -> list[tuple[int, int]]:
    """Split the nxh = nx/2+1 x-wavenumbers over nranks as mgpu_slab_fft_x does: as evenly as
    possible, the first nxh % nranks blocks one wider.  Returns [(first wavenumber, width)]."""
    if nranks > nxh:
        raise ValueError(f"{nxh} x-wavenumbers cannot be split into {nranks} non-empty blocks")
    b, r = divmod(nxh, nranks)
    return [(q * b + min(q, r), b + (1 if q < r else 0)) for q in range(nranks)]


@dataclass(frozen=True)
class SlabGeometry:
    """Sizes of a y-slab decomposition of an nx x ny x nz domain over nranks slabs."""
    nx: int
    ny: int
    nz: int
    nranks: int
    halo: int = 4

    def __post_init__(self):
        if self.ny % self.nranks:
            raise ValueError(f"ny={self.ny} is not a multiple of {self.nranks} slabs")
        nyl = self.ny // self.nranks
        if nyl % 2 or nyl < max(self.halo, 2):
            raise ValueError(f"slabs of {nyl} rows: need an even number >= max(halo={self.halo}, 2)")
        kx_blocks(self.nx // 2 + 1, self.nranks)

    @property
    def nyl(self) -> int:
        return self.ny // self.nranks

    @property
    def nxh(self) -> int:
        return self.nx // 2 + 1

    @property
    def blocks(self) -> list[tuple[int, int]]:
        return kx_blocks(self.nxh, self.nranks)

    def y0(self, rank: int) -> int:
        return rank * self.nyl

    def rows(self, rank: int) -> np.ndarray:
        """Global rows held by a slab model, halo rows included (periodic)."""
        return np.arange(self.y0(rank) - self.halo, self.y0(rank) + self.nyl + self.halo) % self.ny

    # element offsets (complex elements) of the all-to-all blocks
    def xblock(self, q: int) -> tuple[int, int]:
        """Block q of a slab's x-spectrum: (offset, length)."""
        k0, w = self.blocks[q]
        return k0 * self.nz * self.nyl, self.nz * self.nyl * w

    def tblock(self, rank: int, r: int) -> tuple[int, int]:
        """Block r (rows of slab r) of rank's transposed spectrum: (offset, length)."""
        n = self.nz * self.nyl * self.blocks[rank][1]
        return r * n, n


# ---- communicators ------------------------------------------------------------------------
class LoopbackComm:
    """Every slab in this process.  Lists passed to the exchanges hold one entry per slab."""

    def __init__(self, nranks: int):
        self.size = nranks
        self.local_ranks = list(range(nranks))

    @staticmethod
    def _sync(t: torch.Tensor):
        if t.is_cuda:
            torch.cuda.synchronize(t.device)

    def halo_exchange(self, send_lo, send_hi, recv_lo, recv_hi):
        """recv_lo[r] <- send_hi[r-1], recv_hi[r] <- send_lo[r+1] (periodic)."""
        R = self.size
        self._sync(send_lo[0])
        for r in range(R):
            recv_lo[r].copy_(send_hi[(r - 1) % R])
            recv_hi[r].copy_(send_lo[(r + 1) % R])
        self._sync(send_lo[0])

    def all_to_all(self, send, recv):
        """recv[q][r] <- send[r][q] for every pair of slabs."""
        self._sync(send[0][0])
        for r in range(self.size):
            for q in range(self.size):
                recv[q][r].copy_(send[r][q])
        self._sync(send[0][0])

    def allreduce_mean(self, bufs):
        self._sync(bufs[0])
        total = bufs[0].clone()
        for b in bufs[1:]:
            total += b
        total /= self.size
        for b in bufs:
            b.copy_(total)
        self._sync(bufs[0])

    def barrier(self):
        pass

    def allreduce_sum_inplace(self, bufs):
        self._sync(bufs[0])
        total = bufs[0].clone()
        for b in bufs[1:]:
            total += b
        for b in bufs:
            b.copy_(total)
        self._sync(bufs[0])

    def allreduce_max(self, bufs):
        self._sync(bufs[0])
        top = bufs[0].clone()
        for b in bufs[1:]:
            torch.maximum(top, b, out=top)
        for b in bufs:
            b.copy_(top)
        self._sync(bufs[0])

    def gather_rows(self, parts):
        return parts

    def allreduce_sum(self, t: torch.Tensor) -> torch.Tensor:
        """Every slab is local: the local sum is the total."""
        return t


class TorchComm:
    """One slab per process over torch.distributed; collectives run on `stream` (the model's)."""

    def __init__(self, group=None):
        self.group = group
        self.rank = dist.get_rank(group)
        self.size = dist.get_world_size(group)
        self.local_ranks = [self.rank]
        self.stream = None

    def _ctx(self):
        if self.stream is None:
            import contextlib
            return contextlib.nullcontext()
        return torch.cuda.stream(self.stream)

    def _peer(self, r: int) -> int:
        return dist.get_global_rank(self.group, r) if self.group is not None else r

    def halo_exchange(self, send_lo, send_hi, recv_lo, recv_hi):
        R, r = self.size, self.rank
        with self._ctx():
            if R == 1:
                recv_lo[0].copy_(send_hi[0])
                recv_hi[0].copy_(send_lo[0])
                return
            prev, nxt = self._peer((r - 1) % R), self._peer((r + 1) % R)
            # the same order on every rank: with two slabs prev == nxt and the two messages each
            # way are matched by order (NCCL) or by tag (gloo)
            ops = [dist.P2POp(dist.isend, send_lo[0], prev, self.group, 1),
                   dist.P2POp(dist.isend, send_hi[0], nxt, self.group, 2),
                   dist.P2POp(dist.irecv, recv_hi[0], nxt, self.group, 1),
                   dist.P2POp(dist.irecv, recv_lo[0], prev, self.group, 2)]
            for w in dist.batch_isend_irecv(ops):
                w.wait()

    def all_to_all(self, send, recv):
        R, me = self.size, self.rank
        with self._ctx():
            recv[0][me].copy_(send[0][me])
            if R == 1:
                return
            ops = []
            for q in range(R):
                if q != me:
                    ops.append(dist.P2POp(dist.isend, send[0][q], self._peer(q), self.group, 3))
                    ops.append(dist.P2POp(dist.irecv, recv[0][q], self._peer(q), self.group, 3))
            for w in dist.batch_isend_irecv(ops):
                w.wait()

    def allreduce_mean(self, bufs):
        with self._ctx():
            dist.all_reduce(bufs[0], group=self.group)
            bufs[0].div_(self.size)

    def barrier(self):
        dist.barrier(group=self.group)

    def allreduce_sum_inplace(self, bufs):
        with self._ctx():
            dist.all_reduce(bufs[0], group=self.group)

    def allreduce_max(self, bufs):
        with self._ctx():
            dist.all_reduce(bufs[0], op=dist.ReduceOp.MAX, group=self.group)

    def allreduce_sum(self, t: torch.Tensor) -> torch.Tensor:
        """Sum of a host tensor over the ranks (on the device for NCCL)."""
        dev = t.device
        if dist.get_backend(self.group) == "nccl":
            t = t.to(torch.device("cuda", torch.cuda.current_device()))
        with self._ctx():
            dist.all_reduce(t, group=self.group)
        return t.to(dev)

    def gather_rows(self, parts):
        with self._ctx():
            out = [torch.empty_like(parts[0]) for _ in range(self.size)]
            dist.all_gather(out, parts[0].contiguous(), group=self.group)
        return out


# ---- the decomposed model -------------------------------------------------------------------
class _Slab:
    def __init__(self, rank: int, model: api.Model, geo: SlabGeometry, dtype, device):
        self.rank = rank
        self.m = model
        g = geo
        # spectra are interleaved complex: 2 reals per element
        self.spec_x = torch.zeros(2 * g.nz * g.nyl * g.nxh, dtype=dtype, device=device)
        self.spec_t = torch.zeros(2 * g.nz * g.ny * g.blocks[rank][1], dtype=dtype, device=device)
        nf = model.halo_fields(cf.HALO_STATE)
        # send below, send above, received from below, received from above
        self.state_bufs = [torch.zeros(nf * g.nz * g.halo * g.nx, dtype=dtype, device=device) for _ in range(4)]
        # depth-1 sets of one or two fields: p, the iterative solve's vectors
        self.p_bufs = [torch.zeros(2 * g.nz * g.nx, dtype=dtype, device=device) for _ in range(4)]
        # the FP32-mixed refinement's FP64 iterate
        self.x64_bufs = [torch.zeros(g.nz * g.nx, dtype=torch.float64, device=device) for _ in range(4)]
        self.means = torch.zeros((1 + model.cfg.number_q_fields) * (g.nz + 2), dtype=torch.float64, device=device)
        # the mean profiles damping, subsidence and profile_diagnostics read (mgpu_slab_mean_profiles)
        self.profiles = torch.zeros(2 * (3 + model.cfg.number_q_fields) * (g.nz + 2), dtype=torch.float64,
                                    device=device)
        # cfltest's six extrema, every one combined by a maximum (mgpu_slab_cfl_extrema)
        self.cfl = torch.zeros(6, dtype=torch.float64, device=device)
        # the iterative solve's dot products of one step (mgpu_slab_iter)
        self.sums = torch.zeros(3, dtype=torch.float64, device=device)

        def cview(buf, off, n):
            return buf[2 * off:2 * (off + n)]
        self.x_blocks = [cview(self.spec_x, *g.xblock(q)) for q in range(g.nranks)]
        self.t_blocks = [cview(self.spec_t, *g.tblock(rank, r)) for r in range(g.nranks)]


class SlabDomain:
    """A periodic domain of cfg's size split into y-slabs over comm's ranks.

    The slabs local to this process (all of them under LoopbackComm) are models created with
    solver SOLVER_EXTERNAL on `device`.  Fields move in and out as global [nz][ny][nx] arrays."""

    def __init__(self, cfg: cf.MgpuConfig, comm, halo: int = 4, device=None):
        self.cfg = cfg
        self.comm = comm
        self.geo = SlabGeometry(cfg.nx, cfg.ny, cfg.nz, comm.size, halo)
        # the library keeps the mean profiles when damping, mean-profile subsidence or
        # profile_diagnostics reads them
        # the pressure solve: the distributed FFT, or iterativesolver's BiCGStab (FP64)
        self.iterative = cfg.solver == cf.SOLVER_ITERATIVE
        self.mean_profiles = bool(cfg.damping_enabled or cfg.profile_diagnostics_enabled
                                  or (cfg.l_subs_pl_theta and not cfg.subsidence_local_theta)
                                  or (cfg.l_subs_pl_q and not cfg.subsidence_local_q and cfg.number_q_fields > 0))
        g = self.geo
        self.fp32 = cfg.precision == cf.FP32_MIXED
        dtype = torch.float32 if self.fp32 else torch.float64
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.slabs: list[_Slab] = []
        for r in comm.local_ranks:
            c = cf.MgpuConfig.from_buffer_copy(cfg)
            c.ny = g.nyl + 2 * halo
            c.solver = cf.SOLVER_EXTERNAL
            m = api.Model(c)
            m.slab_init(g.ny, halo, max(w for _, w in g.blocks))
            self.slabs.append(_Slab(r, m, g, dtype, self.device))
        if isinstance(comm, TorchComm) and self.device.type == "cuda":
            comm.stream = torch.cuda.ExternalStream(self.slabs[0].m.stream, device=self.device)

    def close(self):
        for s in self.slabs:
            s.m.close()
        self.slabs = []

    # -- fields
    def upload(self, name, arr: np.ndarray):
        a = np.asarray(arr, dtype=np.float64).reshape(self.geo.nz, self.geo.ny, self.geo.nx)
        for s in self.slabs:
            s.m.upload(name, np.ascontiguousarray(a[:, self.geo.rows(s.rank), :]))

    def set_state(self, state: dict):
        for k, v in state.items():
            self.upload(k, v)

    def upload_local(self, name, arrays):
        """Upload each local slab's rows directly: arrays[i] is [nz][nyl + 2*halo][nx] for the i-th
        local slab (the rows SlabGeometry.rows gives), so no process builds the global field."""
        for s, a in zip(self.slabs, arrays):
            s.m.upload(name, a)

    def download(self, name) -> np.ndarray:
        g = self.geo
        parts = [torch.from_numpy(s.m.download(name)[:, g.halo:g.halo + g.nyl, :].copy()) for s in self.slabs]
        if isinstance(self.comm, TorchComm):
            dev = self.device if dist.get_backend(self.comm.group) == "nccl" else torch.device("cpu")
            parts = [p.to(dev) for p in self.comm.gather_rows([parts[0].to(dev)])]
        return np.concatenate([p.cpu().numpy() for p in parts], axis=1)

    def set_timestep(self, ts: int):
        for s in self.slabs:
            s.m.set_timestep(ts)

    # -- stepping
    def _exchange(self, halo_set: int, depth: int):
        # the depth-1 sets (p and the solver vectors) share the pressure buffers
        bufs = [s.state_bufs if halo_set == cf.HALO_STATE else
                (s.x64_bufs if halo_set == cf.HALO_ITER_X64 else s.p_bufs) for s in self.slabs]
        for s, b in zip(self.slabs, bufs):
            s.m.halo_pack(halo_set, depth, b[0].data_ptr(), b[1].data_ptr())
        self.comm.halo_exchange([b[0] for b in bufs], [b[1] for b in bufs], [b[2] for b in bufs],
                                [b[3] for b in bufs])
        for s, b in zip(self.slabs, bufs):
            s.m.halo_unpack(halo_set, depth, b[2].data_ptr(), b[3].data_ptr())

    def step(self, n: int = 1):
        g = self.geo
        for _ in range(n):
            self._exchange(cf.HALO_STATE, g.halo)
            for s in self.slabs:
                s.m.step_phase(cf.PHASE_SUBGRID)
            if self.cfg.cfl_enabled:
                # on cfltest's evaluation steps (the same on every slab) the domain extrema
                gathered = [s.m.slab_cfl_extrema(s.cfl.data_ptr(), False) for s in self.slabs]
                if gathered[0]:
                    self.comm.allreduce_max([s.cfl for s in self.slabs])
                    for s in self.slabs:
                        s.m.slab_cfl_extrema(s.cfl.data_ptr(), True)
            if self.fp32:
                for s in self.slabs:
                    s.m.slab_level_means(s.means.data_ptr())
                self.comm.allreduce_mean([s.means for s in self.slabs])
            for s in self.slabs:
                s.m.step_phase(cf.PHASE_DYNAMICS)
                if not self.iterative:
                    s.m.slab_fft_x(s.spec_x.data_ptr(), g.nranks, False)
            if self.mean_profiles:
                # each slab's means of this step, averaged over the slabs for the next step
                for s in self.slabs:
                    s.m.slab_mean_profiles(s.profiles.data_ptr(), False)
                self.comm.allreduce_mean([s.profiles for s in self.slabs])
                for s in self.slabs:
                    s.m.slab_mean_profiles(s.profiles.data_ptr(), True)
            if self.iterative:
                self._iterative_solve()
            else:
                self.comm.all_to_all([s.x_blocks for s in self.slabs], [s.t_blocks for s in self.slabs])
                for s in self.slabs:
                    k0, w = g.blocks[s.rank]
                    s.m.slab_solve_columns(s.spec_t.data_ptr(), k0, w, g.nyl)
                self.comm.all_to_all([s.t_blocks for s in self.slabs], [s.x_blocks for s in self.slabs])
                for s in self.slabs:
                    s.m.slab_fft_x(s.spec_x.data_ptr(), g.nranks, True)
            self._exchange(cf.HALO_PRESSURE, 1)
            for s in self.slabs:
                s.m.step_phase(cf.PHASE_PSTEP)

    def _reduce_step(self, step: int) -> bool:
        """A reducing BiCGStab step on every slab, its sums added over the slabs, then FINISH."""
        for s in self.slabs:
            s.m.slab_iter(step, s.sums.data_ptr())
        self.comm.allreduce_sum_inplace([s.sums for s in self.slabs])
        done = [s.m.slab_iter(cf.SLAB_ITER_FINISH, s.sums.data_ptr()) for s in self.slabs]
        return done[0]

    def _all(self, step: int):
        for s in self.slabs:
            s.m.slab_iter(step)

    def _iterative_solve(self):
        """iterativesolver over the slabs (mgpu_slab_iter), BiCGStab or conjugate gradients, with
        the FP32-mixed models' iterative refinement around an FP32 solve: halo rows of the vectors
        A is applied to, and every inner product summed over the slabs (inner_prod's allreduce)."""
        self._all(cf.SLAB_ITER_BEGIN)
        if self.fp32:
            self._refinement()
        else:
            self._krylov()
        self._all(cf.SLAB_ITER_END)

    def _refinement(self):
        """The FP32-mixed solve: the compatible right-hand side, then FP64 residuals and FP32
        corrections until the residual meets the tolerance or stops falling (8 at most)."""
        self._reduce_step(cf.SLAB_ITER_COMPAT)
        self._all(cf.SLAB_ITER_SHIFT)
        prev_err = 0.0
        for outer in range(8):
            self._exchange(cf.HALO_ITER_X64, 1)
            if self._reduce_step(cf.SLAB_ITER_REFINE):
                break
            err = self.slabs[0].m.reductions().solver_residual
            if outer > 0 and not err < prev_err:
                self._all(cf.SLAB_ITER_UNCORRECT)
                break
            prev_err = err
            self._all(cf.SLAB_ITER_INNER)
            self._krylov()
            self._all(cf.SLAB_ITER_CORRECT)

    def _krylov(self):
        """BiCGStab or conjugate gradients on the current work vectors."""
        self._exchange(cf.HALO_ITER_X, 1)
        done = self._reduce_step(cf.SLAB_ITER_INIT)
        if self.cfg.solver_type == cf.ITER_CG:
            done = False  # cg_solver runs at least one iteration
            while not done:
                self._reduce_step(cf.SLAB_ITER_PRECOND)
                self._exchange(cf.HALO_ITER_CG, 1)
                self._reduce_step(cf.SLAB_ITER_APPLY)
                done = self._reduce_step(cf.SLAB_ITER_UPDATE)
            return
        while not done:
            self._all(cf.SLAB_ITER_DIRECTION)
            self._exchange(cf.HALO_ITER_PP, 1)
            self._reduce_step(cf.SLAB_ITER_APPLY)
            self._all(cf.SLAB_ITER_HALF_STEP)
            self._exchange(cf.HALO_ITER_CS, 1)
            self._reduce_step(cf.SLAB_ITER_APPLY2)
            done = self._reduce_step(cf.SLAB_ITER_UPDATE)

    def checkpoint_write(self, path: str):
        """One MONC-layout checkpoint of the whole domain: the slabs' interior rows gathered, the
        mean profiles and step state of the first slab (the same on every slab), written by rank 0
        through the host codec."""
        names = api._checkpoint_names(self.cfg)
        fields = {n: self.download(n) for n in names}
        m = self.slabs[0].m
        mean = None
        if self.mean_profiles:
            mean = m.mean_profile_rows()
        meta = m.checkpoint_state()
        if 0 in self.comm.local_ranks:
            api.checkpoint_write_host(self.cfg, path, fields, meta, mean)
        self.comm.barrier()

    def checkpoint_read(self, path: str):
        """Restart every slab from a whole-domain checkpoint (its fields scattered by rows)."""
        fields, mean, meta = api.checkpoint_read_host(self.cfg, path)
        self.set_state(fields)
        for s in self.slabs:
            s.m.restore_state(meta, mean)

    def diagnostics(self):
        """Domain-mean theta and w'^2 per level (mgpu_diagnostics): each slab's means over its
        interior rows, averaged over the slabs."""
        nz = self.geo.nz
        local = torch.zeros(2 * nz, dtype=torch.float64)
        for s in self.slabs:
            th, w2 = s.m.diagnostics()
            local[:nz] += torch.from_numpy(th)
            local[nz:] += torch.from_numpy(w2)
        total = self.comm.allreduce_sum(local) / self.comm.size
        return total[:nz].numpy(), total[nz:].numpy()

    def profile_diagnostics(self) -> dict:
        """profile_diagnostics sums over the whole domain: each slab's totals over its interior rows
        (MONC's <name>_total_local of one rank), summed over the slabs.  The sums read the row
        below each interior row, so the state halos are exchanged first."""
        self._exchange(cf.HALO_STATE, self.geo.halo)
        parts = [s.m.profile_diagnostics() for s in self.slabs]
        names = list(parts[0])
        local = torch.tensor(np.stack([sum(p[n] for p in parts) for n in names]), dtype=torch.float64)
        total = self.comm.allreduce_sum(local)
        return dict(zip(names, total.numpy()))

    def synchronize(self):
        for s in self.slabs:
            torch.cuda.ExternalStream(s.m.stream, device=self.device).synchronize()
