"""Host logic of the y-slab decomposition on CPU: slab geometry, the halo exchange and the two
all-to-all transposes of the pressure solve, over gloo with world size 2 and 4 and through the
in-process loopback communicator.

The GPU kernels that pack halo rows and write the x-spectrum in kx blocks are restated here in
numpy following the layouts include/monc_gpu.h documents (mgpu_halo_pack, mgpu_slab_fft_x,
mgpu_slab_solve_columns); the test checks that, with those layouts, the exchanges deliver
exactly the periodic halo rows and a spectrum equal to the 2-D FFT of the whole domain.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from monc_b200 import decomposition as dc

NX, NY, NZ = 16, 32, 3
HALO = 4


def test_geometry_blocks_and_rows():
    g = dc.SlabGeometry(64, 64, 10, 4)
    assert g.nyl == 16
    assert g.blocks == [(0, 9), (9, 8), (17, 8), (25, 8)]
    assert dc.kx_blocks(33, 8) == [(0, 5)] + [(5 + 4 * q, 4) for q in range(7)]
    # x blocks tile the slab spectrum exactly
    ends = [g.xblock(q)[0] + g.xblock(q)[1] for q in range(4)]
    assert ends[-1] == 10 * 16 * 33 and all(g.xblock(q + 1)[0] == ends[q] for q in range(3))
    assert list(g.rows(0)[:HALO]) == [60, 61, 62, 63]
    assert list(g.rows(3)[-HALO:]) == [0, 1, 2, 3]
    with pytest.raises(ValueError):
        dc.SlabGeometry(64, 64, 10, 3)  # rows do not split
    with pytest.raises(ValueError):
        dc.SlabGeometry(64, 8, 10, 4)  # slabs of 2 rows cannot supply 4 halo rows
    with pytest.raises(ValueError):
        dc.kx_blocks(3, 4)
    assert dc.kx_blocks(5, 1) == [(0, 5)]


def domain(seed=1):
    rng = np.random.RandomState(seed)
    return rng.randn(NZ, NY, NX)


def pack(slab, depth, halo):
    """mgpu_halo_pack: first and last `depth` interior rows of every level -> [nz][depth][nx]."""
    ny = slab.shape[1]
    return slab[:, halo:halo + depth].copy(), slab[:, ny - halo - depth:ny - halo].copy()


def unpack(slab, lo, hi, depth, halo):
    ny = slab.shape[1]
    slab[:, halo - depth:halo] = lo
    slab[:, ny - halo:ny - halo + depth] = hi


def fft_x_blocks(slab, g, halo):
    """mgpu_slab_fft_x: rfft along x of the interior rows, kx blocks [nz][nyl][w_q] end to end."""
    spec = np.fft.rfft(slab[:, halo:halo + g.nyl], axis=2)  # [nz][nyl][nxh]
    out = np.zeros(g.nz * g.nyl * g.nxh, dtype=complex)
    for q, (k0, w) in enumerate(g.blocks):
        off, n = g.xblock(q)
        out[off:off + n] = spec[:, :, k0:k0 + w].reshape(-1)
    return out


def as_real(c):
    return torch.from_numpy(np.ascontiguousarray(c).view(np.float64).copy())


def as_complex(t):
    return t.numpy().view(np.complex128)


def run_slab_checks(comm, ranks):
    """The exchanges for the slabs `ranks` held here; returns nothing, asserts inside."""
    g = dc.SlabGeometry(NX, NY, NZ, comm.size, HALO)
    full = domain()
    # slabs with garbage in the halo rows
    slabs = {r: full[:, g.rows(r)].copy() for r in ranks}
    for r in ranks:
        slabs[r][:, :HALO] = np.nan
        slabs[r][:, -HALO:] = np.nan
    # halo exchange at full depth, then at depth 1 after spoiling the halos again
    for depth in (HALO, 1):
        bufs = {r: [torch.from_numpy(b) for b in pack(slabs[r], depth, HALO)] for r in ranks}
        recv = {r: [torch.empty_like(bufs[r][0]), torch.empty_like(bufs[r][1])] for r in ranks}
        comm.halo_exchange([bufs[r][0] for r in ranks], [bufs[r][1] for r in ranks],
                           [recv[r][0] for r in ranks], [recv[r][1] for r in ranks])
        for r in ranks:
            unpack(slabs[r], recv[r][0].numpy(), recv[r][1].numpy(), depth, HALO)
            lo_rows = slice(HALO - depth, g.nyl + HALO + depth)
            np.testing.assert_array_equal(slabs[r][:, lo_rows], full[:, g.rows(r)][:, lo_rows])
    # forward transpose: rank q gets all rows of kx block q
    spec_x = {r: as_real(fft_x_blocks(slabs[r], g, HALO)) for r in ranks}
    spec_t = {r: torch.zeros(2 * g.nz * g.ny * g.blocks[r][1], dtype=torch.float64) for r in ranks}

    def xb(r):
        return [spec_x[r][2 * o:2 * (o + n)] for o, n in (g.xblock(q) for q in range(g.nranks))]

    def tb(r):
        return [spec_t[r][2 * o:2 * (o + n)] for o, n in (g.tblock(r, s) for s in range(g.nranks))]

    comm.all_to_all([xb(r) for r in ranks], [tb(r) for r in ranks])
    ref = np.fft.fft(np.fft.rfft(full, axis=2), axis=1)  # [nz][ny][nxh]
    for r in ranks:
        k0, w = g.blocks[r]
        t = as_complex(spec_t[r]).reshape(g.nranks, g.nz, g.nyl, w)   # row blocks [b][nz][rpb][w]
        cols = t.transpose(1, 0, 2, 3).reshape(g.nz, g.ny, w)          # [nz][ny][w]
        got = np.fft.fft(cols, axis=1)
        np.testing.assert_allclose(got, ref[:, :, k0:k0 + w], rtol=0, atol=1e-12 * np.abs(ref).max())
        # mgpu_slab_solve_columns stand-in: scale every coefficient by its wavenumber index
        scaled = np.fft.ifft(got * (1.0 + np.arange(k0, k0 + w))[None, None, :], axis=1)
        blocks = scaled.reshape(g.nz, g.nranks, g.nyl, w).transpose(1, 0, 2, 3)
        spec_t[r].copy_(as_real(blocks.reshape(-1)))
    # backward transpose, inverse x-FFT of each slab's rows
    for r in ranks:
        spec_x[r].zero_()
    comm.all_to_all([tb(r) for r in ranks], [xb(r) for r in ranks])
    expect = np.fft.irfft(np.fft.rfft(full, axis=2) * (1.0 + np.arange(g.nxh))[None, None, :], n=NX, axis=2)
    for r in ranks:
        spec = np.zeros((g.nz, g.nyl, g.nxh), dtype=complex)
        flat = as_complex(spec_x[r])
        for q, (k0, w) in enumerate(g.blocks):
            off, n = g.xblock(q)
            spec[:, :, k0:k0 + w] = flat[off:off + n].reshape(g.nz, g.nyl, w)
        rows = np.fft.irfft(spec, n=NX, axis=2)
        np.testing.assert_allclose(rows, expect[:, g.y0(r):g.y0(r) + g.nyl], rtol=0, atol=1e-12)
    # level means: the mean of equal slabs' means is the domain mean
    means = {r: torch.from_numpy(full[:, g.y0(r):g.y0(r) + g.nyl].mean(axis=(1, 2)).copy()) for r in ranks}
    comm.allreduce_mean([means[r] for r in ranks])
    for r in ranks:
        np.testing.assert_allclose(means[r].numpy(), full.mean(axis=(1, 2)), rtol=1e-14, atol=1e-15)
    # cfltest's extrema in max form (minima negated): one maximum gives the domain's min and max
    ext = {r: torch.tensor([-full[:, g.y0(r):g.y0(r) + g.nyl].min(), full[:, g.y0(r):g.y0(r) + g.nyl].max()])
           for r in ranks}
    comm.allreduce_max([ext[r] for r in ranks])
    for r in ranks:
        assert (-ext[r][0].item(), ext[r][1].item()) == (full.min(), full.max())
    # inner products of the iterative solve: the slabs' partial sums add up to the domain's
    dots = {r: torch.tensor([(full[:, g.y0(r):g.y0(r) + g.nyl] ** 2).sum(), float(g.nyl), 0.0]) for r in ranks}
    comm.allreduce_sum_inplace([dots[r] for r in ranks])
    for r in ranks:
        np.testing.assert_allclose(dots[r][0].item(), (full ** 2).sum(), rtol=1e-13)
        assert dots[r][1].item() == NY and dots[r][2].item() == 0.0


@pytest.mark.parametrize("nranks", [1, 2, 4])
def test_loopback_exchanges(nranks):
    run_slab_checks(dc.LoopbackComm(nranks), list(range(nranks)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, errs):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        run_slab_checks(dc.TorchComm(), [rank])
    except Exception as e:  # report to the parent
        errs.put(f"rank {rank}: {type(e).__name__}: {e}")
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 4])
def test_gloo_exchanges(world):
    ctx = mp.get_context("spawn")
    errs = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, errs)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
    alive = [p for p in procs if p.is_alive()]
    for p in alive:
        p.kill()
    assert not alive, "a rank did not finish"
    msgs = []
    while not errs.empty():
        msgs.append(errs.get())
    assert not msgs, msgs
    assert all(p.exitcode == 0 for p in procs)
