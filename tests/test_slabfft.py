"""Slab-decomposed 3D transforms (the reference's FFTW-MPI z-slab decomposition,
fftwlink.F90:63-77 and 324-368).

On CPU: two gloo ranks run SlabFFT3D with stand-in per-rank pieces (torch.fft line transforms
and torch re-arrangements in place of the CUDA kernels), so the decomposition, packing order,
all-to-all and scaling are checked against numpy's fftn without a GPU.  On the GPU: the library's
pieces (bastr_fft_lines, bastr_slab_pack / unpack) against numpy, one rank through SlabFFT3D and
2 and 4 ranks through LocalRanks (all slabs on one device, the exchange a local re-arrangement).
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

TOL = 1e-12


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


class TorchPieces:
    """Stand-ins for the CUDA pieces on CPU tensors (test only)."""

    def lines(self, a, axis, direction, scale=1.0):
        dim = 2 - axis
        f = torch.fft.fft(a, dim=dim) if direction < 0 else torch.fft.ifft(a, dim=dim) * a.shape[dim]
        a.copy_(f * scale)

    def pack(self, slab, blocks, p):
        nzl, ny, nx = slab.shape
        blocks.copy_(slab.reshape(nzl, p, ny // p, nx).permute(1, 0, 2, 3))

    def unpack(self, blocks, slab, p):
        slab.copy_(blocks.permute(1, 0, 2, 3).reshape(slab.shape))


def _grid(n, seed):
    nx, ny, nz = n
    rng = np.random.default_rng(seed)
    return rng.standard_normal((nz, ny, nx)) + 1j * rng.standard_normal((nz, ny, nx))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, n, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime
    import torch.distributed as dist
    from bastr_b200.slabfft import SlabFFT3D
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    nx, ny, nz = n
    u = _grid(n, 5)
    nzl = nz // world
    f = SlabFFT3D(nx, ny, nz, group=dist.group.WORLD, kernels=TorchPieces())
    slab = torch.from_numpy(u[rank * nzl:(rank + 1) * nzl].copy())
    y = f.forward(slab)
    back = f.backward(y)
    q.put((rank, y.numpy(), back.numpy()))
    dist.destroy_process_group()


def test_two_gloo_ranks_match_numpy():
    n = (8, 12, 6)          # nx, ny, nz: every extent differs
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, n, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict((r, (y, b)) for r, y, b in (q.get(timeout=120) for _ in range(world)))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    nx, ny, nz = n
    u = _grid(n, 5)
    want = np.fft.fftn(u) / u.size                  # forward e^{-ikx} scaled by 1/N
    nyl = ny // world
    got = np.concatenate([res[r][0] for r in range(world)], axis=1)   # y-slabs [nz][ny/P][nx]
    assert _rel(got, want) < TOL
    back = np.concatenate([res[r][1] for r in range(world)], axis=0)
    assert _rel(back, u) < TOL
    assert got.shape == (nz, ny, nx) and res[0][0].shape == (nz, nyl, nx)


def test_extents_must_divide_over_ranks():
    from bastr_b200.slabfft import LocalRanks
    with pytest.raises(ValueError):
        LocalRanks(16, 16, 12, 8, kernels=TorchPieces())


@pytest.mark.gpu
def test_lines_match_numpy_on_every_axis(gpu_lib):
    from bastr_b200.slabfft import _Kernels
    k = _Kernels()
    u = _grid((32, 64, 16), 1)
    for axis in range(3):
        a = torch.from_numpy(u.copy()).cuda()
        k.lines(a, axis, -1, 0.5)
        assert _rel(a.cpu().numpy(), 0.5 * np.fft.fft(u, axis=2 - axis)) < 1e-13
        a = torch.from_numpy(u.copy()).cuda()
        k.lines(a, axis, 1)
        assert _rel(a.cpu().numpy(), np.fft.ifft(u, axis=2 - axis) * u.shape[2 - axis]) < 1e-13


@pytest.mark.gpu
def test_pack_unpack_are_exact_rearrangements(gpu_lib):
    from bastr_b200.slabfft import _Kernels
    k = _Kernels()
    u = torch.from_numpy(_grid((16, 32, 4), 2)).cuda()
    for p in (1, 2, 4, 8):
        b = torch.empty((p, 4, 32 // p, 16), dtype=u.dtype, device=u.device)
        k.pack(u, b, p)
        assert torch.equal(b, u.reshape(4, p, 32 // p, 16).permute(1, 0, 2, 3))
        back = torch.empty_like(u)
        k.unpack(b, back, p)
        assert torch.equal(back, u)


@pytest.mark.gpu
@pytest.mark.parametrize("p", [1, 2, 4])
def test_slab_transform_matches_numpy(gpu_lib, p):
    from bastr_b200.slabfft import LocalRanks, SlabFFT3D
    nx, ny, nz = 64, 32, 128
    u = _grid((nx, ny, nz), 3)
    want = np.fft.fftn(u) / u.size
    nzl = nz // p
    slabs = [torch.from_numpy(u[r * nzl:(r + 1) * nzl].copy()).cuda() for r in range(p)]
    if p == 1:
        f = SlabFFT3D(nx, ny, nz)
        ys = [f.forward(slabs[0])]
        backs = [f.backward(ys[0])]
    else:
        f = LocalRanks(nx, ny, nz, p)
        ys = f.forward(slabs)
        backs = f.backward(ys)
    got = np.concatenate([y.cpu().numpy() for y in ys], axis=1)
    assert _rel(got, want) < TOL
    back = np.concatenate([b.cpu().numpy() for b in backs], axis=0)
    assert _rel(back, u) < TOL
