"""Slab-decomposed 3D transforms over several GPUs: one process per GPU, the grid in z-slabs.

The reference distributes its 3D grid in z-slabs over MPI ranks (fftwlink.F90:63-77) and
transforms it with FFTW-MPI (fftwlink.F90:324-368: forward e^{-ikx} scaled by 1/N, backward
e^{+ikx}).  Here rank r of P holds planes z in [r nz/P, (r+1) nz/P) of a complex FP64 grid
[nz][ny][nx] (x fastest) in its own GPU's memory, and

    forward:  x and y lines of the slab (bastr_fft_lines) -> pack (bastr_slab_pack: the block
              for rank q holds the slab's y range q ny/P ..) -> one all-to-all of equal blocks
              (NCCL all_to_all_single) -> z lines of the received y-slab [nz][ny/P][nx], scaled 1/N
    backward: z lines of the y-slab -> all-to-all -> unpack (bastr_slab_unpack) -> y and x lines

so the spectrum stays y-slab distributed between the two (the reference's transposed layout) and
every block crosses NVLink once, into the receiver's own memory.  `exchange` is the only
collective; with one rank it is a copy.

`LocalRanks` runs P ranks' slabs in one process on one GPU, the exchange being a local
re-arrangement of the blocks: it exercises the decomposition, packing and exchange order on a
single device (what one GPU can check); `SlabFFT3D` with a torch.distributed process group is the
multi-GPU form.
"""
from __future__ import annotations

import ctypes as C

from . import BASTR_OK, load_library


def _ptr(t):
    return C.c_void_p(t.data_ptr())


class _Kernels:
    """The library's per-GPU pieces on CUDA complex128 tensors (the caller's stream)."""

    def __init__(self):
        import torch
        self.torch = torch
        self.lib = load_library()

    def _stream(self, t):
        return C.c_void_p(self.torch.cuda.current_stream(t.device).cuda_stream)

    def lines(self, a, axis: int, direction: int, scale: float = 1.0):
        nz, ny, nx = a.shape
        rc = self.lib.bastr_fft_lines(_ptr(a), nx, ny, nz, axis, direction, C.c_double(scale), self._stream(a))
        if rc != BASTR_OK:
            raise RuntimeError(f"bastr_fft_lines: {rc}")

    def pack(self, slab, blocks, nparts: int):
        nzl, ny, nx = slab.shape
        rc = self.lib.bastr_slab_pack(_ptr(slab), _ptr(blocks), nx, ny, nzl, nparts, self._stream(slab))
        if rc != BASTR_OK:
            raise RuntimeError(f"bastr_slab_pack: {rc}")

    def unpack(self, blocks, slab, nparts: int):
        nzl, ny, nx = slab.shape
        rc = self.lib.bastr_slab_unpack(_ptr(blocks), _ptr(slab), nx, ny, nzl, nparts, self._stream(slab))
        if rc != BASTR_OK:
            raise RuntimeError(f"bastr_slab_unpack: {rc}")


def _check_extents(n: tuple, p: int):
    nz, ny, nx = n
    if nz % p or ny % p:
        raise ValueError(f"grid {nx}x{ny}x{nz}: nz and ny must be multiples of the {p} ranks")


class SlabFFT3D:
    """Forward / backward slab transforms of this rank's share of an nx x ny x nz complex grid.

    `group`: a torch.distributed process group of P ranks (one GPU each) or None for one rank;
    `kernels`: the per-GPU pieces (the library's by default; tests on CPU ranks pass stand-ins)."""

    def __init__(self, nx: int, ny: int, nz: int, group=None, kernels=None):
        import torch
        import torch.distributed as dist
        self.torch, self.dist, self.group = torch, dist, group
        self.p = dist.get_world_size(group) if group is not None else 1
        self.rank = dist.get_rank(group) if group is not None else 0
        self.n = (nz, ny, nx)
        _check_extents(self.n, self.p)
        self.k = kernels or _Kernels()

    def exchange(self, send):
        """One all-to-all of P equal blocks along the first axis of `send`."""
        if self.p == 1:
            return send.clone()
        send = send.contiguous()
        recv = self.torch.empty_like(send)
        # as FP64 pairs: every backend moves float64, not every one complex128
        self.dist.all_to_all_single(self.torch.view_as_real(recv), self.torch.view_as_real(send), group=self.group)
        return recv

    def forward(self, slab):
        """slab [nz/P][ny][nx] -> this rank's y-slab of the spectrum [nz][ny/P][nx] (scaled 1/N)."""
        nz, ny, nx = self.n
        p = self.p
        a = slab.clone()
        self.k.lines(a, 0, -1)
        self.k.lines(a, 1, -1)
        blocks = self.torch.empty((p, nz // p, ny // p, nx), dtype=a.dtype, device=a.device)
        self.k.pack(a, blocks, p)
        y = self.exchange(blocks).reshape(nz, ny // p, nx)
        self.k.lines(y, 2, -1, 1.0 / (nx * ny * nz))
        return y

    def backward(self, yslab):
        """This rank's y-slab [nz][ny/P][nx] -> its z-slab of the grid [nz/P][ny][nx] (unscaled)."""
        nz, ny, nx = self.n
        p = self.p
        y = yslab.clone()
        self.k.lines(y, 2, 1)
        blocks = self.exchange(y.reshape(p, nz // p, ny // p, nx))
        a = self.torch.empty((nz // p, ny, nx), dtype=y.dtype, device=y.device)
        self.k.unpack(blocks, a, p)
        self.k.lines(a, 1, 1)
        self.k.lines(a, 0, 1)
        return a


class LocalRanks:
    """P ranks' slabs transformed in one process (one device): the same pieces as SlabFFT3D,
    the all-to-all done as a local re-arrangement of the blocks (rank r's received block q is
    rank q's sent block r)."""

    def __init__(self, nx: int, ny: int, nz: int, p: int, kernels=None):
        import torch
        self.torch = torch
        self.n, self.p = (nz, ny, nx), p
        _check_extents(self.n, p)
        self.k = kernels or _Kernels()

    def _all_to_all(self, sends):
        p = self.p
        return [self.torch.stack([sends[q][r] for q in range(p)]) for r in range(p)]

    def forward(self, slabs):
        nz, ny, nx = self.n
        p = self.p
        sends = []
        for s in slabs:
            a = s.clone()
            self.k.lines(a, 0, -1)
            self.k.lines(a, 1, -1)
            b = self.torch.empty((p, nz // p, ny // p, nx), dtype=a.dtype, device=a.device)
            self.k.pack(a, b, p)
            sends.append(b)
        out = []
        for r in self._all_to_all(sends):
            y = r.reshape(nz, ny // p, nx).contiguous()
            self.k.lines(y, 2, -1, 1.0 / (nx * ny * nz))
            out.append(y)
        return out

    def backward(self, yslabs):
        nz, ny, nx = self.n
        p = self.p
        sends = []
        for y in yslabs:
            y = y.clone()
            self.k.lines(y, 2, 1)
            sends.append(y.reshape(p, nz // p, ny // p, nx))
        out = []
        for r in self._all_to_all(sends):
            a = self.torch.empty((nz // p, ny, nx), dtype=r.dtype, device=r.device)
            self.k.unpack(r.contiguous(), a, p)
            self.k.lines(a, 1, 1)
            self.k.lines(a, 0, 1)
            out.append(a)
        return out
