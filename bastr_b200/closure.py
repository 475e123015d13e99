"""Learned subgrid closure for the coarse 3D solve (the C ABI's ``bastr_net_*`` and
``bastr_closure_apply``).

Data: a fine (DNS) run of the solver; at snapshot times its velocity u and advective term
u.grad u (spectral derivatives through ``bastr_fft``) are box-filtered over r^3 cells onto the
coarse grid, giving the filtered velocity ub and tau = filter(u.grad u) - ub.grad ub (the
second term with spectral derivatives on the coarse grid).  The network (see
``bastr_b200/csrc/closure.cu``) learns tau / tau_rms from ub; it is trained on the GPU by the
library's own forward, backward and Adam kernels.  A coarse run applies it after every step as
one sub-step u <- u - dt * tau_rms * net(u) (Lie splitting), on the device.

PyTorch holds the device buffers here; the arithmetic is the library's.
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np


def _lib():
    from . import load_library
    return load_library()


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def init_weights(seed: int = 0) -> np.ndarray:
    """Deterministic initial FP32 weights: uniform in +-1/sqrt(fan-in), zero biases (the layout
    of bastr_b200/csrc/closure.cu)."""
    c, nin = 32, 81
    rng = np.random.default_rng(seed)
    w = np.zeros(nparams(), dtype=np.float32)
    o = 0
    w[o:o + c * nin] = rng.uniform(-1, 1, c * nin) / np.sqrt(nin)
    o += c * nin + c
    w[o:o + c * c] = rng.uniform(-1, 1, c * c) / np.sqrt(c)
    o += c * c + c
    w[o:o + c * c] = rng.uniform(-1, 1, c * c) / np.sqrt(c)
    o += c * c + c
    w[o:o + 3 * c] = rng.uniform(-1, 1, 3 * c) / np.sqrt(c)
    return w


def nparams() -> int:
    return 32 * 81 + 32 + 32 * 32 + 32 + 32 * 32 + 32 + 3 * 32 + 3


def bf16_bits_torch(w32):
    """BF16 bit patterns (round to nearest even) of an FP32 tensor, as int16."""
    import torch
    b = w32.contiguous().view(torch.int32).to(torch.int64) & 0xFFFFFFFF
    lsb = (b >> 16) & 1
    r = ((b + 0x7FFF + lsb) >> 16) & 0xFFFF
    return r.to(torch.int32).to(torch.int16)


class Net:
    """The closure network on one GPU: FP32 master weights, their BF16 copy and Adam moments as
    torch tensors; forward, loss/gradient and Adam through the library's kernels."""

    def __init__(self, weights: np.ndarray | None = None, seed: int = 0, device: int = 0):
        import torch
        self.torch = torch
        self.lib = _lib()
        self.dev = torch.device("cuda", device)
        w = init_weights(seed) if weights is None else np.asarray(weights, np.float32)
        self.w = torch.tensor(w, device=self.dev)
        self.wb = bf16_bits_torch(self.w)
        self.m = torch.zeros_like(self.w)
        self.v = torch.zeros_like(self.w)
        self.t = 0
        self.nblk = self.lib.bastr_net_grad_blocks()
        self.part = torch.empty((self.nblk, nparams() + 1), dtype=torch.float32, device=self.dev)
        self.grad = torch.empty(nparams(), dtype=torch.float32, device=self.dev)
        self.loss = torch.zeros(1, dtype=torch.float64, device=self.dev)
        self.tau_scale = 1.0

    def _stream(self):
        return C.c_void_p(self.torch.cuda.current_stream(self.dev).cuda_stream)

    def forward(self, u, scale: float = 1.0):
        """scale * net(u) for u [3][nz][ny][nx] (float32 CUDA tensor)."""
        u = u.contiguous()
        out = self.torch.empty_like(u)
        rc = self.lib.bastr_net_forward(u.shape[3], u.shape[2], u.shape[1], _ptr(u), _ptr(self.wb), _ptr(out),
                                        C.c_float(scale), self._stream())
        if rc != 0:
            raise RuntimeError(f"bastr_net_forward: {rc}")
        return out

    def loss_grad(self, u, tau):
        u, tau = u.contiguous(), tau.contiguous()
        rc = self.lib.bastr_net_grad(u.shape[3], u.shape[2], u.shape[1], _ptr(u), _ptr(tau), _ptr(self.wb),
                                     _ptr(self.part), self.nblk, _ptr(self.grad), _ptr(self.loss), self._stream())
        if rc != 0:
            raise RuntimeError(f"bastr_net_grad: {rc}")
        return float(self.loss.item()), self.grad

    def adam(self, lr: float = 1e-3, b1: float = 0.9, b2: float = 0.999, eps: float = 1e-8):
        self.t += 1
        rc = self.lib.bastr_net_adam(_ptr(self.w), _ptr(self.wb), _ptr(self.m), _ptr(self.v), _ptr(self.grad),
                                     self.t, C.c_float(lr), C.c_float(b1), C.c_float(b2), C.c_float(eps),
                                     self._stream())
        if rc != 0:
            raise RuntimeError(f"bastr_net_adam: {rc}")

    def train(self, pairs, iters: int, lr: float = 2e-3, log_every: int = 0, group=None):
        """Adam over the (u, tau/tau_scale) pairs in turn; returns the loss history.  With a
        torch.distributed process group of several ranks (one GPU each, every rank holding its
        own pairs), the gradient is averaged over the ranks before every step (data parallel:
        one all-reduce of the nparams() floats per step)."""
        hist = []
        for it in range(iters):
            u, tau = pairs[it % len(pairs)]
            loss, g = self.loss_grad(u, tau)
            if group is not None:
                average_gradient(g, group)
            self.adam(lr)
            hist.append(loss)
            if log_every and it % log_every == 0:
                print(f"iter {it}: loss {loss:.4e}", flush=True)
        return hist


def average_gradient(g, group=None):
    """In-place mean of a gradient tensor over the ranks of a torch.distributed group (NCCL for
    CUDA tensors, gloo for CPU tensors)."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    if world > 1:
        dist.all_reduce(g, op=dist.ReduceOp.SUM, group=group)
        g.div_(world)
    return g


# ---------------------------------------------------------------------------------------------
# data: filtered fine fields and the subgrid term
# ---------------------------------------------------------------------------------------------
def box_filter(f: np.ndarray, r: int) -> np.ndarray:
    """Mean over r x r x r cells of a [nz][ny][nx] field -> [nz/r][ny/r][nx/r]."""
    nz, ny, nx = f.shape
    return f.reshape(nz // r, r, ny // r, r, nx // r, r).mean(axis=(1, 3, 5))


def wavenumbers(n: int) -> np.ndarray:
    return np.fft.fftfreq(n, 1.0 / n)


def advective_gpu(solver, u) -> list[np.ndarray]:
    """u.grad u of a fine field through the library's full-grid transforms (bastr_fft)."""
    nz, ny, nx = u[0].shape
    ks = [wavenumbers(nx)[None, None, :], wavenumbers(ny)[None, :, None], wavenumbers(nz)[:, None, None]]
    uh = [solver.fft(c.astype(np.complex128), -1) for c in u]
    out = [np.zeros_like(u[0]) for _ in range(3)]
    for j in range(3):
        for i in range(3):
            d = solver.fft(1j * ks[j] * uh[i], +1).real
            out[i] += u[j] * d
    return out


def advective_np(u) -> list[np.ndarray]:
    """u.grad u on a (coarse) periodic grid with spectral derivatives (numpy)."""
    nz, ny, nx = u[0].shape
    ks = [wavenumbers(nx)[None, None, :], wavenumbers(ny)[None, :, None], wavenumbers(nz)[:, None, None]]
    uh = [np.fft.fftn(c) for c in u]
    out = [np.zeros_like(u[0]) for _ in range(3)]
    for j in range(3):
        for i in range(3):
            out[i] += u[j] * np.fft.ifftn(1j * ks[j] * uh[i]).real
    return out


def filtered_pair(solver, u, r: int):
    """(ub, tau) of one fine snapshot u (three [nz][ny][nx] arrays)."""
    adv = advective_gpu(solver, u)
    ub = [box_filter(c, r) for c in u]
    fadv = [box_filter(c, r) for c in adv]
    cadv = advective_np(ub)
    tau = [fa - ca for fa, ca in zip(fadv, cadv)]
    return np.stack(ub), np.stack(tau)


def shell_spectrum(u: np.ndarray, kmax: int) -> np.ndarray:
    """E(k) = sum over |k| in shell nint(|k|) = s of |u^|^2 / 2 (u^ scaled 1/N), s = 0..kmax."""
    nz, ny, nx = u[0].shape
    kk = np.sqrt(wavenumbers(nx)[None, None, :] ** 2 + wavenumbers(ny)[None, :, None] ** 2 +
                 wavenumbers(nz)[:, None, None] ** 2)
    sh = np.floor(kk + 0.5).astype(int).ravel()
    e = sum(np.abs(np.fft.fftn(c) / c.size) ** 2 for c in u).ravel() / 2
    return np.bincount(sh, weights=e, minlength=kmax + 1)[:kmax + 1]


def gpu_seconds(fn):
    """Device seconds of fn() (synchronised before and after)."""
    import torch
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    fn()
    torch.cuda.synchronize()
    return time.perf_counter() - t0
