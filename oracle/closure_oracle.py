"""CPU oracle of the learned subgrid closure (test infrastructure only: the tests use it as the
checker of the CUDA network kernels; nothing in the product calls it).

The network and its parameter layout are the ones the CUDA kernels implement
(bastr_b200/csrc/closure.cu): layer 1 a periodic 3x3x3 stencil 3 -> 32 channels, layers 2 and 3
pointwise 32 -> 32, layer 4 pointwise 32 -> 3, GELU (tanh form) after layers 1-3.  Weights are
used as BF16 (round to nearest even of the FP32 master value), and so are the inputs of every
layer (the taps and the activations h1..h3, rounded FP64 -> FP32 -> BF16 as the kernels round
their FP32 values) unless ``act_bf16=False``; the products and sums are FP64.  The loss is
mean((net(u) - tau)^2) over points and channels; the gradient is back-propagation written out by
hand, passing the rounding of layer inputs through unchanged (its derivative taken as 1, as the
kernels do), and `fd_gradient` differentiates the smooth loss (``act_bf16=False``) numerically
to check it.
There is no reference counterpart: the closure extends the reference's solver.
"""
from __future__ import annotations

import numpy as np

C = 32
NIN = 81
OFF_W1 = 0
OFF_B1 = OFF_W1 + C * NIN
OFF_W2 = OFF_B1 + C
OFF_B2 = OFF_W2 + C * C
OFF_W3 = OFF_B2 + C
OFF_B3 = OFF_W3 + C * C
OFF_W4 = OFF_B3 + C
OFF_B4 = OFF_W4 + 3 * C
NP = OFF_B4 + 3


def bf16_round(w: np.ndarray) -> np.ndarray:
    """FP32 -> BF16 (round to nearest, ties to even) -> back to FP32 values."""
    b = np.asarray(w, dtype=np.float32).view(np.uint32).astype(np.uint64)
    lsb = (b >> 16) & 1
    r = ((b + 0x7FFF + lsb) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def bf16_bits(w: np.ndarray) -> np.ndarray:
    """The uint16 bit patterns of bf16_round(w)."""
    return (bf16_round(w).view(np.uint32) >> 16).astype(np.uint16)


def unpack(w: np.ndarray):
    w = np.asarray(w, dtype=np.float64)
    return (w[OFF_W1:OFF_B1].reshape(C, NIN), w[OFF_B1:OFF_W2], w[OFF_W2:OFF_B2].reshape(C, C), w[OFF_B2:OFF_W3],
            w[OFF_W3:OFF_B3].reshape(C, C), w[OFF_B3:OFF_W4], w[OFF_W4:OFF_B4].reshape(3, C), w[OFF_B4:NP])


def init_weights(seed: int = 0) -> np.ndarray:
    """Deterministic initial FP32 weights (uniform, scaled by 1/sqrt(fan-in); zero biases)."""
    rng = np.random.default_rng(seed)
    w = np.zeros(NP, dtype=np.float32)
    w[OFF_W1:OFF_B1] = rng.uniform(-1, 1, C * NIN) / np.sqrt(NIN)
    w[OFF_W2:OFF_B2] = rng.uniform(-1, 1, C * C) / np.sqrt(C)
    w[OFF_W3:OFF_B3] = rng.uniform(-1, 1, C * C) / np.sqrt(C)
    w[OFF_W4:OFF_B4] = rng.uniform(-1, 1, 3 * C) / np.sqrt(C)
    return w


def gelu(z):
    a, c = np.sqrt(2.0 / np.pi), 0.044715
    t = np.tanh(a * (z + c * z ** 3))
    return 0.5 * z * (1 + t), 0.5 * (1 + t) + 0.5 * z * (1 - t * t) * a * (1 + 3 * c * z * z)


def taps(u: np.ndarray) -> np.ndarray:
    """[n, 81] inputs of every point of u [3][nz][ny][nx]: tap i = c*27 + (dz+1)*9 + (dy+1)*3 + (dx+1)."""
    cols = []
    for c in range(3):
        for dz in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dx in (-1, 0, 1):
                    cols.append(np.roll(u[c], shift=(-dz, -dy, -dx), axis=(0, 1, 2)).ravel())
    return np.stack(cols, axis=1).astype(np.float64)


def _act(h: np.ndarray, act_bf16: bool) -> np.ndarray:
    return bf16_round(h.astype(np.float32)).astype(np.float64) if act_bf16 else h


def forward(u: np.ndarray, w: np.ndarray, keep: bool = False, act_bf16: bool = True):
    """net(u) [3][nz][ny][nx] with BF16-rounded weights (and layer inputs, with act_bf16)."""
    W1, b1, W2, b2, W3, b3, W4, b4 = unpack(bf16_round(w))
    x = _act(taps(u), act_bf16)
    h1, d1 = gelu(x @ W1.T + b1)
    h1 = _act(h1, act_bf16)
    h2, d2 = gelu(h1 @ W2.T + b2)
    h2 = _act(h2, act_bf16)
    h3, d3 = gelu(h2 @ W3.T + b3)
    h3 = _act(h3, act_bf16)
    out = h3 @ W4.T + b4
    res = out.T.reshape((3,) + u.shape[1:])
    if keep:
        return res, (x, h1, d1, h2, d2, h3, d3, out)
    return res


def loss_grad(u: np.ndarray, tau: np.ndarray, w: np.ndarray, act_bf16: bool = True):
    """loss = mean((net(u) - tau)^2) and d loss / d w (with respect to the BF16-rounded weights)."""
    W1, b1, W2, b2, W3, b3, W4, b4 = unpack(bf16_round(w))
    _, (x, h1, d1, h2, d2, h3, d3, out) = forward(u, w, keep=True, act_bf16=act_bf16)
    t = np.stack([tau[c].ravel() for c in range(3)], axis=1).astype(np.float64)
    r = out - t
    n = r.shape[0]
    loss = float(np.sum(r * r) / (3 * n))
    eo = 2.0 * r / (3 * n)
    e3 = (eo @ W4) * d3
    e2 = (e3 @ W3) * d2
    e1 = (e2 @ W2) * d1
    g = np.zeros(NP)
    g[OFF_W1:OFF_B1] = (e1.T @ x).ravel()
    g[OFF_B1:OFF_W2] = e1.sum(0)
    g[OFF_W2:OFF_B2] = (e2.T @ h1).ravel()
    g[OFF_B2:OFF_W3] = e2.sum(0)
    g[OFF_W3:OFF_B3] = (e3.T @ h2).ravel()
    g[OFF_B3:OFF_W4] = e3.sum(0)
    g[OFF_W4:OFF_B4] = (eo.T @ h3).ravel()
    g[OFF_B4:NP] = eo.sum(0)
    return loss, g


def loss_only(u, tau, wv):
    """Loss with the weights taken as given (FP64, no BF16 rounding): for finite differences."""
    W1, b1, W2, b2, W3, b3, W4, b4 = unpack(wv)
    x = taps(u)
    h1, _ = gelu(x @ W1.T + b1)
    h2, _ = gelu(h1 @ W2.T + b2)
    h3, _ = gelu(h2 @ W3.T + b3)
    out = h3 @ W4.T + b4
    t = np.stack([tau[c].ravel() for c in range(3)], axis=1)
    return float(np.sum((out - t) ** 2) / (3 * out.shape[0]))


def fd_gradient(u, tau, w, idx, h=1e-6):
    """Central differences of the loss at the BF16-rounded weights, for parameters idx."""
    w0 = bf16_round(w).astype(np.float64)
    g = []
    for q in idx:
        wp, wm = w0.copy(), w0.copy()
        wp[q] += h
        wm[q] -= h
        g.append((loss_only(u, tau, wp) - loss_only(u, tau, wm)) / (2 * h))
    return np.array(g)


def adam(w, m, v, g, t, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step (Kingma & Ba 2015) in FP32, as k_net_adam does it."""
    w, m, v, g = (np.asarray(a, dtype=np.float32) for a in (w, m, v, g))
    m = (b1 * m + (1 - b1) * g).astype(np.float32)
    v = (b2 * v + (1 - b2) * g * g).astype(np.float32)
    mh = m / np.float32(1 - b1 ** t)
    vh = v / np.float32(1 - b2 ** t)
    w = (w - np.float32(lr) * mh / (np.sqrt(vh) + np.float32(eps))).astype(np.float32)
    return w, m, v
