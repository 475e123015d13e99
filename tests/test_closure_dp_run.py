"""The data-parallel closure training launcher on CPU: two gloo ranks with different shares of the
targets compute the same global tau_rms and, through the same training loop the GPU ranks run
(Net.train with the gradient averaged before every step), end with identical weights, equal to
one rank training on the pooled data.  The network is replaced by a small linear stand-in
(no GPU); the seed split is checked to give every seed exactly once."""
import os
import socket

import numpy as np
import torch
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class LinearNet:
    """Stand-in with Net's training interface: tau ~ w . u per point, squared-error loss."""

    def __init__(self):
        self.w = torch.zeros(3, dtype=torch.float64)
        self.grad = torch.zeros(3, dtype=torch.float64)

    def loss_grad(self, u, tau):
        x = u.reshape(3, -1).double()
        t = tau.reshape(3, -1).double().sum(0)
        r = self.w @ x - t
        self.grad.copy_(2.0 * (x @ r) / r.numel())
        return float(torch.mean(r * r)), self.grad

    def adam(self, lr):
        self.w -= lr * self.grad


def _data(seed):
    g = torch.Generator().manual_seed(seed)
    u = torch.randn(3, 4, 4, 4, generator=g, dtype=torch.float64)
    tau = torch.stack([0.5 * u[0] - u[1], u[2], 0.3 * u[0]]) + 0.1 * torch.randn(3, 4, 4, 4, generator=g,
                                                                                  dtype=torch.float64)
    return u, tau


def _train(net, pairs, group):
    from bastr_b200.closure import Net
    from bastr_b200.closure_dp import global_tau_rms
    tau_rms = global_tau_rms(pairs, group, "cpu")
    train = [(u, t / tau_rms) for u, t in pairs]
    Net.train(net, train, iters=50, lr=0.05, group=group)
    return tau_rms


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime
    import torch.distributed as dist
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    pairs = [_data(10 + rank)]
    net = LinearNet()
    tau_rms = _train(net, pairs, dist.group.WORLD)
    q.put((rank, tau_rms, net.w.numpy().copy()))
    dist.destroy_process_group()


def test_two_ranks_train_identical_weights():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = {r: (s, w) for r, s, w in (q.get(timeout=120) for _ in range(world))}
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (s0, w0), (s1, w1) = res[0], res[1]
    assert s0 == s1
    assert np.array_equal(w0, w1)
    # the same as training one network on both ranks' data with the gradients averaged by hand
    pooled = [_data(10), _data(11)]
    rms = float(torch.sqrt(torch.mean(torch.stack([t for _, t in pooled]) ** 2)))
    assert abs(rms - s0) < 1e-12 * rms
    net = LinearNet()
    scaled = [(u, t / rms) for u, t in pooled]
    for _ in range(50):
        g = sum(net.loss_grad(u, t)[1].clone() for u, t in scaled) / 2
        net.w -= 0.05 * g
    assert np.allclose(net.w.numpy(), w0, rtol=1e-12, atol=1e-14)


def test_seed_shards_cover_every_seed_once():
    from bastr_b200.closure_dp import shard_seeds
    seeds = list(range(8))
    for world in (1, 2, 3, 8):
        got = sorted(s for r in range(world) for s in shard_seeds(seeds, r, world))
        assert got == seeds
