"""The learned closure's CUDA kernels against the CPU oracle (oracle/closure_oracle.py): forward
pass, loss and gradient, Adam step and the closure sub-step on a solver's state; then what the
trained network gains over no closure on filtered DNS data that the solver itself generates."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a, b = np.asarray(a, np.float64).ravel(), np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _weights(seed):
    from oracle import closure_oracle as co
    rng = np.random.default_rng(seed)
    w = co.init_weights(seed)
    w[co.OFF_B1:co.OFF_W2] = rng.uniform(-0.2, 0.2, co.C)
    w[co.OFF_B2:co.OFF_W3] = rng.uniform(-0.2, 0.2, co.C)
    w[co.OFF_B4:co.NP] = rng.uniform(-0.2, 0.2, 3)
    return w


def _tensor(a):
    import torch
    return torch.tensor(np.ascontiguousarray(a, np.float32), device="cuda")


def test_forward_matches_oracle(gpu_lib):
    from bastr_b200.closure import Net
    from oracle import closure_oracle as co
    rng = np.random.default_rng(1)
    u = rng.standard_normal((3, 8, 12, 16)).astype(np.float32)   # [3][nz][ny][nx], all extents differ
    w = _weights(2)
    net = Net(weights=w)
    got = net.forward(_tensor(u), scale=1.5).cpu().numpy()
    # tensor-core forward: BF16 layer inputs, FP32 sums.  The oracle rounds the same inputs from
    # its FP64 values, so an input whose FP32 and FP64 values straddle a BF16 rounding boundary
    # rounds differently (about 6e-5 relative L2 in an FP32 simulation): tolerance 5e-4.
    assert _rel(got, 1.5 * co.forward(u.astype(np.float64), w)) < 5e-4


def test_forward_tiles_and_extents(gpu_lib):
    """Point counts that are not a multiple of the 128-point tile, extents of 3 (every neighbour
    wraps), many tiles per block, and two calls in a row give the same bits."""
    from bastr_b200.closure import Net
    from oracle import closure_oracle as co
    rng = np.random.default_rng(11)
    w = _weights(12)
    net = Net(weights=w)
    for shape in [(3, 3, 3, 3), (3, 5, 7, 9), (3, 24, 40, 36)]:
        u = rng.standard_normal(shape).astype(np.float32)
        got = net.forward(_tensor(u)).cpu().numpy()
        assert np.all(np.isfinite(got))
        assert _rel(got, co.forward(u.astype(np.float64), w)) < 5e-4, shape
        again = net.forward(_tensor(u)).cpu().numpy()
        assert np.array_equal(got, again)


def test_forward_and_training_loss_agree(gpu_lib):
    """The tensor-core forward (inference) and the training kernel's forward use the same
    arithmetic: the loss of one equals the loss of the other up to FP32 summation order."""
    import torch
    from bastr_b200.closure import Net
    rng = np.random.default_rng(13)
    u = rng.standard_normal((3, 16, 16, 16)).astype(np.float32)
    tau = rng.standard_normal((3, 16, 16, 16)).astype(np.float32)
    net = Net(weights=_weights(14))
    loss, _ = net.loss_grad(_tensor(u), _tensor(tau))
    pred = net.forward(_tensor(u))
    l2 = float(torch.mean((pred.double() - _tensor(tau).double()) ** 2))
    assert abs(loss - l2) / l2 < 1e-5


def test_bf16_copy_matches_oracle_rounding(gpu_lib):
    from bastr_b200.closure import Net
    from oracle import closure_oracle as co
    w = _weights(3)
    net = Net(weights=w)
    assert np.array_equal(net.wb.cpu().numpy().view(np.uint16), co.bf16_bits(w))


def test_loss_and_gradient_match_oracle(gpu_lib):
    from bastr_b200.closure import Net
    from oracle import closure_oracle as co
    rng = np.random.default_rng(4)
    u = rng.standard_normal((3, 8, 8, 12)).astype(np.float32)
    tau = (0.5 * rng.standard_normal((3, 8, 8, 12))).astype(np.float32)
    w = _weights(5)
    net = Net(weights=w)
    loss, g = net.loss_grad(_tensor(u), _tensor(tau))
    rl, rg = co.loss_grad(u.astype(np.float64), tau.astype(np.float64), w)
    # BF16 layer inputs rounded from FP32 here and from FP64 in the oracle (see the forward test)
    assert abs(loss - rl) / rl < 1e-4
    assert _rel(g.cpu().numpy(), rg) < 1e-3
    # deterministic: the same call gives the same bits
    _, g2 = net.loss_grad(_tensor(u), _tensor(tau))
    assert np.array_equal(g.cpu().numpy(), g2.cpu().numpy())


def test_adam_matches_oracle(gpu_lib):
    from bastr_b200.closure import Net
    from oracle import closure_oracle as co
    rng = np.random.default_rng(6)
    u = rng.standard_normal((3, 6, 6, 6)).astype(np.float32)
    tau = rng.standard_normal((3, 6, 6, 6)).astype(np.float32)
    w = _weights(7)
    net = Net(weights=w)
    _, g = net.loss_grad(_tensor(u), _tensor(tau))
    gh = g.cpu().numpy()
    net.adam(lr=1e-3)
    w1, _, _ = co.adam(w, np.zeros_like(w), np.zeros_like(w), gh, 1, 1e-3)
    assert _rel(net.w.cpu().numpy(), w1) < 1e-6
    assert np.array_equal(net.wb.cpu().numpy().view(np.uint16), co.bf16_bits(net.w.cpu().numpy()))


def test_training_reduces_loss(gpu_lib):
    """A target the network can represent (a pointwise function of neighbouring velocities)."""
    from bastr_b200.closure import Net
    rng = np.random.default_rng(8)
    u = rng.standard_normal((3, 16, 16, 16)).astype(np.float32)
    tau = np.stack([0.5 * u[0] * np.roll(u[1], 1, axis=2), np.tanh(u[2]), u[0] - np.roll(u[2], -1, axis=0)])
    net = Net(seed=0)
    hist = net.train([(_tensor(u), _tensor(tau))], iters=300, lr=3e-3)
    assert hist[-1] < 0.3 * hist[0]


def test_closure_apply_matches_host(gpu_lib):
    """u <- dealias(u - dt * scale * net(u)) on a 3D solver's state."""
    from bastr_b200 import BastrGPU, seeded_field
    from bastr_b200.closure import Net
    from oracle import closure_oracle as co
    from oracle.bastr_oracle import Params, dealias_mask, generate_wave
    n, dt, scale = 16, 1e-2, 0.7
    u0 = seeded_field(n, n, n, k0=3.0, seed=2)
    w = _weights(9)
    net = Net(weights=w)
    with BastrGPU(n, n, n) as s:
        s.set_state(u0)
        u = np.stack(s.get_state())
        s.closure_apply(net, scale, dt)
        got = np.stack(s.get_state())
    tau = co.forward(u.astype(np.float32).astype(np.float64), w)
    p = Params(ia=n, ja=n, ka=n)
    k1, k2, k3 = generate_wave(p)
    m = dealias_mask(p, np.sqrt(k1 * k1 + k2 * k2 + k3 * k3))
    want = np.stack([np.fft.ifftn(np.fft.fftn(u[c] - dt * scale * tau[c]) * m).real for c in range(3)])
    # the sub-step's change of the state, against the oracle's network (BF16 layer inputs: 5e-4)
    assert _rel(got - u, want - u) < 5e-4


def test_trained_closure_beats_no_closure_on_filtered_dns(gpu_lib):
    """A-priori gain: on held-out filtered DNS data (64^3 -> 16^3, box filter r = 4), the trained
    network's tau has a smaller mean-square error than the no-closure model (tau = 0)."""
    import torch
    from bastr_b200 import BastrGPU, seeded_field
    from bastr_b200.closure import Net, filtered_pair
    n, r = 64, 4
    pairs = []
    with BastrGPU(n, n, n, reynolds=500.0, deltat=2e-3, forcemethod=1, target_energy=1.5, velgrad_every=0) as s:
        s.set_state(seeded_field(n, n, n, k0=3.0, seed=0))
        for _ in range(4):
            s.step(40)
            ub, tau = filtered_pair(s, s.get_state(), r)
            pairs.append((ub, tau))
    scale = float(np.sqrt(np.mean(np.stack([t for _, t in pairs[:3]]) ** 2)))
    train = [(_tensor(ub), _tensor(t / scale)) for ub, t in pairs[:3]]
    net = Net(seed=1)
    net.train(train, iters=600, lr=3e-3)
    ub, tau = pairs[3]
    pred = net.forward(_tensor(ub), scale=scale).cpu().numpy()
    mse_net = float(np.mean((pred - tau) ** 2))
    mse_none = float(np.mean(tau ** 2))
    assert mse_net < 0.7 * mse_none, (mse_net, mse_none)
    torch.cuda.synchronize()


def test_closure_study_runs_from_ensemble_data(gpu_lib):
    """The a-posteriori study end to end at a small size: training pairs from the batched solver
    (bastr_ensemble_subgrid), training by the library's kernels, the held-out filtered DNS against
    the plain and the closure coarse runs, device-timed."""
    import argparse

    from bastr_b200.closure_study import run
    args = argparse.Namespace(fine=64, ratio=4, reynolds=40.0, dt=1e-3, target=1.5, k0=3.0, train_seeds=[0, 1],
                              test_seed=7, spinup=20, every=10, snapshots=2, steps=20, iters=60, lr=2e-3,
                              net_seed=0, batch=10, closure_every=1, group=1)
    res = run(args)
    assert res["pairs"] == 4 and res["training_data"].startswith("batched solver")
    assert res["loss_last"] < res["loss_first"]
    assert res["apriori_held_out"]["mse_closure"] < res["apriori_held_out"]["mse_no_closure"]
    assert res["fine_gpu_ms"] > 0 and res["coarse_closure_gpu_ms"] > 0
    assert len(res["E_dns"]) == len(res["E_closure"]) > 0
