"""CPU checks of the closure oracle (test infrastructure): its hand-written back-propagation
agrees with central finite differences of its own loss, BF16 rounding is round-to-nearest-even,
and the input taps follow the kernels' periodic 3x3x3 ordering."""
import numpy as np

from oracle import closure_oracle as co


def test_bf16_round_to_nearest_even():
    x = np.array([1.0, 1.00390625, 1.005859375, -2.5, 3.0e-3], dtype=np.float32)
    r = co.bf16_round(x)
    assert r[0] == 1.0 and r[1] == 1.0            # 1 + 2^-8 is a tie: even mantissa (1.0)
    assert r[2] == np.float32(1.0078125)          # above the tie: rounds up
    assert r[3] == -2.5
    assert abs(r[4] - 3.0e-3) / 3.0e-3 < 2 ** -8


def test_taps_order():
    u = np.zeros((3, 4, 5, 6))
    u[1, 0, 0, 1] = 7.0                            # channel 1 at (z=0, y=0, x=1)
    x = co.taps(u)
    # point (z=0, y=0, x=0): its neighbour dx = +1 is tap 1*27 + 1*9 + 1*3 + 2 = 41
    assert x[0, 41] == 7.0 and np.count_nonzero(x[0]) == 1
    # periodic: point (z=0, y=0, x=2) sees it at dx = -1 (tap 1*27 + 13 - 1 = 39)
    assert x[2, 39] == 7.0


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    u = rng.standard_normal((3, 4, 5, 6))
    tau = 0.3 * rng.standard_normal((3, 4, 5, 6))
    w = co.init_weights(1)
    w[co.OFF_B1:co.OFF_W2] = rng.uniform(-0.1, 0.1, co.C)   # non-zero biases exercise those paths
    w[co.OFF_B4:co.NP] = rng.uniform(-0.1, 0.1, 3)
    loss, g = co.loss_grad(u, tau, w, act_bf16=False)
    assert loss > 0
    idx = [0, 7, 80, co.OFF_B1 + 3, co.OFF_W2 + 5, co.OFF_B2 + 1, co.OFF_W3 + 100, co.OFF_B3 + 31,
           co.OFF_W4 + 40, co.OFF_B4 + 2]
    fd = co.fd_gradient(u, tau, w, idx)
    assert np.allclose(g[idx], fd, rtol=1e-5, atol=1e-9)


def test_adam_moves_against_gradient():
    w = np.ones(5, np.float32)
    g = np.array([1, -1, 0, 2, -3], np.float32)
    w1, m, v = co.adam(w, np.zeros(5, np.float32), np.zeros(5, np.float32), g, 1, 1e-2)
    assert np.all(np.sign(w - w1) == np.sign(g))


def test_bf16_layer_inputs_change_little():
    """Rounding every layer's input to BF16 moves the output by about the BF16 resolution."""
    rng = np.random.default_rng(5)
    u = rng.standard_normal((3, 4, 5, 6))
    w = co.init_weights(2)
    a, b = co.forward(u, w, act_bf16=True), co.forward(u, w, act_bf16=False)
    rel = np.linalg.norm(a - b) / np.linalg.norm(b)
    assert 1e-5 < rel < 2 ** -6
