"""Closure training data on the device (bastr_subgrid / bastr_ensemble_subgrid) and the device-timed
ensemble run (bastr_ensemble_run).

- bastr_subgrid against a NumPy restatement on the CPU: the box filter of width r of the state u
  read back from the handle, and tau = filter(u.grad u) - ub.grad ub with spectral derivatives
  (numpy.fft) on the fine and the coarse grid; FP32 outputs of FP64 arithmetic: 1e-6;
- an ensemble's realization gives bitwise the data of the same run on its own handle;
- bastr_ensemble_run over k batches leaves every realization bitwise where k calls of
  bastr_ensemble_step leave it.
"""
import numpy as np
import pytest

from tests.parity_util import field, rel_l2

pytestmark = pytest.mark.gpu


def _k(n):
    return np.fft.fftfreq(n, 1.0 / n)


def advective(u):
    """u_j d_j u_i with spectral derivatives on a periodic grid (2D or 3D, C order, x last)."""
    d = len(u)
    shape = u[0].shape
    ks = [_k(shape[-1 - a]).reshape([-1 if b == d - 1 - a else 1 for b in range(d)]) for a in range(d)]
    uh = [np.fft.fftn(c) for c in u]
    return [sum(u[j] * np.fft.ifftn(1j * ks[j] * uh[i]).real for j in range(d)) for i in range(d)]


def box(f, r):
    if f.ndim == 2:
        ny, nx = f.shape
        return f.reshape(ny // r, r, nx // r, r).mean(axis=(1, 3))
    nz, ny, nx = f.shape
    return f.reshape(nz // r, r, ny // r, r, nx // r, r).mean(axis=(1, 3, 5))


def reference(u, r):
    ub = [box(c, r) for c in u]
    fadv = [box(c, r) for c in advective(u)]
    cadv = advective(ub)
    return np.stack(ub), np.stack([a - b for a, b in zip(fadv, cadv)])


CASES = {"2d": (dict(ia=128, ja=128, ka=0, reynolds=500.0, deltat=1e-3, forcemethod=2, forcek=4,
                     target_energy=0.1, lprojectd=True), 4),
         "3d": (dict(ia=64, ja=64, ka=64, reynolds=200.0, deltat=1e-3, forcemethod=1, target_energy=1.5), 4)}


@pytest.mark.parametrize("name", sorted(CASES))
def test_subgrid_matches_numpy(gpu_lib, name):
    from bastr_b200 import BastrGPU
    kw, r = CASES[name]
    with BastrGPU(precision="fp64", velgrad_every=0, **kw) as s:
        s.set_state(field(kw["ia"], kw["ja"], kw["ka"], k0=4.0 if kw["ka"] == 0 else 3.0, seed=2))
        s.step(5)
        ub, tau = s.subgrid(r)
        u = s.get_state()
    rub, rtau = reference(u, r)
    assert rel_l2(ub.cpu().numpy(), rub) <= 1e-6
    assert rel_l2(tau.cpu().numpy(), rtau) <= 1e-6
    assert np.abs(rtau).max() > 1e-3      # a non-trivial subgrid term


def test_ensemble_subgrid_and_run_match_single_handles(gpu_lib):
    from bastr_b200 import BastrEnsemble, BastrGPU
    cfgs = [dict(CASES["2d"][0], seed=3, precision="fp32"), dict(CASES["3d"][0], seed=4, precision="fp32"),
            dict(CASES["2d"][0], seed=5, precision="fp32", forcek=3)]
    fields = [field(c["ia"], c["ja"], c["ka"], k0=4.0 if c["ka"] == 0 else 3.0, seed=c["seed"]) for c in cfgs]
    with BastrEnsemble(cfgs) as ens:
        for i, u in enumerate(fields):
            ens.set_state(i, u)
        ms = ens.run(20, 10)
        assert ms > 0
        data = [ens.subgrid(i, 4) for i in range(len(cfgs))]
        states = [ens.get_state(i) for i in range(len(cfgs))]
    with BastrEnsemble(cfgs) as ens2:
        for i, u in enumerate(fields):
            ens2.set_state(i, u)
        ens2.step(10)
        ens2.step(10)
        states2 = [ens2.get_state(i) for i in range(len(cfgs))]
    for a, b in zip(states, states2):
        assert all(np.array_equal(x, y) for x, y in zip(a, b))
    for c, u, (ub, tau), st in zip(cfgs, fields, data, states):
        kw = {k: v for k, v in c.items() if k != "seed"}
        with BastrGPU(velgrad_every=1, **kw) as s:
            s.set_state(u)
            s.step(20)
            ub1, tau1 = s.subgrid(4)
            assert all(np.array_equal(x, y) for x, y in zip(s.get_state(), st))
        assert np.array_equal(ub.cpu().numpy(), ub1.cpu().numpy())
        assert np.array_equal(tau.cpu().numpy(), tau1.cpu().numpy())
