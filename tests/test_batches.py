"""Batches of steps through the C ABI (the main loop, solution.F90:54-97, run n iterations per
call): bastr_step(h, n) splits n into device chunks of at most 256 steps (the records kept on the
device per batch); the records, the shells, the state and the counters must not depend on how the
steps are grouped into calls or chunks.  bastr_step(h, 0) runs nothing.
"""
import numpy as np
import pytest

from tests.parity_util import field

pytestmark = pytest.mark.gpu

KW = dict(reynolds=2000.0, deltat=2e-4, forcemethod=2, forcek=3, target_energy=0.1, velgrad_every=1)


def _values(recs):
    return np.array([[r.nstep, r.time, r.Esspe, r.Edspe, r.k2Edspe, r.kMEdspe, r.factor, r.E, *r.velgrad]
                     for r in recs])


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_grouping_of_steps_does_not_matter(gpu_lib, prec):
    from bastr_b200 import BastrGPU
    n = 600   # three device chunks: 256 + 256 + 88
    runs = {}
    for grouping in ("one_call", "calls_of_97", "single_steps"):
        with BastrGPU(32, 32, 0, precision=prec, **KW) as s:
            s.set_state(field(32, 32, 0, k0=3.0, seed=12))
            recs, shells = [], []
            sizes = {"one_call": [n], "calls_of_97": [97] * (n // 97) + [n % 97], "single_steps": [1] * n}[grouping]
            for k in sizes:
                r, sh = s.step(k, shells=True)
                recs += r
                shells.append(sh)
            runs[grouping] = (_values(recs), np.concatenate(shells), np.stack(s.get_state()), s.counters())
    ref = runs["one_call"]
    assert ref[0].shape[0] == n and ref[3][0] == n
    for name, got in runs.items():
        assert np.array_equal(got[0], ref[0]), name
        assert np.array_equal(got[1], ref[1]), name
        assert np.array_equal(got[2], ref[2]), name
        assert got[3] == ref[3], name


def test_zero_steps_runs_nothing(gpu_lib):
    from bastr_b200 import BastrGPU
    with BastrGPU(16, 16, 16, precision="fp64", **KW) as s:
        u = field(16, 16, 16, k0=3.0, seed=13)
        s.set_state(u)
        before = np.stack(s.get_state())
        recs, shells = s.step(0, shells=True)
        assert recs == [] and shells.shape[0] == 0
        assert s.counters() == (0, 0.0)
        assert np.array_equal(np.stack(s.get_state()), before)


@pytest.mark.parametrize("dims,method", [((64, 64, 0), 3), ((16, 16, 16), 4)], ids=["2d_m3", "3d_m4"])
def test_restart_continues_the_run(gpu_lib, dims, method):
    """A restart (the reference's read_continue_field, then the main loop from the saved nstep):
    a new handle given the state and counters after 5 steps continues the run, random-phase forcing
    included (its phases follow the step counter), within 1e-11 of the uninterrupted run; the
    state passes through its physical form once, hence not bitwise."""
    from bastr_b200 import BastrGPU
    from tests.parity_util import rel_l2
    kw = dict(KW, forcemethod=method, forcek=2, target_energy=0.2 if method == 3 else 0.05)
    u = field(*dims, k0=3.0, seed=14)
    with BastrGPU(*dims, precision="fp64", **kw) as a:
        a.set_state(u)
        a.step(5)
        mid, (n5, t5) = a.get_state(), a.counters()
        tail = a.step(5)
        end = np.stack(a.get_state())
    with BastrGPU(*dims, precision="fp64", **kw) as b:
        b.set_state(mid)
        b.set_counters(n5, t5)
        again = b.step(5)
        assert [r.nstep for r in again] == [r.nstep for r in tail]
        assert [r.time for r in again] == [r.time for r in tail]
        assert rel_l2(_values(again)[:, 2:], _values(tail)[:, 2:]) <= 1e-11
        assert rel_l2(np.stack(b.get_state()), end) <= 1e-11
