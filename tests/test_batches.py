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
