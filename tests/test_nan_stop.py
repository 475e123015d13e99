"""The NaN stop of the main loop (solution.F90:69-81): when Es+Ed of a step is NaN the reference
dumps that step's field and stops before `nstep = nstep + 1`.

bastr_step must stop at that step also inside a batch of many steps (no kernel of a later step
runs), with that step's record filled, the later records NaN, the counters of that step and the
state that produced the NaN; with out == NULL it must still report the stop.  The failures are
made on the host: a NaN written into the uploaded field, or an inviscid field with a time step far
beyond stability that overflows after a few steps.  No GPU fault is involved.
"""
import ctypes as C
import math
import warnings

import numpy as np
import pytest

from tests.parity_util import field

pytestmark = pytest.mark.gpu

BLOWUP = dict(ia=32, ja=32, ka=0, reynolds=0.0, deltat=0.03, forcemethod=2, forcek=3, target_energy=200.0,
              kmax=10)


def _solver(ia, ja, ka, **kw):
    from bastr_b200 import BastrGPU
    return BastrGPU(ia, ja, ka, precision=kw.pop("precision", "fp64"), velgrad_every=1, **kw)


def _step_raw(s, n, with_out=True):
    """bastr_step through the C ABI: (status, records or None, shells or None)."""
    from bastr_b200 import CStepOut
    out = (CStepOut * n)() if with_out else None
    sh = np.full((n, 2, s.allkmax + 1), 7.0) if with_out else None
    rc = s.lib.bastr_step(s.h, n, out, sh.ctypes.data_as(C.POINTER(C.c_double)) if sh is not None else None)
    recs = [s._rec(out[i]) for i in range(n)] if with_out else None
    return rc, recs, sh


def _blowup_field():
    return [10.0 * c for c in field(32, 32, 0, k0=3.0, seed=5)]


def _nan_step_one_by_one(kw, u, limit=50):
    """Steps one call at a time until the stop: (nan step, records before it, state at it)."""
    from bastr_b200 import BASTR_E_NAN
    with _solver(**kw) as s:
        s.set_state(u)
        recs = []
        for i in range(limit):
            rc, r, _ = _step_raw(s, 1)
            if rc == BASTR_E_NAN:
                n, t = s.counters()
                return i, recs, r[0], n, t, s.get_state()
            assert rc == 0
            recs.append(r[0])
    raise AssertionError("no NaN within the limit")


def test_nan_point_in_initial_field_stops_at_step_zero(gpu_lib):
    from bastr_b200 import BASTR_E_NAN
    for ia, ja, ka in ((64, 64, 0), (16, 16, 16)):
        u = field(ia, ja, ka, k0=4.0 if ka == 0 else 3.0, seed=3)
        u[0].flat[17] = math.nan
        with _solver(ia, ja, ka, reynolds=5000.0, deltat=1e-4, forcemethod=0) as s:
            s.set_state(u)
            rc, recs, sh = _step_raw(s, 12)
            assert rc == BASTR_E_NAN
            assert "NaN at nstep 0" in s._err()
            assert math.isnan(recs[0].Esspe + recs[0].Edspe)
            assert all(math.isnan(r.Esspe) and r.nstep == 0 for r in recs[1:])
            assert np.isnan(sh[1:]).all()
            assert s.counters() == (0, 0.0)
            assert np.isnan(np.stack(s.get_state())).any()
            # out == NULL: the stop is still reported, and a repeated call stops again at once
            rc, _, _ = _step_raw(s, 5, with_out=False)
            assert rc == BASTR_E_NAN
            assert s.counters() == (0, 0.0)


def test_batch_stops_at_the_step_that_one_step_calls_stop_at(gpu_lib):
    """A batch of 20 steps stops exactly where single-step calls stop, with identical records
    before it and the identical state; the oracle stops at the same step."""
    from bastr_b200 import BASTR_E_NAN
    from oracle.bastr_oracle import Oracle
    from tests.parity_util import make_params
    u = _blowup_field()
    k, recs1, nanrec, n1, t1, state1 = _nan_step_one_by_one(BLOWUP, u)
    assert n1 == k and k >= 2
    assert math.isnan(nanrec.Esspe + nanrec.Edspe)
    for with_out in (True, False):
        with _solver(**BLOWUP) as s:
            s.set_state(u)
            rc, recs, sh = _step_raw(s, 20, with_out=with_out)
            assert rc == BASTR_E_NAN
            assert f"NaN at nstep {k}" in s._err()
            assert s.counters() == (n1, t1)
            st = s.get_state()
            for a, b in zip(st, state1):
                assert np.array_equal(a, b, equal_nan=True)
            if with_out:
                for a, b in zip(recs[:k], recs1):
                    assert a.nstep == b.nstep
                    assert np.array_equal([a.Esspe, a.Edspe, a.factor, a.E, *a.velgrad],
                                          [b.Esspe, b.Edspe, b.factor, b.E, *b.velgrad], equal_nan=True)
                assert recs[k].nstep == k and math.isnan(recs[k].Esspe + recs[k].Edspe)
                assert all(math.isnan(r.Esspe) for r in recs[k + 1:])
                assert np.isnan(sh[k + 1:]).all() and np.isfinite(sh[:k]).all()
    # the oracle stops at the same step (it raises there, before nstep advances)
    o = Oracle(make_params(**BLOWUP), u, workers=1)
    o.initial_dealias()
    with np.errstate(all="ignore"), warnings.catch_warnings():
        warnings.simplefilter("ignore")
        with pytest.raises(FloatingPointError):
            for _ in range(20):
                o.step_once(True)
    assert o.nstep == k


def test_async_batch_records_report_the_stop(gpu_lib):
    from bastr_b200 import BASTR_E_NAN, BastrError
    u = _blowup_field()
    k = _nan_step_one_by_one(BLOWUP, u)[0]
    with _solver(**BLOWUP) as s:
        s.set_state(u)
        s.step_async(10)
        with pytest.raises(BastrError) as ei:
            s.records(10)
        assert ei.value.code == BASTR_E_NAN
        assert s.counters()[0] == k
