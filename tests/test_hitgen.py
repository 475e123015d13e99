"""bastr_hitgen (Bastrpp's hitgen2d / hitgen2dbis / hitgen3d) through the C ABI against the
oracle's restatement on the same Philox stream: fields, random_angle and the scalars
(energy before scaling, factor, alpha).  FP64; the transforms differ only in rounding."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a, b = np.asarray(a, np.float64).ravel(), np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("dims,variant", [((64, 64, 0), 0), ((64, 64, 0), 1), ((64, 128, 0), 0), ((64, 128, 0), 1),
                                          ((32, 32, 32), 0), ((16, 32, 64), 0), ((2048, 2048, 0), 0)],
                         ids=["2d", "2d_bis", "2d_nonsquare", "2d_bis_nonsquare", "3d", "3d_nonsquare", "2d2048"])
def test_hitgen_matches_oracle(gpu_lib, dims, variant):
    from bastr_b200 import BastrGPU
    from oracle.bastr_oracle import Params, hitgen
    ia, ja, ka = dims
    seed = 0x1234_5678_9ABC
    p = Params(ia=ia, ja=ja, ka=ka, forcek=5, target_energy=0.075)
    want_u, want_angle, want = hitgen(p, variant, seed)
    with BastrGPU(ia, ja, ka, forcek=5, target_energy=0.075) as s:
        got_u, got_angle, got = s.hitgen(variant, seed)
    assert _rel(np.stack(got_u), np.stack(want_u)) <= 1e-12
    # phases compared on the circle: modes whose transform is real up to rounding may sit at +pi or
    # -pi; the phase of a mode with a small |FFT(r)| carries the transform's rounding over |FFT(r)|
    d = np.angle(np.exp(1j * (got_angle - want_angle)))
    assert np.max(np.abs(d)) <= 1e-8
    for k in ("energy", "factor"):
        assert abs(got[k] - want[k]) <= 1e-12 * abs(want[k])
    if variant == 1:
        assert abs(got["alpha"] - want["alpha"]) <= 1e-9 * abs(want["alpha"])
        for k in ("QX", "QY", "QZ", "QW"):
            assert abs(got[k] - want[k]) <= 1e-10 * max(abs(want[q]) for q in ("QX", "QY", "QZ", "QW"))
    else:
        assert np.isnan(got["alpha"])


def test_hitgen_field_starts_a_run(gpu_lib):
    """The generated field is a valid initial state: set_state, step, finite records."""
    from bastr_b200 import BastrGPU
    with BastrGPU(128, 128, 0, forcek=5, target_energy=0.075, forcemethod=2, lprojectd=True) as s:
        u, _, st = s.hitgen(0, 7)
        s.set_state(u)
        recs = s.step(5)
    assert all(np.isfinite(r.Esspe) for r in recs)
    assert abs(st["factor"] ** 2 * st["energy"] - 0.075) < 1e-15


def test_hitgen_rejects_bad_variants(gpu_lib):
    from bastr_b200 import BastrError, BastrGPU
    with BastrGPU(16, 16, 16) as s:
        with pytest.raises(BastrError, match="two-dimensional"):
            s.hitgen(1, 0)
        with pytest.raises(BastrError, match="variant"):
            s.hitgen(2, 0)
