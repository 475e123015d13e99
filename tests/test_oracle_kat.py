"""Known-answer tests that pin the CPU oracle (the reference ships no tests or fixtures, so the
restatement is pinned by analytic results):

* transforms: normalisation and sign of fft/ifft (fftwlink.F90:324-368) on single modes;
* derivatives and the right-hand side of a single mode (solution.F90:816-863);
* dealias mask and projection (tool.F90:175-270);
* Parseval: Es + Ed = mean(|u|^2)/2 (solution.F90:930-1016);
* linear viscous decay exp(-nu k^2 t) of a small-amplitude mode;
* the 1-D viscous Burgers equation embedded in 2D and 3D against the Cole-Hopf solution;
* the log format (1X,I20,n(1X,E20.13E2)) of listwrite (utility.F90:87-164).
"""
import math

import numpy as np
import pytest

from oracle.bastr_oracle import (Oracle, Params, dealias_mask, fortran_e20_13, generate_wave, kint,
                                 listwrite_line, miucal)


def grid(n):
    return 2 * np.pi * np.arange(n) / n


def test_miucal_is_one_at_unit_temperature():
    assert miucal(1.0, 273.15) == pytest.approx(1.0, abs=1e-15)
    assert Params(ia=16, ja=16, reynolds=5000.0).nu == pytest.approx(2e-4, rel=1e-15)
    assert Params(ia=16, ja=16, reynolds=0.0).nu == 0.0


def test_wavenumbers_and_nyquist_sign():
    k1, k2 = generate_wave(Params(ia=8, ja=8))
    assert list(k1[0]) == [0, 1, 2, 3, 4, -3, -2, -1]   # Nyquist index carries +ia/2
    assert list(k2[:, 0]) == [0, 1, 2, 3, 4, -3, -2, -1]


def test_kint_rounds_half_away_from_zero():
    assert list(kint(np.array([0.0, 0.49, 0.5, 1.5, 2.5, 2.49]))) == [0, 0, 1, 2, 3, 2]


def test_fft_normalisation_and_sign():
    p = Params(ia=16, ja=16)
    o = Oracle(p, [np.zeros(p.shape)] * 2)
    x = grid(16)[None, :].repeat(16, 0)
    f = o.fft(np.cos(3 * x) + 2 * np.sin(2 * x))
    assert f[0, 3] == pytest.approx(0.5) and f[0, 13] == pytest.approx(0.5)
    assert f[0, 2] == pytest.approx(-1j) and f[0, 14] == pytest.approx(1j)   # e^{-ikx} convention
    assert np.allclose(o.ifft(f).real, np.cos(3 * x) + 2 * np.sin(2 * x))


def test_dealias_mask_counts():
    p = Params(ia=12, ja=12)
    k1, k2 = generate_wave(p)
    kk = np.sqrt(k1 ** 2 + k2 ** 2)
    keep = dealias_mask(p, kk)
    # cutoff floor(12/3) = 4: kept modes are the integer points strictly inside radius 4
    expect = sum(1 for a in range(-5, 7) for b in range(-5, 7) if a * a + b * b < 16)
    assert keep.sum() == expect


def test_single_mode_rhs():
    """u = (sin x, 0): u_t = -u u_x + nu u_xx = -sin(2x)/2 - nu sin x."""
    n = 16
    p = Params(ia=n, ja=n, reynolds=100.0)
    x = grid(n)[None, :].repeat(n, 0)
    u = [np.sin(x), np.zeros_like(x)]
    for proj in (False, True):
        p.lprojectd = proj
        o = Oracle(p, u)
        ut, _ = o.compute_ut([o.fft(c) for c in o.u])
        assert np.allclose(ut[0].real, -0.5 * np.sin(2 * x) - p.nu * np.sin(x), atol=1e-14)
        assert np.allclose(ut[1].real, 0.0, atol=1e-14)


def test_projection_keeps_only_dilatational_part():
    n = 16
    p = Params(ia=n, ja=n, lprojectd=True)
    x = grid(n)[None, :].repeat(n, 0)
    y = x.T
    # solenoidal (sin y, 0) + dilatational (sin x, 0)
    o = Oracle(p, [np.sin(y) + np.sin(x), np.zeros((n, n))])
    s = o.projection([o.fft(c) for c in o.u])
    assert np.allclose(o.ifft(s[0]).real, np.sin(x), atol=1e-14)
    assert np.allclose(o.ifft(s[1]).real, 0.0, atol=1e-14)


def test_parseval_and_single_mode_spectra():
    n = 32
    p = Params(ia=n, ja=n, kmax=10)
    x = grid(n)[None, :].repeat(n, 0)
    y = x.T
    o = Oracle(p, [np.cos(3 * x), np.cos(3 * x)])   # (cos 3x, cos 3x): d-part in x, s-part in y
    sp = o.spectra_compute([o.fft(c) for c in o.u])
    assert sp["Ed"][3] == pytest.approx(0.25, abs=1e-14)
    assert sp["Es"][3] == pytest.approx(0.25, abs=1e-14)
    assert sp["Esspe"] + sp["Edspe"] == pytest.approx(0.5, abs=1e-14)
    rng = np.random.default_rng(0)
    o = Oracle(p, [rng.standard_normal((n, n)), rng.standard_normal((n, n))])
    o.initial_dealias()
    sp = o.spectra_compute([o.fft(c) for c in o.u])
    # the k = 0 mode carries no Es/Ed (|k| <= dk/2, solution.F90:957-972)
    mean_sq = np.mean(o.u[0]) ** 2 + np.mean(o.u[1]) ** 2
    assert sp["Esspe"] + sp["Edspe"] == pytest.approx(np.mean(o.u[0] ** 2 + o.u[1] ** 2) / 2 - mean_sq / 2,
                                                      rel=1e-13)
    # shell counts: Ecount(s) = #integer points with nint(|k|) = s
    for s in range(1, 11):
        cnt = sum(1 for a in range(-16, 16) for b in range(-16, 16)
                  if math.floor(math.sqrt(a * a + b * b) + 0.5) == s)
        assert sp["Ecount"][s] == cnt


def test_linear_viscous_decay():
    n, eps = 32, 1e-9
    p = Params(ia=n, ja=n, reynolds=50.0, deltat=1e-3)
    x = grid(n)[None, :].repeat(n, 0)
    y = x.T
    u = [eps * np.sin(3 * x) * np.cos(2 * y), eps * np.cos(3 * x) * np.sin(2 * y)]
    o = Oracle(p, u)
    o.initial_dealias()
    for _ in range(50):
        o.step_once(False)
    decay = math.exp(-p.nu * 13 * 50 * p.deltat)
    assert np.allclose(o.u[0], u[0] * decay, atol=eps * 1e-6)
    assert np.allclose(o.u[1], u[1] * decay, atol=eps * 1e-6)


def cole_hopf(x, t, nu, nterms=60):
    """Exact 1-D viscous Burgers solution for u0 = sin x (Cole 1951, Hopf 1950)."""
    from scipy.special import ive
    a = 1.0 / (2.0 * nu)
    num = np.zeros_like(x)
    den = np.full_like(x, ive(0, a))
    for m in range(1, nterms):
        w = ive(m, a) * math.exp(-nu * m * m * t)
        num += 4.0 * nu * m * w * np.sin(m * x)
        den += 2.0 * w * np.cos(m * x)
    return num / den


@pytest.mark.parametrize("proj", [False, True])
def test_cole_hopf_2d(proj):
    n = 64
    p = Params(ia=n, ja=n, reynolds=10.0, deltat=1e-3, lprojectd=proj)
    x = grid(n)[None, :].repeat(n, 0)
    o = Oracle(p, [np.sin(x), np.zeros((n, n))])
    o.initial_dealias()
    for _ in range(100):
        o.step_once(False)
    exact = cole_hopf(grid(n), 0.1, p.nu)
    assert np.max(np.abs(o.u[0] - exact[None, :])) < 1e-7
    assert np.max(np.abs(o.u[1])) < 1e-14


def test_cole_hopf_3d_cn():
    n = 32
    p = Params(ia=n, ja=n, ka=n, reynolds=10.0, deltat=5e-4, timemethod=2)
    x = np.broadcast_to(grid(n)[None, None, :], (n, n, n))
    o = Oracle(p, [np.sin(x), np.zeros((n, n, n)), np.zeros((n, n, n))])
    o.initial_dealias()
    for _ in range(40):
        o.step_once(False)
    exact = cole_hopf(grid(n), 40 * p.deltat, p.nu)
    # Crank-Nicolson fixed point: second order in time
    assert np.max(np.abs(o.u[0] - exact[None, None, :])) < 1e-6


def test_band_forcing_reaches_target():
    n = 32
    p = Params(ia=n, ja=n, forcemethod=2, forcek=3, target_energy=0.3, deltat=1e-4)
    rng = np.random.default_rng(1)
    o = Oracle(p, [rng.standard_normal((n, n)), rng.standard_normal((n, n))])
    o.initial_dealias()
    rec, _ = o.step_once(False)
    factor, E = rec.forcing
    # after forcing, mean(f^2) over the band equals target (band energy rescaled by (1+factor)^2)
    assert E * (1 + factor) ** 2 == pytest.approx(0.3, rel=1e-12)


def test_listwrite_format():
    assert fortran_e20_13(1.0) == " 0.1000000000000E+01"
    assert fortran_e20_13(-0.075) == "-0.7500000000000E-01"
    assert fortran_e20_13(0.0) == " 0.0000000000000E+00"
    assert fortran_e20_13(1.5e-120) == " 0.1500000000000-119"
    line = listwrite_line(3, 3e-4, 1.0, 2.0)
    assert line == "                    3  0.3000000000000E-03  0.1000000000000E+01  0.2000000000000E+01"


def test_philox_known_answers():
    """Philox-4x32-10 against the published known-answer vectors (Salmon et al. 2011)."""
    import numpy as np
    from oracle.bastr_oracle import philox4x32_10
    cases = [((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
             ((0xFFFFFFFF,) * 4, (0xFFFFFFFF, 0xFFFFFFFF), (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
             ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
              (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1))]
    for c, k, want in cases:
        out = philox4x32_10([np.array([x], np.uint64) for x in c], *k)
        assert tuple(int(o[0]) for o in out) == want


def test_random_phase_force_is_real_and_in_band():
    import numpy as np
    from oracle.bastr_oracle import Params, band_phases, generate_wave
    for p in (Params(ia=32, ja=32, ka=0, forcek=4), Params(ia=16, ja=16, ka=16, forcek=3)):
        ks = generate_wave(p)
        kk = np.sqrt(sum(k * k for k in ks))
        band = np.abs(kk - p.forcek) < 0.5
        phi = band_phases(p, 7, band)
        safe = np.where(band, kk, 1.0)
        e = np.sin(phi) + 1j * np.cos(phi)
        for k in ks:
            f = np.fft.ifftn(np.where(band, k / safe * e, 0.0))
            assert np.max(np.abs(f.imag)) < 1e-14 * max(1.0, np.max(np.abs(f.real)))
        assert np.all(phi[~band] == 0) and np.all(np.abs(phi[band]) <= np.pi)
        assert not np.array_equal(band_phases(p, 8, band), phi)   # a new draw every call


def _hitgen_amplitude(p, bis):
    """var2(|k|) of the generators (Bastrpp.F90:650-657 2D, 757-762 3D, 861-862 bis)."""
    ks = generate_wave(p)
    kk = np.sqrt(sum(k * k for k in ks))
    kks = np.where(kk == 0, 1.0, kk)
    fk = float(p.forcek)
    var1 = kks ** 4 * np.exp(-2 * (kks / fk) ** 2)
    if not bis:
        var1 = np.where(kks >= fk, var1, fk ** 6 / kks ** 2 * math.exp(-2.0))
    var2 = np.sqrt(var1 / (2 * np.pi * kks)) if p.ndims == 2 else np.sqrt(var1 / (4 * np.pi * kks ** 2))
    return ks, kk, np.where(kk == 0, 0.0, var2)


def _off_nyquist(p):
    """Modes with no index at the Nyquist position: there the generators' wavenumber (+n/2 on
    both partners) breaks the Hermitian pairing and the real part halves the mode."""
    axes = [p.ia, p.ja] + ([p.ka] if p.ndims == 3 else [])
    masks = [np.arange(n) != n // 2 for n in axes]
    m = masks[0][None, :] & masks[1][:, None] if p.ndims == 2 else \
        masks[0][None, None, :] & masks[1][None, :, None] & masks[2][:, None, None]
    return m


@pytest.mark.parametrize("dims", [(64, 64, 0), (32, 64, 0), (16, 16, 16)], ids=["2d", "2d_nonsquare", "3d"])
def test_hitgen_spectrum_is_the_generators_and_energy_is_target(dims):
    """The random phases do not touch the amplitudes: away from the Nyquist lines every mode of
    the generated field has |u^|^2 = factor^2 var2(|k|)^2, whatever the random numbers; the
    field is dilatational (u^ parallel to k) and mean |u|^2 = target_energy."""
    from oracle.bastr_oracle import hitgen
    p = Params(ia=dims[0], ja=dims[1], ka=dims[2], forcek=5, target_energy=0.075)
    u, angle, st = hitgen(p, 0, seed=11)
    n = p.npts
    assert abs(sum(np.mean(c * c) for c in u) - 0.075) < 1e-15
    us = [np.fft.fftn(c) / n for c in u]
    ks, kk, var2 = _hitgen_amplitude(p, False)
    m = _off_nyquist(p)
    e = sum(np.abs(c) ** 2 for c in us)
    want = (st["factor"] * var2) ** 2
    assert np.max(np.abs(e - want)[m]) <= 1e-12 * want.max()
    # curl-free: k_i u^_j - k_j u^_i = 0
    for i in range(p.ndims):
        for j in range(i + 1, p.ndims):
            assert np.max(np.abs(ks[i] * us[j] - ks[j] * us[i])[m]) <= 1e-12 * np.sqrt(want.max()) * kk.max()
    # random_angle is a phase in [-pi, pi] everywhere but k = 0, which keeps a uniform number
    assert np.all(np.abs(angle) <= np.pi)
    assert 0.0 < angle.flat[0] < 1.0


def test_hitgen_bis_cancels_u2_theta():
    """hitgen2dbis picks alpha so that <|u|^2 theta> = 0 for u = uA + alpha uB."""
    from oracle.bastr_oracle import hitgen
    p = Params(ia=64, ja=64, ka=0, forcek=5, target_energy=0.075)
    u, _, st = hitgen(p, 1, seed=3)
    n = p.npts
    ks = generate_wave(p)
    us = [np.fft.fftn(c) / n for c in u]
    theta = (np.fft.ifftn(1j * (ks[0] * us[0] + ks[1] * us[1])) * n).real
    w = (u[0] ** 2 + u[1] ** 2) * theta
    assert abs(np.mean(w)) <= 1e-12 * np.mean(np.abs(w))
    assert abs(st["residual"]) <= 1e-9 * max(abs(st[q]) for q in ("QX", "QY", "QZ", "QW")) * max(1.0, abs(st["alpha"])) ** 3
    assert abs(sum(np.mean(c * c) for c in u) - 0.075) < 1e-15


def test_hitgen_alpha_root_forms():
    """Both branches of the reference's cubic formula give a root."""
    from oracle.bastr_oracle import hitgen_alpha
    for q in [(1.0, 2.0, 3.0, 4.0), (-6.0, 11.0, -6.0, 1.0), (0.3, -2.0, 0.1, 1.5)]:
        a = hitgen_alpha(*q)
        assert abs(q[0] + q[1] * a + q[2] * a * a + q[3] * a ** 3) < 1e-9


def test_hitgen_uniform_stream():
    """53-bit uniforms in (0, 1), distinct per draw and seed, reproducible."""
    from oracle.bastr_oracle import hitgen_uniform
    p = Params(ia=64, ja=64, ka=0)
    a, b, c = hitgen_uniform(p, 0, 5), hitgen_uniform(p, 1, 5), hitgen_uniform(p, 0, 6)
    assert np.array_equal(a, hitgen_uniform(p, 0, 5))
    assert a.min() > 0.0 and a.max() < 1.0 and abs(a.mean() - 0.5) < 0.02
    assert not np.array_equal(a, b) and not np.array_equal(a, c)


def test_nan_energy_stops_before_the_step_advances():
    """solution.F90:69-84: a NaN Es+Ed dumps the field of that step and stops before nstep and
    time advance, so the dumped state is the one that produced the NaN."""
    import warnings

    from bastr_b200.initfield import seeded_field
    p = Params(ia=32, ja=32, ka=0, reynolds=0.0, deltat=0.03, forcemethod=2, forcek=3, target_energy=200.0,
               kmax=10)
    o = Oracle(p, [10.0 * c for c in seeded_field(32, 32, 0, k0=3.0, seed=5)], workers=1)
    o.initial_dealias()
    n_ok = 0
    with np.errstate(all="ignore"), warnings.catch_warnings():
        warnings.simplefilter("ignore")
        with pytest.raises(FloatingPointError):
            for _ in range(20):
                o.step_once(True)
                n_ok += 1
    assert o.nstep == n_ok and n_ok >= 2
    assert o.time == pytest.approx(n_ok * p.deltat)
    fnum, nstep, time, dumped = o.dumps[-1]
    assert nstep == o.nstep
    assert all(a is not b and np.array_equal(a, b, equal_nan=True) for a, b in zip(dumped, o.u))
