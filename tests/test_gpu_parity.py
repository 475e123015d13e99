"""GPU parity: the CUDA library (through its C ABI) against the FP64 CPU oracle.

Tolerances are the ones the reference's FP64 path is held to: relative L2 <= 1e-12 after one
step and <= 1e-9 after many steps, for the velocity, the per-step energy/dissipation
sequences, the velocity-gradient statistics, the forcing factors and every spectrum shell.
The FP32 form is held to <= 1e-5 relative L2 against the same oracle.
"""
import pytest

from tests.parity_util import compare, field, make_params, run_gpu, run_oracle

pytestmark = pytest.mark.gpu

CASES_2D = [
    # name, params, k0
    ("decay", dict(reynolds=5000.0, deltat=1e-4), 4.0),
    ("band_proj", dict(reynolds=5000.0, deltat=1e-4, forcemethod=2, forcek=5, target_energy=0.075,
                       lprojectd=True), 4.0),
    ("linear", dict(reynolds=1000.0, deltat=2e-4, forcemethod=1, target_energy=1.0), 3.0),
    ("band5_proj", dict(reynolds=2000.0, deltat=1e-4, forcemethod=5, forcek=4, target_energy=1.5,
                        lprojectd=True), 4.0),
    ("cn", dict(reynolds=5000.0, deltat=1e-4, timemethod=2), 4.0),
    ("inviscid", dict(reynolds=0.0, deltat=1e-4), 2.0),
]


def _check(err, tol):
    bad = {k: v for k, v in err.items() if not (v <= tol)}
    assert not bad, f"above {tol}: {bad}"


@pytest.mark.parametrize("name,kw,k0", CASES_2D, ids=[c[0] for c in CASES_2D])
def test_2d_fp64_one_step(gpu_lib, name, kw, k0):
    p = make_params(64, 64, 0, kmax=100, **kw)
    u = field(64, 64, 0, k0=k0, seed=1)
    vg = name != "inviscid"
    err = compare(run_oracle(p, u, 1, vg), run_gpu(p, u, 1, "fp64", vg), vg)
    _check(err, 1e-12)


@pytest.mark.parametrize("name,kw,k0", CASES_2D[:4], ids=[c[0] for c in CASES_2D[:4]])
def test_2d_fp64_many_steps(gpu_lib, name, kw, k0):
    p = make_params(128, 128, 0, kmax=100, **kw)
    u = field(128, 128, 0, k0=k0, seed=2)
    err = compare(run_oracle(p, u, 30), run_gpu(p, u, 30, "fp64"))
    _check(err, 1e-9)


@pytest.mark.parametrize("dims,kw", [
    ((128, 128, 0), dict(reynolds=5000.0, deltat=1e-4, timemethod=2, forcemethod=2, forcek=5, target_energy=0.075,
                         lprojectd=True)),
    ((32, 32, 32), dict(reynolds=2000.0, deltat=5e-4, timemethod=2, forcemethod=1, target_energy=1.5)),
], ids=["2d_band_proj", "3d_linear"])
def test_cn_many_steps(gpu_lib, dims, kw):
    """Crank-Nicolson (six sweeps per step, solution.F90:205-231, 272-301) over many steps, with
    forcing: the sweeps' fixed-point iterates stay at FP64 parity."""
    ia, ja, ka = dims
    p = make_params(ia, ja, ka, kmax=100, **kw)
    u = field(ia, ja, ka, k0=4.0 if ka == 0 else 3.0, seed=6)
    n = 30 if ka == 0 else 20
    err = compare(run_oracle(p, u, n), run_gpu(p, u, n, "fp64"))
    _check(err, 1e-9)


def test_2d_nonsquare(gpu_lib):
    p = make_params(64, 128, 0, reynolds=3000.0, deltat=1e-4, forcemethod=2, forcek=3, target_energy=0.1)
    u = field(64, 128, 0, k0=3.0, seed=3)
    err = compare(run_oracle(p, u, 5), run_gpu(p, u, 5, "fp64"))
    _check(err, 1e-10)


@pytest.mark.parametrize("dims,kw", [
    ((32, 128, 0), dict(reynolds=2000.0, deltat=1e-4, timemethod=2, forcemethod=1, target_energy=1.0)),
    ((128, 256, 0), dict(reynolds=5000.0, deltat=1e-4, forcemethod=5, forcek=4, target_energy=1.5, lprojectd=True)),
], ids=["32x128_cn_linear", "128x256_band5_proj"])
def test_2d_nonsquare_forms(gpu_lib, dims, kw):
    """More non-square 2D grids: Crank-Nicolson with linear forcing and RK3 with projected band
    forcing; FP64 over 10 steps at 1e-9 and the FP32 form at 1e-5."""
    ia, ja, ka = dims
    p = make_params(ia, ja, ka, **kw)
    u = field(ia, ja, ka, k0=3.0, seed=8)
    ref = run_oracle(p, u, 10)
    _check(compare(ref, run_gpu(p, u, 10, "fp64")), 1e-9)
    err = compare(ref, run_gpu(p, u, 10, "fp32"))
    _check({k: v for k, v in err.items() if k != "eta_min"}, 1e-5)
    assert err["eta_min"] <= 1e-4


def test_2d_512_hundred_steps(gpu_lib):
    """The 512^2 decaying configuration (Re 5000, dt 1e-4, spectra to kmax 170), 100 steps."""
    p = make_params(512, 512, 0, reynolds=5000.0, deltat=1e-4, kmax=170)
    u = field(512, 512, 0, k0=4.0, seed=0)
    err = compare(run_oracle(p, u, 100), run_gpu(p, u, 100, "fp64"))
    _check(err, 1e-9)


CASES_3D = [
    ("linear", dict(reynolds=5000.0, deltat=5e-4, forcemethod=1, target_energy=1.5), 3.0),
    ("decay_proj", dict(reynolds=2000.0, deltat=5e-4, lprojectd=True), 3.0),
    ("band", dict(reynolds=2000.0, deltat=5e-4, forcemethod=2, forcek=3, target_energy=0.2), 3.0),
    ("band5", dict(reynolds=2000.0, deltat=5e-4, forcemethod=5, forcek=3, target_energy=2.0), 3.0),
    ("cn", dict(reynolds=2000.0, deltat=5e-4, timemethod=2), 3.0),
]


@pytest.mark.parametrize("name,kw,k0", CASES_3D, ids=[c[0] for c in CASES_3D])
def test_3d_fp64_one_step(gpu_lib, name, kw, k0):
    p = make_params(32, 32, 32, **kw)
    u = field(32, 32, 32, k0=k0, seed=4)
    err = compare(run_oracle(p, u, 1), run_gpu(p, u, 1, "fp64"))
    _check(err, 1e-12)


@pytest.mark.parametrize("name,kw,k0", CASES_3D[:2], ids=[c[0] for c in CASES_3D[:2]])
def test_3d_fp64_many_steps(gpu_lib, name, kw, k0):
    p = make_params(32, 32, 32, **kw)
    u = field(32, 32, 32, k0=k0, seed=5)
    err = compare(run_oracle(p, u, 20), run_gpu(p, u, 20, "fp64"))
    _check(err, 1e-9)


@pytest.mark.parametrize("dims,kw", [
    ((32, 64, 32), dict(reynolds=2000.0, deltat=5e-4, forcemethod=2, forcek=3, target_energy=0.2, lprojectd=True)),
    ((32, 32, 64), dict(reynolds=2000.0, deltat=5e-4, forcemethod=1, target_energy=1.5)),
    ((16, 32, 64), dict(reynolds=1000.0, deltat=5e-4, timemethod=2, forcemethod=5, forcek=2, target_energy=2.0)),
], ids=["32x64x32_band_proj", "32x32x64_linear", "16x32x64_cn_band5"])
def test_3d_noncubic(gpu_lib, dims, kw):
    """Grids whose three extents differ (ja, ka >= 2*floor(ia/3)): the truncated layout keeps
    2K-1 modes along y and z whatever ja and ka are, and the passes transform ja and ka points.
    FP64 over 10 steps at 1e-9, the FP32 form at 1e-5."""
    ia, ja, ka = dims
    p = make_params(ia, ja, ka, **kw)
    u = field(ia, ja, ka, k0=3.0, seed=7)
    ref = run_oracle(p, u, 10)
    _check(compare(ref, run_gpu(p, u, 10, "fp64")), 1e-9)
    err = compare(ref, run_gpu(p, u, 10, "fp32"))
    _check({k: v for k, v in err.items() if k != "eta_min"}, 1e-5)
    assert err["eta_min"] <= 1e-4


@pytest.mark.parametrize("dims,kw", [
    ((16, 16, 0), dict(reynolds=1000.0, deltat=2e-4, forcemethod=2, forcek=2, target_energy=0.1, lprojectd=True)),
    ((32, 32, 0), dict(reynolds=1000.0, deltat=2e-4, timemethod=2, forcemethod=1, target_energy=1.0)),
    ((16, 16, 16), dict(reynolds=1000.0, deltat=5e-4, forcemethod=5, forcek=2, target_energy=2.0)),
    ((16, 16, 32), dict(reynolds=1000.0, deltat=5e-4, timemethod=2, lprojectd=True)),
], ids=["16x16_band_proj", "32x32_cn_linear", "16x16x16_band5", "16x16x32_cn_proj"])
def test_smallest_grids(gpu_lib, dims, kw):
    """The smallest extents the library builds (16 points: K = 5, transforms of 16 points), where
    every line holds few modes and most lanes of a line group are idle; FP64 over 10 steps at
    1e-9 and the FP32 form at 1e-5."""
    ia, ja, ka = dims
    p = make_params(ia, ja, ka, **kw)
    u = field(ia, ja, ka, k0=2.0, seed=9)
    ref = run_oracle(p, u, 10)
    _check(compare(ref, run_gpu(p, u, 10, "fp64")), 1e-9)
    err = compare(ref, run_gpu(p, u, 10, "fp32"))
    _check({k: v for k, v in err.items() if k != "eta_min"}, 1e-5)
    assert err["eta_min"] <= 1e-4


def test_kernel_shared_memory_limit_never_shrinks(gpu_lib):
    """Grids with the same ja share the 3D y-forward kernel instance, whose shared memory follows
    KY: a 32^3 handle, then a 16x32x64 one (smaller KY, smaller request), then 32^3 again must
    all run (the kernel's shared-memory limit is set per kernel and must not drop under the
    first, larger request)."""
    import numpy as np
    from bastr_b200 import BastrGPU
    for dims in ((32, 32, 32), (16, 32, 64), (32, 32, 32)):
        with BastrGPU(*dims, precision="fp64", velgrad_every=1) as s:
            s.set_state(field(*dims, k0=3.0, seed=1))
            recs = s.step(2)
            assert np.isfinite(recs[-1].Esspe)


def test_interleaved_handles_match_solo_runs(gpu_lib):
    """Handles of different shapes and forms alive at once, stepped in turn on their own streams
    (they share kernel instances, launch caches and twiddle tables): every handle's records and
    state are bitwise those of the same handle run alone."""
    import numpy as np
    from bastr_b200 import BastrGPU
    cases = [((32, 32, 32), "fp64"), ((16, 32, 64), "fp64"), ((64, 128, 0), "fp32"), ((32, 32, 32), "fp32")]
    kw = dict(reynolds=2000.0, deltat=5e-4, forcemethod=2, forcek=2, target_energy=0.3, velgrad_every=1)

    def values(recs, state):
        return np.concatenate([np.array([[r.Esspe, r.Edspe, r.factor, *r.velgrad] for r in recs]).ravel(),
                               np.stack(state).ravel()])

    solo = []
    for dims, prec in cases:
        with BastrGPU(*dims, precision=prec, **kw) as s:
            s.set_state(field(*dims, k0=3.0, seed=2))
            recs = s.step(3) + s.step(3)
            solo.append(values(recs, s.get_state()))
    handles = [BastrGPU(*dims, precision=prec, **kw) for dims, prec in cases]
    try:
        for (dims, _), s in zip(cases, handles):
            s.set_state(field(*dims, k0=3.0, seed=2))
        recs = [[] for _ in cases]
        for _ in range(2):
            for i, s in enumerate(handles):
                recs[i] += s.step(3)
        for i, s in enumerate(handles):
            assert np.array_equal(values(recs[i], s.get_state()), solo[i]), cases[i]
    finally:
        for s in handles:
            s.close()


@pytest.mark.parametrize("dims,every", [((64, 64, 0), 3), ((32, 32, 32), 2)], ids=["2d_every3", "3d_every2"])
def test_velgrad_every_n_steps(gpu_lib, dims, every):
    """Statistics every n steps (velgrad_every = n; the reference computes them every step): the
    steps with nstep % n == 0 carry the oracle's eight statistics, the others NaN, and the
    dynamics (state, spectra, forcing) are those of the every-step run."""
    import numpy as np
    from bastr_b200 import BastrGPU
    from tests.parity_util import rel_l2
    ia, ja, ka = dims
    kw = dict(reynolds=2000.0, deltat=2e-4 if ka == 0 else 5e-4, forcemethod=2, forcek=3, target_energy=0.2)
    p = make_params(ia, ja, ka, **kw)
    u = field(ia, ja, ka, k0=3.0, seed=10)
    rrec, rsh, ru = run_oracle(p, u, 7)
    with BastrGPU(ia, ja, ka, precision="fp64", velgrad_every=every, **kw) as s:
        s.set_state(u)
        recs, shells = s.step(7, shells=True)
        ug = s.get_state()
    assert rel_l2(np.stack(ug), np.stack(ru)) <= 1e-10
    for name in ("Esspe", "Edspe", "factor"):
        got = [getattr(r, name) for r in recs]
        want = [getattr(r, name) if name != "factor" else r.forcing[0] for r in rrec]
        assert rel_l2(got, want) <= 1e-10, name
    for i, (g, r) in enumerate(zip(recs, rrec)):
        if i % every == 0:
            assert rel_l2(g.velgrad, r.velgrad) <= 1e-10, i
        else:
            assert all(np.isnan(v) for v in g.velgrad), i


def test_3d_64_ten_steps(gpu_lib):
    p = make_params(64, 64, 64, reynolds=5000.0, deltat=5e-4, forcemethod=1, target_energy=1.5, kmax=21)
    u = field(64, 64, 64, k0=3.0, seed=0)
    err = compare(run_oracle(p, u, 10), run_gpu(p, u, 10, "fp64"))
    _check(err, 1e-10)


@pytest.mark.parametrize("dims", [(128, 128, 0), (32, 32, 32)], ids=["2d", "3d"])
def test_fp32_form(gpu_lib, dims):
    ia, ja, ka = dims
    kw = dict(reynolds=5000.0, deltat=1e-4 if ka == 0 else 5e-4, forcemethod=1 if ka else 2, forcek=5,
              target_energy=1.5 if ka else 0.075, lprojectd=ka == 0)
    p = make_params(ia, ja, ka, **kw)
    u = field(ia, ja, ka, k0=4.0 if ka == 0 else 3.0, seed=6)
    err = compare(run_oracle(p, u, 30), run_gpu(p, u, 30, "fp32"))
    # eta_min is a pointwise extremum of sqrt(nu/|div|): FP32 round-off of div enters unsmoothed
    _check({k: v for k, v in err.items() if k != "eta_min"}, 1e-5)
    assert err["eta_min"] <= 1e-4


@pytest.mark.parametrize("dims", [(64, 64, 0), (16, 16, 16)], ids=["2d", "3d"])
def test_linear_forcing_state_between_steps(gpu_lib, dims):
    """Linear forcing scales the whole field after each step; the state read between batches of
    steps, and the steps that follow that read, must match the oracle at both points."""
    import numpy as np
    from bastr_b200 import BastrGPU
    from oracle.bastr_oracle import Oracle
    from tests.parity_util import rel_l2
    ia, ja, ka = dims
    p = make_params(ia, ja, ka, reynolds=1000.0, deltat=2e-4, forcemethod=1, target_energy=1.0)
    u = field(ia, ja, ka, k0=3.0, seed=4)
    o = Oracle(p, u)
    o.initial_dealias()
    with BastrGPU(ia, ja, ka, reynolds=p.reynolds, deltat=p.deltat, forcemethod=1, target_energy=1.0,
                  precision="fp64") as s:
        s.set_state(u)
        for n in (3, 2):
            recs, _ = s.step(n, shells=True)
            ref = [o.step_once(True)[0] for _ in range(n)]
            assert rel_l2([r.Esspe for r in recs], [r.Esspe for r in ref]) <= 1e-12
            assert rel_l2([r.factor for r in recs], [r.forcing[0] for r in ref]) <= 1e-12
            assert rel_l2(np.stack(s.get_state()), np.stack(o.u)) <= 1e-12


@pytest.mark.parametrize("dims", [(64, 64, 0), (32, 32, 32)], ids=["2d", "3d"])
def test_transfer_spectra_match_oracle(gpu_lib, dims):
    """bastr_transfer (Bastrpp transfer2d/transfer3d) against the oracle's restatement on the
    state after a few steps: every shell 1..allkmax of T, T1, T2 within 1e-12 relative L2."""
    import numpy as np
    from bastr_b200 import BastrGPU
    from oracle.bastr_oracle import transfer
    from tests.parity_util import rel_l2
    ia, ja, ka = dims
    p = make_params(ia, ja, ka, reynolds=2000.0, deltat=1e-3, forcemethod=1, target_energy=1.0)
    u = field(ia, ja, ka, k0=3.0, seed=5)
    with BastrGPU(ia, ja, ka, reynolds=p.reynolds, deltat=p.deltat, forcemethod=1, target_energy=1.0) as s:
        s.set_state(u)
        s.step(3)
        uf = s.get_state()
        got = s.transfer()
    ref = transfer(p, uf)
    for g, r in zip(got, ref):
        assert rel_l2(g[1:], r[1:]) <= 1e-12, (g[1:6], r[1:6])


@pytest.mark.parametrize("dims,method", [((64, 64, 0), 3), ((64, 64, 0), 4), ((16, 16, 16), 3), ((16, 16, 16), 4)],
                         ids=["2d_m3", "2d_m4", "3d_m3", "3d_m4"])
def test_random_phase_forcing_matches_oracle(gpu_lib, dims, method):
    """Forcing methods 3 and 4 (random phases from the shared Philox stream): velocity, spectra,
    factor, E, energy and Fen of 1 and of 10 steps."""
    ia, ja, ka = dims
    target = 1.0 if method == 3 else 1e-3
    p = make_params(ia, ja, ka, reynolds=1000.0, deltat=1e-3, forcemethod=method, forcek=3,
                    target_energy=target, kmax=100)
    u = field(ia, ja, ka, k0=3.0, seed=6)
    for n, tol in ((1, 1e-12), (10, 1e-9)):
        err = compare(run_oracle(p, u, n), run_gpu(p, u, n, "fp64"))
        _check(err, tol)


@pytest.mark.parametrize("dims,kw", [
    ((64, 64, 0), dict(forcemethod=2, lprojectd=True)), ((64, 64, 0), dict(forcemethod=0)),
    ((64, 64, 0), dict(forcemethod=1, timemethod=2)), ((32, 32, 32), dict(forcemethod=1)),
    ((32, 32, 32), dict(forcemethod=3)), ((32, 32, 32), dict(forcemethod=0))],
    ids=["2d_band", "2d_none", "2d_linear_cn", "3d_linear", "3d_random", "3d_none"])
def test_launch_count_matches_profiled_launches(gpu_lib, dims, kw):
    """The launches per step the library reports (the bench's gpu_launches) are the kernels a
    step actually launches, counted by the per-launch profiler."""
    from bastr_b200 import BastrGPU
    ia, ja, ka = dims
    with BastrGPU(ia, ja, ka, target_energy=1.0, **kw) as s:
        s.set_state(field(ia, ja, ka, k0=3.0, seed=1))
        stats = s.profile(3)
        assert sum(k["launches"] for k in stats) == 3 * s.info()["launches_per_step"]
