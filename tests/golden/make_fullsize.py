"""Generates the full-size parity fixtures ``tests/golden/fullsize_*.npz`` from the CPU oracle.

The step throughput is quoted on 2048^2 (band forcing, projection) and 256^3 (linear forcing).
Running the FP64 oracle for 100 steps there takes minutes (2048^2) to about an hour (256^3) on
the host cores, too long for a GPU test, so this script runs it once and freezes what the GPU
test compares against:

- the per-step record of every step (Esspe, Edspe, k2Edspe, kMEdspe, the 8 velocity-gradient
  statistics, forcing factor and E);
- both shell spectra (Es, Ed, every shell 0..allkmax) of every step (3D) or of steps
  1-5, 10, 20, ..., 100 (2D, 683 shells each);
- the state after step 1 and after the last step, reduced to: the normalised spectrum
  (fft/N) on the box |kx|, |ky|[, |kz|] <= KB, the velocity at NS seeded random points (an
  unbiased sample of the relative L2 error of the whole field), and the sum of u_c^2 over all
  points per component;
- the sum and sum of squares of the seeded initial field, so a test can tell that it rebuilt
  the same field.

The oracle is oracle/bastr_oracle.py (the FP64 restatement of solution.F90 / tool.F90 /
fftwlink.F90 with complex-to-complex transforms).

    python tests/golden/make_fullsize.py [2d2048] [3d256]
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from bastr_b200.initfield import seeded_field  # noqa: E402
from oracle.bastr_oracle import Oracle, Params  # noqa: E402

# the step-throughput workloads (the same parameters as bench.py)
CASES = {
    "2d2048": dict(params=dict(ia=2048, ja=2048, ka=0, reynolds=5000.0, deltat=1e-4, forcemethod=2, forcek=5,
                               target_energy=0.075, lprojectd=True, kmax=1 << 30),
                   k0=4.0, nsteps=100, box=16, shell_steps=[1, 2, 3, 4, 5] + list(range(10, 101, 10))),
    "3d256": dict(params=dict(ia=256, ja=256, ka=256, reynolds=5000.0, deltat=5e-4, forcemethod=1, forcek=5,
                              target_energy=1.5, lprojectd=False, kmax=85),
                  k0=3.0, nsteps=100, box=5, shell_steps=list(range(1, 101))),
}
NS = 2048          # sampled points per state
SAMPLE_SEED = 20251204


def sample_index(npts):
    return np.sort(np.random.default_rng(SAMPLE_SEED).choice(npts, NS, replace=False))


def box_modes(u, box):
    """Normalised spectrum fft(u)/N of each component on |k_i| <= box, axes in array order."""
    out = []
    for c in u:
        s = np.fft.fftn(c) / c.size
        idx = np.r_[0:box + 1, -box:0]
        sel = s
        for ax in range(c.ndim):
            sel = np.take(sel, idx, axis=ax)
        out.append(sel)
    return np.stack(out)


def reduce_state(u, box):
    u = [np.asarray(c, np.float64) for c in u]
    ix = sample_index(u[0].size)
    return dict(box=box_modes(u, box), samples=np.stack([c.ravel()[ix] for c in u]),
                sumsq=np.array([float(np.sum(c * c)) for c in u]))


def record_row(r):
    fo = r.forcing if r.forcing is not None else ()
    return [r.Esspe, r.Edspe, r.k2Edspe, r.kMEdspe, *r.velgrad,
            fo[0] if len(fo) > 0 else np.nan, fo[1] if len(fo) > 1 else np.nan]


def generate(name):
    cfg = CASES[name]
    p = Params(**cfg["params"])
    u0 = seeded_field(p.ia, p.ja, p.ka, k0=cfg["k0"], seed=0)
    o = Oracle(p, u0)
    o.initial_dealias()
    recs, shells = [], []
    st1 = None
    t0 = time.perf_counter()
    for i in range(1, cfg["nsteps"] + 1):
        r, sp = o.step_once(True)
        recs.append(record_row(r))
        if i in cfg["shell_steps"]:
            shells.append(np.stack([sp["Es"], sp["Ed"]]))
        if i == 1:
            st1 = reduce_state(o.u, cfg["box"])
        print(f"{name}: step {i} ({time.perf_counter() - t0:.0f} s)", flush=True)
    stn = reduce_state(o.u, cfg["box"])
    out = dict(records=np.array(recs), shells=np.array(shells), shell_steps=np.array(cfg["shell_steps"]),
               nsteps=cfg["nsteps"], box=cfg["box"], sample_seed=SAMPLE_SEED, nsamples=NS,
               u0_sum=np.array([float(np.sum(c)) for c in u0]),
               u0_sumsq=np.array([float(np.sum(c * c)) for c in u0]))
    for tag, st in (("step1", st1), ("last", stn)):
        for k, v in st.items():
            out[f"{tag}_{k}"] = v
    return out


if __name__ == "__main__":
    names = [a for a in sys.argv[1:] if a in CASES] or list(CASES)
    for name in names:
        path = os.path.join(HERE, f"fullsize_{name}.npz")
        np.savez_compressed(path, **generate(name))
        print("wrote", path, os.path.getsize(path), "bytes", flush=True)
