"""Generates the golden fixtures of tests/golden/ from the CPU oracle.

The reference (Fortran + FFTW-MPI + HDF5) has no tests, fixtures or golden outputs and cannot
be built here, so the fixtures come from the oracle itself (oracle/bastr_oracle.py, pinned by
the analytic tests in tests/test_oracle_kat.py).  They freeze the oracle's outputs on small
seeded cases so that GPU runs and later oracle edits are checked against the same numbers.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from bastr_b200.initfield import seeded_field  # noqa: E402
from oracle.bastr_oracle import Oracle, Params  # noqa: E402

CASES = {
    "2d_band_proj_32": (dict(ia=32, ja=32, ka=0, reynolds=5000.0, deltat=1e-4, forcemethod=2, forcek=3,
                             target_energy=0.075, lprojectd=True, kmax=10), 4.0, 7, 5),
    "2d_linear_cn_32": (dict(ia=32, ja=32, ka=0, reynolds=1000.0, deltat=2e-4, forcemethod=1,
                             target_energy=1.0, timemethod=2, kmax=10), 3.0, 8, 4),
    "3d_linear_16": (dict(ia=16, ja=16, ka=16, reynolds=5000.0, deltat=5e-4, forcemethod=1,
                          target_energy=1.5, kmax=5), 3.0, 9, 3),
    "3d_band5_16": (dict(ia=16, ja=16, ka=16, reynolds=2000.0, deltat=5e-4, forcemethod=5, forcek=2,
                         target_energy=2.0, kmax=5), 3.0, 10, 3),
}


def generate(name):
    kw, k0, seed, nsteps = CASES[name]
    p = Params(**kw)
    u0 = seeded_field(p.ia, p.ja, p.ka, k0=k0, seed=seed)
    o = Oracle(p, u0, workers=1)
    o.initial_dealias()
    recs, shells = [], []
    for _ in range(nsteps):
        r, sp = o.step_once(True)
        fo = r.forcing if r.forcing is not None else ()
        recs.append([r.Esspe, r.Edspe, r.k2Edspe, r.kMEdspe, *r.velgrad,
                     fo[0] if len(fo) > 0 else np.nan, fo[1] if len(fo) > 1 else np.nan])
        shells.append(np.stack([sp["Es"], sp["Ed"]]))
    return dict(u0=np.stack(u0), u=np.stack(o.u), records=np.array(recs), shells=np.array(shells),
                nsteps=nsteps)


if __name__ == "__main__":
    for name in CASES:
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **generate(name))
        print("wrote", name)
