"""Runs a fixed set of solver cases (small grids and the two measured sizes) through one build
of the library and saves every result: ``python -m tests.checked_cases <library.so> <out.npz>``.

Used by tests/test_checked_build.py to run the same cases through the normal library and the
index-checking one (``-DBASTR_CHECKED``) in separate processes (a process loads one library).
Each case: seeded field, a few steps with the shell spectra and velocity-gradient statistics
every step, then the state, the standalone spectra and (up to 2^21 points) the transfer spectra.
"""
from __future__ import annotations

import sys

import numpy as np

# (name, ia, ja, ka, precision, solver keywords)
CASES = [
    ("2d16_rk3_band", 16, 16, 0, "fp64", dict(forcemethod=2, forcek=2, target_energy=0.075, lprojectd=True)),
    ("2d32x64_cn_linear", 32, 64, 0, "fp64", dict(timemethod=2, forcemethod=1, target_energy=1.0)),
    ("2d64_fp32_rand", 64, 64, 0, "fp32", dict(forcemethod=3, forcek=4, target_energy=0.5)),
    ("2d128_fp32_band5", 128, 128, 0, "fp32", dict(forcemethod=5, forcek=4, target_energy=1.5, lprojectd=True)),
    ("3d16_fp64_linear", 16, 16, 16, "fp64", dict(forcemethod=1, target_energy=1.5)),
    ("3d32x16x64_fp64_cn", 32, 32, 64, "fp64", dict(timemethod=2, forcemethod=4, forcek=3, target_energy=0.1)),
    ("3d32_fp32_band", 32, 32, 32, "fp32", dict(forcemethod=2, forcek=3, target_energy=0.5)),
    ("3d64_fp32_decay", 64, 64, 64, "fp32", dict()),
    # the measured sizes: several TMA boxes per line in 2D (K = 682), the TMA-staged 3D passes
    ("2d2048_fp32_band", 2048, 2048, 0, "fp32", dict(forcemethod=2, forcek=5, target_energy=0.075, lprojectd=True)),
    ("3d256_fp32_linear", 256, 256, 256, "fp32", dict(forcemethod=1, target_energy=1.5)),
]
NSTEPS = 3
BIG = 1 << 21   # grids with more points: no transfer spectra (their work grids take gigabytes)


def run(lib_path: str) -> dict:
    import bastr_b200
    bastr_b200.load_library(lib_path)
    from bastr_b200 import BastrGPU, seeded_field
    out = {}
    for name, ia, ja, ka, prec, kw in CASES:
        u = seeded_field(ia, ja, ka, k0=3.0 if ka else 4.0, seed=11)
        with BastrGPU(ia, ja, ka, reynolds=2000.0, deltat=2e-4, kmax=1 << 30, precision=prec,
                      velgrad_every=1, **kw) as s:
            s.set_state(u)
            recs, shells = s.step(NSTEPS, shells=True)
            state = np.stack(s.get_state())
            sp = s.spectra()
            tr = s.transfer() if ia * ja * max(ka, 1) <= BIG else (np.zeros(1),)
        out[f"{name}/records"] = np.array([[r.Esspe, r.Edspe, r.k2Edspe, r.kMEdspe, *r.velgrad, r.factor, r.E,
                                            r.energy, r.Fen] for r in recs])
        out[f"{name}/shells"] = shells
        out[f"{name}/state"] = state
        out[f"{name}/spectra"] = np.concatenate([np.ravel(np.asarray(x, dtype=np.float64)) for x in sp])
        out[f"{name}/transfer"] = np.concatenate([np.ravel(x) for x in tr])
    return out


if __name__ == "__main__":
    np.savez(sys.argv[2], **run(sys.argv[1]))
