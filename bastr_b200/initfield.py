"""Seeded synthetic initial velocity fields for the Burgers solver.

The reference makes its initial fields with ``Bastrpp hitgen2d/3d`` (Bastrpp.F90:601-808),
seeded from the system clock, so they cannot be reproduced.  This generator is seeded
instead: NumPy ``default_rng(seed)`` (PCG64) draws a complex Gaussian amplitude for every
Fourier mode, shaped so that the shell spectrum follows ``E(k) ~ k^4 exp(-2 (k/k0)^2)``;
the real part of the inverse transform gives a real (Hermitian) field; the mean is removed
and every component is scaled to rms ``rms``.

Arrays are C order ``(ny, nx)`` / ``(nz, ny, nx)``, x fastest, i.e. the bytes of the
reference's Fortran ``u(1:ia,1:ja[,1:ka])``.
"""
from __future__ import annotations

import numpy as np


def _wavenumbers(n: int) -> np.ndarray:
    i = np.arange(n)
    return np.where(i <= n // 2, i, i - n).astype(np.float64)


def seeded_field(ia: int, ja: int, ka: int = 0, k0: float = 4.0, seed: int = 0,
                 rms: float = 1.0) -> list[np.ndarray]:
    """Returns ``[u1, u2]`` (2D, ``ka == 0``) or ``[u1, u2, u3]`` (3D) as float64 arrays."""
    rng = np.random.default_rng(seed)
    if ka == 0:
        shape = (ja, ia)
        kx = _wavenumbers(ia)[None, :]
        ky = _wavenumbers(ja)[:, None]
        kk = np.sqrt(kx * kx + ky * ky)
        ncomp = 2
    else:
        shape = (ka, ja, ia)
        kx = _wavenumbers(ia)[None, None, :]
        ky = _wavenumbers(ja)[None, :, None]
        kz = _wavenumbers(ka)[:, None, None]
        kk = np.sqrt(kx * kx + ky * ky + kz * kz)
        ncomp = 3
    shell = np.floor(kk + 0.5).astype(np.int64)
    count = np.bincount(shell.ravel())
    spec = kk ** 4 * np.exp(-2.0 * (kk / k0) ** 2)
    amp = np.sqrt(spec / count[shell])
    amp[kk == 0] = 0.0
    npts = float(np.prod(shape))
    out = []
    for _ in range(ncomp):
        z = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) * amp
        u = np.fft.ifftn(z).real * npts
        u -= u.mean()
        u *= rms / np.sqrt(np.mean(u * u))
        out.append(np.ascontiguousarray(u))
    return out
