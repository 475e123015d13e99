"""CPU oracle for the Bastr pseudo-spectral Burgers time step (test infrastructure only).

This module is the checker, not the product.  Only ``tests/``, ``__graft_entry__.smoke()``
and the CPU-baseline legs of ``bench.py`` may import it.  The product path (the CUDA
library under ``bastr_b200/csrc``) never calls into it.

It is a line-by-line FP64 restatement of the reference's Fortran hot path, with the same
complex-to-complex transforms, normalisation and quirks:

* ``fft``/``ifft``           -- fftwlink.F90:324-368 (forward e^{-ikx} scaled by 1/N, backward raw)
* ``generate_wave``          -- tool.F90:17-96
* ``kint``                   -- tool.F90:126-147 (method 2: nint(k/dk))
* ``dealiasing``             -- tool.F90:149-217 (zero where |k| >= floor(ia/3), all axes use ia)
* ``projection``             -- tool.F90:219-270
* ``compute_ut``             -- solution.F90:816-928
* ``rk3`` / ``cn``           -- solution.F90:172-301
* ``forcing``                -- solution.F90:303-814 (methods 0-5; the random phases of methods
  3/4 come from Philox-4x32-10 here and in the library, from gfortran's random_number in the
  reference: equal in distribution, not in value)
* ``spectra_compute``        -- solution.F90:930-1108
* ``velgrad_calculate``      -- solution.F90:1110-1286
* ``quantity_prepare``/``miucal`` -- solution.F90:1288-1329
* ``readinput`` derivations  -- readwrite.F90:69-83 (ndims, allkmax)
* ``mainloop``               -- solution.F90:20-170
* ``listwrite`` format       -- utility.F90:87-164 ``(1X,I20,n(1X,E20.13E2))``
* ``transfer``               -- Bastrpp.F90:174-305, 418-599 (transfer2d / transfer3d)
* ``hitgen``                 -- Bastrpp.F90:601-1005 (hitgen2d / hitgen3d / hitgen2dbis; the uniform
  numbers come from Philox-4x32-10 here and in the library, from random_number in the reference)

Layout: fields are NumPy arrays in C order ``(ny, nx)`` for 2D and ``(nz, ny, nx)`` for 3D,
i.e. the same bytes as the reference's Fortran ``u(1:im,1:jm[,1:km])`` with x fastest.

Parity status: unpinned.  The reference ships no tests, fixtures or golden outputs, and it
cannot be built here (no Fortran compiler, MPI, FFTW or HDF5).  The restatement is pinned only
by analytic known-answer tests (single-mode transforms and derivatives, Parseval, linear
viscous decay, the 1-D Burgers Cole-Hopf solution embedded in 2D/3D) in ``tests/``.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np

try:  # scipy's pocketfft runs multi-threaded; numpy's is the fallback
    import scipy.fft as _sfft

    def _fftn(a, workers):
        return _sfft.fftn(a, workers=workers)

    def _ifftn(a, workers):
        return _sfft.ifftn(a, workers=workers)
except ImportError:  # pragma: no cover
    def _fftn(a, workers):
        return np.fft.fftn(a)

    def _ifftn(a, workers):
        return np.fft.ifftn(a)


# ---------------------------------------------------------------------------------------
# parameters (commvar.F90:16-66, readwrite.F90:19-112, solution.F90:1288-1329)
# ---------------------------------------------------------------------------------------
@dataclass
class Params:
    """The ``datin/input.dat`` values the hot path reads (readwrite.F90:35-44)."""
    ia: int
    ja: int
    ka: int = 0
    ref_tem: float = 273.15
    reynolds: float = 5000.0
    maxstep: int = 10
    deltat: float = 1e-4
    lwsequ: bool = False
    feqwsequ: int = 1000000
    lwspectra: bool = True
    feqwspe: int = 50
    kmax: int = 1 << 30
    timemethod: int = 1
    forcemethod: int = 0
    forcek: int = 5
    target_energy: float = 0.075
    lprojectd: bool = False

    @property
    def ndims(self) -> int:
        """readwrite.F90:69-80."""
        if self.ka == 0:
            if self.ja == 0:
                raise ValueError("1D case is not implemented yet!")
            return 2
        return 3

    @property
    def allkmax(self) -> int:
        """readwrite.F90:75-83: min(int(ia/3), kmax)."""
        return min(self.ia // 3, self.kmax)

    @property
    def nu(self) -> float:
        """solution.F90:1306-1310 with miucal (solution.F90:1315-1329) at T=1."""
        if self.reynolds == 0.0:
            return 0.0
        return miucal(1.0, self.ref_tem) / self.reynolds

    @property
    def shape(self):
        return (self.ja, self.ia) if self.ndims == 2 else (self.ka, self.ja, self.ia)

    @property
    def npts(self) -> int:
        return int(np.prod(self.shape))


def miucal(temper: float, ref_tem: float) -> float:
    """Sutherland law, solution.F90:1315-1329 (equals 1 at temper=1)."""
    tempconst = 110.4 / ref_tem
    tempconst1 = 1.0 + tempconst
    return temper * math.sqrt(temper) * tempconst1 / (temper + tempconst)


# ---------------------------------------------------------------------------------------
# spectral tools (tool.F90)
# ---------------------------------------------------------------------------------------
def wavenumbers_1d(n: int) -> np.ndarray:
    """tool.F90:31-37: index i (1-based) <= n/2+1 -> i-1, else i-n-1 (Nyquist is +n/2)."""
    i = np.arange(n)
    return np.where(i <= n // 2, i, i - n).astype(np.float64)


def generate_wave(p: Params):
    """tool.F90:17-96.  Returns k1, k2[, k3] broadcast to the field shape."""
    kx = wavenumbers_1d(p.ia)
    ky = wavenumbers_1d(p.ja)
    if p.ndims == 2:
        k1 = np.broadcast_to(kx[None, :], p.shape).copy()
        k2 = np.broadcast_to(ky[:, None], p.shape).copy()
        return k1, k2
    kz = wavenumbers_1d(p.ka)
    k1 = np.broadcast_to(kx[None, None, :], p.shape).copy()
    k2 = np.broadcast_to(ky[None, :, None], p.shape).copy()
    k3 = np.broadcast_to(kz[:, None, None], p.shape).copy()
    return k1, k2, k3


def kint(k, dk=1.0):
    """tool.F90:126-147, method 2: Fortran NINT (half away from zero; k >= 0 here)."""
    return np.floor(np.asarray(k) / dk + 0.5).astype(np.int64)


def dealias_mask(p: Params, kk: np.ndarray, factor: int = 3) -> np.ndarray:
    """tool.F90:185-193 / 206-214: True where the mode is KEPT (|k| < floor(ia/factor))."""
    cutoff = math.floor(float(p.ia) / float(factor))
    return ~(kk >= cutoff)


# ---------------------------------------------------------------------------------------
# the solver state, a restatement of the reference's module globals
# ---------------------------------------------------------------------------------------
@dataclass
class StepRecord:
    nstep: int
    time: float
    Esspe: float
    Edspe: float
    k2Edspe: float
    kMEdspe: float
    velgrad: tuple            # umumtheta2, umumijji, u2theta, dissp, eta_min, Tay, ReTay, Kol
    forcing: tuple | None     # (factor[, E]) written after the RK step, or None
    spect: tuple | None       # (kn, Es, Ed) shells 1..allkmax when written, else None


class Oracle:
    """Restatement of mainloop2D/3D and everything it calls, in FP64 with c2c transforms."""

    def __init__(self, p: Params, u, workers: int | None = None):
        if p.timemethod not in (1, 2):
            raise ValueError("Undefined time method")  # readwrite.F90:98-104
        self.p = p
        self.workers = workers if workers is not None else (os.cpu_count() or 1)
        self.ks = generate_wave(p)
        self.kk2 = sum(k * k for k in self.ks)
        self.kk = np.sqrt(self.kk2)
        self.nu = p.nu
        self.u = [np.array(c, dtype=np.float64, copy=True).reshape(p.shape) for c in u]
        if len(self.u) != p.ndims:
            raise ValueError("need one velocity component per dimension")
        # quantity_prepare (solution.F90:1288-1313)
        self.nstep = 0
        self.time = 0.0
        self.nxtwsequ = min(p.feqwsequ, p.maxstep)
        self.nxtwspe = 0
        self.filenumb = 1
        self.N = float(p.npts)
        self._mask = dealias_mask(p, self.kk)
        self.dumps = []

    # -- fftwlink.F90:324-368 ------------------------------------------------------------
    def fft(self, a):
        return _fftn(np.asarray(a, dtype=np.complex128), self.workers) / (1.0 * self.N)

    def ifft(self, a):
        return _ifftn(np.asarray(a, dtype=np.complex128), self.workers) * self.N

    # -- tool.F90 -------------------------------------------------------------------------
    def dealiasing(self, f):
        return np.where(self._mask, f, 0.0)

    def projection(self, fs):
        kk = self.kk
        big = kk > 0.5
        safe = np.where(big, kk, 1.0)
        ud = sum(f * k / safe for f, k in zip(fs, self.ks))
        return [np.where(big, ud * k / safe, 0.0) for k in self.ks]

    # -- solution.F90:816-928 -------------------------------------------------------------
    def compute_ut(self, uspe):
        """Returns (u_t list, physical uspe list); both complex like the reference."""
        p, ks, nu = self.p, self.ks, self.nu
        I = 1j
        d = p.ndims
        grads = [[self.ifft(I * uspe[i] * ks[j]) for j in range(d)] for i in range(d)]
        lap = [self.ifft(-uspe[i] * self.kk2) for i in range(d)]
        uphys = [self.ifft(uspe[i]) for i in range(d)]
        if d == 2:
            # solution.F90:841-846 uses dreal() of every factor
            ut = []
            for i in range(2):
                t = (-uphys[0].real * grads[i][0].real
                     - uphys[1].real * grads[i][1].real
                     + nu * lap[i].real)
                ut.append(t.astype(np.complex128))
        else:
            # solution.F90:903-908 multiplies the COMPLEX physical u by dreal(derivatives)
            ut = []
            for i in range(3):
                t = (-uphys[0] * grads[i][0].real - uphys[1] * grads[i][1].real
                     - uphys[2] * grads[i][2].real + nu * lap[i].real)
                ut.append(t)
        ut = [self.dealiasing(self.fft(t)) for t in ut]
        if p.lprojectd:
            ut = self.projection(ut)
        ut = [self.ifft(t) for t in ut]
        return ut, uphys

    # -- solution.F90:172-203, 233-270 ----------------------------------------------------
    def rk3(self):
        dt = self.p.deltat
        uspe = [self.fft(c) for c in self.u]
        kA, _ = self.compute_ut(uspe)
        uspe = [self.fft((c + dt * a.real / 2.0).astype(np.complex128)) for c, a in zip(self.u, kA)]
        kB, _ = self.compute_ut(uspe)
        uspe = [self.fft((c - dt * a.real + 2.0 * dt * b.real).astype(np.complex128))
                for c, a, b in zip(self.u, kA, kB)]
        kC, _ = self.compute_ut(uspe)
        self.u = [c + dt * (a.real + 4.0 * b.real + cc.real) / 6.0
                  for c, a, b, cc in zip(self.u, kA, kB, kC)]

    # -- solution.F90:205-231, 272-301 ----------------------------------------------------
    def cn(self):
        dt = self.p.deltat
        uold = [c.copy() for c in self.u]
        uspe = [self.fft(c) for c in self.u]
        for step in range(1, 7):
            kA, _ = self.compute_ut(uspe)
            self.u = [o + dt * a.real for o, a in zip(uold, kA)]
            if step == 6:
                break
            uspe = [self.fft(0.5 * (c + o)) for c, o in zip(self.u, uold)]

    # -- solution.F90:303-814 -------------------------------------------------------------
    def forcing(self):
        p = self.p
        m = p.forcemethod
        N = self.N
        if m == 0:
            return None
        if m == 1:
            energy = float(np.sum(sum(c ** 2 for c in self.u) / 2.0)) / N
            factor = math.sqrt(p.target_energy / energy)
            self.u = [factor * c for c in self.u]
            return (factor,)
        if m in (2, 5):
            dk = 0.5
            uspe = [self.fft(c) for c in self.u]
            kk = self.kk
            band = ((kk - dk) < p.forcek) & ((kk + dk) > p.forcek)
            if m == 5 and p.ndims == 2 and p.lprojectd:
                safe = np.where(band, kk, 1.0)
                ud = uspe[0] * self.ks[0] / safe + uspe[1] * self.ks[1] / safe
                force = [np.where(band, ud * k / safe, 0.0) for k in self.ks]
            else:
                force = [np.where(band, s, 0.0) for s in uspe]
            # the 3D method-5 path calls ifft2d on force1/2; both wrap backward_plan (fftwlink.F90:350-368)
            force = [self.ifft(f) for f in force]
            E = float(np.sum(sum(f.real ** 2 for f in force))) / N
            if m == 2:
                factor = math.sqrt(p.target_energy / E) - 1.0
            else:
                energy = float(np.sum(sum(c ** 2 for c in self.u))) / N
                if p.target_energy > energy:
                    factor = math.sqrt((p.target_energy - energy) / E + 1.0) - 1.0
                else:
                    factor = 0.0
            self.u = [c + factor * f.real for c, f in zip(self.u, force)]
            return (factor, E)
        if m in (3, 4):
            # solution.F90:379-482 (2D), 631-753 (3D): unit dilatational modes k/|k| (sin phi +
            # i cos phi) on the band; E = mean(f.u), energy = mean(|u|^2), Fen = mean(|f|^2)
            dk = 0.5
            kk = self.kk
            band = ((kk - dk) < p.forcek) & ((kk + dk) > p.forcek)
            phi = band_phases(p, self.nstep - 1, band)
            safe = np.where(band, kk, 1.0)
            e = np.sin(phi) + 1j * np.cos(phi)
            force = [self.ifft(np.where(band, k / safe * e, 0.0)) for k in self.ks]
            E = float(np.sum(sum(f.real * c for f, c in zip(force, self.u)))) / N
            energy = float(np.sum(sum(c ** 2 for c in self.u))) / N
            Fen = float(np.sum(sum(f.real ** 2 for f in force))) / N
            if m == 3:
                factor = (math.sqrt(max((p.target_energy - energy) * Fen + E * E, 0.0)) - E) / Fen
            else:
                factor = p.target_energy
            self.u = [c + factor * f.real for c, f in zip(self.u, force)]
            return (factor, E, energy, Fen)
        raise NotImplementedError(f"forcemethod {m}")

    # -- solution.F90:930-1108 ------------------------------------------------------------
    def spectra_compute(self, uspe):
        p = self.p
        kk = self.kk
        big = kk > 0.5
        safe = np.where(big, kk, 1.0)
        if p.ndims == 2:
            k1, k2 = self.ks
            us = np.where(big, uspe[0] * k2 / safe - uspe[1] * k1 / safe, 0.0)
            ud = np.where(big, uspe[0] * k1 / safe + uspe[1] * k2 / safe, 0.0)
            es_mode = (us * np.conj(us)).real / 2
        else:
            ud = np.where(big, sum(s * k / safe for s, k in zip(uspe, self.ks)), 0.0)
            es_mode = 0.0
            for s, k in zip(uspe, self.ks):
                usi = np.where(big, s - ud * k / safe, 0.0)
                es_mode = es_mode + (usi * np.conj(usi)).real / 2
        ed_mode = (ud * np.conj(ud)).real / 2
        kMEd = float(np.sum(np.where(big, ed_mode / safe, 0.0)))
        sh = kint(kk, 1.0).ravel()
        am = p.allkmax
        sel = sh <= am
        Ecount = np.bincount(sh[sel], minlength=am + 1)[: am + 1].astype(np.int64)
        Es = np.bincount(sh[sel], weights=np.ravel(es_mode)[sel], minlength=am + 1)[: am + 1]
        Ed = np.bincount(sh[sel], weights=np.ravel(ed_mode)[sel], minlength=am + 1)[: am + 1]
        kn = np.bincount(sh[sel], weights=kk.ravel()[sel], minlength=am + 1)[: am + 1]
        kn = kn.copy()
        for i in range(1, am + 1):  # solution.F90:991-996: shells 1..allkmax are normalised
            kn[i] = kn[i] / Ecount[i] if Ecount[i] else float("nan")
        return dict(Es=Es, Ed=Ed, kn=kn, Ecount=Ecount,
                    Edspe=float(np.sum(ed_mode)), Esspe=float(np.sum(es_mode)),
                    k2Edspe=float(np.sum(ed_mode * kk * kk)), kMEdspe=kMEd)

    # -- solution.F90:1110-1286 -----------------------------------------------------------
    def velgrad_calculate(self, uspe):
        p, nu = self.p, self.nu
        d = p.ndims
        I = 1j
        ks = self.ks
        kk2 = self.kk2
        g = [[self.ifft(I * uspe[i] * ks[j]).real for j in range(d)] for i in range(d)]
        lap = [self.ifft(-uspe[i] * kk2).real for i in range(d)]
        th = self.ifft(-I * sum(uspe[i] * ks[i] * kk2 for i in range(d))).real
        u = self.u
        N = self.N
        div = sum(g[i][i] for i in range(d))
        uu = sum(c ** 2 for c in u)
        umumtheta2 = float(np.sum(div ** 2 * uu)) / N
        ijji = sum(g[i][i] ** 2 for i in range(d))
        for i in range(d):
            for j in range(i + 1, d):
                ijji = ijji + 2.0 * g[i][j] * g[j][i]
        umumijji = float(np.sum(ijji * uu)) / N
        u2theta = float(np.sum(div * uu)) / N
        dissp = sum(2.0 * u[i] * div * lap[i] for i in range(d)) + uu * th
        dissp = float(np.sum(dissp)) / N
        eps = nu * div ** 2
        for (i, j) in ([(0, 1)] if d == 2 else [(0, 1), (1, 2), (0, 2)]):
            eps = eps + nu * (g[i][j] - g[j][i]) ** 2
        epsilon = float(np.sum(eps)) / N
        # eta_min starts at the default-real literal 2*3.14 (solution.F90:1145, 1236)
        eta0 = float(np.float32(2) * np.float32(3.14))
        with np.errstate(divide="ignore", invalid="ignore"):
            eta_pts = np.sqrt(nu / np.abs(div))
        eta_min = min(eta0, float(np.nanmin(eta_pts))) if eta_pts.size else eta0
        urms = math.sqrt(float(np.sum(uu)) / N)
        dudx2 = float(np.sum(sum(g[i][i] ** 2 for i in range(d)))) / N
        ufluc = urms / math.sqrt(float(d))
        with np.errstate(divide="ignore", invalid="ignore"):
            tay = ufluc / math.sqrt(dudx2 / float(d)) if dudx2 > 0 else float("inf")
            retay = ufluc * tay / nu if nu != 0 else float("inf")
            kol = math.sqrt(math.sqrt(nu ** 3 / epsilon)) if epsilon > 0 else float("inf")
        return (umumtheta2, umumijji, u2theta, dissp, eta_min, tay, retay, kol)

    # -- solution.F90:36-170 --------------------------------------------------------------
    def initial_dealias(self):
        """solution.F90:41-52 / 106-122."""
        self.u = [self.ifft(self.dealiasing(self.fft(c))).real for c in self.u]

    def step_once(self, do_velgrad: bool = True) -> StepRecord:
        """One iteration of the `do while(nstep<=maxstep)` body."""
        p = self.p
        uspe = [self.fft(c) for c in self.u]
        sp = self.spectra_compute(uspe)
        spect = None
        if p.lwspectra and self.nstep == self.nxtwspe:
            spect = (sp["kn"][1:].copy(), sp["Es"][1:].copy(), sp["Ed"][1:].copy())
            self.nxtwspe = min(self.nxtwspe + p.feqwspe, p.maxstep)
        vg = self.velgrad_calculate(uspe) if do_velgrad else None
        rec_n, rec_t = self.nstep, self.time
        E = sp["Esspe"] + sp["Edspe"]
        if (p.lwsequ and self.nstep == self.nxtwsequ) or math.isnan(E):
            self.dumps.append((self.filenumb, self.nstep, self.time, [c.copy() for c in self.u]))
            self.filenumb += 1
            self.nxtwsequ = min(self.nxtwsequ + p.feqwsequ, p.maxstep)
        if math.isnan(E):
            raise FloatingPointError('"E" is a NaN')
        self.nstep += 1
        self.time += p.deltat
        if p.timemethod == 1:
            self.rk3()
        else:
            self.cn()
        fo = self.forcing()
        return StepRecord(rec_n, rec_t, sp["Esspe"], sp["Edspe"], sp["k2Edspe"], sp["kMEdspe"],
                          vg, fo, spect), sp

    def mainloop(self, nsteps: int | None = None, do_velgrad: bool = True):
        """Runs the loop; ``nsteps`` bounds the number of iterations (default: maxstep+1)."""
        self.initial_dealias()
        recs = []
        n = 0
        while self.nstep <= self.p.maxstep and (nsteps is None or n < nsteps):
            rec, _ = self.step_once(do_velgrad)
            recs.append(rec)
            n += 1
        return recs


# ---------------------------------------------------------------------------------------
# log format (utility.F90:87-164)
# ---------------------------------------------------------------------------------------
def fortran_e20_13(x: float) -> str:
    """Fortran ``E20.13E2``: ' 0.ddddddddddddd E+ee' right-justified in 20 columns."""
    if x != x:
        return "NaN".rjust(20)
    if math.isinf(x):
        return ("-Infinity" if x < 0 else "Infinity").rjust(20)
    if x == 0.0:
        s = "0.0000000000000E+00"
        return (("-" + s) if math.copysign(1.0, x) < 0 else s).rjust(20)
    m, e = f"{abs(x):.12e}".split("e")  # d.dddddddddddd (13 significant digits)
    e = int(e) + 1
    digits = m.replace(".", "")
    if abs(e) <= 99:
        es = f"E{'+' if e >= 0 else '-'}{abs(e):02d}"
    else:
        es = f"{'+' if e >= 0 else '-'}{abs(e):03d}"
    s = f"0.{digits}{es}"
    if x < 0:
        s = "-" + s
    return s.rjust(20)


def listwrite_line(nstep: int, time: float, *vals: float) -> str:
    """utility.F90:87-164: ``(1X,I20,n(1X,E20.13E2))`` with time/ref_tim (ref_tim = 1)."""
    return " " + f"{nstep:20d}" + "".join(" " + fortran_e20_13(v) for v in (time, *vals))


# ---------------------------------------------------------------------------------------
# post-processing: energy transfer spectra (Bastrpp)
# ---------------------------------------------------------------------------------------
def transfer(p: Params, u):
    """transfer2d / transfer3d, Bastrpp.F90:174-305 / 418-599, on the physical field u (list of
    d real arrays): complex-to-complex transforms with the reference's scaling (forward 1/N,
    backward unscaled), products in physical space kept complex as the reference keeps them,
    per-mode trans, trans1, trans2 summed over the full grid into shells kint(|k|) <= allkmax.
    Returns T, T1, T2 for shells 0..allkmax."""
    d = p.ndims
    n = p.npts
    ks = generate_wave(p)
    fwd = lambda a: np.fft.fftn(a) / n        # noqa: E731  fft2d/fft3d (fftwlink.F90:324-347)
    bwd = lambda a: np.fft.ifftn(a) * n       # noqa: E731  ifft2d/ifft3d (fftwlink.F90:349-368)
    uspe = [fwd(np.asarray(c, dtype=np.complex128)) for c in u]
    ux = [[bwd(1j * uspe[c] * ks[j]) for j in range(d)] for c in range(d)]
    uph = [bwd(uspe[c]) for c in range(d)]
    tA = [-sum(uph[j] * ux[c][j].real for j in range(d)) for c in range(d)]
    div = sum(ux[j][j] for j in range(d)).real
    tC = [uph[c] * div for c in range(d)]
    P = [[uph[c] * uph[j] for j in range(d)] for c in range(d)]
    tA = [fwd(a) for a in tA]
    us2 = [fwd(a) for a in uph]
    tC = [fwd(a) for a in tC]
    P = [[fwd(a) for a in row] for row in P]
    trans = sum(np.real(np.conj(us2[c]) * tA[c]) for c in range(d))
    trans1 = np.imag(sum(ks[j] * P[c][j] * np.conj(us2[c]) for c in range(d) for j in range(d)))
    trans2 = sum(np.real(np.conj(us2[c]) * tC[c]) for c in range(d))
    kk = np.sqrt(sum(k * k for k in ks))
    sh = kint(kk).ravel()
    am = p.allkmax
    sel = sh <= am
    out = [np.bincount(sh[sel], weights=t.ravel()[sel], minlength=am + 1) for t in (trans, trans1, trans2)]
    return tuple(out)


# ---------------------------------------------------------------------------------------
# random phases of forcing methods 3/4 (Philox-4x32-10, Salmon et al. SC 2011)
# ---------------------------------------------------------------------------------------
PHILOX_KEY = (0xB5A57F01, 0x7E5D0C2B)


def philox4x32_10(c, k0, k1):
    """Ten Philox rounds on the 4-word counter c (numpy uint32 arrays) with key (k0, k1)."""
    c = [np.asarray(x, dtype=np.uint64) & 0xFFFFFFFF for x in c]
    k0, k1 = np.uint64(k0), np.uint64(k1)
    m = np.uint64(0xFFFFFFFF)
    for _ in range(10):
        p0 = np.uint64(0xD2511F53) * c[0]
        p1 = np.uint64(0xCD9E8D57) * c[2]
        hi0, lo0, hi1, lo1 = p0 >> np.uint64(32), p0 & m, p1 >> np.uint64(32), p1 & m
        c = [(hi1 ^ c[1] ^ k0) & m, lo1, (hi0 ^ c[3] ^ k1) & m, lo0]
        k0 = (k0 + np.uint64(0x9E3779B9)) & m
        k1 = (k1 + np.uint64(0xBB67AE85)) & m
    return [x.astype(np.uint32) for x in c]


def band_phases(p: Params, ctr: int, band: np.ndarray) -> np.ndarray:
    """Phase of every grid mode for forcing call ctr (zero off the band): each mode's canonical
    half (kx > 0, or kx = 0 with (ky, kz) > 0) draws phi = 2 pi (u - 1/2) from Philox of
    (kx | (ky+1024) << 11, kz + 1024, ctr lo, ctr hi); the other half takes -phi(-k)."""
    ks = generate_wave(p)
    kx = ks[0].astype(np.int64)
    ky = ks[1].astype(np.int64)
    kz = ks[2].astype(np.int64) if p.ndims == 3 else np.zeros_like(kx)
    neg = (kx < 0) | ((kx == 0) & ((ky < 0) | ((ky == 0) & (kz < 0))))
    sgn = np.where(neg, -1.0, 1.0)
    ax, ay, az = np.where(neg, -kx, kx), np.where(neg, -ky, ky), np.where(neg, -kz, kz)
    c0 = (ax | ((ay + 1024) << 11)).astype(np.uint64)
    c1 = (az + 1024).astype(np.uint64)
    c2 = np.full_like(c0, ctr & 0xFFFFFFFF)
    c3 = np.full_like(c0, (ctr >> 32) & 0xFFFFFFFF)
    out = philox4x32_10([c0, c1, c2, c3], *PHILOX_KEY)
    u = (out[0].astype(np.float64) + 0.5) / 4294967296.0
    return np.where(band, sgn * (2.0 * np.pi * u - np.pi), 0.0)


# ---------------------------------------------------------------------------------------
# initial-field generators of Bastrpp (hitgen2d / hitgen2dbis / hitgen3d)
# ---------------------------------------------------------------------------------------
HITGEN_TAG = 0x48475431


def hitgen_uniform(p: Params, draw: int, seed: int) -> np.ndarray:
    """Uniform (0,1) field (53-bit) for draw `draw`: Philox-4x32-10 keyed by the 64-bit seed on the
    counter (point index lo, hi, draw, tag), point index x fastest.  Stands in for gfortran's
    random_number(random_angle) (Bastrpp.F90:637, 737, 849, 889)."""
    idx = np.arange(p.npts, dtype=np.uint64)
    c = [idx & np.uint64(0xFFFFFFFF), idx >> np.uint64(32), np.full_like(idx, draw), np.full_like(idx, HITGEN_TAG)]
    out = philox4x32_10(c, seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF)
    x = (out[0].astype(np.uint64) << np.uint64(32)) | out[1].astype(np.uint64)
    u = ((x >> np.uint64(11)).astype(np.float64) + 0.5) * (1.0 / 9007199254740992.0)
    return u.reshape(p.shape)


def hitgen_modes(p: Params, r: np.ndarray, bis: bool):
    """One draw of the generators (Bastrpp.F90:641-666 2D, 741-771 3D, 853-876 / 893-916 bis):
    theta = atan2 of FFT(r), u^_c = var2 k_c/|k| (sin theta + i cos theta); for bis also
    theta^ = i (kx u^_1 + ky u^_2).  Returns (u^ list, theta^ or None, random_angle)."""
    d = p.ndims
    n = p.npts
    ks = generate_wave(p)
    R = np.fft.fftn(r.astype(np.complex128)) / n
    kk = np.sqrt(sum(k * k for k in ks))
    zero = kk == 0
    kks = np.where(zero, 1.0, kk)
    fk = float(p.forcek)
    if bis:
        var1 = kks ** 4 * np.exp(-2.0 * (kks / fk) ** 2)
    else:
        var1 = np.where(kks >= fk, kks ** 4 * np.exp(-2.0 * (kks / fk) ** 2), fk ** 6 / kks ** 2 * np.exp(-2.0))
    var2 = np.sqrt(var1 / 2.0 / np.pi / kks) if d == 2 else np.sqrt(var1 / 4.0 / np.pi / kks ** 2)
    th = np.arctan2(R.imag, R.real)
    angle = np.where(zero, r, th)
    ph = np.sin(th) + 1j * np.cos(th)
    us = [np.where(zero, 0.0, var2 * ks[c] / kks * ph) for c in range(d)]
    thspe = (1j * (ks[0] * us[0] + ks[1] * us[1])) if bis else None
    return us, thspe, angle


def hitgen_alpha(QX, QY, QZ, QW):
    """The real root of QX + QY a + QZ a^2 + QW a^3 = 0 the reference takes (Bastrpp.F90:951-973)."""
    QP = QY / QW - (1.0 / 3.0) * (QZ / QW) ** 2
    QQ = 2.0 / 27.0 * (QZ / QW) ** 3 - (1.0 / 3.0) * (QZ * QY) / QW ** 2 + QX / QW
    QDELTA = (QQ / 2.0) ** 2 + (QP / 3.0) ** 3
    if QDELTA >= 0.0:
        t1 = -QQ / 2.0 + math.sqrt(QDELTA)
        t2 = -QQ / 2.0 - math.sqrt(QDELTA)
        return math.copysign(abs(t1) ** (1.0 / 3.0), t1) + math.copysign(abs(t2) ** (1.0 / 3.0), t2) - QZ / (3.0 * QW)
    return 2.0 * math.sqrt(-QP / 3.0) * math.cos((1.0 / 3.0) * math.acos(3.0 * QQ / (2.0 * QP) * math.sqrt(-3.0 / QP))) \
        - QZ / (3.0 * QW)


def hitgen(p: Params, variant: int, seed: int):
    """create_initial_field_2d / _3d (variant 0; Bastrpp.F90:601-808) and create_initial_field_2d_bis
    (variant 1; :810-1005) with p.forcek and p.target_energy.  Returns (u list, random_angle,
    stats dict: energy before scaling, factor, alpha, residual, QX..QW)."""
    n = p.npts
    bwd = lambda a: np.fft.ifftn(a) * n       # noqa: E731  ifft2d/ifft3d (fftwlink.F90:349-368)
    us, th, angle = hitgen_modes(p, hitgen_uniform(p, 0, seed), variant == 1)
    uA = [bwd(c).real for c in us]
    st = {"alpha": float("nan"), "residual": float("nan"), "QX": 0.0, "QY": 0.0, "QZ": 0.0, "QW": 0.0}
    if variant == 1:
        thA = bwd(th).real
        us, th, angle = hitgen_modes(p, hitgen_uniform(p, 1, seed), True)
        uB = [bwd(c).real for c in us]
        thB = bwd(th).real
        aa = uA[0] ** 2 + uA[1] ** 2
        bb = uB[0] ** 2 + uB[1] ** 2
        ab = uB[0] * uA[0] + uB[1] * uA[1]
        QX = float(np.sum(aa * thA)) / n
        QY = float(np.sum(2 * ab * thA + aa * thB)) / n
        QZ = float(np.sum(2 * ab * thB + bb * thA)) / n
        QW = float(np.sum(bb * thB)) / n
        a = hitgen_alpha(QX, QY, QZ, QW)
        st.update(alpha=a, residual=QX + a * QY + a * a * QZ + a ** 3 * QW, QX=QX, QY=QY, QZ=QZ, QW=QW)
        u = [uA[c] + a * uB[c] for c in range(2)]
    else:
        u = uA
    energy = float(sum(np.sum(c * c) for c in u)) / n
    factor = math.sqrt(p.target_energy / energy)
    st.update(energy=energy, factor=factor)
    return [c * factor for c in u], angle, st
