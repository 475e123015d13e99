"""Python host binding of the B200 Burgers time step (``libbastr_gpu.so``, C ABI in
``include/bastr_gpu.h``).

``BastrGPU`` mirrors what the reference's Fortran driver does around the hot path:
``readinput`` parameters in, ``set_state`` for ``read_initial_field`` plus the initial dealias
of ``mainloop`` (solution.F90:41-52), ``step`` for iterations of the main loop
(solution.F90:54-97), ``get_state`` for the fields ``writeflfed`` dumps, and ``mainloop`` for
the whole loop with the reference's log lines.  Errors raise ``BastrError`` carrying the
library's message, like the reference's ``stop 'message'``.

There is no CPU fallback: constructing a solver without the built library or without a CUDA
device raises.
"""
from __future__ import annotations

import ctypes as C
import math
import os
from dataclasses import dataclass

import numpy as np

from .initfield import seeded_field  # noqa: F401  (re-export)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbastr_gpu.so")

BASTR_OK = 0
BASTR_E_INVALID = -1
BASTR_E_UNSUPPORTED = -2
BASTR_E_CUDA = -3
BASTR_E_NAN = -4
BASTR_E_STATE = -5
BASTR_FP64 = 0
BASTR_FP32 = 1

EXPORTED = [
    "bastr_create", "bastr_destroy", "bastr_set_state", "bastr_get_state", "bastr_set_counters",
    "bastr_get_counters", "bastr_step", "bastr_step_async", "bastr_step_records", "bastr_spectra",
    "bastr_fft", "bastr_set_stream", "bastr_sync", "bastr_info", "bastr_last_error", "bastr_profile",
    "bastr_spectra_noalloc", "bastr_set_plan",
    "bastr_ensemble_create", "bastr_ensemble_destroy", "bastr_ensemble_size", "bastr_ensemble_set_state",
    "bastr_ensemble_get_state", "bastr_ensemble_step", "bastr_ensemble_set_plan", "bastr_ensemble_get_plan",
    "bastr_ensemble_tune", "bastr_ensemble_last_error",
    "bastr_net_nparams", "bastr_net_grad_blocks", "bastr_net_forward", "bastr_net_grad", "bastr_net_adam",
    "bastr_closure_apply", "bastr_transfer", "bastr_hitgen",
    "bastr_h5_write", "bastr_h5_read", "bastr_h5_write_field", "bastr_h5_read_field", "bastr_h5_last_error",
    "bastr_subgrid", "bastr_ensemble_subgrid", "bastr_ensemble_run",
    "bastr_fft_lines", "bastr_slab_pack", "bastr_slab_unpack",
]
BASTR_H5_F64 = 0
BASTR_H5_I32 = 1
BASTR_E_TOO_LARGE = -6


class BastrError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"bastr error {code}: {msg}")
        self.code = code


class CParams(C.Structure):
    _fields_ = [
        ("ia", C.c_int32), ("ja", C.c_int32), ("ka", C.c_int32),
        ("ref_tem", C.c_double), ("reynolds", C.c_double), ("deltat", C.c_double),
        ("kmax", C.c_int32), ("timemethod", C.c_int32), ("forcemethod", C.c_int32),
        ("forcek", C.c_int32), ("target_energy", C.c_double), ("lprojectd", C.c_int32),
        ("precision", C.c_int32), ("device", C.c_int32), ("velgrad_every", C.c_int32),
    ]


class CStepOut(C.Structure):
    _fields_ = [
        ("nstep", C.c_int64), ("time", C.c_double),
        ("Esspe", C.c_double), ("Edspe", C.c_double), ("k2Edspe", C.c_double), ("kMEdspe", C.c_double),
        ("velgrad", C.c_double * 8), ("factor", C.c_double), ("E", C.c_double),
        ("energy", C.c_double), ("Fen", C.c_double),
    ]


class CH5Dataset(C.Structure):
    _fields_ = [("name", C.c_char_p), ("type", C.c_int32), ("rank", C.c_int32), ("dims", C.c_int64 * 4),
                ("data", C.c_void_p)]


class CKernelStat(C.Structure):
    _fields_ = [("name", C.c_char * 48), ("launches", C.c_int32), ("total_ms", C.c_double),
                ("bytes_per_launch", C.c_double)]


_lib = None


def load_library(path: str = LIB_PATH) -> C.CDLL:
    """Loads the CUDA library; raises if it has not been built (no fallback exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is missing: run `python -m bastr_b200.build`")
    lib = C.CDLL(path)
    P = C.c_void_p
    D = C.POINTER(C.c_double)
    lib.bastr_create.argtypes = [C.POINTER(CParams), C.POINTER(P)]
    lib.bastr_destroy.argtypes = [P]
    lib.bastr_set_state.argtypes = [P, D, D, D]
    lib.bastr_get_state.argtypes = [P, D, D, D]
    lib.bastr_set_counters.argtypes = [P, C.c_int64, C.c_double]
    lib.bastr_get_counters.argtypes = [P, C.POINTER(C.c_int64), D]
    lib.bastr_step.argtypes = [P, C.c_int32, C.POINTER(CStepOut), D]
    lib.bastr_step_async.argtypes = [P, C.c_int32]
    lib.bastr_step_records.argtypes = [P, C.c_int32, C.POINTER(CStepOut), D]
    lib.bastr_spectra.argtypes = [P, D, D, D, C.POINTER(C.c_int64)]
    lib.bastr_fft.argtypes = [P, D, C.c_int32]
    lib.bastr_set_stream.argtypes = [P, P]
    lib.bastr_sync.argtypes = [P]
    lib.bastr_info.argtypes = [P, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int64)]
    lib.bastr_last_error.argtypes = [P, C.c_char_p, C.c_int32]
    lib.bastr_profile.argtypes = [P, C.c_int32, C.POINTER(CKernelStat), C.c_int32, C.POINTER(C.c_int32)]
    lib.bastr_spectra_noalloc.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_int32, P, P, P, P, P, P, P]
    lib.bastr_fft_lines.argtypes = [P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_double, P]
    lib.bastr_slab_pack.argtypes = [P, P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, P]
    lib.bastr_slab_unpack.argtypes = [P, P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, P]
    lib.bastr_set_plan.argtypes = [P, C.c_int32]
    lib.bastr_ensemble_create.argtypes = [C.POINTER(CParams), C.c_int32, C.POINTER(P)]
    lib.bastr_ensemble_destroy.argtypes = [P]
    lib.bastr_ensemble_size.argtypes = [P, C.POINTER(C.c_int32)]
    lib.bastr_ensemble_set_state.argtypes = [P, C.c_int32, D, D, D]
    lib.bastr_ensemble_get_state.argtypes = [P, C.c_int32, D, D, D]
    lib.bastr_ensemble_step.argtypes = [P, C.c_int32, C.POINTER(CStepOut)]
    lib.bastr_ensemble_set_plan.argtypes = [P, C.c_int32, C.c_int32]
    lib.bastr_ensemble_get_plan.argtypes = [P, C.POINTER(C.c_int32)]
    lib.bastr_ensemble_tune.argtypes = [P, C.c_int32, C.c_int32, C.c_int32, D]
    lib.bastr_ensemble_last_error.argtypes = [P, C.c_char_p, C.c_int32]
    lib.bastr_net_nparams.argtypes = []
    lib.bastr_net_grad_blocks.argtypes = []
    lib.bastr_net_forward.argtypes = [C.c_int32, C.c_int32, C.c_int32, P, P, P, C.c_float, P]
    lib.bastr_net_grad.argtypes = [C.c_int32, C.c_int32, C.c_int32, P, P, P, P, C.c_int32, P, P, P]
    lib.bastr_net_adam.argtypes = [P, P, P, P, P, C.c_int32, C.c_float, C.c_float, C.c_float, C.c_float, P]
    lib.bastr_closure_apply.argtypes = [P, P, C.c_float, C.c_double]
    lib.bastr_transfer.argtypes = [P, D, D, D]
    lib.bastr_hitgen.argtypes = [P, C.c_int32, C.c_uint64, D, D, D, D, D]
    lib.bastr_h5_write.argtypes = [C.c_char_p, C.POINTER(CH5Dataset), C.c_int32]
    lib.bastr_h5_read.argtypes = [C.c_char_p, C.c_char_p, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int64),
                                  P, C.c_int64]
    lib.bastr_h5_write_field.argtypes = [C.c_char_p, C.c_int32, C.c_int32, C.c_int32, D, D, D, C.c_int64, C.c_double]
    lib.bastr_h5_read_field.argtypes = [C.c_char_p, C.c_int32, C.c_int32, C.c_int32, D, D, D,
                                        C.POINTER(C.c_int64), D]
    lib.bastr_h5_last_error.argtypes = [C.c_char_p, C.c_int32]
    lib.bastr_subgrid.argtypes = [P, C.c_int32, P, P]
    lib.bastr_ensemble_subgrid.argtypes = [P, C.c_int32, C.c_int32, P, P]
    lib.bastr_ensemble_run.argtypes = [P, C.c_int32, C.c_int32, D]
    for name in EXPORTED:
        getattr(lib, name).restype = C.c_int
    _lib = lib
    return lib


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


@dataclass
class StepRecord:
    nstep: int
    time: float
    Esspe: float
    Edspe: float
    k2Edspe: float
    kMEdspe: float
    velgrad: tuple
    factor: float
    E: float
    energy: float = float("nan")
    Fen: float = float("nan")


def miucal(temper: float, ref_tem: float) -> float:
    """Sutherland viscosity law (solution.F90:1315-1329)."""
    tc = 110.4 / ref_tem
    return temper * math.sqrt(temper) * (1.0 + tc) / (temper + tc)


def make_cparams(ia: int, ja: int, ka: int = 0, *, ref_tem: float = 273.15, reynolds: float = 5000.0,
                 deltat: float = 1e-4, kmax: int = 1 << 30, timemethod: int = 1, forcemethod: int = 0,
                 forcek: int = 5, target_energy: float = 0.075, lprojectd: bool = False,
                 precision: str = "fp64", device: int = 0, velgrad_every: int = 1) -> CParams:
    """The ``bastr_params`` of one field (the ``datin/input.dat`` values the hot path reads)."""
    return CParams(ia, ja, ka, ref_tem, reynolds, deltat, kmax, timemethod, forcemethod, forcek,
                   target_energy, 1 if lprojectd else 0,
                   BASTR_FP32 if precision == "fp32" else BASTR_FP64, device, velgrad_every)


class BastrGPU:
    """One solver handle on one GPU (see module docstring)."""

    def __init__(self, ia: int, ja: int, ka: int = 0, *, ref_tem: float = 273.15,
                 reynolds: float = 5000.0, deltat: float = 1e-4, kmax: int = 1 << 30,
                 timemethod: int = 1, forcemethod: int = 0, forcek: int = 5,
                 target_energy: float = 0.075, lprojectd: bool = False,
                 precision: str = "fp64", device: int = 0, velgrad_every: int = 1):
        self.lib = load_library()
        p = make_cparams(ia, ja, ka, ref_tem=ref_tem, reynolds=reynolds, deltat=deltat, kmax=kmax,
                         timemethod=timemethod, forcemethod=forcemethod, forcek=forcek,
                         target_energy=target_energy, lprojectd=lprojectd, precision=precision,
                         device=device, velgrad_every=velgrad_every)
        self._p = p
        self.h = C.c_void_p()
        rc = self.lib.bastr_create(C.byref(p), C.byref(self.h))
        if rc != BASTR_OK:
            msg = self._err()
            self.close()
            raise BastrError(rc, msg)
        self.ndims = 2 if ka == 0 else 3
        self.shape = (ja, ia) if ka == 0 else (ka, ja, ia)
        self.deltat = deltat
        self.forcemethod = forcemethod
        a = C.c_int32()
        self.lib.bastr_info(self.h, C.byref(a), None, None)
        self.allkmax = a.value

    # -- plumbing ------------------------------------------------------------------------
    def _err(self) -> str:
        buf = C.create_string_buffer(1024)
        if self.h:
            self.lib.bastr_last_error(self.h, buf, 1024)
        return buf.value.decode(errors="replace")

    def _check(self, rc: int):
        if rc != BASTR_OK:
            raise BastrError(rc, self._err())

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            self.lib.bastr_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def info(self):
        a, n, b = C.c_int32(), C.c_int32(), C.c_int64()
        self._check(self.lib.bastr_info(self.h, C.byref(a), C.byref(n), C.byref(b)))
        return {"allkmax": a.value, "launches_per_step": n.value, "device_bytes": b.value}

    # -- state ---------------------------------------------------------------------------
    def set_state(self, u):
        arrs = [np.ascontiguousarray(c, dtype=np.float64).reshape(self.shape) for c in u]
        if len(arrs) != self.ndims:
            raise ValueError("one array per velocity component")
        u3 = arrs[2] if self.ndims == 3 else arrs[0]
        self._check(self.lib.bastr_set_state(self.h, _dptr(arrs[0]), _dptr(arrs[1]), _dptr(u3)))

    def get_state(self, out=None):
        """The physical velocity components; into `out` (one C-contiguous float64 array of the
        grid's shape per component, e.g. pinned host memory) when given."""
        if out is None:
            out = [np.empty(self.shape, dtype=np.float64) for _ in range(self.ndims)]
        elif len(out) != self.ndims or any(o.shape != self.shape or o.dtype != np.float64 or
                                           not o.flags.c_contiguous for o in out):
            raise ValueError("get_state(out=...): one C-contiguous float64 array of the grid's shape per component")
        u3 = out[2] if self.ndims == 3 else out[0]
        self._check(self.lib.bastr_get_state(self.h, _dptr(out[0]), _dptr(out[1]), _dptr(u3)))
        return out

    def set_counters(self, nstep: int, time: float):
        self._check(self.lib.bastr_set_counters(self.h, nstep, time))

    def counters(self):
        n, t = C.c_int64(), C.c_double()
        self._check(self.lib.bastr_get_counters(self.h, C.byref(n), C.byref(t)))
        return n.value, t.value

    # -- stepping ------------------------------------------------------------------------
    @staticmethod
    def _rec(o: CStepOut) -> StepRecord:
        return StepRecord(o.nstep, o.time, o.Esspe, o.Edspe, o.k2Edspe, o.kMEdspe,
                          tuple(o.velgrad), o.factor, o.E, o.energy, o.Fen)

    def step(self, nsteps: int = 1, shells: bool = False):
        """Runs nsteps main-loop iterations; returns records (and per-step Es/Ed shells)."""
        out = (CStepOut * max(nsteps, 1))()
        sh = np.empty((max(nsteps, 1), 2, self.allkmax + 1), dtype=np.float64) if shells else None
        rc = self.lib.bastr_step(self.h, nsteps, out, _dptr(sh) if sh is not None else None)
        recs = [self._rec(out[i]) for i in range(nsteps)]
        if rc != BASTR_OK:
            raise BastrError(rc, self._err())
        return (recs, sh[:nsteps]) if shells else recs

    def step_async(self, nsteps: int):
        self._check(self.lib.bastr_step_async(self.h, nsteps))

    def records(self, nsteps: int):
        out = (CStepOut * max(nsteps, 1))()
        self._check(self.lib.bastr_step_records(self.h, nsteps, out, None))
        return [self._rec(out[i]) for i in range(nsteps)]

    def sync(self):
        self._check(self.lib.bastr_sync(self.h))

    def transfer(self):
        """Transfer spectra T, T1, T2 of the current state, shells 0..allkmax (Bastrpp's
        transfer2d/transfer3d)."""
        n = self.allkmax + 1
        t, t1, t2 = (np.empty(n) for _ in range(3))
        self._check(self.lib.bastr_transfer(self.h, _dptr(t), _dptr(t1), _dptr(t2)))
        return t, t1, t2

    def hitgen(self, variant: int = 0, seed: int = 0):
        """Bastrpp's initial-field generators (hitgen2d / hitgen3d = variant 0, hitgen2dbis =
        variant 1) on this handle's grid, forcek and target_energy.  Returns (fields, angle,
        stats): the physical u1, u2[, u3], the random_angle field and a dict of energy (before
        scaling), factor, alpha, residual, QX, QY, QZ, QW.  The state is not changed."""
        out = [np.empty(self.shape, dtype=np.float64) for _ in range(self.ndims)]
        angle = np.empty(self.shape, dtype=np.float64)
        st = np.empty(8, dtype=np.float64)
        u3 = out[2] if self.ndims == 3 else None
        self._check(self.lib.bastr_hitgen(self.h, variant, seed & 0xFFFFFFFFFFFFFFFF, _dptr(out[0]), _dptr(out[1]),
                                          _dptr(u3) if u3 is not None else None, _dptr(angle), _dptr(st)))
        names = ("energy", "factor", "alpha", "residual", "QX", "QY", "QZ", "QW")
        return out, angle, dict(zip(names, st.tolist()))

    def subgrid(self, r: int):
        """(ub, tau) of the current state as float32 CUDA tensors [d][...coarse grid] (bastr_subgrid):
        the box-filtered velocity and the subgrid term filter(u.grad u) - ub.grad ub."""
        import torch
        shape = [self.ndims] + [n // r for n in self.shape]
        ub = torch.empty(shape, dtype=torch.float32, device="cuda")
        tau = torch.empty_like(ub)
        self._check(self.lib.bastr_subgrid(self.h, r, C.c_void_p(ub.data_ptr()), C.c_void_p(tau.data_ptr())))
        return ub, tau

    def closure_apply(self, net, scale: float, dt: float):
        """One closure sub-step u <- u - dt * scale * net(u) on this (3D) solver's state; `net` is
        a bastr_b200.closure.Net."""
        self._check(self.lib.bastr_closure_apply(self.h, C.c_void_p(net.wb.data_ptr()), C.c_float(scale), dt))

    def set_plan(self, share_log2: int):
        """Persistent grids on 1/2**share_log2 of the resident blocks (0 = all)."""
        self._check(self.lib.bastr_set_plan(self.h, share_log2))

    def set_stream(self, stream_ptr: int):
        self._check(self.lib.bastr_set_stream(self.h, C.c_void_p(stream_ptr)))

    def spectra(self):
        n = self.allkmax + 1
        kn, es, ed = (np.empty(n) for _ in range(3))
        ec = np.empty(n, dtype=np.int64)
        self._check(self.lib.bastr_spectra(self.h, _dptr(kn), _dptr(es), _dptr(ed),
                                           ec.ctypes.data_as(C.POINTER(C.c_int64))))
        return kn, es, ed, ec

    def profile(self, nsteps: int):
        """Per-kernel device time over nsteps iterations (CUDA events around every launch)."""
        stats = (CKernelStat * 64)()
        n = C.c_int32()
        self._check(self.lib.bastr_profile(self.h, nsteps, stats, 64, C.byref(n)))
        return [{"name": stats[i].name.decode(), "launches": stats[i].launches,
                 "total_ms": stats[i].total_ms, "bytes_per_launch": stats[i].bytes_per_launch}
                for i in range(min(n.value, 64))]

    def fft(self, array: np.ndarray, direction: int) -> np.ndarray:
        """fft2d/fft3d (direction -1, scaled 1/N) or ifft2d/ifft3d (+1) of a full complex grid."""
        a = np.ascontiguousarray(array, dtype=np.complex128).reshape(self.shape).copy()
        self._check(self.lib.bastr_fft(self.h, a.view(np.float64).ctypes.data_as(C.POINTER(C.c_double)),
                                       direction))
        return a


# -------------------------------------------------------------------------------------------
# Field files without libhdf5 (the HDF5 subset of hdf5io.F90's field files; host code only)
# -------------------------------------------------------------------------------------------
def _h5_check(lib, rc: int):
    if rc != BASTR_OK:
        buf = C.create_string_buffer(512)
        lib.bastr_h5_last_error(buf, 512)
        raise BastrError(rc, buf.value.decode(errors="replace"))


def h5_write(path: str, datasets: dict):
    """Writes {name: array} (float64 or int32 arrays, C order) as the root-group datasets of an
    HDF5 file (bastr_h5_write)."""
    lib = load_library()
    keep, sets = [], []
    for name, a in datasets.items():
        a = np.ascontiguousarray(a)
        if a.dtype == np.float64:
            t = BASTR_H5_F64
        elif a.dtype == np.int32:
            t = BASTR_H5_I32
        else:
            raise ValueError(f"{name}: only float64 and int32 datasets")
        if a.ndim == 0:
            a = a.reshape(1)
        dims = (C.c_int64 * 4)(*(list(a.shape) + [0] * (4 - a.ndim)))
        keep.append(a)
        sets.append(CH5Dataset(name.encode(), t, a.ndim, dims, a.ctypes.data))
    arr = (CH5Dataset * max(len(sets), 1))(*sets)
    _h5_check(lib, lib.bastr_h5_write(path.encode(), arr, len(sets)))


def h5_read(path: str, name: str, dtype=np.float64) -> np.ndarray:
    """One dataset of an HDF5 field file (bastr_h5_read), as a C-order array."""
    lib = load_library()
    t = BASTR_H5_I32 if np.dtype(dtype) == np.int32 else BASTR_H5_F64
    rank = C.c_int32()
    dims = (C.c_int64 * 4)()
    _h5_check(lib, lib.bastr_h5_read(path.encode(), name.encode(), t, C.byref(rank), dims, None, 0))
    out = np.empty([dims[i] for i in range(rank.value)], dtype=np.int32 if t == BASTR_H5_I32 else np.float64)
    _h5_check(lib, lib.bastr_h5_read(path.encode(), name.encode(), t, C.byref(rank), dims,
                                     C.c_void_p(out.ctypes.data), out.nbytes))
    return out


def write_field(path: str, u, nstep: int | None = None, time: float = 0.0):
    """The reference's field file (writeflfed, readwrite.F90:222-257): u = [u1, u2(, u3)] arrays of
    shape (ja, ia) or (ka, ja, ia), x fastest; nstep and time are written when nstep is given."""
    lib = load_library()
    arrs = [np.ascontiguousarray(c, dtype=np.float64) for c in u]
    if arrs[0].ndim == 2:
        ka, (ja, ia) = 0, arrs[0].shape
    else:
        ka, ja, ia = arrs[0].shape
    u3 = arrs[2] if ka else arrs[0]
    _h5_check(lib, lib.bastr_h5_write_field(path.encode(), ia, ja, ka, _dptr(arrs[0]), _dptr(arrs[1]), _dptr(u3),
                                            -1 if nstep is None else int(nstep), float(time)))


def read_field(path: str, ia: int, ja: int, ka: int = 0, counters: bool = False):
    """u1, u2(, u3) of a field file on an ia x ja (x ka) grid (read_initial_field /
    read_continue_field, readwrite.F90:114-220); with counters, also (nstep, time)."""
    lib = load_library()
    shape = (ja, ia) if ka == 0 else (ka, ja, ia)
    out = [np.empty(shape) for _ in range(2 if ka == 0 else 3)]
    n, t = C.c_int64(), C.c_double()
    u3 = out[2] if ka else out[0]
    _h5_check(lib, lib.bastr_h5_read_field(path.encode(), ia, ja, ka, _dptr(out[0]), _dptr(out[1]), _dptr(u3),
                                           C.byref(n) if counters else None,
                                           C.byref(t) if counters else None))
    return (out, n.value, t.value) if counters else out


from .ensemble import BastrEnsemble, ensemble_configs, partition_by_cost  # noqa: E402,F401
