"""Builds the in-tree CUDA library ``bastr_b200/libbastr_gpu.so`` for sm_100a.

Run ``python -m bastr_b200.build`` (or ``__graft_entry__.build()``).  nvcc cross-compiles,
so no GPU is needed.  The library is split into translation units (the C ABI, the 2D and 3D
step schedules per compute precision, the allocation-free spectra) that compile in parallel
into ``bastr_b200/_build/``; an object is rebuilt only when one of its sources is newer than it,
and the library is relinked when an object is newer than it.

``build(checked=True)`` (``python -m bastr_b200.build --checked``) makes the index-checking
variant ``bastr_b200/libbastr_gpu_checked.so`` (``-DBASTR_CHECKED``, objects in
``bastr_b200/_build_checked/``): the same entry points, with the kernels' staging copies,
output stores, state accesses and gathers checked against the handle's buffers.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJDIR = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libbastr_gpu.so")
OBJDIR_CHECKED = os.path.join(HERE, "_build_checked")
LIB_CHECKED = os.path.join(HERE, "libbastr_gpu_checked.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
HEADER = os.path.join(ROOT, "include", "bastr_gpu.h")

_COMMON = ["handle.cuh", "solver.cuh", "fft_engine.cuh", "regfft.cuh", "tma.cuh", "umma.cuh"]
# translation unit -> the sources it includes
UNITS = {
    "capi.cu": _COMMON + ["diag.cu", "fullfft.cu", "closure.cu", "transfer.cu", "hitgen.cu", "subgrid.cu",
                         "ensemble.cu", "slab.cu"],
    "steps2d_f32.cu": _COMMON + ["pass2d.cu", "steps2d.cuh"],
    "steps2d_f64.cu": _COMMON + ["pass2d.cu", "steps2d.cuh"],
    "steps3d_f32.cu": _COMMON + ["pass2d.cu", "pass3d.cu", "steps3d.cuh"],
    "steps3d_f64.cu": _COMMON + ["pass2d.cu", "pass3d.cu", "steps3d.cuh"],
    "noalloc.cu": ["solver.cuh", "fft_engine.cuh"],
    "h5field.cpp": [],
}
# every source file of the library (for callers that check staleness as a whole)
DEPS = sorted({d for u, ds in UNITS.items() for d in ds + [u]})
FLAGS = ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
         "--expt-relaxed-constexpr"]


def _obj(unit: str, objdir: str = OBJDIR) -> str:
    return os.path.join(objdir, os.path.splitext(unit)[0] + ".o")


def _mtime(p: str) -> float:
    return os.path.getmtime(p) if os.path.exists(p) else float("inf")


def _unit_stale(unit: str, objdir: str = OBJDIR) -> bool:
    o = _obj(unit, objdir)
    if not os.path.exists(o):
        return True
    t = os.path.getmtime(o)
    srcs = [os.path.join(CSRC, d) for d in UNITS[unit] + [unit]] + [HEADER]
    return any(_mtime(s) > t for s in srcs)


def _stale(lib: str = LIB, objdir: str = OBJDIR) -> bool:
    if not os.path.exists(lib):
        return True
    t = os.path.getmtime(lib)
    return any(_unit_stale(u, objdir) or os.path.getmtime(_obj(u, objdir)) > t for u in UNITS)


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None, jobs: int | None = None,
          checked: bool = False) -> str:
    """Compiles the stale translation units in parallel and links the library.  `extra` flags
    (e.g. -D overrides) apply to every unit and force a full rebuild.  `checked`: the
    index-checking variant (its own objects and library file)."""
    objdir, lib = (OBJDIR_CHECKED, LIB_CHECKED) if checked else (OBJDIR, LIB)
    flags = list(extra or []) + (["-DBASTR_CHECKED"] if checked else [])
    if extra:
        force = True
    if not force and not _stale(lib, objdir):
        return lib
    os.makedirs(objdir, exist_ok=True)
    todo = [u for u in UNITS if force or _unit_stale(u, objdir)]

    def compile_unit(unit):
        obj = _obj(unit, objdir)
        cmd = [NVCC, *ARCH, *FLAGS, "-I", os.path.join(ROOT, "include"), "-c", os.path.join(CSRC, unit),
               "-o", obj + ".tmp", *flags]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode == 0:
            os.replace(obj + ".tmp", obj)
        return unit, r

    njobs = jobs or min(len(todo), max(1, os.cpu_count() or 1)) or 1
    failed = []
    with ThreadPoolExecutor(max_workers=njobs) as ex:
        for unit, r in ex.map(compile_unit, todo):
            if r.returncode != 0:
                failed.append(unit)
                sys.stderr.write(r.stdout + r.stderr)
    if failed:
        raise RuntimeError(f"nvcc failed for {', '.join(failed)}")
    link = [NVCC, *ARCH, "--shared", "-Xcompiler", "-fPIC", "-o", lib + ".tmp", *[_obj(u, objdir) for u in UNITS]]
    if verbose:
        print(" ".join(link), flush=True)
    r = subprocess.run(link, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"link of {os.path.basename(lib)} failed")
    os.replace(lib + ".tmp", lib)
    return lib


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True, checked="--checked" in sys.argv))
