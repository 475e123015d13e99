"""Builds the in-tree CUDA library ``bastr_b200/libbastr_gpu.so`` for sm_100a.

Run ``python -m bastr_b200.build`` (or ``__graft_entry__.build()``).  nvcc cross-compiles,
so no GPU is needed.  The library is rebuilt only when a source is newer than it.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libbastr_gpu.so")
SOURCES = ["capi.cu", "noalloc.cu"]
DEPS = ["capi.cu", "pass2d.cu", "pass3d.cu", "diag.cu", "ensemble.cu", "fullfft.cu", "closure.cu", "transfer.cu", "hitgen.cu", "noalloc.cu", "fft_engine.cuh", "regfft.cuh",
        "solver.cuh"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, d) for d in DEPS] + [os.path.join(ROOT, "include", "bastr_gpu.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> str:
    if not force and not _stale():
        return LIB
    cmd = [NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "--shared", "-Xcompiler", "-fPIC",
           "-Xcompiler", "-fvisibility=hidden", "--expt-relaxed-constexpr",
           "-I", os.path.join(ROOT, "include"),
           "-o", LIB + ".tmp", *[os.path.join(CSRC, s) for s in SOURCES], *(extra or [])]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed for libbastr_gpu.so")
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
