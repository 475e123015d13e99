"""The index-checking build (``-DBASTR_CHECKED``, ``bastr_b200/libbastr_gpu_checked.so``): the
library's memory checker, since no sanitizer runs on this pool.

Every device buffer a handle allocates is registered; in the checked build the kernels' staging
copies (``cp.async`` and line staging), their output stores, the stage epilogue's state reads
and writes, and the spectra and forcing gathers verify that each access lies inside one
registered buffer.  An access that does not sets a bit in the handle's error word, goes to a
scratch line instead (no fault), and the next ``bastr_step`` returns BASTR_E_CUDA.  The tensor
maps of the TMA staging are checked against the buffers at creation in every build.

CPU: the checked library exports the same entry points as the normal one.  GPU: the cases of
tests/checked_cases.py (2D and 3D, square and not, FP64 and FP32, RK3 and Crank-Nicolson, forcing
methods 1-5, statistics every step, spectra and transfer spectra, and the measured sizes 2048^2
and 256^3) run
through both libraries in separate processes: the checked run reports no bad access, and its
results are bitwise those of the normal build (the checks never change an in-bounds access).
"""
import ctypes
import os
import re
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    text = open(os.path.join(ROOT, "include", "bastr_gpu.h")).read()
    return sorted(set(re.findall(r"BASTR_API\s+int\s+(bastr_\w+)\s*\(", text)))


def test_checked_library_exports_the_header():
    from bastr_b200 import build
    if not os.path.exists(build.LIB_CHECKED):
        pytest.skip("the checked variant is not built (python -m bastr_b200.build --checked)")
    lib = ctypes.CDLL(build.LIB_CHECKED)
    missing = [name for name in _declared() if not hasattr(lib, name)]
    assert not missing, missing


@pytest.mark.gpu
def test_checked_build_matches_and_reports_nothing(tmp_path):
    from bastr_b200 import build
    libs = {"normal": build.build(), "checked": build.build(checked=True)}
    res = {}
    for kind, lib in libs.items():
        out = tmp_path / f"{kind}.npz"
        r = subprocess.run([sys.executable, "-m", "tests.checked_cases", lib, str(out)], cwd=ROOT,
                           capture_output=True, text=True, timeout=900)
        assert r.returncode == 0, f"{kind} run failed:\n{r.stdout[-2000:]}\n{r.stderr[-4000:]}"
        res[kind] = dict(np.load(out))
    assert res["normal"].keys() == res["checked"].keys()
    differ = [k for k in res["normal"] if not np.array_equal(res["normal"][k], res["checked"][k], equal_nan=True)]
    assert not differ, differ


_PLANTED = """
import sys
import bastr_b200
bastr_b200.load_library(sys.argv[1])
from bastr_b200 import BastrError, BastrGPU, seeded_field
with BastrGPU(16, 16, 0, reynolds=2000.0, deltat=2e-4, precision=sys.argv[2], velgrad_every=1) as s:
    s.set_state(seeded_field(16, 16, 0, k0=4.0, seed=3))
    try:
        s.step(1)
        print("no error")
    except BastrError as e:
        print("code", e.code, str(e))
"""


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_checked_build_reports_a_planted_table_error(precision):
    """The mistake is planted in the checker's own table, on the host: with BASTR_CHECK_SHRINK=16
    every registered buffer loses its last 16 bytes, so accesses to the last state modes (in
    bounds; nothing leaves its buffer) are reported and redirected to the scratch line.  The
    batch must return BASTR_E_CUDA naming the index check; the normal library ignores the
    variable."""
    from bastr_b200 import BASTR_E_CUDA, build
    env = dict(os.environ, BASTR_CHECK_SHRINK="16")
    for lib, want_error in ((build.build(checked=True), True), (build.build(), False)):
        r = subprocess.run([sys.executable, "-c", _PLANTED, lib, precision], cwd=ROOT, env=env,
                           capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr[-3000:]
        out = r.stdout.strip().splitlines()[-1]
        if want_error:
            assert out.startswith(f"code {BASTR_E_CUDA}") and "index check" in out, out
        else:
            assert out == "no error", out


def _calls(text, name):
    """The argument text of every call `name(...)` in `text` (balanced parentheses)."""
    out, i = [], 0
    while True:
        j = text.find(name + "(", i)
        if j < 0:
            return out
        k, depth = j + len(name) + 1, 1
        while depth:
            depth += {"(": 1, ")": -1}.get(text[k], 0)
            k += 1
        out.append(text[j + len(name) + 1:k - 1])
        i = k


def test_pass_kernels_route_their_global_accesses_through_the_checks():
    """Source guard for the checked build's coverage: in the pass kernels every cp.async source,
    every line staging and every paired vector store goes through BASTR_CHK (or passes the
    geometry that carries the table), so a new access of these kinds cannot skip the checker."""
    csrc = os.path.join(ROOT, "bastr_b200", "csrc")
    for fname in ("pass2d.cu", "pass3d.cu"):
        text = open(os.path.join(csrc, fname)).read()
        for name in ("cp_async16", "cp_async8"):
            for args in _calls(text, name):
                assert "BASTR_CHK" in args, (fname, name, args)
        for args in _calls(text, "stage_line"):
            assert args.rstrip().endswith(", g"), (fname, args)
        for args in _calls(text, "st2<T>"):
            assert args.lstrip().startswith("BASTR_CHK("), (fname, args)
