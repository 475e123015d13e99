"""bastr_spectra_noalloc: shell spectra of a spectrum held in the caller's own device memory.

It exists for callers that cannot let the library call cudaMalloc (GPU memory owned by CUDA
Fortran / OpenACC data regions, memory-capped pools), so they cannot create a solver handle.
These tests call it through the C ABI on a spectrum this test owns and check it against the
existing handle-based entry points (bastr_spectra for the shells, the step record for the
totals) on two calls in a row, within the FP64 parity tolerance of the other GPU tests.

This file is collected last so that a failure here never hides the rest of the suite.
"""
import ctypes as C
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _rel(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("dims,kmax", [((64, 64, 0), 100), ((64, 128, 0), 100), ((32, 32, 32), 100),
                                       ((64, 64, 0), 5), ((32, 64, 32), 100), ((16, 32, 64), 3)],
                         ids=["2d", "2d_rect", "3d", "2d_kmax5", "3d_rect", "3d_rect_kmax3"])
def test_noalloc_spectra_match_handle(gpu_lib, dims, kmax):
    """kmax below ia/3 truncates allkmax (the shells past it are not returned, the totals still
    cover every mode); non-cubic 3D grids have per-axis Nyquist limits."""
    import torch

    from bastr_b200 import BASTR_OK, BastrGPU, load_library, seeded_field
    ia, ja, ka = dims
    u = seeded_field(ia, ja, ka, k0=4.0 if ka == 0 else 3.0, seed=11)
    with BastrGPU(ia, ja, ka, kmax=kmax, reynolds=5000.0, deltat=1e-4, precision="fp64") as s:
        s.set_state(u)                   # dealiases, as mainloop does before its first step
        ud = s.get_state()
        _, es_ref, ed_ref, _ = s.spectra()
        rec = s.step(1)[0]              # its spectra line is computed on the same state
    tot_ref = [rec.Esspe, rec.Edspe, rec.k2Edspe, rec.kMEdspe]

    # the caller's own spectra: fft2d/fft3d of the dealiased field (forward scaled by 1/N)
    dev = torch.device("cuda", 0)
    n = ud[0].size
    spe = [torch.from_numpy(np.ascontiguousarray(np.fft.fftn(c) / n)).to(dev) for c in ud]
    allkmax = min(ia // 3, kmax)
    d_es = torch.empty(allkmax + 1, dtype=torch.float64, device=dev)
    d_ed = torch.empty(allkmax + 1, dtype=torch.float64, device=dev)
    d_tot = torch.empty(4, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()

    lib = load_library()
    results = []
    for call in range(2):
        for t in (d_es, d_ed, d_tot):
            t.fill_(math.nan)
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info(dev)[0]
        rc = lib.bastr_spectra_noalloc(ia, ja, ka, kmax, _ptr(spe[0]), _ptr(spe[1]),
                                       _ptr(spe[2] if ka else spe[0]), _ptr(d_es), _ptr(d_ed),
                                       _ptr(d_tot), None)
        assert rc == BASTR_OK
        torch.cuda.synchronize()
        if call == 1:
            # the first call may load the kernels' module; the second allocates no device memory
            assert torch.cuda.mem_get_info(dev)[0] == free0
        es, ed, tot = d_es.cpu().numpy(), d_ed.cpu().numpy(), d_tot.cpu().numpy()
        assert _rel(es, es_ref) <= TOL
        assert _rel(ed, ed_ref) <= TOL
        for got, ref in zip(tot, tot_ref):
            assert abs(got - ref) <= TOL * abs(ref)
        results.append((es.copy(), ed.copy(), tot.copy()))
    # the shared workspace keeps the last call's contents; a repeated call gives the same bits
    for a, b in zip(results[0], results[1]):
        assert np.array_equal(a, b)
    # without the totals array: the shells alone, the same values
    d_es.fill_(math.nan)
    d_ed.fill_(math.nan)
    rc = lib.bastr_spectra_noalloc(ia, ja, ka, kmax, _ptr(spe[0]), _ptr(spe[1]), _ptr(spe[2] if ka else spe[0]),
                                   _ptr(d_es), _ptr(d_ed), None, None)
    assert rc == BASTR_OK
    torch.cuda.synchronize()
    assert np.array_equal(d_es.cpu().numpy(), results[0][0])
    assert np.array_equal(d_ed.cpu().numpy(), results[0][1])


def test_noalloc_rejects_grids_beyond_its_workspace(gpu_lib):
    import torch

    from bastr_b200 import BASTR_E_INVALID, BASTR_E_TOO_LARGE, load_library
    lib = load_library()
    t = torch.zeros(8, dtype=torch.float64, device="cuda")
    p = _ptr(t)
    # 8192^2: nint(|k|max) = 5793 shells needed, the fixed workspace holds 4096
    assert lib.bastr_spectra_noalloc(8192, 8192, 0, 100, p, p, p, p, p, p, None) == BASTR_E_TOO_LARGE
    assert lib.bastr_spectra_noalloc(96, 96, 0, 100, p, p, p, p, p, p, None) == BASTR_E_INVALID
    assert lib.bastr_spectra_noalloc(64, 64, 0, 100, None, p, p, p, p, p, None) == BASTR_E_INVALID
