"""bastr_fft (the fft2d/fft3d/ifft2d/ifft3d replacement, fftwlink.F90:324-368) against numpy's
FFT of the same complex grid: forward e^{-ikx} scaled by 1/N, backward e^{+ikx} unscaled, in
place on [nz][ny][nx] with x fastest.  FP64; relative L2 within 1e-13."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("dims", [(64, 128, 0), (256, 256, 0), (2048, 2048, 0), (16, 32, 64), (128, 128, 128)],
                         ids=["2d_64x128", "2d_256", "2d_2048", "3d_16x32x64", "3d_128"])
def test_fft_matches_numpy(gpu_lib, dims):
    from bastr_b200 import BastrGPU
    ia, ja, ka = dims
    shape = (ja, ia) if ka == 0 else (ka, ja, ia)
    rng = np.random.default_rng(7)
    a = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    n = a.size
    with BastrGPU(ia, ja, ka) as s:
        f = s.fft(a, -1)
        b = s.fft(a, +1)
        back = s.fft(f, +1)
    assert _rel(f, np.fft.fftn(a) / n) < 1e-13
    assert _rel(b, np.fft.ifftn(a) * n) < 1e-13
    assert _rel(back, a) < 1e-13


def test_fft_rejects_bad_direction(gpu_lib):
    from bastr_b200 import BastrError, BastrGPU
    with BastrGPU(64, 64, 0) as s:
        with pytest.raises(BastrError):
            s.fft(np.zeros((64, 64), complex), 0)
