"""The oracle's own FFT against numpy.fft (pocketfft)."""
import numpy as np
import pytest

LENGTHS = [24, 32, 36, 48, 72, 96, 144, 192, 288, 384, 768, 1536, 7, 30, 125]


@pytest.mark.parametrize("n", LENGTHS)
def test_fft1d(n, oracle_lib):
    import oracle as O
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    ref_f, ref_b = np.fft.fft(x), np.fft.ifft(x) * n
    scale = np.abs(ref_f).max()
    assert np.abs(O.fft1d(x, -1) - ref_f).max() / scale < 5e-15 * max(1, np.log2(n))
    assert np.abs(O.fft1d(x, +1) - ref_b).max() / scale < 5e-15 * max(1, np.log2(n))


@pytest.mark.parametrize("shape", [(24, 36, 48), (48, 48, 48), (16, 12, 10)])
def test_rfft3d_roundtrip(shape, oracle_lib):
    import oracle as O
    rng = np.random.default_rng(1)
    x = rng.standard_normal(shape)
    X = O.rfft3d(x)
    Xr = np.fft.rfftn(x, axes=(0, 1, 2))
    assert np.abs(X - Xr).max() / np.abs(Xr).max() < 1e-14
    y = O.irfft3d(Xr, shape[2]) / np.prod(shape)
    assert np.abs(y - x).max() < 1e-13
