"""Batched 1-D FFT building block of libspns against numpy.fft, every compiled length."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LENGTHS = [48, 72, 96, 144, 192, 288, 384, 768, 1536]


@pytest.mark.parametrize("n", LENGTHS)
@pytest.mark.parametrize("sign", [-1, 1])
def test_fft1d_batch(n, sign):
    import torch
    from spns_b200 import hit
    rng = np.random.default_rng(n)
    batch = 37
    x = rng.standard_normal((batch, n)) + 1j * rng.standard_normal((batch, n))
    d = torch.from_numpy(x.copy()).to("cuda")
    hit.fft1d_batch_f64(d.data_ptr(), n, batch, sign)
    y = d.cpu().numpy()
    ref = np.fft.fft(x, axis=1) if sign < 0 else np.fft.ifft(x, axis=1) * n
    err = np.abs(y - ref).max() / np.abs(ref).max()
    assert err < 1e-14, err


def test_unsupported_length_is_an_error():
    import torch
    from spns_b200 import hit
    d = torch.zeros(100, dtype=torch.complex128, device="cuda")
    with pytest.raises(hit.SpnsError) as ei:
        hit.fft1d_batch_f64(d.data_ptr(), 100, 1, -1)
    assert ei.value.status == -2
