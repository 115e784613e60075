"""The engine's 2-D FFT (row transform + transposed store, twice) against numpy.fft, through pty_fft2_dev."""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N", [32, 64, 128, 256, 512])
@pytest.mark.parametrize("inverse", [False, True])
def test_fft2_matches_numpy(N, inverse):
    import torch

    from ptychopy_b200 import abi

    rng = np.random.default_rng(N + inverse)
    a = (rng.standard_normal((3, N, N)) + 1j * rng.standard_normal((3, N, N))).astype(np.complex64)
    d = torch.from_numpy(a.view(np.float32)).cuda()
    w = torch.empty_like(d)
    abi.fft2_dev(d.data_ptr(), w.data_ptr(), 3, N, inverse=inverse)
    torch.cuda.synchronize()
    got = d.cpu().numpy().view(np.complex64)
    ref = np.fft.ifft2(a.astype(np.complex128)) * N * N if inverse else np.fft.fft2(a.astype(np.complex128))
    assert rel_err(got, ref) < 3e-6


def test_fft2_roundtrip_identity():
    import torch

    from ptychopy_b200 import abi

    N = 256
    rng = np.random.default_rng(7)
    a = (rng.standard_normal((2, N, N)) + 1j * rng.standard_normal((2, N, N))).astype(np.complex64)
    d = torch.from_numpy(a.view(np.float32).copy()).cuda()
    w = torch.empty_like(d)
    abi.fft2_dev(d.data_ptr(), w.data_ptr(), 2, N)
    abi.fft2_dev(d.data_ptr(), w.data_ptr(), 2, N, inverse=True)
    torch.cuda.synchronize()
    got = d.cpu().numpy().view(np.complex64) / (N * N)
    assert rel_err(got, a) < 3e-6
