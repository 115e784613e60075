"""Split-BF16 tensor-core 2-D FFT (pty_fft2_tc) against numpy's FP64 FFT, beside the engine's FP32 FFT: the
mixed-precision result is reported with its measured error, not held to the FP32 bound."""
import ctypes

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


def _run(a, inverse):
    import torch

    from ptychopy_b200 import abi

    L = abi.lib()
    batch, N = a.shape[0], a.shape[1]
    d = torch.from_numpy(a.view(np.float32).copy()).cuda()
    w = torch.empty_like(d)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    abi.check(L.pty_fft2_tc(ctypes.c_void_p(d.data_ptr()), ctypes.c_void_p(w.data_ptr()), batch, N, int(inverse),
                            ctypes.c_void_p(err.data_ptr()), None))
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    tc = d.cpu().numpy().view(np.complex64)
    ref32 = torch.from_numpy(a.view(np.float32).copy()).cuda()
    abi.fft2_dev(ref32.data_ptr(), w.data_ptr(), batch, N, inverse=inverse)
    torch.cuda.synchronize()
    return tc, ref32.cpu().numpy().view(np.complex64)


@pytest.mark.parametrize("inverse", [False, True])
def test_fft2_tc_error_vs_fp64(inverse):
    rng = np.random.default_rng(40 + int(inverse))
    a = (rng.standard_normal((3, 256, 256)) + 1j * rng.standard_normal((3, 256, 256))).astype(np.complex64)
    tc, f32 = _run(a, inverse)
    a64 = a.astype(np.complex128)
    exact = np.fft.ifft2(a64) * 256 * 256 if inverse else np.fft.fft2(a64)
    e_tc, e_32 = rel_err(tc, exact), rel_err(f32, exact)
    print(f"inverse={inverse}: split-BF16 tensor-core FFT rel err {e_tc:.2e}, FP32 FFT {e_32:.2e}")
    assert e_32 < 3e-6
    assert e_tc < 5e-5  # ~16 mantissa bits per operand through four GEMM stages


def test_fft2_tc_pattern_like_data():
    """Diffraction-like dynamic range: an exit wave of a probe on a random object, forward then inverse."""
    from ptychopy_b200 import synth

    rng = np.random.default_rng(3)
    N = 256
    dx_s = synth.sample_pixel(1.409e-10, 1.92, 75e-6, N)
    probe = synth.make_probe(N, dx_s, K=1)[0]
    obj = synth.make_object(N, N, rng)
    psi = (probe * obj)[None].astype(np.complex64)
    tc, f32 = _run(psi, False)
    exact = np.fft.fft2(psi.astype(np.complex128))
    assert rel_err(tc, exact) < 5e-5
    back, _ = _run(tc.astype(np.complex64), True)
    assert rel_err(back / (N * N), psi.astype(np.complex128)) < 1e-4
