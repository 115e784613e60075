"""pty_fft2_dev_noalloc: the batched 2-D FFT without any device allocation.

For callers that cannot call cudaMalloc (a host that owns all device memory up front and forbids allocation
afterwards): the entry point keeps its work buffer in a static device array of the library.  These tests call it
through the C ABI and check it against the allocating entry point pty_fft2_dev on two calls in a row, against numpy
at every supported size (one call on a non-default stream) with the device's free memory unchanged across a round
of calls, and that a request larger than the 8 MiB scratch is refused.  The file is collected last.
"""
import ctypes

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


def _random(batch, N, seed):
    rng = np.random.default_rng(seed)
    return (rng.standard_normal((batch, N, N)) + 1j * rng.standard_normal((batch, N, N))).astype(np.complex64)


def test_no_alloc_fft_matches_allocating_entry_point():
    import torch

    from ptychopy_b200 import abi

    lib = abi.lib()
    for k, (N, batch, inverse) in enumerate([(256, 3, False), (512, 2, True)]):  # two calls in a row
        a = _random(batch, N, 100 + k)
        ref = torch.from_numpy(a.view(np.float32).copy()).cuda()
        work = torch.empty_like(ref)
        abi.fft2_dev(ref.data_ptr(), work.data_ptr(), batch, N, inverse=inverse)
        got = torch.from_numpy(a.view(np.float32).copy()).cuda()
        rc = lib.pty_fft2_dev_noalloc(ctypes.c_void_p(got.data_ptr()), batch, N, int(inverse), None)
        assert rc == abi.PTY_OK, lib.pty_last_error().decode()
        torch.cuda.synchronize()
        g = got.cpu().numpy().view(np.complex64)
        r = ref.cpu().numpy().view(np.complex64)
        assert rel_err(g, r) < 3e-6
        exact = np.fft.ifft2(a.astype(np.complex128)) * N * N if inverse else np.fft.fft2(a.astype(np.complex128))
        assert rel_err(g, exact) < 3e-6


def test_no_alloc_fft_all_sizes_leave_device_memory_unchanged():
    """A first round of calls, one per size, brings the static scratch and each size's kernels onto the GPU (CUDA
    loads device code lazily); a second round, one call on a non-default stream, then changes the device's free
    memory by nothing: nothing is allocated.  The second round's results are checked against numpy."""
    import torch

    from ptychopy_b200 import abi

    lib = abi.lib()
    cases = [(32, 40, False), (64, 20, True), (128, 9, False), (256, 4, True), (512, 2, False)]

    def upload():
        return [torch.from_numpy(_random(b, N, 200 + N).view(np.float32).copy()).cuda() for N, b, _ in cases]

    def run(datas, side=None):
        for k, ((N, batch, inverse), d) in enumerate(zip(cases, datas)):
            stream = ctypes.c_void_p(side.cuda_stream) if side is not None and k == 2 else None
            if stream is not None:
                # calls share the static scratch, so they must not overlap: the side stream (non-blocking) waits
                # for the calls already queued on the default stream
                side.wait_stream(torch.cuda.current_stream())
            rc = lib.pty_fft2_dev_noalloc(ctypes.c_void_p(d.data_ptr()), batch, N, int(inverse), stream)
            assert rc == abi.PTY_OK, lib.pty_last_error().decode()
            if stream is not None:
                side.synchronize()
        torch.cuda.synchronize()

    run(upload())
    datas = upload()
    side = torch.cuda.Stream()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    run(datas, side)
    assert torch.cuda.mem_get_info()[0] == free0
    for (N, batch, inverse), d in zip(cases, datas):
        a = _random(batch, N, 200 + N).astype(np.complex128)
        exact = np.fft.ifft2(a) * N * N if inverse else np.fft.fft2(a)
        assert rel_err(d.cpu().numpy().view(np.complex64), exact) < 3e-6, N


def test_no_alloc_fft_rejects_oversize_requests():
    import torch

    from ptychopy_b200 import abi

    lib = abi.lib()
    d = torch.zeros((5, 512, 512, 2), dtype=torch.float32, device="cuda")  # 10 MiB > 8 MiB
    rc = lib.pty_fft2_dev_noalloc(ctypes.c_void_p(d.data_ptr()), 5, 512, 0, None)
    assert rc == abi.PTY_ERR_INVALID
    assert b"8 MiB" in lib.pty_last_error()
