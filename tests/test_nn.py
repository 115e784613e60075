"""The warm-start network's CPU reference (oracle/nn_ref.py) against finite differences, and the ctypes surface of
its CUDA kernels (loaded, no GPU needed)."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "oracle"))
import nn_ref  # noqa: E402


def _fd(f, a, eps=1e-6):
    g = np.zeros_like(a)
    it = np.nditer(a, flags=["multi_index"])
    for _ in it:
        i = it.multi_index
        old = a[i]
        a[i] = old + eps
        fp = f()
        a[i] = old - eps
        fm = f()
        a[i] = old
        g[i] = (fp - fm) / (2 * eps)
    return g


def test_conv3x3_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    x = rng.standard_normal((2, 3, 5, 6))
    w = rng.standard_normal((4, 3, 3, 3))
    b = rng.standard_normal(4)
    r = rng.standard_normal((2, 4, 5, 6))
    f = lambda: float((nn_ref.conv3x3(x, w, b) * r).sum())  # noqa: E731
    dx, dw, db = nn_ref.conv3x3_bwd(x, w, r)
    assert np.allclose(dx, _fd(f, x), atol=1e-6)
    assert np.allclose(dw, _fd(f, w), atol=1e-6)
    assert np.allclose(db, _fd(f, b), atol=1e-6)


def test_pool_up_mse_gradients():
    rng = np.random.default_rng(1)
    x = rng.standard_normal((1, 2, 4, 6))
    r = rng.standard_normal((1, 2, 2, 3))
    assert np.allclose(nn_ref.pool2_bwd(r), _fd(lambda: float((nn_ref.pool2(x) * r).sum()), x), atol=1e-7)
    r2 = rng.standard_normal((1, 2, 8, 12))
    assert np.allclose(nn_ref.up2_bwd(r2), _fd(lambda: float((nn_ref.up2(x) * r2).sum()), x), atol=1e-7)
    t = rng.standard_normal(x.shape)
    loss, g = nn_ref.mse(x, t)
    assert np.allclose(g, _fd(lambda: nn_ref.mse(x, t)[0], x), atol=1e-7)


def test_kernel_symbols_exported():
    from ptychopy_b200 import abi

    L = abi.lib()
    for name in ["pty_nn_conv3x3", "pty_nn_conv3x3_bwd", "pty_nn_relu", "pty_nn_relu_bwd", "pty_nn_pool2",
                 "pty_nn_pool2_bwd", "pty_nn_up2", "pty_nn_up2_bwd", "pty_nn_mse", "pty_nn_adam"]:
        assert hasattr(L, name)


def test_kernel_entry_points_reject_bad_arguments():
    """Null pointers and empty sizes are refused before any launch (no GPU needed)."""
    import ctypes

    from ptychopy_b200 import abi

    L = abi.lib()
    assert L.pty_nn_relu(None, 10, None) == abi.PTY_ERR_INVALID
    assert L.pty_nn_pool2(None, None, 1, 2, 2, None) == abi.PTY_ERR_INVALID
    assert L.pty_nn_conv3x3(None, None, None, None, 1, 1, 1, 4, 4, 0, None) == abi.PTY_ERR_INVALID
    assert L.pty_nn_adam(None, None, None, None, 0, 1e-3, 0.9, 0.999, 1e-8, 1, None) == abi.PTY_ERR_INVALID
    assert L.pty_tc_conv3x3(None, None, None, None, 1, 16, 16, 8, 8, 0, 0, 0, 1.0, None, None) == abi.PTY_ERR_INVALID
    assert L.pty_tc_pool2(None, None, 1, 2, 2, 8, None) == abi.PTY_ERR_INVALID
    assert L.pty_tc_weights_size(16, 300) == -1  # Cout above 256
    assert L.pty_warm_stitch(None, None, 0, None, 32, 128, 0.9, 0.1, 0.2, None, 10, 10, None) == abi.PTY_ERR_INVALID
    assert L.pty_fft2_tc(None, None, 1, 128, 0, None, None) == abi.PTY_ERR_INVALID
    assert b"bad argument" in L.pty_last_error()
    codes = (ctypes.c_int * 4)()
    assert L.pty_selftest_bounded_waits(None) == abi.PTY_ERR_INVALID
    del codes
