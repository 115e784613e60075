"""Forward model of simulation mode (pty_simulate) against the oracle's bilinear patch and numpy's FFT."""
import numpy as np
import pytest

from conftest import rel_err
from ptychopy_b200 import abi, synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N", [32, 128, 256])
def test_simulate_matches_oracle(oracle, N):
    rng = np.random.default_rng(N)
    X = Y = N + 40
    obj = synth.make_object(X, Y, rng)
    probe = synth.make_probe(N, 10e-9, K=1, fwhm=8 * 10e-9)[0]
    pos = (rng.random((7, 2)) * 39).astype(np.float32)  # fractional positions inside the object
    amp = abi.simulate(obj, probe, pos)
    assert amp.shape == (7, N, N)
    for i, (qx, qy) in enumerate(pos):
        patch = oracle.extract_patch(obj, float(qx), float(qy), N)
        ref = np.abs(np.fft.fft2(patch * probe.astype(np.complex128)))
        assert rel_err(amp[i], ref) < 1e-5


def test_simulate_rejects_negative_positions():
    obj = np.ones((64, 64), np.complex64)
    probe = np.ones((32, 32), np.complex64)
    with pytest.raises(abi.PtyError):
        abi.simulate(obj, probe, np.array([[-1.0, 0.0]], np.float32))
