"""Reference DM on the GPU against the FP64 oracle (relative object/probe error <= 1e-4)."""
import numpy as np
import pytest

from conftest import rel_err
from gpu_helpers import dataset, gpu_session

pytestmark = pytest.mark.gpu
TOL = 1e-4


@pytest.mark.parametrize("N,nx", [(64, 5), (128, 4), (32, 6)])
def test_dm_matches_oracle(oracle, N, nx):
    d = dataset(N=N, nx=nx, algorithm="DM")
    s = gpu_session(d, probe=d["probe"], updateProbe=3, phaseConstraint=1)
    pos = s.positions()
    assert np.array_equal(pos, d["pos"])
    o = oracle.OracleSession("DM", d["amp"], pos, np.zeros((d["X"], d["Y"])), d["probe"], probe_guess_path=False,
                             updateProbe=3, phaseConstraint=1)
    for it in range(1, 7):
        s.step()
        o.step()
        if it in (1, 2, 3, 6):
            ob, pr, _ = o.state()
            assert rel_err(s.object(), ob) < TOL, f"object, iteration {it}"
            assert rel_err(s.probe(), pr) < TOL, f"probe, iteration {it}"


def test_dm_probe_guess_and_wave_split(oracle):
    # probe guess on the device vs the oracle's, then DM with a wave size that does not divide the pattern count.
    # The DM run starts both sides from the device's guess: the reference's phase constraint clamps increments
    # with arg > 0 (discontinuous at arg = pi), and the guess has near-zero regions whose phase is set by
    # round-off, so FP32 and FP64 guesses would legitimately diverge there in the first iteration.
    d = dataset(N=64, nx=5, algorithm="DM")
    s = gpu_session(d, wave=7, updateProbe=2)
    g = oracle.probe_guess(d["amp"], d["kw"]["beamSize"], d["dx_s"], K=1)
    assert rel_err(s.probe(), g) < 1e-5
    o = oracle.OracleSession("DM", d["amp"], d["pos"], np.zeros((d["X"], d["Y"])), s.probe(), probe_guess_path=True,
                             updateProbe=2)
    for _ in range(4):
        s.step()
        o.step()
    ob, pr, _ = o.state()
    assert rel_err(s.object(), ob) < TOL and rel_err(s.probe(), pr) < TOL


def test_dm_full_window_512(oracle):
    # full detector size of the DM configuration (512^2), fewer positions so the oracle finishes in seconds
    d = dataset(N=512, nx=3, step=50e-9, algorithm="DM", fwhm_px=39.0)
    s = gpu_session(d, probe=d["probe"], updateProbe=2)
    o = oracle.OracleSession("DM", d["amp"], d["pos"], np.zeros((d["X"], d["Y"])), d["probe"],
                             probe_guess_path=False, updateProbe=2, nthreads=8)
    for _ in range(3):
        s.step()
        o.step()
    ob, pr, _ = o.state()
    assert rel_err(s.object(), ob) < TOL and rel_err(s.probe(), pr) < TOL


def test_dm_config_size_first_iteration():
    # 30x30 positions at 512^2 (the DM benchmark size): the first iteration has the closed form
    # O_1 = sum_j clamp(conj(P) IFFT2(A_j)) at the rounded offsets (zero object, zero exit waves, probeMax = 1)
    from ptychopy_b200 import synth

    ds = synth.make_dataset("dm512", seed=3)
    s = gpu_session(dict(amp=ds["amp"], kw=dict(ds["kwargs"], algorithm="DM")), probe=ds["probe_true"])
    s.step()
    got = s.object()
    N = 512
    P = np.conj(ds["probe_true"][0]).astype(np.complex128)
    exp = np.zeros((ds["X"], ds["Y"]), np.complex128)
    for j, q in enumerate(ds["pos"]):
        ox, oy = np.round(q).astype(int)
        inc = P * np.fft.ifft2(ds["amp"][j].astype(np.float64))
        inc = np.where(np.angle(inc) > 0, np.abs(inc), inc)
        exp[ox:ox + N, oy:oy + N] += inc
    assert np.isfinite(got).all()
    assert rel_err(got, exp) < TOL
