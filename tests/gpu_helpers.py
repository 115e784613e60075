"""Shared set-up of the GPU parity tests: seeded small datasets and matching GPU / oracle sessions."""
import numpy as np

from ptychopy_b200 import abi, synth


def dataset(N=64, nx=5, step=40e-9, K=1, seed=11, photons=1e6, fwhm_px=10.0, algorithm="ePIE"):
    rng = np.random.default_rng(seed)
    lambd, z, dx_d = 2.48e-10, 1.0, 172e-6
    dx_s = synth.sample_pixel(lambd, z, dx_d, N)
    pos, X, Y = synth.raster_positions(nx, nx, step, step, dx_s, N)
    obj = synth.make_object(X, Y, rng, corr_px=4.0)
    probe = synth.make_probe(N, dx_s, K=K, fwhm=fwhm_px * dx_s)
    amp = synth.make_patterns(obj, probe, pos, N, photons, rng)
    kw = dict(size=N, scanDimsx=nx, scanDimsy=nx, stepx=step, stepy=step, lambd=lambd, z=z, dx_d=dx_d,
              beamSize=fwhm_px * dx_s, probeModes=K, algorithm=algorithm)
    return dict(amp=amp, pos=pos, X=X, Y=Y, obj=obj, probe=probe, dx_s=dx_s, kw=kw)


def gpu_session(d, probe=None, obj=None, **params):
    kw = dict(d["kw"])
    kw.update(params)
    s = abi.Session(**kw)
    s.set_patterns(d["amp"])
    if probe is not None:
        s.set_probe(probe)
    if obj is not None:
        s.set_object(obj)
    s.init()
    return s


def subpixel_shifts(raw, X, Y, N):
    """Row and column remainders of the ML positions after rounding to the window grid (find_reconstruction_ROI)."""
    cvx = np.float32(np.ceil(X / 2 - N / 2))
    cvy = np.float32(np.ceil(Y / 2 - N / 2))
    p1 = raw[:, 0].astype(np.float32) + cvx
    p2 = raw[:, 1].astype(np.float32) + cvy
    sy = (p1 - np.sign(p1) * np.floor(np.abs(p1) + 0.5)).astype(np.float64)
    sx = (p2 - np.sign(p2) * np.floor(np.abs(p2) + 0.5)).astype(np.float64)
    return sx, sy


def shifted_probe(probe, sx, sy):
    """probe(r - sy, c - sx) by the Fourier shift theorem (shift_probe)."""
    N = probe.shape[-1]
    f = np.fft.fftfreq(N)
    return np.fft.ifft2(np.fft.fft2(probe) * np.exp(-2j * np.pi * (sx * f[None, :] + sy * f[:, None])))


def mls_dataset(oracle, N=64, nx=5, step=40e-9, seed=3, pert=0.1, shifted=False, probe=None):
    """Noise-free MLs case on the ML mesh: intensities |FFT2(P O_true[window])|^2 at the ML window starts, the
    start object O_true with a smooth perturbation of relative size `pert`.  Data consistent with the model keep
    |Psi| far above FFT round-off wherever the data are non-zero, so FP32 and FP64 runs stay within round-off of each
    other; with Poisson data and a flat start the modulus step A/(|Psi| + 1e-9) turns the round-off phase of
    near-zero Psi into O(1) differences.  shifted=True: the probe of each window is shifted by the position's
    sub-pixel remainder, the forward model of the reference's default MLs path."""
    rng = np.random.default_rng(seed)
    lambd, z, dx_d = 2.48e-10, 1.0, 172e-6
    dx_s = synth.sample_pixel(lambd, z, dx_d, N)
    raw = oracle.mls_raw_positions(nx, nx, step, step, dx_s)
    X, Y, starts, roi = oracle.mls_geometry(raw, N)
    o_true = synth.make_object(X, Y, rng, corr_px=4.0).astype(np.complex128)
    if probe is None:
        probe = synth.make_probe(N, dx_s, K=1, fwhm=10 * dx_s)[0]
    probe = np.asarray(probe, np.complex128)
    if shifted:
        sx, sy = subpixel_shifts(raw, X, Y, N)
        intens = np.stack([np.abs(np.fft.fft2(shifted_probe(probe, sx[k], sy[k]) * o_true[r:r + N, c:c + N])) ** 2
                           for k, (r, c) in enumerate(starts)])
    else:
        intens = np.stack([np.abs(np.fft.fft2(probe * o_true[r:r + N, c:c + N])) ** 2 for r, c in starts])
    o0 = (o_true * (1 + pert * synth.make_object(X, Y, rng, corr_px=8.0) - pert)).astype(np.complex64)
    kw = dict(size=N, scanDimsx=nx, scanDimsy=nx, stepx=step, stepy=step, lambd=lambd, z=z, dx_d=dx_d,
              beamSize=10 * dx_s, probeModes=1, algorithm="MLs")
    return dict(intens=intens.astype(np.float32), raw=raw, X=X, Y=Y, starts=starts, roi=roi, obj=o0,
                probe=probe.astype(np.complex64), dx_s=dx_s, kw=kw)
