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
