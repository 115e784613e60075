"""Regenerates the golden fixtures in this directory from the oracle (oracle/oracle.cpp).

    python tests/golden/make_golden.py

Each .npz holds the inputs (seeded synthetic amplitudes, positions, starting probe) and the oracle's FP64 results
after a few iterations.  The reference ships no golden vectors and does not build, so these fixtures pin the
restatement itself: tests/test_golden.py re-runs the oracle on the stored inputs (CPU) and checks the CUDA path
against the stored results (GPU).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import pyoracle  # noqa: E402

from ptychopy_b200 import synth  # noqa: E402

CASES = {
    # name: (algorithm, N, nx, K, iterations, schedule, given modes)
    "epie_n32": ("ePIE", 32, 4, 1, 3, dict(updateProbe=2, calculateRMS=1, seed=99), False),
    "dm_n32": ("DM", 32, 4, 1, 3, dict(updateProbe=2), False),
    "epie_modes_n32": ("ePIE", 32, 4, 2, 3, dict(updateProbe=2, updateModes=2, calculateRMS=1, seed=5), True),
    "epie_guess_n64": ("ePIE", 64, 3, 1, 2, dict(updateProbe=1, seed=1), None),
}


# MLs on the reference's default path: name -> (N, nx, probe modes, PPS, iterations)
MLS_CASES = {
    "mls_default_n32": (32, 6, 2, 2, 4),
}


def inputs(N, nx, K, seed=4242):
    rng = np.random.default_rng(seed)
    lambd, z, dx_d, step = 2.48e-10, 1.0, 172e-6, 40e-9
    dx_s = synth.sample_pixel(lambd, z, dx_d, N)
    pos, X, Y = synth.raster_positions(nx, nx, step, step, dx_s, N)
    obj = synth.make_object(X, Y, rng, corr_px=3.0)
    probe = synth.make_probe(N, dx_s, K=K, fwhm=6 * dx_s)
    amp = synth.make_patterns(obj, probe, pos, N, 1e5, rng)
    params = dict(size=N, scanDimsx=nx, scanDimsy=nx, stepx=step, stepy=step, lambd=lambd, z=z, dx_d=dx_d,
                  beamSize=6 * dx_s, probeModes=K)
    return amp, pos, X, Y, probe, params, dx_s


def make(name):
    algo, N, nx, K, iters, sched, modes = CASES[name]
    amp, pos, X, Y, probe, params, dx_s = inputs(N, nx, K)
    if modes is None:  # probe from the guess
        start = pyoracle.probe_guess(amp, params["beamSize"], dx_s, K=K)
        guess = True
    else:
        start = probe.astype(np.complex128) if modes else np.concatenate(
            [probe[:1], np.zeros_like(probe[1:])]).astype(np.complex128)
        guess = False
    kw = {k: v for k, v in sched.items()}
    o = pyoracle.OracleSession(algo, amp, pos, np.zeros((X, Y)), start, probe_guess_path=guess,
                               modes_given=bool(modes), **kw)
    errs = [o.step() for _ in range(iters)]
    ob, pr, sc = o.state()
    np.savez_compressed(os.path.join(HERE, name + ".npz"), amp=amp, pos=pos, probe_start=start.astype(np.complex128),
                        object=ob, probe=pr, errors=np.array(errs), scalars=sc, algorithm=algo,
                        iterations=iters, guess=guess, modes_given=bool(modes),
                        params=np.array(repr(dict(params, algorithm=algo, **sched))))


def make_mls(name):
    """Noise-free intensities of the shifted-probe model (gpu_helpers.mls_dataset), the oracle's default MLs path with
    probe modes, the position search from iteration PPS and the variable-probe update from iteration 3."""
    sys.path.insert(0, os.path.dirname(HERE))
    from gpu_helpers import mls_dataset

    N, nx, K, pps, iters = MLS_CASES[name]
    d = mls_dataset(pyoracle, N=N, nx=nx, shifted=True, seed=8)
    o = pyoracle.OracleMls(d["raw"], d["intens"], d["probe"], obj=d["obj"], variable=1, PPS=pps, K=K)
    errs = [o.step() for _ in range(iters)]
    ob, pr, _ = o.state()
    E, e0, e1, pos = o.variable_state()
    np.savez_compressed(os.path.join(HERE, name + ".npz"), intens=d["intens"], raw=d["raw"],
                        probe_start=d["probe"].astype(np.complex64), obj_start=d["obj"], object=ob, probe=pr,
                        extra_mode=E, evo0=e0, evo1=e1, positions=pos, errors=np.array(errs), iterations=iters,
                        params=np.array(repr(dict(d["kw"], probeModes=K, PPS=pps, calculateRMS=1))))


if __name__ == "__main__":
    for n in CASES:
        make(n)
        print("wrote", n)
    for n in MLS_CASES:
        make_mls(n)
        print("wrote", n)
