"""The benchmark configurations at their full sizes against the FP64 oracle (multithreaded over the host's cores).

config 0: ePIE, 10 x 10 raster at 128^2, 20 iterations, the probe updating from iteration 10 (the reference
          defaults), starting from the mean-amplitude probe guess;
config 1: DM, 30 x 30 raster (900 positions) at 512^2, the probe updating from iteration 2, three iterations;
config 2: ePIE with 5 Hermite-Gauss probe modes, 51 x 51 raster (2601 positions) at 256^2, one iteration with the
          modes and the probe updating, FP32 (1e-4) and the split-BF16 tensor-core transforms (error stated);
MLs:      the reference's default path (variable probe, position search) at the DM configuration's 512^2 window.
Patterns are simulated on the device (synth.make_patterns_torch) and Poisson-sampled.

Where the reference's method itself amplifies round-off (measured with the oracle's own FP32 instance against its
FP64 one), the tests say so and bound the engine by that amplification instead of by TOL.
"""
import os

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-4
NT = max(1, os.cpu_count() or 1)


def _dataset(name, seed=20261203, **override):
    from ptychopy_b200 import synth

    cfg = dict(synth.CONFIGS[name])
    cfg.update(override)
    rng = np.random.default_rng(seed)
    N = cfg["N"]
    dx_s = synth.sample_pixel(cfg["lambd"], cfg["z"], cfg["dx_d"], N)
    pos, X, Y = synth.raster_positions(cfg["nx"], cfg["ny"], cfg["step"], cfg["step"], dx_s, N)
    obj = synth.make_object(X, Y, rng)
    probe = synth.make_probe(N, dx_s, K=cfg["K"])
    amp = synth.make_patterns_torch(obj, probe, pos, N, cfg["photons"], seed,
                                    intensities=cfg["algorithm"] == "MLs").cpu().numpy()
    kw = dict(size=N, scanDimsx=cfg["nx"], scanDimsy=cfg["ny"], stepx=cfg["step"], stepy=cfg["step"],
              lambd=cfg["lambd"], z=cfg["z"], dx_d=cfg["dx_d"], beamSize=synth.BEAM_FWHM, probeModes=cfg["K"],
              algorithm=cfg["algorithm"])
    return dict(cfg=cfg, amp=amp, pos=pos, X=X, Y=Y, obj=obj, probe=probe, dx_s=dx_s, kw=kw)


def _session(d, probe=None, obj=None, **params):
    from ptychopy_b200 import abi

    s = abi.Session(**dict(d["kw"], **params))
    s.set_patterns(d["amp"])
    if probe is not None:
        s.set_probe(probe)
    if obj is not None:
        s.set_object(obj)
    s.init()
    return s


def test_config0_epie_full_run(oracle):
    """20 iterations from the probe guess and a zero object, as the reference runs them by default.  Until the probe
    starts updating (iteration 10) the engine matches the FP64 oracle to TOL.  From there on the method amplifies
    round-off (the probe update on Poisson data: the oracle's own FP32 instance departs from its FP64 one by ~1e-3
    at iteration 10 and ~1e-2 by iteration 20), so the engine is held to three times the FP32 oracle's own
    departure (floors TOL for object and probe, 1e-5 for the error metric): numerically equivalent to an FP32
    implementation of the same equations."""
    d = _dataset("epie128")
    s = _session(d, calculateRMS=1, seed=41)
    assert np.array_equal(s.positions(), d["pos"])
    guess = s.probe()
    runs = {fp32: oracle.OracleSession("ePIE", d["amp"], d["pos"], np.zeros((d["X"], d["Y"])),
                                       guess.astype(np.complex64) if fp32 else guess, probe_guess_path=True,
                                       calculateRMS=1, seed=41, nthreads=NT, fp32=fp32) for fp32 in (False, True)}
    for it in range(1, 21):
        e = s.step()
        eo = {fp32: o.step() for fp32, o in runs.items()}
        if it in (1, 5, 9, 10, 11, 15, 20):
            (ob, pr, _), (ob32, pr32, _) = runs[False].state(), runs[True].state()
            dev = (rel_err(s.object(), ob), rel_err(s.probe(), pr), abs(e - eo[False]) / eo[False])
            dev32 = (rel_err(ob32, ob), rel_err(pr32, pr), abs(eo[True] - eo[False]) / eo[False])
            print(f"config 0 iteration {it}: engine vs FP64 object {dev[0]:.2e} probe {dev[1]:.2e} error metric "
                  f"{dev[2]:.2e}; FP32 oracle vs FP64 {dev32[0]:.2e} {dev32[1]:.2e} {dev32[2]:.2e}")
            if it < 10:
                assert dev[0] < TOL and dev[1] < TOL and dev[2] < 1e-6, f"iteration {it}"
            else:
                for a, b, floor in zip(dev, dev32, (TOL, TOL, 1e-5)):
                    assert a <= max(floor, 3 * b), f"iteration {it}"
    s.close()
    for o in runs.values():
        o.close()


def test_config1_dm_full_size(oracle):
    """900 patterns of 512^2, three iterations, the probe updating from iteration 2.  Without the phase constraint
    the iteration is well conditioned (the oracle's FP32 instance stays within 3e-6 of FP64) and the engine is held
    to TOL.  The phase constraint clamps increments with arg > 0 to the positive real axis, a jump at arg = pi that
    FP32 round-off decides for the few increments lying within round-off of it (the oracle's FP32 instance departs by
    ~7e-5 from FP64 in its first iteration at this size); that run is checked to 1e-3."""
    d = _dataset("dm512")
    for pc, tol, iters in ((0, TOL, 3), (1, 1e-3, 1)):
        s = _session(d, probe=d["probe"], updateProbe=2, phaseConstraint=pc)
        o = oracle.OracleSession("DM", d["amp"], d["pos"], np.zeros((d["X"], d["Y"])), d["probe"],
                                 probe_guess_path=False, updateProbe=2, phaseConstraint=pc, nthreads=NT)
        for it in range(1, iters + 1):
            s.step()
            o.step()
            ob, pr, _ = o.state()
            eo_, ep_ = rel_err(s.object(), ob), rel_err(s.probe(), pr)
            print(f"config 1 (900 x 512^2) phaseConstraint={pc} iteration {it}: object {eo_:.2e}, probe {ep_:.2e}")
            assert eo_ < tol and ep_ < tol, f"phaseConstraint={pc}, iteration {it}"
        s.close()
        o.close()


def test_config2_epie_five_modes_full_size(oracle):
    """2601 patterns of 256^2 with 5 probe modes, one iteration with the modes and the probe updating, from the
    object 0.5 (O_true + 1) (far-from-solution starts put many pixels where |Psi| is at round-off level, whose phase
    the modulus step then copies into the update: there the method itself is chaotic), no phase constraint."""
    d = _dataset("epie256k5")
    kw = dict(updateProbe=1, updateModes=1, calculateRMS=1, seed=13, phaseConstraint=0)
    start = (0.5 * d["obj"] + 0.5).astype(np.complex64)
    runs = {prec: _session(d, probe=d["probe"], obj=start, precision=prec, **kw) for prec in (0, 1)}
    o = oracle.OracleSession("ePIE", d["amp"], d["pos"], start, d["probe"], probe_guess_path=False, modes_given=True,
                             nthreads=NT, **kw)
    errs = {prec: s.step() for prec, s in runs.items()}
    eo = o.step()
    ob, pr, _ = o.state()
    res = {prec: (rel_err(s.object(), ob), rel_err(s.probe(), pr), abs(errs[prec] - eo) / eo)
           for prec, s in runs.items()}
    print(f"config 2 (2601 x 256^2, 5 modes), one iteration vs FP64: FP32 object {res[0][0]:.2e} probe "
          f"{res[0][1]:.2e} error metric {res[0][2]:.2e}; split-BF16 tensor-core transforms object {res[1][0]:.2e} "
          f"probe {res[1][1]:.2e} error metric {res[1][2]:.2e}")
    assert res[0][0] < TOL and res[0][1] < TOL and res[0][2] < 1e-6
    assert res[1][0] < 2e-3 and res[1][1] < 2e-3 and res[1][2] < 2e-3
    for s in runs.values():
        s.close()
    o.close()


def test_mls_default_path_512(oracle):
    """The reference's default MLs path at the 512^2 window (model-consistent data; see test_gpu_mls.py)."""
    from gpu_helpers import gpu_session, mls_dataset

    d = mls_dataset(oracle, N=512, nx=3, step=50e-9, shifted=True)
    s = gpu_session(dict(amp=d["intens"], kw=d["kw"]), probe=d["probe"], obj=d["obj"], calculateRMS=1, PPS=2)
    o = oracle.OracleMls(d["raw"], d["intens"], d["probe"], obj=d["obj"], variable=1, PPS=2)
    for it in range(1, 4):
        e = s.step()
        eo = o.step()
        ob, pr, _ = o.state()
        eo_, ep_ = rel_err(s.object(), ob), rel_err(s.probe(), pr)
        print(f"MLs 512^2 iteration {it}: object {eo_:.2e}, probe {ep_:.2e}, error metric {abs(e - eo) / eo:.2e}")
        assert eo_ < TOL and ep_ < TOL, f"iteration {it}"
        assert abs(e - eo) <= 1e-5 * abs(eo)
    s.close()
