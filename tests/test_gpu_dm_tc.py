"""DM with precision=1 at 512^2: the column pass (forward transform along x, modulus step, inverse transform along x)
computes its 32-point DFT stages as FP16-split tcgen05 GEMMs (kernels_dm_tc.cu).  The iteration is checked against
the FP64 oracle to the same 1e-4 as the FP32 path, and the departures of both paths are printed side by side."""
import os
import time

import numpy as np
import pytest

from conftest import rel_err
from test_gpu_configs import _dataset, _session

pytestmark = pytest.mark.gpu
TOL = 1e-4
NT = max(1, os.cpu_count() or 1)


@pytest.mark.parametrize("nx", [3, 30])
def test_dm_precision1_vs_fp64(oracle, nx):
    d = _dataset("dm512", nx=nx, ny=nx)
    iters = 3 if nx == 3 else 1
    o = oracle.OracleSession("DM", d["amp"], d["pos"], np.zeros((d["X"], d["Y"])), d["probe"],
                             probe_guess_path=False, updateProbe=2, phaseConstraint=0, nthreads=NT)
    runs = {pr: _session(d, probe=d["probe"], updateProbe=2, phaseConstraint=0, precision=pr) for pr in (0, 1)}
    for it in range(1, iters + 1):
        o.step()
        ob, pb, _ = o.state()
        for pr, s in runs.items():
            s.step()
            eo_, ep_ = rel_err(s.object(), ob), rel_err(s.probe(), pb)
            print(f"DM {nx}x{nx} x 512^2 precision={pr} iteration {it}: object {eo_:.2e}, probe {ep_:.2e}")
            assert eo_ < TOL and ep_ < TOL, f"precision={pr}, iteration {it}"
    for s in runs.values():
        s.close()
    o.close()


def test_dm_precision1_phase_constraint():
    """With the phase constraint the two paths agree to the constraint's round-off conditioning (1e-3, as for the
    FP32 path against the oracle)."""
    d = _dataset("dm512", nx=6, ny=6)
    runs = {pr: _session(d, probe=d["probe"], updateProbe=2, phaseConstraint=1, precision=pr) for pr in (0, 1)}
    for s in runs.values():
        s.run(2)
    e = rel_err(runs[1].object(), runs[0].object())
    print(f"DM 6x6 x 512^2 phaseConstraint=1, 2 iterations: precision=1 vs precision=0 object {e:.2e}")
    assert e < 1e-3
    for s in runs.values():
        s.close()


def test_dm_precision1_iteration_time():
    """Both paths on the 900 x 512^2 configuration: iteration time (CUDA-graph replays, device-synchronised)."""
    d = _dataset("dm512")
    out = {}
    for pr in (0, 1):
        s = _session(d, probe=d["probe"], updateProbe=2, phaseConstraint=0, precision=pr)
        s.run(3)
        t0 = time.perf_counter()
        s.run(10)
        out[pr] = (time.perf_counter() - t0) / 10 * 1e3
        s.close()
    print(f"DM 900 x 512^2 iteration: precision=0 {out[0]:.3f} ms, precision=1 {out[1]:.3f} ms")
    assert out[1] > 0 and out[0] > 0


def test_dm_precision1_refused_off_512():
    from ptychopy_b200 import abi

    d = _dataset("dm512", N=256, nx=3, ny=3)
    with pytest.raises(abi.PtyError, match="512"):
        _session(d, probe=d["probe"], precision=1)
