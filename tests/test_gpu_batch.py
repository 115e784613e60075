"""Batched reconstructions (pty_batch_run): several independent scans of uneven sizes interleaved on their own
streams give the same objects and probes as running each scan alone."""
import numpy as np
import pytest

from conftest import rel_err
from gpu_helpers import dataset, gpu_session, mls_dataset
from ptychopy_b200 import abi

pytestmark = pytest.mark.gpu
TOL = 1e-5  # float atomics accumulate in a different order when scans overlap on the GPU


def _scans(oracle):
    d1 = dataset(N=64, nx=5, algorithm="DM")
    d2 = dataset(N=128, nx=3, algorithm="DM", seed=5)
    d3 = dataset(N=64, nx=3, algorithm="DM", seed=7)
    d4 = dataset(N=64, nx=4, algorithm="DM", seed=8)
    m1 = mls_dataset(oracle, N=32, nx=11)
    m2 = mls_dataset(oracle, N=64, nx=4, seed=9)
    e1 = dataset(N=32, nx=4, algorithm="ePIE", seed=6)

    def make():
        # three DM scans of one size with different phase-constraint and probe schedules; d4 runs in four waves
        # (5 + 5 + 5 + 1 patterns)
        return [gpu_session(d1, probe=d1["probe"], updateProbe=2),
                gpu_session(d2, probe=d2["probe"]),
                gpu_session(d3, probe=d3["probe"], updateProbe=2, phaseConstraint=2),
                gpu_session(d4, probe=d4["probe"], updateProbe=3, wave=5),
                gpu_session(dict(amp=m1["intens"], kw=m1["kw"]), probe=m1["probe"], obj=m1["obj"]),
                gpu_session(dict(amp=m2["intens"], kw=m2["kw"]), probe=m2["probe"], obj=m2["obj"]),
                gpu_session(e1, probe=e1["probe"], updateProbe=2)]
    return make


def test_batch_matches_individual_runs(oracle):
    # the lone MLs sessions run each group's transforms as one cluster launch per window, the batched ones as
    # separate passes, so this also compares the two forms of the MLs group
    make = _scans(oracle)
    alone = make()
    for s in alone:
        s.run(4)
    batch = make()
    abi.batch_run(batch, 4)
    for a, b in zip(alone, batch):
        assert b.dims()["iters"] == 4
        assert rel_err(b.object(), a.object()) < TOL
        assert rel_err(b.probe(), a.probe()) < TOL


def test_batch_then_step_continues(oracle):
    # a batch advances each session's iteration counter, so a later single step continues the schedule
    make = _scans(oracle)
    alone, batch = make(), make()
    for s in alone:
        s.run(3)
    abi.batch_run(batch, 2)
    for s in batch:
        s.step()
    for a, b in zip(alone, batch):
        assert rel_err(b.object(), a.object()) < TOL


def test_batch_rejects_uninitialised():
    d = dataset(N=32, nx=3, algorithm="DM")
    s = abi.Session(**d["kw"])
    s.set_patterns(d["amp"])
    with pytest.raises(abi.PtyError):
        abi.batch_run([s], 1)
