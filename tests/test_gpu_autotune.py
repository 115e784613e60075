"""pty_autotune: times the launch variants on temporary sessions before pty_init and keeps the fastest; a tuned
session reconstructs the same as an untuned one."""
import numpy as np
import pytest

from conftest import rel_err
from gpu_helpers import dataset

pytestmark = pytest.mark.gpu


def _session(d, tune, **params):
    from ptychopy_b200 import abi

    s = abi.Session(**dict(d["kw"], **params))
    s.set_patterns(d["amp"])
    s.set_probe(d["probe"])
    rep = s.autotune(iters=1) if tune else None
    s.init()
    return s, rep


@pytest.mark.parametrize("alg,N,nx,K", [("DM", 64, 6, 1), ("ePIE", 256, 3, 1), ("ePIE", 128, 3, 1), ("ePIE", 256, 4, 3)])
def test_autotune_keeps_results(alg, N, nx, K):
    d = dataset(N=N, nx=nx, algorithm=alg, K=K)
    kw = dict(algorithm=alg, seed=5, updateProbe=1, updateModes=2) if K > 1 else dict(algorithm=alg, seed=5)
    tuned, rep = _session(d, True, **kw)
    plain, _ = _session(d, False, **kw)
    if alg == "ePIE":
        assert "kernel chain" in rep  # the per-position chain is one of the timed variants
    print(rep)
    assert rep.startswith(alg) and "ms/iteration" in rep
    for _ in range(3):
        tuned.step()
        plain.step()
    assert rel_err(tuned.object(), plain.object()) < 1e-5
    assert rel_err(tuned.probe(), plain.probe()) < 1e-5
    tuned.close()
    plain.close()


def test_autotune_after_init_is_an_error():
    from ptychopy_b200 import abi

    d = dataset(N=64, nx=3)
    s, _ = _session(d, False, algorithm="ePIE")
    with pytest.raises(abi.PtyError):
        s.autotune()
    s.close()
