"""Committed golden fixtures (tests/golden/*.npz, made by tests/golden/make_golden.py from the oracle).

CPU: the oracle reproduces its stored results (regression pin of the restatement).
GPU: the CUDA path matches the stored FP64 results (relative object/probe error <= 1e-4, error metric 1e-6).
"""
import ast
import glob
import os

import numpy as np
import pytest

from conftest import rel_err

HERE = os.path.dirname(os.path.abspath(__file__))
ALL = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(HERE, "golden", "*.npz")))
CASES = [c for c in ALL if not c.startswith("mls_")]
MLS_CASES = [c for c in ALL if c.startswith("mls_")]


def load(name):
    z = np.load(os.path.join(HERE, "golden", name + ".npz"))
    params = ast.literal_eval(str(z["params"]))
    return z, params


def test_fixtures_present():
    assert {"epie_n32", "dm_n32", "epie_modes_n32", "epie_guess_n64"} <= set(CASES)
    assert {"mls_default_n32"} <= set(MLS_CASES)


def _mls_oracle(oracle, z, params):
    return oracle.OracleMls(z["raw"], z["intens"], z["probe_start"], obj=z["obj_start"], variable=1,
                            PPS=params["PPS"], K=params["probeModes"])


@pytest.mark.parametrize("name", MLS_CASES)
def test_oracle_reproduces_mls_fixture(oracle, name):
    z, params = load(name)
    o = _mls_oracle(oracle, z, params)
    errs = [o.step() for _ in range(int(z["iterations"]))]
    ob, pr, _ = o.state()
    E, e0, e1, pos = o.variable_state()
    for got, want in ((ob, z["object"]), (pr, z["probe"]), (E, z["extra_mode"]), (e0, z["evo0"]), (e1, z["evo1"])):
        assert rel_err(got, want) < 1e-12
    assert np.array_equal(pos, z["positions"])
    assert np.allclose(errs, z["errors"], rtol=1e-12, atol=0)


@pytest.mark.gpu
@pytest.mark.parametrize("name", MLS_CASES)
def test_cuda_matches_mls_fixture(name):
    """The default MLs path (modes, position search, variable probe) against the stored FP64 results: object and the
    dominant mode 1e-4, the weaker mode, the extra mode and the refined positions as in test_gpu_mls."""
    from gpu_helpers import gpu_session

    z, params = load(name)
    s = gpu_session(dict(amp=z["intens"], kw=params), probe=z["probe_start"], obj=z["obj_start"])
    errs = [s.step() for _ in range(int(z["iterations"]))]
    gp = s.probe()
    assert rel_err(s.object(), z["object"]) < 1e-4
    assert rel_err(gp[0], z["probe"][0]) < 1e-4
    assert rel_err(gp[1], z["probe"][1]) < 1e-3
    E, e0, e1 = s.mls_state()
    assert rel_err(E, z["extra_mode"]) < 1e-3 and rel_err(e0, z["evo0"]) < 1e-5 and rel_err(e1, z["evo1"]) < 1e-2
    assert np.abs(s.positions() - z["positions"]).max() < 1e-4
    assert np.allclose(errs, z["errors"], rtol=1e-3)
    s.close()


@pytest.mark.parametrize("name", CASES)
def test_oracle_reproduces_fixture(oracle, name):
    z, params = load(name)
    X, Y = z["object"].shape
    sched = {k: params[k] for k in ("updateProbe", "updateModes", "calculateRMS", "seed", "phaseConstraint")
             if k in params}
    o = oracle.OracleSession(str(z["algorithm"]), z["amp"], z["pos"], np.zeros((X, Y)), z["probe_start"],
                             probe_guess_path=bool(z["guess"]), modes_given=bool(z["modes_given"]), **sched)
    errs = [o.step() for _ in range(int(z["iterations"]))]
    ob, pr, _ = o.state()
    assert rel_err(ob, z["object"]) < 1e-12
    assert rel_err(pr, z["probe"]) < 1e-12
    assert np.allclose(errs, z["errors"], rtol=1e-12, atol=0)


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_cuda_matches_fixture(name):
    from ptychopy_b200 import abi

    z, params = load(name)
    kw = {k: v for k, v in params.items()}
    s = abi.Session(**kw)
    s.set_patterns(z["amp"])
    if not bool(z["guess"]):
        pstart = z["probe_start"]
        if not bool(z["modes_given"]):
            pstart = pstart[:1]
        s.set_probe(pstart)
    s.init()
    if bool(z["guess"]):
        assert rel_err(s.probe(), z["probe_start"]) < 1e-5
    errs = [s.step() for _ in range(int(z["iterations"]))]
    tol = 1e-4 if not (params.get("probeModes", 1) > 1 and not bool(z["modes_given"])) else 1e-3
    assert rel_err(s.object(), z["object"]) < tol
    assert rel_err(s.probe(), z["probe"]) < tol
    if params.get("calculateRMS"):
        assert np.allclose(errs, z["errors"], rtol=1e-6, atol=1e-9)
