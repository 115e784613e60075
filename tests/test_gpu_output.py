"""Result files and checkpoints: the reference's text format (re+imj cells joined by ", ", 6 significant digits,
src/Cuda2DArray.cpp:46-52, src/Cuda2DArray.hpp:439-464) and raw complex64 binary output, the `save` checkpoints
written every `save` iterations (src/IPhaser.cpp:384-385), and the objectGuess / probeGuess readers on those files."""
import os

import numpy as np
import pytest

import pyoracle as po
from gpu_helpers import dataset

pytestmark = pytest.mark.gpu


def _kw(d, **extra):
    kw = dict(d["kw"])
    kw.pop("algorithm")
    kw.update(updateProbe=2, seed=11, jobID="job", **extra)
    return kw


def test_text_results_checkpoints_and_guess_round_trip(tmp_path):
    import ptychopy_b200
    from ptychopy_b200 import abi

    pt = ptychopy_b200.import_ptychopy()
    d = dataset(N=64, nx=4)
    out = str(tmp_path)
    obj, probe = pt.epienp(diffractionNP=d["amp"], iter=4, save=2, outputDir=out, returnResults=1, **_kw(d))
    files = sorted(os.listdir(out))
    assert files == ["job_object_0.csv", "job_object_1.csv", "job_object_2.csv",
                     "job_probes_0.csv", "job_probes_1.csv", "job_probes_2.csv"]
    text = open(os.path.join(out, "job_object_0.csv")).read()
    assert text == po.format_complex_csv(obj)
    assert open(os.path.join(out, "job_probes_0.csv")).read() == po.format_complex_csv(probe)
    assert open(os.path.join(out, "job_object_2.csv")).read() == text  # iteration 4 = the final state
    # checkpoint 1 holds iteration 2: the same run stopped after two iterations
    o2, p2 = pt.epienp(diffractionNP=d["amp"], iter=2, writeResults=0, returnResults=1, **_kw(d))
    assert open(os.path.join(out, "job_object_1.csv")).read() == po.format_complex_csv(o2)
    # the files read back as objectGuess / probeGuess: the values at 6 significant digits
    s = abi.Session(**dict(d["kw"], objectGuess=os.path.join(out, "job_object_0.csv"),
                           probeGuess=os.path.join(out, "job_probes_0.csv")))
    s.set_patterns(d["amp"])
    s.init()
    assert np.array_equal(s.object(), po.parse_complex_csv(text))
    assert np.array_equal(s.probe()[0], po.parse_complex_csv(open(os.path.join(out, "job_probes_0.csv")).read()))
    s.close()


def test_binary_results(tmp_path):
    import ptychopy_b200

    pt = ptychopy_b200.import_ptychopy()
    d = dataset(N=64, nx=4, algorithm="DM")
    out = str(tmp_path)
    kw = _kw(d)
    obj, probe = pt.dmnp(diffractionNP=d["amp"], iter=3, binaryOutput=1, outputDir=out, returnResults=1, **kw)
    o = np.fromfile(os.path.join(out, "job_object_0.bin"), np.complex64).reshape(obj.shape)
    p = np.fromfile(os.path.join(out, "job_probes_0.bin"), np.complex64).reshape(probe.shape)
    assert np.array_equal(o, obj) and np.array_equal(p, probe)
