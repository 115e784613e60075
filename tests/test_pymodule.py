"""The CPython module surface: the reference's method names and keyword arguments (no GPU needed)."""
import numpy as np
import pytest

REFERENCE_METHODS = ["helloworld", "epie", "dm", "mls", "epienp", "dmnp", "mlsnp", "epiecmdstr", "dmcmdstr",
                     "mlscmdstr", "epieinit", "epiepost", "epiestep", "epieresobj", "epieresprobe", "epienpinit",
                     "mlsinit", "mlspost", "mlsstep", "mlsresobj", "mlsresprobe"]


@pytest.fixture(scope="module")
def ptychopy():
    import ptychopy_b200

    return ptychopy_b200.import_ptychopy()


def test_module_has_reference_methods(ptychopy):
    import sys

    for m in REFERENCE_METHODS:
        assert callable(getattr(ptychopy, m)), m
    assert sys.modules["ptychopy"] is ptychopy


def test_hdf5_files_raise_not_implemented(ptychopy):
    # .bin / .csv pattern files are read (tests/test_ingest.py, tests/test_gpu_ingest.py); .h5 needs the HDF5
    # library, which this build does not link, also when a command string names them
    with pytest.raises(NotImplementedError):
        ptychopy.epie(jobID="x", fp="/data/scan#.h5", size=256)
    with pytest.raises(NotImplementedError):
        ptychopy.dmcmdstr(cmdstr="./ptycho -jobID=x -fp=/data/scan#.h5")


def test_unknown_keyword_is_a_type_error(ptychopy):
    with pytest.raises(TypeError):
        ptychopy.epienp(jobID="x", notakeyword=3)


def test_missing_patterns_is_a_value_error(ptychopy):
    with pytest.raises(ValueError):
        ptychopy.dmnp(jobID="x")


def test_wrong_pattern_rank_is_a_value_error(ptychopy):
    with pytest.raises(ValueError):
        ptychopy.epienp(diffractionNP=np.zeros((4, 4)))


def test_step_without_session(ptychopy):
    with pytest.raises(RuntimeError):
        ptychopy.epiestep()


def test_helloworld(ptychopy):
    assert ptychopy.helloworld([1.0, 2.0, 3.0], [[1.0]], [[[1.0]]]) is None
