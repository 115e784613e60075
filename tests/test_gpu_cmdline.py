"""The command-string entry points on the GPU: epiecmdstr / dmcmdstr give the object of the keyword run with the
same options (the command line's defaults written out as keywords), write their result files, and epieinit +
epiestep continue like the whole run.  Simulation mode, on synthetic PGM images written by the test."""
import os

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

CMD = ("./ptycho -jobID=cmd{algo} -algorithm=MLs -size=64 -scanDims=4,4 -step=60e-9,60e-9 -lambda=2.48e-10 -z=1 "
       "-dx_d=172e-6 -beamSize=110e-9 -i=3 -updateProbe=2 -simulate=1")
# the same run as keywords; PPS and delta_p are the command line's defaults (MLs only)
KW = dict(size=64, scanDimsx=4, scanDimsy=4, stepx=60e-9, stepy=60e-9, lambd=2.48e-10, z=1.0, dx_d=172e-6,
          beamSize=110e-9, iter=3, updateProbe=2, PPS=5)


@pytest.fixture
def sim_dir(tmp_path, monkeypatch):
    N = 64
    yy, xx = np.mgrid[0:N, 0:N]
    images = {"lena": 128 + 100 * np.sin(xx / 5.0) * np.cos(yy / 7.0), "baboon": 255 * (xx + yy) / (2 * N - 2)}
    (tmp_path / "data").mkdir()
    for name, img in images.items():
        with open(tmp_path / "data" / f"{name}{N}.pgm", "wb") as f:
            f.write(f"P5\n{N} {N}\n255\n".encode())
            f.write(img.round().clip(0, 255).astype(np.uint8).tobytes())
    monkeypatch.chdir(tmp_path)
    return tmp_path


@pytest.mark.parametrize("algo", ["ePIE", "DM"])
def test_command_string_run_equals_keyword_run(sim_dir, algo):
    import ptychopy_b200

    pt = ptychopy_b200.import_ptychopy()
    run = pt.epiecmdstr if algo == "ePIE" else pt.dmcmdstr
    o = run(CMD.format(algo=algo))  # the entry point's algorithm, whatever -algorithm says
    assert o.dtype == np.complex64 and o.ndim == 2
    for part in ("object", "probes"):
        assert os.path.getsize(sim_dir / "data" / f"cmd{algo}_{part}_0.csv") > 0
    keyword_run = pt.epie if algo == "ePIE" else pt.dm
    o2, _ = keyword_run(simulate=1, returnResults=1, writeResults=0, **KW)
    if algo == "ePIE":
        assert np.array_equal(o, o2)
    else:  # DM sums the object increments of a wave with atomics: two runs agree to rounding
        assert rel_err(o, o2) < 1e-5


def test_step_mode_from_a_command_string(sim_dir):
    import ptychopy_b200

    pt = ptychopy_b200.import_ptychopy()
    whole = pt.epiecmdstr(CMD.format(algo="ePIE"))
    assert pt.epieinit(CMD.format(algo="Step") + " -binaryOutput=1") is True
    for _ in range(3):
        pt.epiestep()
    o = pt.epieresobj()
    assert o.shape == whole.shape and rel_err(o, whole) < 1e-6
    assert pt.epieresprobe().shape == (64, 64)
    assert pt.epiepost() is True
    # epiepost writes in the session's format: raw complex64 with -binaryOutput=1
    assert os.path.getsize(sim_dir / "data" / "cmdStep_object_0.bin") == o.nbytes
