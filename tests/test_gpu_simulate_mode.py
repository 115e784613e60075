"""Simulation mode (simulate=1): the reference's PGM object (data/lena<N>.pgm, data/baboon<N>.pgm relative to the
working directory), the simulated probe and the forward model, against the oracle's restatement; then a whole run
through ptychopy.epie(simulate=1) equals ptychopy.epienp on those patterns.  The images are synthetic, written by the
test."""
import numpy as np
import pytest

import pyoracle as po
from conftest import rel_err

pytestmark = pytest.mark.gpu


def _write_pgm(path, img, binary=True):
    h, w = img.shape
    with open(path, "wb") as f:
        if binary:
            f.write(f"P5\n# synthetic\n{w} {h}\n255\n".encode())
            f.write(img.astype(np.uint8).tobytes())
        else:
            f.write(f"P2\n{w} {h}\n255\n".encode())
            f.write(" ".join(str(int(v)) for v in img.ravel()).encode())


@pytest.fixture
def images(tmp_path, monkeypatch):
    N = 64
    rng = np.random.default_rng(4)
    yy, xx = np.mgrid[0:N, 0:N]
    lena = (128 + 100 * np.sin(xx / 5.0) * np.cos(yy / 7.0) + rng.integers(0, 20, (N, N))).clip(0, 255)
    baboon = (255 * (xx + yy) / (2 * N - 2)).round()
    (tmp_path / "data").mkdir()
    _write_pgm(tmp_path / "data" / f"lena{N}.pgm", lena)
    _write_pgm(tmp_path / "data" / f"baboon{N}.pgm", baboon, binary=False)
    monkeypatch.chdir(tmp_path)
    return N, lena.astype(np.uint8), baboon.astype(np.uint8)


@pytest.mark.parametrize("algo", ["ePIE", "DM"])
def test_simulated_patterns_match_oracle(images, algo):
    from ptychopy_b200 import abi

    N, lena, baboon = images
    kw = dict(size=N, scanDimsx=4, scanDimsy=4, stepx=60e-9, stepy=60e-9, lambd=2.48e-10, z=1.0, dx_d=172e-6,
              beamSize=110e-9, algorithm=algo, simulate=1, seed=99)
    s = abi.Session(**kw)
    s.init()
    amp = s.patterns()
    pos, d = s.positions(), s.dims()
    assert np.array_equal(po.read_pgm("data/lena64.pgm"), lena)
    obj = po.sim_object(lena, baboon, d["X"], d["Y"])
    dx_s = po.sample_pixel(kw["lambd"], kw["z"], kw["dx_d"], N)
    probe = po.sim_probe(N, kw["beamSize"], dx_s, 99)
    want = po.simulate_amplitudes(obj, probe, pos)
    assert rel_err(amp, want) < 2e-5
    # the run starts from the probe guess of the simulated patterns, as the reference's prePhase does
    g = po.probe_guess(amp.astype(np.float64), kw["beamSize"], dx_s, K=1)
    assert rel_err(s.probe(), g) < 1e-5
    s.close()


def test_simulate_mode_run_equals_numpy_run(images):
    import ptychopy_b200
    from ptychopy_b200 import abi

    N = images[0]
    pt = ptychopy_b200.import_ptychopy()
    kw = dict(size=N, scanDimsx=4, scanDimsy=4, stepx=60e-9, stepy=60e-9, lambd=2.48e-10, z=1.0, dx_d=172e-6,
              beamSize=110e-9, iter=3, updateProbe=2, seed=99, returnResults=1, writeResults=0)
    sess_kw = {k: v for k, v in kw.items() if k not in ("returnResults", "writeResults")}
    s = abi.Session(**dict(sess_kw, algorithm="ePIE", simulate=1))
    s.init()
    amp = s.patterns()
    s.close()
    o1, p1 = pt.epie(simulate=1, **kw)
    o2, p2 = pt.epienp(diffractionNP=amp, **kw)
    assert np.array_equal(o1, o2) and np.array_equal(p1, p2)


def test_simulate_mode_errors(tmp_path, monkeypatch):
    import ptychopy_b200

    pt = ptychopy_b200.import_ptychopy()
    monkeypatch.chdir(tmp_path)
    kw = dict(size=64, scanDimsx=2, scanDimsy=2, iter=1, returnResults=1, writeResults=0)
    with pytest.raises(OSError):  # no data/lena64.pgm here
        pt.epie(simulate=1, **kw)
    with pytest.raises(NotImplementedError):
        pt.mls(simulate=1, **kw)
