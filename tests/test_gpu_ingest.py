"""Whole-mode pattern ingest on the GPU.

(1) The reference's own preprocessing kernels (d_symmetrizeDiffraction, d_rot90, d_shiftX / d_shiftY, compiled
unchanged into oracle/_ref) composed as DiffractionLoader::run (src/DiffractionLoader.cpp:55-131) against the
oracle's restatement, bit for bit; (2) the engine's one-pass preprocessing kernel against the oracle, bit for bit;
(3) ptychopy.epie / dm reading .bin and .csv files equal ptychopy.epienp / dmnp on the oracle's ingested patterns."""
import ctypes

import numpy as np
import pytest

import pyoracle as po
from conftest import rel_err

pytestmark = pytest.mark.gpu

# (raw rows, raw cols, size, qx, qy): crop inside, zero padding on both sides, window past the far edges, direct copy
CASES = [(300, 280, 256, 150, 140), (200, 220, 256, 100, 110), (400, 400, 256, 300, 310), (256, 256, 256, 40, 90),
         (100, 90, 64, 50, 45)]


def _reference_chain(raw, S, qx, qy, rot, shift):
    """The reference's DiffractionLoader::run with its own kernels (in-bounds cases only)."""
    import torch

    import pyref

    rows, cols = raw.shape
    out = torch.zeros((S, S), dtype=torch.float32, device="cuda")
    if rows == S and cols == S:
        out.copy_(torch.from_numpy(raw))
    else:
        d = torch.from_numpy(raw).cuda()
        dx, dy = qx - S // 2, qy - S // 2
        oox, dox = (-dx, 0) if dx < 0 else (0, dx)
        ooy, doy = (-dy, 0) if dy < 0 else (0, dy)
        numX = S if qx + S // 2 < rows else rows - dox
        numY = S if qy + S // 2 < cols else cols - doy
        assert oox + numX <= S and ooy + numY <= S  # the reference's launch writes inside the pattern
        pyref.call("ref_symmetrize", pyref.ptr(d), pyref.ptr(out), dox, doy, cols, oox, ooy, S, numX, numY)
    temp = out.clone()
    if rot > 0:
        pyref.call("ref_rotate90", pyref.ptr(temp), pyref.ptr(out), S, rot)
    if shift:
        pyref.call("ref_shift_fft", pyref.ptr(out), pyref.ptr(temp), S)
    return out.cpu().numpy()


@pytest.mark.parametrize("rot,shift", [(0, 0), (1, 0), (0, 1), (1, 1), (2, 1)])
def test_reference_preprocessing_matches_oracle_and_engine(rot, shift):
    import torch

    from ptychopy_b200 import abi

    rng = np.random.default_rng(7)
    for rows, cols, S, qx, qy in CASES:
        raw = rng.random((rows, cols)).astype(np.float32) * 100
        want = po.preprocess_pattern(raw, S, qx, qy, rot, shift)
        assert np.array_equal(_reference_chain(raw, S, qx, qy, rot, shift), want), (rows, cols, S, qx, qy)
        d = torch.from_numpy(np.stack([raw, raw[::-1].copy()])).cuda()
        out = torch.zeros((2, S, S), dtype=torch.float32, device="cuda")
        rc = abi.lib().pty_preprocess_patterns(ctypes.c_void_p(d.data_ptr()), 2, rows, cols, S, qx, qy, rot, shift,
                                               ctypes.c_void_p(out.data_ptr()), None)
        assert rc == abi.PTY_OK
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.array_equal(got[0], want)
        assert np.array_equal(got[1], po.preprocess_pattern(raw[::-1].copy(), S, qx, qy, rot, shift))


@pytest.mark.parametrize("algo,ext", [("ePIE", "bin"), ("DM", "csv")])
def test_file_mode_equals_numpy_mode(tmp_path, algo, ext):
    import ptychopy_b200
    from gpu_helpers import dataset

    pt = ptychopy_b200.import_ptychopy()
    d = dataset(N=64, nx=4, algorithm=algo)
    P = d["amp"].shape[0]
    # raw 80 x 72 detector frames holding the patterns rotated back, shifted back and padded around (40, 36)
    frames = np.zeros((P, 80, 72), np.float32)
    for i in range(P):
        frames[i, 8:72, 4:68] = np.rot90(np.fft.ifftshift(d["amp"][i]), -1)
    dpf, fs = 5, 3
    for f in range((P + dpf - 1) // dpf):
        chunk = frames[f * dpf:(f + 1) * dpf]
        name = tmp_path / f"frames_{f + fs:04d}.{ext}"
        if ext == "bin":
            chunk.tofile(name)
        else:
            with open(name, "w") as fh:
                for fr in chunk:
                    for row in fr:
                        fh.write(",".join(repr(float(v)) for v in row) + "\n")
    fp = str(tmp_path / f"frames_#04d.{ext}")
    amp = po.ingest(fp, P, 64, 80, 72, 40, 36, fs=fs, dpf=dpf, rotate90_times=1, fft_shift_data=1)
    assert np.array_equal(amp, d["amp"])
    kw = dict(d["kw"])
    kw.pop("algorithm")
    kw.update(iter=3, updateProbe=2, seed=5, calculateRMS=0, returnResults=1, writeResults=0)
    run_files = {"ePIE": pt.epie, "DM": pt.dm}[algo]
    run_np = {"ePIE": pt.epienp, "DM": pt.dmnp}[algo]
    o1, p1 = run_files(fp=fp, fs=fs, dpf=dpf, nx=80, ny=72, qx=40, qy=36, rotate90=1, fftShiftData=1, **kw)
    o2, p2 = run_np(diffractionNP=amp, **kw)
    if algo == "ePIE":  # deterministic
        assert np.array_equal(o1, o2) and np.array_equal(p1, p2)
    else:  # DM sums its increments with float atomics, whose order varies from run to run
        assert rel_err(o1, o2) < 1e-5 and rel_err(p1, p2) < 1e-5


def test_file_mode_errors(tmp_path):
    import ptychopy_b200

    pt = ptychopy_b200.import_ptychopy()
    kw = dict(size=64, scanDimsx=2, scanDimsy=2, nx=64, ny=64, returnResults=1, writeResults=0, iter=1)
    with pytest.raises(OSError):
        pt.epie(fp=str(tmp_path / "missing_#d.bin"), **kw)
    np.zeros((3, 64, 64), np.float32).tofile(tmp_path / "short_0.bin")  # 3 patterns where 4 are needed
    with pytest.raises(ValueError):
        pt.epie(fp=str(tmp_path / "short_#d.bin"), dpf=4, **kw)
    with pytest.raises(NotImplementedError):
        pt.epie(fp=str(tmp_path / "scan_#d.h5"), **kw)
