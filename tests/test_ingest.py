"""Whole-mode pattern ingest, CPU side: the oracle's restatement of the reference's readers and preprocessing
(src/FileManager.cpp:145-216, src/DiffractionLoader.cpp:55-131) against known answers.  No GPU needed."""
import numpy as np

import pyoracle as po


def test_quarter_turn_and_quadrant_swap_known_answers():
    a = np.arange(64 * 64, dtype=np.float32).reshape(64, 64)
    assert np.array_equal(po.rotate90(a, 1), np.rot90(a))   # d_rot90: out[S-1-c][r] = in[r][c]
    assert np.array_equal(po.rotate90(a, 5), np.rot90(a))
    for t in (0, 2, 3, 4):                                   # other values move nothing in the reference
        assert np.array_equal(po.rotate90(a, t), a)
    assert np.array_equal(po.fft_shift(a), np.fft.fftshift(a))


def test_symmetrize_crop_and_pad():
    raw = np.arange(300 * 280, dtype=np.float32).reshape(300, 280)
    out = po.symmetrize(raw, 256, 150, 140)                  # window inside: plain crop
    assert np.array_equal(out, raw[22:278, 12:268])
    raw2 = np.arange(200 * 220, dtype=np.float32).reshape(200, 220)
    out = po.symmetrize(raw2, 256, 100, 110)                 # window past both edges: zero padding
    assert np.array_equal(out[28:228, 18:238], raw2) and out[:28].sum() == 0 and out[:, :18].sum() == 0
    raw3 = np.ones((256, 256), np.float32)
    assert np.array_equal(po.symmetrize(raw3, 256, 10, 10), raw3)   # already size x size: copied as it is


def test_readers_and_file_index_pattern(tmp_path):
    rng = np.random.default_rng(1)
    data = rng.random((6, 5, 7)).astype(np.float32)
    data[:3].tofile(tmp_path / "scan_002.bin")
    data[3:].tofile(tmp_path / "scan_003.bin")
    got = po.ingest(str(tmp_path / "scan_#03d.bin"), 6, 8, 5, 7, 2, 3, fs=2, dpf=3)
    want = np.stack([po.preprocess_pattern(d, 8, 2, 3) for d in data])
    assert np.array_equal(got, want)
    with open(tmp_path / "p.csv", "w") as f:
        for k in range(2):
            for r in range(5):
                f.write(", ".join(repr(float(v)) for v in data[k, r]) + "\n")
    assert np.array_equal(po.read_pattern_file(str(tmp_path / "p.csv"), 5, 7), data[:2])
