"""The persistent ePIE kernel against the FP64 oracle: same seeded visiting order, same update schedule."""
import numpy as np
import pytest

from conftest import rel_err
from gpu_helpers import dataset, gpu_session

pytestmark = pytest.mark.gpu
TOL = 1e-4


@pytest.mark.parametrize("N,nx", [(64, 5), (128, 4), (32, 6), (256, 3), (512, 2)])
def test_epie_matches_oracle(oracle, N, nx):
    d = dataset(N=N, nx=nx)
    s = gpu_session(d, probe=d["probe"], updateProbe=2, calculateRMS=1, seed=77)
    o = oracle.OracleSession("ePIE", d["amp"], d["pos"], np.zeros((d["X"], d["Y"])), d["probe"],
                             probe_guess_path=False, updateProbe=2, calculateRMS=1, seed=77)
    for it in range(1, 5):
        eg = s.step()
        eo = o.step()
        ob, pr, _ = o.state()
        assert rel_err(s.object(), ob) < TOL, f"object, iteration {it}"
        assert rel_err(s.probe(), pr) < TOL, f"probe, iteration {it}"
        assert abs(eg - eo) <= 1e-6 * max(abs(eo), 1e-12) + 1e-7, f"error metric, iteration {it}"


def test_epie_probe_guess(oracle):
    d = dataset(N=64, nx=5)
    s = gpu_session(d, updateProbe=1, seed=3)
    g = oracle.probe_guess(d["amp"], d["kw"]["beamSize"], d["dx_s"], K=1)
    assert rel_err(s.probe(), g) < 1e-5
    o = oracle.OracleSession("ePIE", d["amp"], d["pos"], np.zeros((d["X"], d["Y"])), g, probe_guess_path=True,
                             updateProbe=1, seed=3)
    for _ in range(3):
        s.step()
        o.step()
    ob, pr, _ = o.state()
    assert rel_err(s.object(), ob) < TOL and rel_err(s.probe(), pr) < TOL


def test_epie_given_modes(oracle):
    # probeNP with K modes (extension): single-mode iterations until updateModes, modal afterwards
    d = dataset(N=64, nx=5, K=3)
    s = gpu_session(d, probe=d["probe"], updateProbe=2, updateModes=3, calculateRMS=1, seed=9)
    o = oracle.OracleSession("ePIE", d["amp"], d["pos"], np.zeros((d["X"], d["Y"])), d["probe"],
                             probe_guess_path=False, modes_given=True, updateProbe=2, updateModes=3,
                             calculateRMS=1, seed=9)
    for it in range(1, 6):
        s.step()
        o.step()
    ob, pr, _ = o.state()
    assert rel_err(s.object(), ob) < TOL and rel_err(s.probe(), pr) < TOL


@pytest.mark.parametrize("N,K,bits,sq", [(64, 1, 10, 1), (64, 3, 5, 0), (256, 3, 10, 1), (512, 1, 8, 1)])
def test_epie_saturated_pixels_float(oracle, N, K, bits, sq):
    """bitDepth (with sqrtData) sets the modulus step's saturation level; pixels at or above it float (one mode
    keeps Psi, several take the modal factor with 1 for A: src/utilitiesKernels.cu:634-682).  Every ePIE variant
    against the oracle with the same level: the shared-memory kernel (64^2, one mode), the cluster kernel (64^2,
    modes from iteration 3), the kernel chain (256^2, modes from iteration 3; 512^2 with the modulus step in its
    transform pass)."""
    d = dataset(N=N, nx=3, K=K)
    level = oracle.saturation_level(bits, 0, sq)
    assert 0 < (d["amp"] >= level).mean() < 0.05  # a few pixels float
    kw = dict(updateProbe=2, updateModes=3, calculateRMS=1, seed=9)
    s = gpu_session(d, probe=d["probe"], bitDepth=bits, sqrtData=sq, **kw)
    runs = [oracle.OracleSession("ePIE", d["amp"], d["pos"], np.zeros((d["X"], d["Y"])), d["probe"],
                                 probe_guess_path=False, modes_given=K > 1, saturation=sat, **kw)
            for sat in (level, None)]
    for _ in range(4):
        s.step()
        for o in runs:
            o.step()
    (ob, pr, _), (ob0, _, _) = (o.state() for o in runs)
    assert rel_err(s.object(), ob) < TOL and rel_err(s.probe(), pr) < TOL
    assert rel_err(ob0, ob) > 10 * TOL  # the floating pixels changed the reconstruction
    s.close()


def test_epie_mode_initialisation(oracle):
    # modes created at updateModes from 0.05 * P0 and Gram-Schmidt: mode 0 and the object stay at parity
    # (the extra modes start at round-off level, so they are compared loosely)
    d = dataset(N=64, nx=5, K=2)
    p0 = d["probe"][:1]
    s = gpu_session(d, probe=p0, updateProbe=2, updateModes=2, seed=5)
    o = oracle.OracleSession("ePIE", d["amp"], d["pos"], np.zeros((d["X"], d["Y"])),
                             np.concatenate([p0, np.zeros_like(p0)]), probe_guess_path=False, updateProbe=2,
                             updateModes=2, seed=5)
    for _ in range(3):
        s.step()
        o.step()
    ob, pr, _ = o.state()
    assert rel_err(s.probe()[0], pr[0]) < 1e-3
    assert rel_err(s.object(), ob) < 1e-3


def test_epie_negative_position_is_an_error():
    from ptychopy_b200 import abi

    d = dataset(N=32, nx=3)
    s = abi.Session(**d["kw"])
    s.set_patterns(d["amp"])
    xy = np.zeros((9, 2))
    xy[:, 0] = np.arange(9) * 1e-8
    s.set_positions(xy)
    # list positions are shifted by their minimum, so they are valid; a too-small object is rejected instead
    s.init()
    s.close()
    s2 = abi.Session(**d["kw"])
    s2.set_patterns(d["amp"])
    s2.set_object(np.ones((10, 10), np.complex64))
    with pytest.raises(abi.PtyError):
        s2.init()


def test_scan_meshes_match_oracle(oracle, tmp_path):
    # spiral scan, jittered raster and a position list file: session geometry == oracle geometry, bit for bit
    from gpu_helpers import dataset, gpu_session

    d = dataset(N=64, nx=5, algorithm="ePIE")
    kw = d["kw"]
    lam, z, dxd = kw["lambd"], kw["z"], kw["dx_d"]
    s = gpu_session(d, probe=d["probe"], spiralScan=1, seed=3)
    pos, X, Y = oracle.spiral_mesh(25, kw["stepx"], kw["stepy"], lam, z, dxd, 64)
    assert np.array_equal(s.positions(), pos) and (s.dims()["X"], s.dims()["Y"]) == (X, Y)
    s = gpu_session(d, probe=d["probe"], jitterRadius=2, seed=11)
    pos, X, Y = oracle.cartesian_mesh(5, 5, kw["stepx"], kw["stepy"], lam, z, dxd, 64, jitter=2, seed=11)
    assert np.array_equal(s.positions(), pos) and (s.dims()["X"], s.dims()["Y"]) == (X, Y)
    xy = (np.random.default_rng(1).random((25, 2)) * 0.4e-6).astype(np.float64)
    f = tmp_path / "positions.csv"
    f.write_text("".join(f"{float(a)!r},{float(b)!r}\n" for a, b in xy))
    s = gpu_session(d, probe=d["probe"], lf=str(f))
    pos, X, Y = oracle.list_mesh(xy, lam, z, dxd, 64)
    assert np.array_equal(s.positions(), pos) and (s.dims()["X"], s.dims()["Y"]) == (X, Y)
    s.step()
    assert np.isfinite(s.object()).all()


def test_scan_drift_matches_oracle(oracle, tmp_path):
    """The scan drift (the reference's command-line `drift`): raster, spiral and position-list sessions with a drift
    place their positions where the oracle does, bit for bit, and the object grows to hold them."""
    from gpu_helpers import dataset, gpu_session

    d = dataset(N=64, nx=5, algorithm="ePIE")
    kw = d["kw"]
    lam, z, dxd = kw["lambd"], kw["z"], kw["dx_d"]
    dr = (3e-9, -2e-9)
    s = gpu_session(d, probe=d["probe"], driftx=dr[0], drifty=dr[1])
    pos, X, Y = oracle.cartesian_mesh(5, 5, kw["stepx"], kw["stepy"], lam, z, dxd, 64, drift=dr)
    assert np.array_equal(s.positions(), pos) and (s.dims()["X"], s.dims()["Y"]) == (X, Y)
    assert (X, Y) != (d["X"], d["Y"])
    s.close()
    s = gpu_session(d, probe=d["probe"], spiralScan=1, seed=3, driftx=dr[0], drifty=dr[1])
    pos, X, Y = oracle.spiral_mesh(25, kw["stepx"], kw["stepy"], lam, z, dxd, 64, drift=dr)
    assert np.array_equal(s.positions(), pos) and (s.dims()["X"], s.dims()["Y"]) == (X, Y)
    s.close()
    xy = (np.random.default_rng(1).random((25, 2)) * 0.4e-6).astype(np.float64)
    f = tmp_path / "positions.csv"
    f.write_text("".join(f"{float(a)!r},{float(b)!r}\n" for a, b in xy))
    s = gpu_session(d, probe=d["probe"], lf=str(f), driftx=dr[0], drifty=dr[1])
    pos, X, Y = oracle.list_mesh(xy, lam, z, dxd, 64, drift=dr)
    assert np.array_equal(s.positions(), pos) and (s.dims()["X"], s.dims()["Y"]) == (X, Y)
    s.step()
    assert np.isfinite(s.object()).all()
    s.close()


@pytest.mark.parametrize("K", [1, 3])
def test_epie_tensor_core_fft_chain(oracle, K):
    """precision=1: ePIE as a per-position kernel chain whose transforms run as split-BF16 tensor-core stages
    (256^2); FP32 fused kernel and the chain both against the FP64 oracle, error stated, with the probe updating
    from iteration 2 and (K = 3) the modes from iteration 3."""
    d = dataset(N=256, nx=3, K=K)
    kw = dict(updateProbe=2, updateModes=3, calculateRMS=1, seed=21)
    runs = {prec: gpu_session(d, probe=d["probe"], precision=prec, **kw) for prec in (0, 1)}
    o = oracle.OracleSession("ePIE", d["amp"], d["pos"], np.zeros((d["X"], d["Y"])), d["probe"],
                             probe_guess_path=False, modes_given=K > 1, **kw)
    errs = {0: [], 1: []}
    for _ in range(4):
        for prec, s in runs.items():
            errs[prec].append(s.step())
        eo = o.step()
    ob, pr, _ = o.state()
    e32, etc = rel_err(runs[0].object(), ob), rel_err(runs[1].object(), ob)
    p32, ptc = rel_err(runs[0].probe(), pr), rel_err(runs[1].probe(), pr)
    print(f"ePIE 256^2 K={K}, 4 iterations vs FP64: object FP32 {e32:.2e}, TC chain {etc:.2e}; "
          f"probe {p32:.2e}, {ptc:.2e}; error metric {errs[0][-1]:.6e} / {errs[1][-1]:.6e} / {eo:.6e}")
    assert e32 < TOL and p32 < TOL
    assert etc < 2e-3 and ptc < 2e-3
    assert abs(errs[1][-1] - eo) <= 2e-3 * abs(eo)
    for s in runs.values():
        s.close()
