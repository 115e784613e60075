"""MLs (LSQ-ML with random groups, one probe mode) on the GPU against the FP64 oracle: the reference's default path
(variable probe and intensity, sub-pixel probe shift, position search from PPS) and the fixed-probe core (mlsCore=1).

Both sides start from the same intensities, probe, object, group stream and draws (SplitMix64 seed).  Parity cases use
noise-free data consistent with the model (gpu_helpers.mls_dataset), where the iteration is well conditioned; the
Poisson / flat-start case is chaotic in the reference algorithm itself (FFT round-off of near-zero Psi decides the
phase the modulus step gives to non-zero data), so it is checked through the error metric only."""
import numpy as np
import pytest

from conftest import rel_err
from gpu_helpers import dataset, gpu_session, mls_dataset

pytestmark = pytest.mark.gpu
TOL = 1e-4
# The error metric sums sqrt(sum (A - |Psi|)^2 / 4 / N^2) over the positions.  On these noise-free, model-consistent
# data A and |Psi| agree to a few percent, so the FP32 residual A - |Psi| keeps ~5 of FP32's 7 digits: measured
# engine-vs-FP64 differences are 4e-8 .. 4e-6 (32^2 .. 512^2).
ERR_TOL = 1e-5


def _pair(oracle, d, **params):
    s = gpu_session(dict(amp=d["intens"], kw=d["kw"]), probe=d["probe"], obj=d["obj"], calculateRMS=1, mlsCore=1,
                    **params)
    o = oracle.OracleMls(d["raw"], d["intens"], d["probe"], obj=d["obj"], delta_p=params.get("delta_p", 0.1),
                         seed=params.get("seed", 0x5EED5EED))
    return s, o


def _pair_default(oracle, d, PPS, **params):
    s = gpu_session(dict(amp=d["intens"], kw=d["kw"]), probe=d["probe"], obj=d["obj"], calculateRMS=1, PPS=PPS,
                    **params)
    o = oracle.OracleMls(d["raw"], d["intens"], d["probe"], obj=d["obj"], delta_p=params.get("delta_p", 0.1),
                         seed=params.get("seed", 0x5EED5EED), variable=1, PPS=PPS)
    return s, o


def _check_default(s, o, what):
    ob, pr, _ = o.state()
    E, e0, e1, pos = o.variable_state()
    gE, g0, g1 = s.mls_state()
    assert rel_err(s.object(), ob) < TOL, f"object, {what}"
    assert rel_err(s.probe(), pr) < TOL, f"probe, {what}"
    # E moves only by steps built from the residuals of the probe directions (one per group: 484 steps after four
    # iterations of 121 groups of one), so FP32 rounding of those residuals accumulates in it: bound 1e-3
    assert rel_err(gE, E) < 1e-3, f"extra mode, {what}"
    assert rel_err(g0, e0) < 1e-5, f"intensity weights, {what}"
    # the extra-mode weights (~1e-6..1e-5) are sums of Re(chi conj(O E)) over the residual chi, which carries the FP32
    # cancellation of a small difference of large terms: bound 1e-2 (their effect on the probes, E evo1, is ~1e-5 of P)
    assert rel_err(g1, e1) < 1e-2, f"extra-mode weights, {what}"
    assert np.abs(s.positions() - pos).max() < 1e-4, f"positions, {what}"
    return pos


@pytest.mark.parametrize("N,nx,PPS", [(64, 6, 3), (32, 11, 2), (128, 4, 3), (64, 2, 1)])
def test_mls_default_path_matches_oracle(oracle, N, nx, PPS):
    """The reference's default MLs path: windows and sub-pixel shifts from the positions, the shifted position
    probes P evo0 + E evo1, the extra-mode and weight updates from iteration 3, the position search from PPS."""
    d = mls_dataset(oracle, N=N, nx=nx, shifted=True)
    s, o = _pair_default(oracle, d, PPS)
    assert np.array_equal(s.positions(), d["raw"])
    _check_default(s, o, "set-up")
    for it in range(1, 6):
        e = s.step()
        eo = o.step()
        pos = _check_default(s, o, f"iteration {it}")
        print(f"MLs default path N={N} iteration {it}: error metric rel diff {abs(e - eo) / abs(eo):.2e}")
        assert abs(e - eo) <= ERR_TOL * abs(eo), f"error, iteration {it}"
        moved = np.abs(pos - d["raw"]).max()
        if it < PPS:
            assert moved == 0.0, "positions move only from PPS"
    assert moved > 0.0
    s.close()


def test_mls_zone_plate_probe_start(oracle):
    """No probe given: MLs starts from the zone-plate guess of initMLH (the ePIE paths use the mean-amplitude guess).
    The data are made with that probe, so the run is consistent with its model."""
    from ptychopy_b200 import synth

    N, lambd = 64, 2.48e-10
    dx_s = synth.sample_pixel(lambd, 1.0, 172e-6, N)
    beam = 10 * dx_s
    fzp = oracle.mls_zone_plate_probe(N, lambd, dx_s, beam)
    d = mls_dataset(oracle, N=N, nx=5, shifted=True, probe=fzp / np.abs(fzp).max())
    s = gpu_session(dict(amp=d["intens"], kw=d["kw"]), obj=d["obj"], calculateRMS=1, PPS=3)
    o = oracle.OracleMls(d["raw"], d["intens"], fzp, obj=d["obj"], variable=1, PPS=3)
    _check_default(s, o, "set-up")
    for it in range(1, 4):
        s.step()
        o.step()
        _check_default(s, o, f"iteration {it}")
    s.close()


def test_mls_default_path_tensor_core_fft(oracle):
    """precision=1 on the default path: the transforms run as split-BF16 tensor-core stages with the pointwise steps
    as separate kernels (the FP32 path fuses them into its FFT passes); both against the FP64 oracle."""
    d = mls_dataset(oracle, N=256, nx=3, shifted=True)
    runs = {prec: gpu_session(dict(amp=d["intens"], kw=d["kw"]), probe=d["probe"], obj=d["obj"], calculateRMS=1,
                              PPS=2, precision=prec) for prec in (0, 1)}
    o = oracle.OracleMls(d["raw"], d["intens"], d["probe"], obj=d["obj"], variable=1, PPS=2)
    for _ in range(3):
        for s in runs.values():
            s.step()
        o.step()
    ob, pr, _ = o.state()
    e32, etc = rel_err(runs[0].object(), ob), rel_err(runs[1].object(), ob)
    p32, ptc = rel_err(runs[0].probe(), pr), rel_err(runs[1].probe(), pr)
    print(f"MLs default path 256^2, 3 iterations vs FP64: object FP32 {e32:.2e}, TC {etc:.2e}; probe {p32:.2e}, {ptc:.2e}")
    assert e32 < TOL and p32 < TOL
    assert etc < 2e-3 and ptc < 2e-3
    for s in runs.values():
        s.close()


@pytest.mark.parametrize("K", [2, 3])
def test_mls_probe_modes_match_oracle(oracle, K):
    """probeModes > 1: modes 1..K-1 from phase tilts of mode 0 recombined by the eigenvectors of their Gram matrix,
    the modal modulus over sum |Psi_k|^2, per-mode probe steps, and ortho_modes after each iteration."""
    d = mls_dataset(oracle, N=64, nx=6, shifted=True)
    s = gpu_session(dict(amp=d["intens"], kw=d["kw"]), probe=d["probe"], obj=d["obj"], calculateRMS=1, PPS=3,
                    probeModes=K)
    o = oracle.OracleMls(d["raw"], d["intens"], d["probe"], obj=d["obj"], variable=1, PPS=3, K=K)
    for it in range(0, 5):
        if it:
            e = s.step()
            eo = o.step()
            print(f"MLs K={K} iteration {it}: error metric rel diff {abs(e - eo) / abs(eo):.2e}")
            assert abs(e - eo) <= ERR_TOL * abs(eo), f"error, iteration {it}"
        ob, pr, _ = o.state()
        gp = s.probe()
        assert gp.shape == (K, 64, 64)
        assert rel_err(s.object(), ob) < TOL, f"object, iteration {it}"
        for k in range(K):  # the weaker modes carry a few % of the power: each checked on its own scale
            assert rel_err(gp[k], pr[k]) < (TOL if k == 0 else 1e-3), f"mode {k}, iteration {it}"
        G = np.einsum("kxy,lxy->kl", gp.conj().astype(np.complex128), gp.astype(np.complex128))
        off = np.abs(G - np.diag(np.diag(G))).max() / np.abs(np.diag(G)).max()
        assert off < 1e-5, f"modes not orthogonal, iteration {it}"
    s.close()


def test_mls_default_path_groups_of_several(oracle):
    # 15x15 = 225 positions: groups of 2 and one of 1, delta_p 0.2, another seed; position search from iteration 2
    d = mls_dataset(oracle, N=32, nx=15, seed=4, shifted=True)
    s, o = _pair_default(oracle, d, 2, delta_p=0.2, seed=77)
    for it in range(4):
        s.step()
        o.step()
    _check_default(s, o, "iteration 4")
    s.close()


@pytest.mark.parametrize("N,nx", [(64, 6), (32, 11), (128, 4), (64, 2)])
def test_mls_matches_oracle(oracle, N, nx):
    d = mls_dataset(oracle, N=N, nx=nx)
    s, o = _pair(oracle, d)
    dims = s.dims()
    assert (dims["X"], dims["Y"]) == (d["X"], d["Y"])
    assert np.array_equal(s.positions(), d["raw"])
    ob, pr, _ = o.state()
    assert rel_err(s.object(), ob) < TOL, "set-up object"
    assert rel_err(s.probe(), pr) < TOL, "set-up probe"
    for it in range(1, 5):
        e = s.step()
        eo = o.step()
        ob, pr, _ = o.state()
        print(f"MLs core N={N} iteration {it}: error metric rel diff {abs(e - eo) / abs(eo):.2e}")
        assert rel_err(s.object(), ob) < TOL, f"object, iteration {it}"
        assert rel_err(s.probe(), pr) < TOL, f"probe, iteration {it}"
        assert abs(e - eo) <= ERR_TOL * abs(eo), f"error, iteration {it}"


def test_mls_groups_of_several_and_delta_p(oracle):
    # 15x15 = 225 positions: groups of 2 (P // 100) and one of 1; delta_p 0.2; another seed
    d = mls_dataset(oracle, N=32, nx=15, seed=4)
    s, o = _pair(oracle, d, delta_p=0.2, seed=77)
    for _ in range(3):
        s.step()
        o.step()
    ob, pr, _ = o.state()
    assert rel_err(s.object(), ob) < TOL and rel_err(s.probe(), pr) < TOL


def test_mls_flat_start_poisson_data(oracle):
    # Poisson data and a flat object: compare the Fourier-error trajectory, which is stable, and its decrease
    d = dataset(N=64, nx=8, algorithm="MLs")
    intens = (d["amp"].astype(np.float64) ** 2).astype(np.float32)
    raw = oracle.mls_raw_positions(8, 8, d["kw"]["stepx"], d["kw"]["stepy"], d["dx_s"])
    for core in (1, 0):
        s = gpu_session(dict(d, amp=intens), probe=d["probe"], calculateRMS=1, mlsCore=core, PPS=4)
        o = oracle.OracleMls(raw, intens, d["probe"][0], variable=1 - core, PPS=4)
        errs = [s.step() for _ in range(6)]
        errs_o = [o.step() for _ in range(6)]
        assert np.isfinite(errs).all() and errs[-1] < errs[0]
        np.testing.assert_allclose(errs, errs_o, rtol=2e-2)
        s.close()


def test_mls_tensor_core_fft_precision(oracle):
    """precision=1: the group FFTs run as split-BF16 tensor-core stages; error vs the FP64 oracle stated beside the
    FP32 run's (the mixed-precision result is reported with its error, not held to the FP32 bound)."""
    from ptychopy_b200 import abi

    d = mls_dataset(oracle, N=256, nx=3)
    runs = {}
    for prec in (0, 1):
        runs[prec] = gpu_session(dict(amp=d["intens"], kw=d["kw"]), probe=d["probe"], obj=d["obj"], calculateRMS=1,
                                 precision=prec, mlsCore=1)
    o = oracle.OracleMls(d["raw"], d["intens"], d["probe"], obj=d["obj"])
    for _ in range(3):
        for s in runs.values():
            s.step()
        o.step()
    ob, pr, _ = o.state()
    e32, etc = rel_err(runs[0].object(), ob), rel_err(runs[1].object(), ob)
    p32, ptc = rel_err(runs[0].probe(), pr), rel_err(runs[1].probe(), pr)
    print(f"MLs 256^2 after 3 iterations vs FP64: object FP32 {e32:.2e}, split-BF16 TC FFT {etc:.2e}; "
          f"probe {p32:.2e}, {ptc:.2e}")
    assert e32 < TOL and p32 < TOL
    assert etc < 2e-3 and ptc < 2e-3
    for s in runs.values():
        s.close()
    # DM fuses its FP32 transforms: precision=1 is refused; ePIE takes it at 256^2 only
    dd = dataset(N=64, nx=3)
    with pytest.raises(abi.PtyError):
        gpu_session(dict(dd, kw=dict(dd["kw"], algorithm="DM")), probe=dd["probe"], precision=1)
    with pytest.raises(abi.PtyError):
        gpu_session(dict(dd, kw=dict(dd["kw"], algorithm="ePIE")), probe=dd["probe"], precision=1)
