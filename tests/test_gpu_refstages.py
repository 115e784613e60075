"""The oracle pinned to the reference's own code.

oracle/_ref/libptyref.so holds the reference's hot-path device functions, compiled unchanged from the reference's
sources by oracle/ref_build.py (d_calculatePsi / d_modulusConstraint / d_updateObject, d_adjustFFT[Modal],
d_updateObjectArray[M], d_updateProbe[M], d_calculateER, the texture gather d_extractObjectArray and d_simulatePSI,
d_get_optimal_step_lsq, d_modulus_amplitude, d_generateMesh).  These tests run them on the GPU, launched as the
reference's host code launches them, and compare with the FP64 oracle (oracle/oracle.cpp), stage by stage and as
whole iterations composed the way the reference's host code composes them (src/DM.cu:80-128,
src/ePIE.cpp:65-129).  The FFTs between the stages are FP64 numpy transforms rounded to complex64 (cuFFT in the
reference).  Tolerances: FP32 reference code against the FP64 oracle.
"""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


def _torch():
    import torch

    return torch


def _dev(a, dtype=None):
    torch = _torch()
    return torch.from_numpy(np.ascontiguousarray(a, dtype)).cuda()


def _pitched(obj):
    """Object in the reference's pitched layout (rows of alignUp(Y, 32) complex64), as a CUDA tensor."""
    import pyref

    X, Y = obj.shape
    a = np.zeros((X, pyref.align32(Y)), np.complex64)
    a[:, :Y] = obj
    return _dev(a)


def _fft2(t, inverse=False):
    """FP64 2-D FFT of the last two axes of a complex64 CUDA tensor, unnormalised both ways, rounded to complex64."""
    a = t.cpu().numpy().astype(np.complex128)
    b = np.fft.ifft2(a) * a.shape[-1] * a.shape[-2] if inverse else np.fft.fft2(a)
    return _dev(b, np.complex64)


@pytest.fixture(scope="module")
def ref():
    import pyref

    pyref.lib()  # fails loudly when the library is missing
    return pyref


def test_ref_cartesian_mesh_bit_exact(ref, oracle):
    torch = _torch()
    for nx, ny, step, N, mx, my in [(10, 10, 50e-9, 128, 0, 0), (30, 30, 50e-9, 512, 0, 0), (51, 51, 100e-9, 256, 0, 0),
                                    (7, 13, 35e-9, 128, 1, 0), (5, 40, 80e-9, 64, 0, 1)]:
        lambd, z, dx_d = 2.48e-10, 1.0, 172e-6
        dx_s = np.float32(oracle.sample_pixel(lambd, z, dx_d, N))
        inv = np.float32(1.0 / np.float64(dx_s))
        ay = ref.align32(ny)
        pos = torch.zeros((nx * ay, 2), dtype=torch.float32, device="cuda")
        ref.call("ref_cartesian_mesh", ref.ptr(pos), nx, ny, float(np.float32(step)), float(np.float32(step)),
                 float(inv), mx, my)
        got = pos.cpu().numpy().reshape(nx, ay, 2)[:, :ny].reshape(-1, 2)
        want = oracle.cartesian_mesh_raw(nx, ny, step, step, lambd, z, dx_d, N, mx, my)
        assert np.array_equal(got, want), (nx, ny, N)


def test_ref_mesh_drift(ref, oracle):
    """d_generateMesh with a scan drift, Cartesian (several shapes, mirrored too), list and spiral (1100 points: two
    1024-wide mesh rows), against the oracle's restatement.  Cartesian and list positions are bit-exact; the
    spiral's cos/sin are CUDA's single-precision functions in the reference and double-precision ones rounded to
    float in the oracle, so those positions agree to a few units in the last place."""
    torch = _torch()
    lambd, z, dx_d, N = 2.48e-10, 1.0, 172e-6, 128
    inv = float(np.float32(1.0 / np.float64(np.float32(oracle.sample_pixel(lambd, z, dx_d, N)))))
    for drift in [(3.1e-9, -1.7e-9), (-2.5e-10, 4.25e-9)]:
        dr = tuple(float(np.float32(v)) for v in drift)
        for nx, ny, step, mx, my in [(7, 13, 35e-9, 0, 0), (30, 30, 50e-9, 1, 0), (5, 40, 80e-9, 0, 1)]:
            ay = ref.align32(ny)
            pos = torch.zeros((nx * ay, 2), dtype=torch.float32, device="cuda")
            s32 = float(np.float32(step))
            ref.call("ref_mesh", 1, ref.ptr(pos), nx, ny, s32, s32, inv, mx, my, dr[0], dr[1])
            got = pos.cpu().numpy().reshape(nx, ay, 2)[:, :ny].reshape(-1, 2)
            want = oracle.mesh_raw_drift("cartesian", lambd, z, dx_d, N, dr, nx=nx, ny=ny, stepx=step, stepy=step,
                                         mirrorX=mx, mirrorY=my)
            assert np.array_equal(got, want), (nx, ny, drift)
        xy = np.random.default_rng(5).random((1100, 2)) * 1e-6
        buf = np.zeros((2048, 2), np.float32)
        buf[:1100] = xy.astype(np.float32)
        pos = _dev(buf)
        ref.call("ref_mesh", 2, ref.ptr(pos), 2, 1024, 0.0, 0.0, inv, 0, 0, dr[0], dr[1])
        want = oracle.mesh_raw_drift("list", lambd, z, dx_d, N, dr, xy_m=xy)
        assert np.array_equal(pos.cpu().numpy(), want), drift
        pos = torch.zeros((2048, 2), dtype=torch.float32, device="cuda")
        s32 = float(np.float32(50e-9))
        ref.call("ref_mesh", 3, ref.ptr(pos), 2, 1024, s32, s32, inv, 0, 0, dr[0], dr[1])
        want = oracle.mesh_raw_drift("spiral", lambd, z, dx_d, N, dr, P=1100, stepx=50e-9, stepy=50e-9)
        assert np.abs(pos.cpu().numpy() - want).max() <= 4e-6 * np.abs(want).max(), drift


# The texture unit filters float texels with weights of 8 fractional bits (rounded to the nearest 1/256, pinned
# bit-exactly below) but with arithmetic of about 12 significant bits: gathered values differ from an exact FP32
# bilinear interpolation with the same weights by up to ~6e-4 of the object's magnitude (measured on B200).  The
# oracle and the engine interpolate exactly with the hardware's weights; where the texture's own arithmetic shows,
# the tests allow TEX_TOL for a gather and TEX_ITER_TOL for an ePIE iteration built on such gathers.
TEX_TOL = 1e-3
TEX_ITER_TOL = 2e-3


def test_ref_texture_weights_bit_exact(ref, oracle):
    """Ramps along each axis expose the filter weight alone (neighbours differ by exactly 1): the hardware's
    weight equals the oracle's round(frac * 256) / 256 at every coordinate, bit for bit."""
    torch = _torch()
    X, Y, N = 64, 64, 32
    out = torch.zeros((N, N), dtype=torch.complex64, device="cuda")
    for axis in (0, 1):
        ramp = np.zeros((X, Y), np.complex64)
        ramp += (np.arange(X, dtype=np.float32)[:, None] if axis == 0 else np.arange(Y, dtype=np.float32)[None, :])
        od = _pitched(ramp)
        for k in range(0, 2048, 3):
            q = np.float32(k / 2048.0 * 29.0)
            qx, qy = (float(q), 0.0) if axis == 0 else (0.0, float(q))
            ref.call("ref_extract_patch", ref.ptr(od), X, Y, ref.align32(Y), qx, qy, N, ref.ptr(out))
            want = oracle.extract_patch(ramp, np.float32(qx), np.float32(qy), N).astype(np.complex64)
            assert np.array_equal(out.cpu().numpy(), want), (axis, qx, qy)


def test_ref_texture_gather_matches_oracle(ref, oracle):
    """Random object: exact at integer positions (the filter weights are 0), within the texture unit's filter
    precision at fractional and edge positions."""
    from ptychopy_b200 import synth

    rng = np.random.default_rng(5)
    X, Y, N = 150, 170, 64
    obj = synth.make_object(X, Y, rng, corr_px=3.0).astype(np.complex64)
    od = _pitched(obj)
    torch = _torch()
    out = torch.zeros((N, N), dtype=torch.complex64, device="cuda")
    integral = [(0.0, 0.0), (3.0, 17.0), (X - N + 0.0, Y - N + 0.0)]
    fractional = [(12.37, 40.81), (55.5, 70.25), (X - N - 0.9, 0.3)]
    fractional += [tuple(map(float, rng.uniform(0, [X - N - 1, Y - N - 1]).astype(np.float32))) for _ in range(20)]
    scale = float(np.max(np.abs(obj)))
    for group, tol in ((integral, 1e-7), (fractional, TEX_TOL)):
        for qx, qy in group:
            ref.call("ref_extract_patch", ref.ptr(od), X, Y, ref.align32(Y), float(qx), float(qy), N, ref.ptr(out))
            want = oracle.extract_patch(obj, np.float32(qx), np.float32(qy), N)
            worst = float(np.max(np.abs(out.cpu().numpy() - want))) / scale
            assert worst < tol, (qx, qy, worst)


def test_ref_simulate_psi_matches_oracle(ref, oracle):
    from ptychopy_b200 import synth

    rng = np.random.default_rng(6)
    X, Y, N = 160, 160, 64
    obj = synth.make_object(X, Y, rng, corr_px=3.0).astype(np.complex64)
    probe = synth.make_probe(N, 1e-8, K=1, fwhm=10e-8)[0].astype(np.complex64)
    od, pd = _pitched(obj), _dev(probe)
    torch = _torch()
    out = torch.zeros((N, N), dtype=torch.complex64, device="cuda")
    for qx, qy, tol in [(10.0, 20.0, 1e-7), (33.6, 51.2, TEX_TOL), (80.25, 0.75, TEX_TOL)]:
        ref.call("ref_simulate_psi", ref.ptr(od), X, Y, ref.align32(Y), ref.ptr(pd), qx, qy, N, ref.ptr(out))
        want = oracle.extract_patch(obj, np.float32(qx), np.float32(qy), N) * probe
        assert rel_err(out.cpu().numpy(), want) < tol


def _factor_after_check_cache(cached, maxval):
    """DM::checkCache (src/DM.cu:54-73): the cached factor moves to 1/max only if it changed by more than 1e-3."""
    passed = np.float32(1.0 / np.float32(maxval))
    return passed if abs(np.float32(cached) - passed) > 1e-3 else np.float32(cached)


@pytest.mark.parametrize("pc,up", [(0, 1), (1, 1), (1, 0)])
def test_ref_dm_iteration_matches_oracle(ref, oracle, pc, up):
    """One reference DM iteration from the reference's own callbacks (forward load d_calculatePsi, forward store
    d_modulusConstraint, inverse store d_updateObject) against the oracle's, from the oracle's state after one
    iteration (non-zero exit waves).  Each position's callback increments go to its own copy of O and P (snapshot
    semantics, which the reference approximates with racing atomics)."""
    from gpu_helpers import dataset

    torch = _torch()
    d = dataset(N=64, nx=4, algorithm="DM")
    X, Y, N, P = d["X"], d["Y"], 64, d["amp"].shape[0]
    # the probe updates from iteration 2: in iteration 1 the object factor is 1/0 (the object starts at zero)
    o = oracle.OracleSession("DM", d["amp"], d["pos"], np.zeros((X, Y)), d["probe"], probe_guess_path=False,
                             updateProbe=2 if up else 99, phaseConstraint=2 if pc else 0)
    o.step()
    O1, P1, sc1 = o.state()
    psi1 = o.psi()
    o.step()
    O2, P2, _ = o.state()
    psi2 = o.psi()
    o.close()

    f0 = _factor_after_check_cache(sc1[2], sc1[0])
    f1 = _factor_after_check_cache(sc1[3], sc1[1])
    ay = ref.align32(Y)
    pos = _dev(d["pos"], np.float32)
    od = _pitched(O1.astype(np.complex64))
    pd = _dev(P1[0], np.complex64)
    psi = _dev(psi1, np.complex64)
    A = _dev(d["amp"], np.float32)
    u = torch.empty_like(psi)
    ref.call("ref_dm_calc_psi", ref.ptr(psi), ref.ptr(od), ref.ptr(pd), ref.ptr(pos), P, N, X, Y, ay, ref.ptr(u))
    Psi = _fft2(u)
    Psim = torch.empty_like(Psi)
    ref.call("ref_dm_modulus", ref.ptr(Psi), ref.ptr(A), P, N, ref.ptr(Psim))
    Pf = _fft2(Psim, inverse=True)
    ocopies = od.unsqueeze(0).repeat(P, 1, 1).contiguous()
    pcopies = pd.unsqueeze(0).repeat(P, 1, 1).contiguous()
    flags = torch.tensor([bool(pc), bool(up)], dtype=torch.bool, device="cuda")
    factors = torch.tensor([f0, f1], dtype=torch.float32, device="cuda")
    out = torch.empty_like(psi)
    ref.call("ref_dm_update", ref.ptr(Pf), ref.ptr(psi), ref.ptr(ocopies), ref.ptr(pcopies), ref.ptr(pos),
             ref.ptr(flags), ref.ptr(factors), P, N, X, Y, ay, ref.ptr(out))
    O1p = od.cpu().numpy().astype(np.complex128)
    O_ref = O1p + (ocopies.cpu().numpy().astype(np.complex128) - O1p[None]).sum(0)
    P_ref = P1[0] + (pcopies.cpu().numpy().astype(np.complex128) - P1[0].astype(np.complex64)[None]).sum(0)
    assert rel_err(O_ref[:, :Y], O2) < 1e-5
    assert rel_err(P_ref, P2[0]) < 1e-5
    assert rel_err(psi.cpu().numpy(), psi2) < 1e-5
    assert np.array_equal(out.cpu().numpy(), psi.cpu().numpy())


def _modal_max(cache, use_all):
    """Probe::getModalDoubleMax (src/utilities.cpp:204-216)."""
    if use_all and cache.shape[0] > 1:
        return float(cache.sum(0).max())
    return float(cache.max())


@pytest.mark.parametrize("K,fractional", [(1, False), (2, False), (1, True), (2, True)])
def test_ref_epie_iteration_matches_oracle(ref, oracle, K, fractional):
    """Two ePIE iterations composed from the reference's kernels in the order of src/ePIE.cpp:65-129 (texture
    gather, mode products, d_adjustFFT[Modal], d_updateObjectArray[M], d_updateProbe[M], d_calculateER), with the
    oracle's seeded visiting order, against the oracle's iterations: object, probe and the error metric.  At
    integer positions the gather is exact and the tolerance is FP32 round-off; at the raster's fractional positions
    the texture unit's filter arithmetic shows (TEX_TOL)."""
    from gpu_helpers import dataset
    from ptychopy_b200 import synth

    torch = _torch()
    d = dataset(N=64, nx=4, K=K, algorithm="ePIE")
    X, Y, N, P = d["X"], d["Y"], 64, d["amp"].shape[0]
    if not fractional:
        d["pos"] = np.floor(d["pos"] + 0.5).astype(np.float32)
    tol = TEX_ITER_TOL if fractional else 1e-5
    seed = 0x1234
    probe0 = d["probe"].astype(np.complex64)
    # a non-zero start object: from a zero object the reference's modal modulus divides 0 by 0 (NaN), which the
    # oracle pins to 0
    obj0 = synth.make_object(X, Y, np.random.default_rng(99), corr_px=6.0).astype(np.complex64)
    # modes switch on from iteration 1 only for K > 1 with given modes: for one mode, beginModalReconstruction
    # re-reads the probe maximum from its intensity cache, which a given probe leaves at zero (1/0 in the update)
    upd_modes = 1 if K > 1 else 99
    o = oracle.OracleSession("ePIE", d["amp"], d["pos"], obj0, probe0, probe_guess_path=False,
                             modes_given=K > 1, seed=seed, updateProbe=1, updateModes=upd_modes, phaseConstraint=1,
                             calculateRMS=1)
    ay = ref.align32(Y)
    O = _pitched(obj0)
    Oc = torch.zeros((X, ay), dtype=torch.float32, device="cuda")
    Pr = _dev(probe0.reshape(K, N, N))
    Pc = torch.zeros((K, N, N), dtype=torch.float32, device="cuda")
    A = _dev(d["amp"], np.float32)
    sqsum = d["amp"].astype(np.float32).sum(axis=(1, 2), dtype=np.float32)
    patch = torch.zeros((N, N), dtype=torch.complex64, device="cuda")
    partial = torch.zeros(N, dtype=torch.float32, device="cuda")
    obj_max, probe_max = 0.0, 1.0  # Sample starts at 0 (src/Sample.cpp:216-220); a given probe keeps 1
    state = seed
    for it in (1, 2):
        pc, use_all = it <= 1, it >= upd_modes
        order, state = oracle.visiting_order(state, P)
        err = 0.0
        for i in order:
            qx, qy = float(d["pos"][i, 0]), float(d["pos"][i, 1])
            ref.call("ref_extract_patch", ref.ptr(O), X, Y, ay, qx, qy, N, ref.ptr(patch))
            psi_old = (patch.unsqueeze(0) * Pr).contiguous()
            Psi = _fft2(psi_old)
            Psim = torch.empty_like(Psi)
            ref.call("ref_adjust_fft", ref.ptr(Psi), ref.ptr(Psim), ref.ptr(A[i]), None, float("inf"), K, N)
            psi = _fft2(Psim, inverse=True)
            ox, oy = int(np.floor(qx + 0.5)), int(np.floor(qy + 0.5))  # roundf of positive positions
            ref.call("ref_update_object", ref.ptr(O), ref.ptr(Pr), ref.ptr(psi), ref.ptr(psi_old), ref.ptr(Oc), ox, oy,
                     float(np.float32(1.0 / probe_max)), K, N, X, Y, ay, int(pc))
            obj_max = float(Oc.max())
            ref.call("ref_update_probe", ref.ptr(Pr), ref.ptr(O), ref.ptr(psi), ref.ptr(psi_old), ref.ptr(Pc), ox, oy,
                     float(np.float32(1.0 / obj_max)), K, N, X, Y, ay)
            probe_max = _modal_max(Pc.cpu().numpy(), use_all)
            ref.call("ref_calculate_er", ref.ptr(Psi), ref.ptr(A[i]), K, N, ref.ptr(partial))
            err += float(partial.sum().item()) / K / float(sqsum[i])
        err /= P
        e_orc = o.step()
        Oo, Po, _ = o.state()
        assert rel_err(O.cpu().numpy()[:, :Y], Oo) < tol, f"object, iteration {it}"
        assert rel_err(Pr.cpu().numpy(), Po) < tol, f"probe, iteration {it}"
        assert abs(err - e_orc) <= tol * abs(e_orc), f"error metric, iteration {it}: {err} vs {e_orc}"
    o.close()


def test_ref_mls_stage_terms_match_oracle(ref, oracle):
    """The MLs modulus factor (d_modulus_amplitude) and step-length system terms (d_get_optimal_step_lsq)."""
    torch = _torch()
    rng = np.random.default_rng(9)
    N = 64

    def c64():
        return (rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N))).astype(np.complex64)

    chi, oup, dPO, probe = c64(), c64(), c64(), c64()
    lam = np.float32(np.finfo(np.float32).eps / (N * N))
    dev = [_dev(v) for v in (chi, oup, dPO, probe)]
    AA1, AA4, Atb1, Atb2 = (torch.zeros((N, N), dtype=torch.float32, device="cuda") for _ in range(4))
    AA2 = torch.zeros((N, N), dtype=torch.complex64, device="cuda")
    ref.call("ref_lsq_terms", *(ref.ptr(t) for t in dev), float(lam), N, ref.ptr(AA1), ref.ptr(AA2), ref.ptr(AA4),
             ref.ptr(Atb1), ref.ptr(Atb2))
    want = oracle.mls_lsq_terms(chi, oup, dPO, probe, float(lam))
    for got, w in zip((AA1, AA2, AA4, Atb1, Atb2), want):
        assert rel_err(got.cpu().numpy().ravel(), w) < 1e-6
    A = np.abs(rng.standard_normal((N, N))).astype(np.float32)
    ap = np.abs(rng.standard_normal((N, N))).astype(np.float32) + 0.05
    res = torch.zeros((N, N), dtype=torch.float32, device="cuda")
    Ad, apd = _dev(A), _dev(ap)  # held: a temporary's memory could be handed to the next allocation
    ref.call("ref_modulus_amplitude", ref.ptr(Ad), ref.ptr(apd), ref.ptr(res), 1.0, N)
    assert rel_err(res.cpu().numpy().ravel(), oracle.mls_modulus_factor(A, ap)) < 1e-6
