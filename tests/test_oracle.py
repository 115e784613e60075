"""The oracle against numpy.fft, hand-derived known answers and the reference's geometry (CPU only)."""
import numpy as np
import pytest

from conftest import rel_err


@pytest.mark.parametrize("N", [8, 32, 64, 128])
def test_fft_matches_numpy(oracle, N):
    rng = np.random.default_rng(N)
    a = rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N))
    assert rel_err(oracle.fft2(a), np.fft.fft2(a)) < 1e-13
    assert rel_err(oracle.fft2(a, inverse=True), np.fft.ifft2(a) * N * N) < 1e-13


def test_fft_known_answers(oracle):
    N = 16
    d = np.zeros((N, N), complex)
    d[0, 0] = 1
    assert np.allclose(oracle.fft2(d), 1.0)  # delta -> flat
    x = np.arange(N)
    pw = np.exp(2j * np.pi * (3 * x[:, None] + 5 * x[None, :]) / N)  # plane wave -> single bin (3, 5)
    F = oracle.fft2(pw)
    assert abs(F[3, 5] - N * N) < 1e-9 and np.abs(np.delete(F.ravel(), 3 * N + 5)).max() < 1e-9


# object sizes and raster steps of the configurations (dx_s = lambda*z/(N*dx_d), object ceil(extent + N))
@pytest.mark.parametrize("nx,step,lam,z,dxd,N,X,step_px", [
    (10, 50e-9, 2.48e-10, 1.0, 172e-6, 128, 168, 4.4386),
    (30, 50e-9, 2.48e-10, 1.0, 172e-6, 512, 1027, 17.7548),
    (51, 100e-9, 1.409e-10, 1.92, 75e-6, 256, 611, 7.0972),
    (64, 50e-9, 2.48e-10, 1.0, 172e-6, 128, 408, 4.4386),
])
def test_geometry_configs(oracle, nx, step, lam, z, dxd, N, X, step_px):
    pos, gx, gy = oracle.cartesian_mesh(nx, nx, step, step, lam, z, dxd, N)
    assert (gx, gy) == (X, X)
    assert pos.min() == 0.0
    assert abs(pos[1, 1] - pos[0, 1] - step_px) < 1e-3
    assert abs(pos[nx, 0] - pos[0, 0] - step_px) < 1e-3


def test_geometry_matches_synth(oracle):
    from ptychopy_b200 import synth

    dx_s = synth.sample_pixel(2.48e-10, 1.0, 172e-6, 128)
    assert dx_s == oracle.sample_pixel(2.48e-10, 1.0, 172e-6, 128)
    p1, X1, Y1 = synth.raster_positions(10, 7, 50e-9, 60e-9, dx_s, 128)
    p2, X2, Y2 = oracle.cartesian_mesh(10, 7, 50e-9, 60e-9, 2.48e-10, 1.0, 172e-6, 128)
    assert (X1, Y1) == (X2, Y2)
    assert np.array_equal(p1, p2)


def test_list_mesh_zero_padding(oracle):
    # positions all > 0: the (0,0) padding entries of the 1024-wide list mesh join the min (P % 1024 != 0)
    xy = np.array([[1e-6, 2e-6], [1.5e-6, 2.5e-6]])
    pos, X, Y = oracle.list_mesh(xy, 2.48e-10, 1.0, 172e-6, 128)
    dx_s = oracle.sample_pixel(2.48e-10, 1.0, 172e-6, 128)
    assert abs(pos[0, 0] - 1e-6 / dx_s) < 1e-2
    assert X == int(np.ceil(np.float32(1.5e-6 / dx_s) + 128))


def test_patch_integer_and_half_offsets(oracle):
    rng = np.random.default_rng(1)
    O = rng.standard_normal((20, 24)) + 1j * rng.standard_normal((20, 24))
    p = oracle.extract_patch(O, 3.0, 5.0, 8)
    assert np.allclose(p, O[3:11, 5:13])
    h = oracle.extract_patch(O, 3.0, 5.5, 8)  # weight exactly 1/2 between columns
    assert np.allclose(h, 0.5 * (O[3:11, 5:13] + O[3:11, 6:14]))


def test_patch_weights_quantised(oracle):
    O = np.zeros((10, 10), complex)
    O[:, 5] = 1.0
    p = oracle.extract_patch(O, 0.0, 4.3, 4)  # fraction 0.3 -> round(0.3*256)/256 = 77/256
    assert abs(p[0, 0].real - 77 / 256) < 1e-12


def test_visiting_order_is_a_permutation(oracle):
    order, s2 = oracle.visiting_order(1234, 50)
    assert sorted(order.tolist()) == list(range(50))
    order2, _ = oracle.visiting_order(s2, 50)
    assert not np.array_equal(order, order2)
    again, _ = oracle.visiting_order(1234, 50)
    assert np.array_equal(order, again)


def _toy(N=16, nx=3, seed=0, K=1):
    from ptychopy_b200 import synth

    rng = np.random.default_rng(seed)
    dx_s = synth.sample_pixel(2.48e-10, 1.0, 172e-6, N)
    pos, X, Y = synth.raster_positions(nx, nx, 30e-9, 30e-9, dx_s, N)
    obj = synth.make_object(X, Y, rng, corr_px=3.0)
    probe = synth.make_probe(N, dx_s, K=K, fwhm=8 * dx_s)
    return pos, X, Y, obj, probe


def test_epie_fixed_point(oracle):
    # amplitudes generated from the current object and probe: the modulus projection is the identity and an
    # iteration leaves object and probe unchanged
    N = 16
    pos, X, Y, obj, probe = _toy(N)
    obj, probe = obj.astype(np.complex128), probe.astype(np.complex128)
    amp = []
    for q in pos:
        o = np.round(q).astype(int)
        amp.append(np.abs(np.fft.fft2(obj[o[0]:o[0] + N, o[1]:o[1] + N] * probe[0])))
    amp = np.array(amp)
    s = oracle.OracleSession("ePIE", amp, np.round(pos), obj, probe, probe_guess_path=False, updateProbe=1,
                             phaseConstraint=0)
    s.step()
    o2, p2, _ = s.state()
    assert rel_err(o2, obj) < 1e-12 and rel_err(p2, probe) < 1e-12


def test_dm_first_iteration_known_answer(oracle):
    # From a zero object and zero exit waves: Psi = 0, so Psi' = A/N^2 (phase 0), psi_1 = IFFT2(A)/N^2 and
    # O_1 = (1/probeMax) * sum_j conj(P) psi_1,j placed at the rounded offsets (phase-clamped increments).
    N = 16
    pos, X, Y, obj, probe = _toy(N, seed=3)
    rng = np.random.default_rng(5)
    amp = rng.uniform(0.0, 2.0, size=(pos.shape[0], N, N))
    s = oracle.OracleSession("DM", amp, pos, np.zeros((X, Y)), probe, probe_guess_path=False)
    s.step()
    o1, _, sc = s.state()
    expect = np.zeros((X, Y), complex)
    for j, q in enumerate(pos):
        ox, oy = np.round(q).astype(int)
        psi1 = np.fft.ifft2(amp[j])  # = IFFT_unnormalised(A)/N^2
        inc = np.conj(probe[0]) * psi1 * 1.0  # probeMax = 1 for a supplied probe
        inc = np.where(np.angle(inc) > 0, np.abs(inc), inc)  # phaseConstraint = 1 at iteration 1
        expect[ox:ox + N, oy:oy + N] += inc
    assert rel_err(o1, expect) < 1e-12
    assert abs(sc[0] - np.sum(np.abs(expect) ** 2)) / sc[0] < 1e-12
    psi = s.psi()
    assert rel_err(psi[0], np.fft.ifft2(amp[0])) < 1e-12


def test_probe_guess_matches_mean_amplitude(oracle):
    rng = np.random.default_rng(2)
    N = 32
    amp = rng.uniform(0.1, 1.0, size=(6, N, N))
    dx_s = oracle.sample_pixel(2.48e-10, 1.0, 172e-6, N)
    P = oracle.probe_guess(amp, 110e-9, dx_s, K=2)
    assert abs(np.abs(P[0]).max() - 1.0) < 1e-12 and np.abs(P[1]).max() == 0
    F = np.abs(np.fft.fft2(P[0]))
    avg = amp.mean(0)
    ratio = F / avg
    assert ratio.std() / ratio.mean() < 1e-10


def test_mls_geometry_holds_every_window(oracle):
    import math

    from ptychopy_b200 import synth

    N = 64
    dx_s = synth.sample_pixel(2.48e-10, 1.0, 172e-6, N)
    raw = oracle.mls_raw_positions(7, 5, 40e-9, 55e-9, dx_s)
    assert raw.dtype == np.float32 and raw.shape == (35, 2)
    assert abs(raw[:, 0].mean()) < 1e-4 and abs(raw[:, 1].mean()) < 1e-4
    X, Y, starts, roi = oracle.mls_geometry(raw, N)
    # object = ceil(1.2 * extent); the extent of axis x is measured on the positions' y and vice versa
    ext_x = np.round(raw[:, 1]).max() - np.round(raw[:, 1]).min() + N - 1
    ext_y = np.round(raw[:, 0]).max() - np.round(raw[:, 0]).min() + N - 1
    assert abs(X - math.ceil(1.2 * ext_x)) <= 1 and abs(Y - math.ceil(1.2 * ext_y)) <= 1
    assert starts.min() >= 0 and (starts[:, 0] + N).max() <= X and (starts[:, 1] + N).max() <= Y
    assert roi[2] > 0 and roi[3] > 0 and roi[0] >= 0 and roi[1] >= 0


def test_mls_oracle_reduces_the_fourier_error(oracle):
    from gpu_helpers import dataset

    d = dataset(N=32, nx=6, algorithm="MLs")
    intens = d["amp"].astype(np.float64) ** 2
    raw = oracle.mls_raw_positions(6, 6, d["kw"]["stepx"], d["kw"]["stepy"], d["dx_s"])
    m = oracle.OracleMls(raw, intens, d["probe"][0])
    errs = [m.step() for _ in range(8)]
    assert np.isfinite(errs).all() and errs[-1] < 0.8 * errs[0]


def test_mls_default_path_forward_model_matches_numpy_shift(oracle):
    """The default MLs path shifts each position's probe by its sub-pixel remainder.  On data made with numpy's
    Fourier-shift model (gpu_helpers.shifted_probe) it converges far below the same data without the shift in the
    model (the core path), and below its own error on unshifted data: the shift's sign and axes match numpy's."""
    from gpu_helpers import mls_dataset

    res = {}
    for shifted in (True, False):
        d = mls_dataset(oracle, N=32, nx=6, shifted=shifted, pert=0.0)
        for var in (1, 0):
            m = oracle.OracleMls(d["raw"], d["intens"], d["probe"], obj=d["obj"], variable=var, PPS=100)
            res[shifted, var] = [m.step() for _ in range(8)][-1]
    assert res[True, 1] < 0.3 * res[True, 0], res
    assert res[True, 1] < 0.3 * res[False, 1], res


def test_mls_default_path_position_search_starts_at_pps(oracle):
    from gpu_helpers import mls_dataset

    d = mls_dataset(oracle, N=32, nx=5, shifted=True)
    for pps in (3, 100):
        m = oracle.OracleMls(d["raw"], d["intens"], d["probe"], obj=d["obj"], variable=1, PPS=pps)
        moved = []
        for _ in range(4):
            m.step()
            moved.append(float(np.abs(m.variable_state()[3] - d["raw"]).max()))
        if pps == 3:
            assert moved[0] == moved[1] == 0.0 and moved[2] > 0.0, moved
            assert max(moved) < 0.2 * 4 * d["raw"].shape[0]  # at most 0.2 px per visit
        else:
            assert max(moved) == 0.0, moved
        E, e0, e1, _ = m.variable_state()
        assert abs(np.sqrt(np.mean(np.abs(E) ** 2)) - 1.0) < 1e-6  # unit-RMS extra mode after each update
        assert np.isfinite(e0).all() and np.isfinite(e1).all()


def test_spiral_mesh(oracle):
    lam, z, dxd, N = 2.48e-10, 1.0, 172e-6, 128
    dx_s = oracle.lib().orc_sample_pixel(lam, z, dxd, N)
    P = 100
    pos, X, Y = oracle.spiral_mesh(P, 50e-9, 50e-9, lam, z, dxd, N)
    # point i sits at sqrt(i)*(cos, sin)(4 sqrt(i))*step/dx_s before the shift; point 0 is the centre
    i = np.arange(P, dtype=np.float64)
    r = np.sqrt(i) * 50e-9 / dx_s
    ref = np.stack([r * np.cos(4 * np.sqrt(i)), r * np.sin(4 * np.sqrt(i))], 1)
    d = pos - pos[0]
    assert np.allclose(d, ref - ref[0], atol=1e-3)
    # the object covers the whole 1024-point spiral of the mesh array, not only the first P points
    i2 = np.arange(1024, dtype=np.float64)
    r2 = np.sqrt(i2) * 50e-9 / dx_s
    ext = (r2 * np.cos(4 * np.sqrt(i2))).max() - (r2 * np.cos(4 * np.sqrt(i2))).min()
    assert abs(X - np.ceil(ext + N)) <= 1
    assert pos.min() >= 0 and (pos + N).max() <= max(X, Y) + 1


def test_jitter_stream_and_bounds(oracle):
    j1 = oracle.mesh_jitter(7, 500, 3)
    j2 = oracle.mesh_jitter(7, 500, 3)
    assert np.array_equal(j1, j2)
    assert (np.abs(j1) <= 3).all() and j1.std() > 1.0
    assert not np.array_equal(j1, oracle.mesh_jitter(8, 500, 3))
    assert (oracle.mesh_jitter(7, 10, 0) == 0).all()
    p0, X0, Y0 = oracle.cartesian_mesh(6, 6, 50e-9, 50e-9, 2.48e-10, 1.0, 172e-6, 64)
    p1, X1, Y1 = oracle.cartesian_mesh(6, 6, 50e-9, 50e-9, 2.48e-10, 1.0, 172e-6, 64, jitter=2, seed=7)
    # jitter moves each point by at most the radius relative to the others (the -min shift moves all together)
    d = (p1 - p1[0]) - (p0 - p0[0])
    assert np.abs(d).max() <= 4.0 + 1e-4 and np.abs(d).max() > 0.1


def test_list_mesh_padding_joins_extent(oracle):
    # positions far from the origin: the (0, 0) padding of the 1024-wide mesh array enlarges the object
    xy = np.stack([np.linspace(1e-6, 2e-6, 20), np.linspace(1e-6, 1.5e-6, 20)], 1)
    pos, X, Y = oracle.list_mesh(xy, 2.48e-10, 1.0, 172e-6, 64)
    dx_s = oracle.lib().orc_sample_pixel(2.48e-10, 1.0, 172e-6, 64)
    assert X == int(np.ceil(np.float32(2e-6 / dx_s) + 64))
    # shifted by the padding's minimum (0), not by the list's own minimum
    assert abs(pos[:, 0].min() - 1e-6 / dx_s) < 1e-3 and abs(pos[:, 1].min() - 1e-6 / dx_s) < 1e-3


def test_mls_default_path_position_steps_are_clamped(oracle):
    """Each iteration moves every position by one common recentring shift (positions minus their mean drift from
    the originals) plus its own least-squares step, clamped to 0.2 px per axis: per axis, the moves of one iteration
    spread over at most 0.4 px.  The data are made at positions up to 1 px away from the nominal ones, so the search
    takes steps near the clamp."""
    from gpu_helpers import mls_dataset, shifted_probe, subpixel_shifts

    N = 32
    d = mls_dataset(oracle, N=N, nx=5, shifted=True, pert=0.0)
    sx, sy = subpixel_shifts(d["raw"], d["X"], d["Y"], N)
    ex, ey = np.random.default_rng(7).uniform(-1.0, 1.0, (2, len(sx)))
    o, p = d["obj"].astype(np.complex128), np.asarray(d["probe"], np.complex128)
    intens = np.stack([np.abs(np.fft.fft2(shifted_probe(p, sx[k] + ex[k], sy[k] + ey[k]) * o[r:r + N, c:c + N])) ** 2
                       for k, (r, c) in enumerate(d["starts"])]).astype(np.float32)
    m = oracle.OracleMls(d["raw"], intens, d["probe"], obj=d["obj"], variable=1, PPS=2)
    prev = m.variable_state()[3].astype(np.float64)
    spreads = []
    for _ in range(5):
        m.step()
        cur = m.variable_state()[3].astype(np.float64)
        step = cur - prev
        spreads.append(float((step.max(axis=0) - step.min(axis=0)).max()))
        prev = cur
    assert spreads[0] == 0.0, spreads  # no search before iteration PPS
    assert max(spreads) <= 0.4 + 1e-4, spreads
    assert max(spreads) > 0.2, spreads  # the search takes steps of the clamp's order


def test_scan_drift(oracle):
    """The scan drift adds row * driftx and column * drifty metres before the pixel conversion
    (src/ScanMeshKernels.cu:86-87): raster rows move by i * driftx / dx_s; list and spiral points by their row
    (index / 1024) and column (index % 1024) of the mesh array.  A zero drift changes nothing."""
    lam, z, dxd, N = 2.48e-10, 1.0, 172e-6, 64
    dx_s = oracle.lib().orc_sample_pixel(lam, z, dxd, N)
    dr = (3e-9, -2e-9)
    raw0 = oracle.mesh_raw_drift("cartesian", lam, z, dxd, N, (0.0, 0.0), nx=5, ny=7, stepx=50e-9, stepy=40e-9)
    assert np.array_equal(raw0, oracle.cartesian_mesh_raw(5, 7, 50e-9, 40e-9, lam, z, dxd, N))
    raw = oracle.mesh_raw_drift("cartesian", lam, z, dxd, N, dr, nx=5, ny=7, stepx=50e-9, stepy=40e-9)
    i, j = np.divmod(np.arange(35), 7)
    assert np.allclose(raw - raw0, np.stack([i * dr[0], j * dr[1]], 1) / dx_s, atol=1e-4)
    p0, X0, Y0 = oracle.cartesian_mesh(5, 7, 50e-9, 40e-9, lam, z, dxd, N)
    p1, X1, Y1 = oracle.cartesian_mesh(5, 7, 50e-9, 40e-9, lam, z, dxd, N, drift=dr)
    assert (X1, Y1) != (X0, Y0) and p1.min() >= 0
    xy = np.random.default_rng(2).random((1100, 2)) * 1e-6
    l0 = oracle.mesh_raw_drift("list", lam, z, dxd, N, (0.0, 0.0), xy_m=xy)
    l1 = oracle.mesh_raw_drift("list", lam, z, dxd, N, dr, xy_m=xy)
    assert l1.shape == (2048, 2) and np.array_equal(l0[1100:], np.zeros((948, 2), np.float32))
    r, c = np.divmod(np.arange(2048), 1024)
    assert np.allclose(l1 - l0, np.stack([r * dr[0], c * dr[1]], 1) / dx_s, atol=1e-4)
    assert np.array_equal(oracle.list_mesh(xy, lam, z, dxd, N)[0], oracle.list_mesh(xy, lam, z, dxd, N, drift=(0, 0))[0])
    s0 = oracle.mesh_raw_drift("spiral", lam, z, dxd, N, (0.0, 0.0), P=1100, stepx=50e-9, stepy=50e-9)
    s1 = oracle.mesh_raw_drift("spiral", lam, z, dxd, N, dr, P=1100, stepx=50e-9, stepy=50e-9)
    assert np.allclose(s1 - s0, np.stack([r * dr[0], c * dr[1]], 1) / dx_s, atol=1e-3)


def test_saturation_level(oracle):
    """Parameters::updatePixelSaturation (src/Parameters.cpp:54-62): 2^bitDepth - 1 - threshold, square-rooted with
    sqrtData, truncated at each step; no level (inf) unless one of the three is given."""
    assert oracle.saturation_level() == np.inf
    assert oracle.saturation_level(16, 0, 1) == 255.0  # floor(sqrt(65535)) = 255, not 255.998
    assert oracle.saturation_level(8, 5, 0) == 250.0
    assert oracle.saturation_level(0, 0, 1) == 65535.0
    assert oracle.saturation_level(0, 7, 0) == float(np.float32(2.0 ** 32 - 8))
    assert oracle.saturation_level(4, 100, 0) == 0.0  # a threshold above the range: every pixel floats


def test_oracle_floating_pixels(oracle):
    """An oracle ePIE iteration with a saturation level above every amplitude equals one without; a level inside
    the data's range changes it."""
    rng = np.random.default_rng(3)
    N, X = 32, 48
    amp = rng.random((4, N, N)) * 10
    pos = np.array([[0, 0], [8, 4], [16, 16], [3, 11]], np.float32)
    probe = (rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N))) * 0.1
    obj = np.ones((X, X), np.complex128)
    runs = [oracle.OracleSession("ePIE", amp, pos, obj, probe, probe_guess_path=False, saturation=sat)
            for sat in (None, 11.0, 5.0)]
    for o in runs:
        o.step()
    (o0, _, _), (o1, _, _), (o2, _, _) = (o.state() for o in runs)
    assert np.array_equal(o0, o1) and not np.allclose(o0, o2)
