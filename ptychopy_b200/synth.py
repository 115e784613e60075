"""Seeded synthetic ptychography data (the stand-in for the reference's APS beamline data, which is not public).

Object: amplitude uniform in [0.8, 1.0], phase a Gaussian random field (Gaussian-filtered white noise,
correlation length 8 px) rescaled to [-pi/2, pi/2], sized to the scan extent plus the window.
Probe: 110 nm FWHM Gaussian-apodised focused beam with a weak defocus phase; for K > 1 orthonormalised
Hermite-Gauss modes HG(0,0), (1,0), (0,1), (1,1), (2,0), ... carrying the given power weights.
Patterns: I = sum_k |FFT2(O_patch * P_k)|^2 (no fftshift, like the reference's simulate mode,
src/Diffractions.cpp:80-117), scaled so the mean pattern holds `photons` counts, Poisson-sampled; ePIE/DM take
sqrt(counts), MLs takes counts.
Scan: the reference's Cartesian raster in FP32 (src/ScanMeshKernels.cu:46-93, src/IPtychoScanMesh.cpp:86-109).
"""
import numpy as np

# name: (alg, N, lambda, z, dx_d, nx, ny, step, photons, iters, K)
CONFIGS = {
    "epie128": dict(algorithm="ePIE", N=128, lambd=2.48e-10, z=1.0, dx_d=172e-6, nx=10, ny=10, step=50e-9,
                    photons=1e6, iters=20, K=1),
    "dm512": dict(algorithm="DM", N=512, lambd=2.48e-10, z=1.0, dx_d=172e-6, nx=30, ny=30, step=50e-9,
                  photons=1e7, iters=100, K=1),
    "epie256k5": dict(algorithm="ePIE", N=256, lambd=1.409e-10, z=1.92, dx_d=75e-6, nx=51, ny=51, step=100e-9,
                      photons=1e6, iters=100, K=5),
    "warm128": dict(algorithm="ePIE", N=128, lambd=2.48e-10, z=1.0, dx_d=172e-6, nx=64, ny=64, step=50e-9,
                    photons=1e5, iters=100, K=1),
}
MODE_WEIGHTS = (0.6, 0.2, 0.1, 0.06, 0.04)
BEAM_FWHM = 110e-9


def sample_pixel(lambd, z, dx_d, N):
    """Object pixel size dx_s = lambda*z/(N*dx_d), rounded to float32 as the reference returns it."""
    return float(np.float32(lambd * z / (N * dx_d)))


def raster_positions(nx, ny, stepx, stepy, dx_s, N):
    """(P, 2) float32 pixel positions in raster order i*ny+j after the -min shift, and the object size."""
    f = np.float32
    inv, sx, sy = f(1.0 / dx_s), f(stepx), f(stepy)
    mdx, mdy = f(nx - 1) * f(0.5), f(ny - 1) * f(0.5)
    px = ((np.arange(nx, dtype=f) - mdx) * sx) * inv
    py = ((np.arange(ny, dtype=f) - mdy) * sy) * inv
    pos = np.stack([np.repeat(px, ny), np.tile(py, nx)], axis=1).astype(f)
    mn, mx = pos.min(0), pos.max(0)
    X = int(np.ceil((mx[0] - mn[0]) + f(N)))
    Y = int(np.ceil((mx[1] - mn[1]) + f(N)))
    return (pos - mn).astype(f), X, Y


def gaussian_random_field(shape, corr_px, rng):
    w = rng.standard_normal(shape)
    kx = np.fft.fftfreq(shape[0])[:, None]
    ky = np.fft.fftfreq(shape[1])[None, :]
    filt = np.exp(-2.0 * (np.pi * corr_px) ** 2 * (kx ** 2 + ky ** 2))
    return np.real(np.fft.ifft2(np.fft.fft2(w) * filt))


def make_object(X, Y, rng, corr_px=8.0):
    amp = rng.uniform(0.8, 1.0, size=(X, Y))
    f = gaussian_random_field((X, Y), corr_px, rng)
    ph = (f - f.min()) / (f.max() - f.min()) * np.pi - np.pi / 2
    return (amp * np.exp(1j * ph)).astype(np.complex64)


def make_probe(N, dx_s, K=1, weights=MODE_WEIGHTS, fwhm=BEAM_FWHM, total_power=None):
    """(K, N, N) complex64 probe modes, mode k carrying weights[k] of the power."""
    s = (fwhm / dx_s) / 2.3548  # Gaussian sigma in pixels
    c = np.arange(N) - N / 2
    x, y = np.meshgrid(c, c, indexing="ij")
    r2 = x ** 2 + y ** 2
    env = np.exp(-r2 / (2 * s * s)) * np.exp(1j * (np.pi / 2) * r2 / (2.3548 * s) ** 2)
    env[r2 > (N / 2) ** 2] = 0
    orders = [(0, 0), (1, 0), (0, 1), (1, 1), (2, 0), (0, 2), (2, 1), (1, 2)]
    if K > len(orders):
        raise ValueError("at most %d modes" % len(orders))
    modes = []
    for (m, n) in orders[:K]:
        hm = np.polynomial.hermite.hermval(x / s, [0] * m + [1])
        hn = np.polynomial.hermite.hermval(y / s, [0] * n + [1])
        modes.append(hm * hn * env)
    # Gram-Schmidt to orthonormal modes, then the power weights
    out = []
    for v in modes:
        v = v.astype(np.complex128)
        for u in out:
            v = v - np.vdot(u, v) * u
        out.append(v / np.linalg.norm(v))
    if total_power is None:
        total_power = float(N * N) * 0.01
    w = np.asarray(weights[:K], dtype=np.float64) if K > 1 else np.ones(1)
    w = w / w.sum()
    return np.stack([np.sqrt(total_power * wk) * m for wk, m in zip(w, out)]).astype(np.complex64)


def make_patterns(obj, probe, pos, N, photons, rng, intensities=False, chunk=64):
    """(P, N, N) float32 amplitudes (or intensities) from rounded positions."""
    P = pos.shape[0]
    off = np.round(pos).astype(np.int64)
    out = np.empty((P, N, N), np.float32)
    scale = None
    for c0 in range(0, P, chunk):
        c1 = min(P, c0 + chunk)
        I = np.zeros((c1 - c0, N, N), np.float32)
        for k in range(probe.shape[0]):
            ex = np.stack([obj[o[0]:o[0] + N, o[1]:o[1] + N] for o in off[c0:c1]]) * probe[k][None]
            F = np.fft.fft2(ex.astype(np.complex64))
            I += (F.real ** 2 + F.imag ** 2).astype(np.float32)
        if scale is None:  # global scale fixed from the first chunk's mean pattern total
            scale = photons / float(I.sum(axis=(1, 2)).mean())
        counts = rng.poisson(I.astype(np.float64) * scale).astype(np.float32)
        out[c0:c1] = counts if intensities else np.sqrt(counts)
    return out


def make_dataset(name="epie128", seed=20261203, **override):
    """Everything a reconstruction needs for one named configuration (overrides: N, nx, ny, photons, K ...)."""
    cfg = dict(CONFIGS[name])
    cfg.update(override)
    rng = np.random.default_rng(seed)
    N = cfg["N"]
    dx_s = sample_pixel(cfg["lambd"], cfg["z"], cfg["dx_d"], N)
    pos, X, Y = raster_positions(cfg["nx"], cfg["ny"], cfg["step"], cfg["step"], dx_s, N)
    obj = make_object(X, Y, rng)
    probe = make_probe(N, dx_s, K=cfg["K"])
    amp = make_patterns(obj, probe, pos, N, cfg["photons"], rng, intensities=(cfg["algorithm"] == "MLs"))
    kwargs = dict(size=N, scanDimsx=cfg["nx"], scanDimsy=cfg["ny"], stepx=cfg["step"], stepy=cfg["step"],
                  lambd=cfg["lambd"], z=cfg["z"], dx_d=cfg["dx_d"], beamSize=BEAM_FWHM, probeModes=cfg["K"],
                  iter=cfg["iters"])
    return dict(cfg=cfg, amp=amp, obj_true=obj, probe_true=probe, pos=pos, X=X, Y=Y, dx_s=dx_s, kwargs=kwargs)


def phase_nrmse(obj, ref, mask=None):
    """Phase NRMSE after removing the global phase offset and a linear phase ramp (least squares)."""
    a = np.angle(obj * np.conj(ref))
    if mask is None:
        mask = np.abs(obj) > 0
    xs, ys = np.nonzero(mask)
    v = a[xs, ys]
    A = np.stack([np.ones_like(xs, dtype=np.float64), xs, ys], axis=1)
    coef, *_ = np.linalg.lstsq(A, v, rcond=None)
    resid = v - A @ coef
    rng = np.angle(ref[xs, ys]).max() - np.angle(ref[xs, ys]).min()
    return float(np.sqrt(np.mean(resid ** 2)) / max(rng, 1e-12))


def make_patterns_torch(obj, probe, pos, N, photons, seed, device="cuda", intensities=False, chunk=64):
    """GPU variant of make_patterns (torch FFT and Poisson on the device), for large benchmark datasets.
    Returns a (P, N, N) float32 CUDA tensor.  Same forward model and scaling; a different random stream."""
    import torch

    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    o = torch.from_numpy(obj).to(device)
    pr = torch.from_numpy(probe).to(device)
    off = np.round(pos).astype(np.int64)
    P = pos.shape[0]
    out = torch.empty((P, N, N), dtype=torch.float32, device=device)
    scale = None
    for c0 in range(0, P, chunk):
        c1 = min(P, c0 + chunk)
        patches = torch.stack([o[a:a + N, b:b + N] for a, b in off[c0:c1]])
        I = torch.zeros((c1 - c0, N, N), dtype=torch.float32, device=device)
        for k in range(pr.shape[0]):
            F = torch.fft.fft2(patches * pr[k][None])
            I += F.real ** 2 + F.imag ** 2
        if scale is None:
            scale = photons / float(I.sum(dim=(1, 2)).mean())
        counts = torch.poisson(I * scale, generator=g)
        out[c0:c1] = counts if intensities else torch.sqrt(counts)
    return out
