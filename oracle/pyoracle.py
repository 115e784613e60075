"""ctypes wrapper of the oracle (oracle/oracle.cpp).  TEST INFRASTRUCTURE ONLY: imported by tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg as the checker; never by the product.

Parity status: pinned to the reference's own device functions, compiled unchanged by oracle/ref_build.py and
compared stage by stage and iteration by iteration in tests/test_gpu_refstages.py; also pinned to numpy.fft,
hand-derived known answers and the committed fixtures under tests/golden/.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "oracle.cpp")
LIB = os.path.join(HERE, "liboracle.so")


def build(force=False, verbose=False):
    """Compile the oracle (g++ only; no GPU needed)."""
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(SRC):
        cmd = ["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-o", LIB, SRC, "-lpthread"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB)
        vp, i, d, f = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_float
        u64 = ctypes.c_uint64
        sig = {
            "orc_fft2": ([vp, i, i], i),
            "orc_sample_pixel": ([d, d, d, i], d),
            "orc_cartesian_mesh": ([i, i, d, d, d, d, d, i, i, i, i, vp, vp], i),
            "orc_list_mesh": ([vp, i, d, d, d, i, i, vp, vp], i),
            "orc_cartesian_mesh_j": ([i, i, d, d, d, d, d, i, i, i, i, ctypes.c_uint, u64, vp, vp], i),
            "orc_list_mesh_j": ([vp, i, d, d, d, i, i, ctypes.c_uint, u64, vp, vp], i),
            "orc_spiral_mesh": ([i, d, d, d, d, d, i, i, ctypes.c_uint, u64, vp, vp], i),
            "orc_cartesian_mesh_jd": ([i, i, d, d, d, d, d, i, i, i, i, ctypes.c_uint, u64, d, d, vp, vp], i),
            "orc_list_mesh_jd": ([vp, i, d, d, d, i, i, ctypes.c_uint, u64, d, d, vp, vp], i),
            "orc_spiral_mesh_d": ([i, d, d, d, d, d, i, i, ctypes.c_uint, u64, d, d, vp, vp], i),
            "orc_mesh_raw_drift": ([i, i, i, vp, d, d, d, d, d, i, i, i, d, d, vp], i),
            "orc_mesh_jitter": ([u64, i, ctypes.c_uint, vp], i),
            "orc_set_dm_reduce": ([vp, vp, vp], i),
            "orc_set_saturation": ([vp, d], i),
            "orc_probe_guess": ([vp, i, i, d, d, i, vp], i),
            "orc_visiting_order": ([ctypes.POINTER(u64), i, vp], None),
            "orc_extract_patch": ([vp, i, i, f, f, i, vp], i),
            "orc_create": ([i, i, i, i, i, i, vp, vp, vp, vp, i, i, u64, i, i, i, i, i], vp),
            "orc_create2": ([i, i, i, i, i, i, i, vp, vp, vp, vp, i, i, u64, i, i, i, i, i], vp),
            "orc_step": ([vp, ctypes.POINTER(d)], i),
            "orc_get": ([vp, vp, vp, vp], i),
            "orc_get_psi": ([vp, vp], i),
            "orc_destroy": ([vp], None),
            "orc_dm_baseline_f32": ([i, i, i, i, vp, vp, vp, i, i, vp], d),
            "orc_mls_geometry": ([vp, i, i, vp, vp, vp], i),
            "orc_mls_create": ([vp, i, i, vp, vp, vp, u64, d, i, i, i], vp),
            "orc_mls_get_var": ([vp, vp, vp, vp, vp], i),
            "orc_mls_step": ([vp, ctypes.POINTER(d)], i),
            "orc_mls_get": ([vp, vp, vp, vp], i),
            "orc_mls_destroy": ([vp], None),
            "orc_cartesian_mesh_raw": ([i, i, d, d, d, d, d, i, i, i, vp], i),
            "orc_mls_modulus_factor": ([vp, vp, i, vp], i),
            "orc_mls_lsq_terms": ([vp, vp, vp, vp, d, i, vp, vp, vp, vp, vp], i),
        }
        for name, (a, r) in sig.items():
            fn = getattr(L, name)
            fn.argtypes = a
            fn.restype = r
        _lib = L
    return _lib


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


def fft2(a, inverse=False):
    b = np.ascontiguousarray(a, dtype=np.complex128).copy()
    assert lib().orc_fft2(_p(b), b.shape[0], int(inverse)) == 0
    return b


def sample_pixel(lambd, z, dx_d, N):
    return lib().orc_sample_pixel(lambd, z, dx_d, N)


def cartesian_mesh(nx, ny, stepx, stepy, lambd, z, dx_d, N, mirrorX=0, mirrorY=0, flip=0, jitter=0, seed=0,
                   drift=(0.0, 0.0)):
    """Raster positions (nx*ny, 2) in pixels after the -min shift, and the object size; drift in metres per raster
    row / column."""
    pos = np.zeros((nx * ny, 2), np.float32)
    xy = np.zeros(2, np.int32)
    assert lib().orc_cartesian_mesh_jd(nx, ny, stepx, stepy, lambd, z, dx_d, N, mirrorX, mirrorY, flip, jitter, seed,
                                       drift[0], drift[1], _p(pos), _p(xy)) == 0
    return pos, int(xy[0]), int(xy[1])


def mesh_raw_drift(kind, lambd, z, dx_d, N, drift, nx=0, ny=0, xy_m=None, P=0, stepx=0.0, stepy=0.0, mirrorX=0,
                   mirrorY=0):
    """The mesh array before jitter and the -min shift, in pixels, with the scan drift: kind "cartesian" (nx*ny, 2),
    "list" (xy_m in metres) or "spiral" (P points), the last two (ceil(P/1024)*1024, 2) in 1024-wide rows."""
    if kind == "cartesian":
        t, a, b, n, xp = 1, nx, ny, nx * ny, None
    else:
        t = 2 if kind == "list" else 3
        if t == 2:
            xp = np.ascontiguousarray(xy_m, np.float64)
            P = xp.shape[0]
        else:
            xp = None
        a, b, n = P, 0, (P + 1023) // 1024 * 1024
    raw = np.zeros((n, 2), np.float32)
    assert lib().orc_mesh_raw_drift(t, a, b, None if xp is None else _p(xp), stepx, stepy, lambd, z, dx_d, N, mirrorX,
                                    mirrorY, drift[0], drift[1], _p(raw)) == 0
    return raw


def cartesian_mesh_raw(nx, ny, stepx, stepy, lambd, z, dx_d, N, mirrorX=0, mirrorY=0):
    """Raw raster positions (nx*ny, 2) float32 in pixels, before the -min shift."""
    raw = np.zeros((nx * ny, 2), np.float32)
    assert lib().orc_cartesian_mesh_raw(nx, ny, stepx, stepy, lambd, z, dx_d, N, mirrorX, mirrorY, _p(raw)) == 0
    return raw


def mls_modulus_factor(A, ap):
    """A / (|Psi| + 1e-9) - 1 per pixel (the oracle's MLs modulus helper)."""
    A = np.ascontiguousarray(A, np.float64).ravel()
    ap = np.ascontiguousarray(ap, np.float64).ravel()
    out = np.zeros_like(A)
    assert lib().orc_mls_modulus_factor(_p(A), _p(ap), A.size, _p(out)) == 0
    return out


def mls_lsq_terms(chi, oup, dPO, probe, lam):
    """Per-pixel (AA1, AA2, AA4, Atb1, Atb2) of the MLs step-length system (the oracle's helper)."""
    c = [np.ascontiguousarray(v, np.complex128).ravel() for v in (chi, oup, dPO, probe)]
    n = c[0].size
    a1, a4, b1, b2 = (np.zeros(n) for _ in range(4))
    a2 = np.zeros(n, np.complex128)
    assert lib().orc_mls_lsq_terms(*(_p(v) for v in c), lam, n, _p(a1), _p(a2), _p(a4), _p(b1), _p(b2)) == 0
    return a1, a2, a4, b1, b2


def list_mesh(xy_m, lambd, z, dx_d, N, flip=0, jitter=0, seed=0, drift=(0.0, 0.0)):
    xy_m = np.ascontiguousarray(xy_m, np.float64)
    pos = np.zeros((xy_m.shape[0], 2), np.float32)
    xy = np.zeros(2, np.int32)
    assert lib().orc_list_mesh_jd(_p(xy_m), xy_m.shape[0], lambd, z, dx_d, N, flip, jitter, seed, drift[0], drift[1],
                                  _p(pos), _p(xy)) == 0
    return pos, int(xy[0]), int(xy[1])


def spiral_mesh(P, stepx, stepy, lambd, z, dx_d, N, flip=0, jitter=0, seed=0, drift=(0.0, 0.0)):
    """Spiral scan positions (P, 2) in pixels after the -min shift, and the object size."""
    pos = np.zeros((P, 2), np.float32)
    xy = np.zeros(2, np.int32)
    assert lib().orc_spiral_mesh_d(P, stepx, stepy, lambd, z, dx_d, N, flip, jitter, seed, drift[0], drift[1],
                                   _p(pos), _p(xy)) == 0
    return pos, int(xy[0]), int(xy[1])


def saturation_level(bitDepth=0, threshold=0, sqrtData=0):
    """The ePIE saturation level of Parameters::updatePixelSaturation (src/Parameters.cpp:54-62): 2^bitDepth - 1 -
    threshold (bitDepth 0: 32), square-rooted with sqrtData, each step truncated to the integer the reference holds
    it in; inf (no pixel floats) unless one of the three is given."""
    if bitDepth <= 0 and threshold <= 0 and not sqrtData:
        return np.inf
    v = max(np.floor(2.0 ** (bitDepth if bitDepth > 0 else 32) - 1 - max(threshold, 0)), 0.0)
    return float(np.float32(np.floor(np.sqrt(v)) if sqrtData else v))


def mesh_jitter(seed, n, radius):
    """The seeded jitter stream: (n, 2) float32 offsets in pixels."""
    out = np.zeros((n, 2), np.float32)
    lib().orc_mesh_jitter(seed, n, radius, _p(out))
    return out


def probe_guess(amp, beamSize, dx_s, K=1):
    amp = np.ascontiguousarray(amp, np.float64)
    P, N = amp.shape[0], amp.shape[1]
    out = np.zeros((K, N, N), np.complex128)
    assert lib().orc_probe_guess(_p(amp), P, N, beamSize, dx_s, K, _p(out)) == 0
    return out


def visiting_order(state, P):
    s = ctypes.c_uint64(state)
    order = np.zeros(P, np.int32)
    lib().orc_visiting_order(ctypes.byref(s), P, _p(order))
    return order, s.value


def extract_patch(obj, qx, qy, N):
    o = np.ascontiguousarray(obj, np.complex128)
    out = np.zeros((N, N), np.complex128)
    assert lib().orc_extract_patch(_p(o), o.shape[0], o.shape[1], qx, qy, N, _p(out)) == 0
    return out


class OracleSession:
    """FP64 restatement of one reconstruction (algo 'ePIE' or 'DM'), stepped one iteration at a time."""

    def __init__(self, algo, amp, pos, obj, probe, *, probe_guess_path, modes_given=False, seed=0x5EED5EED,
                 phaseConstraint=1, updateProbe=10, updateModes=20, calculateRMS=0, nthreads=1, fp32=False,
                 saturation=None):
        self.amp = np.ascontiguousarray(amp, np.float64)
        self.pos = np.ascontiguousarray(pos, np.float32)
        obj = np.ascontiguousarray(obj, np.complex128)
        probe = np.ascontiguousarray(probe, np.complex128)
        if probe.ndim == 2:
            probe = probe[None]
        self.X, self.Y = obj.shape
        self.K, self.N = probe.shape[0], probe.shape[1]
        self.P = self.amp.shape[0]
        self.h = lib().orc_create2(int(fp32), 0 if algo == "ePIE" else 1, self.N, self.K, self.P, self.X, self.Y, _p(self.amp),
                                  _p(self.pos), _p(obj), _p(probe), int(probe_guess_path), int(modes_given),
                                  seed, phaseConstraint, updateProbe, updateModes, calculateRMS, nthreads)
        if not self.h:
            raise ValueError("oracle rejected the configuration")
        if saturation is not None:  # ePIE: pixels with amplitude >= saturation float
            lib().orc_set_saturation(self.h, float(saturation))

    # DM position shards: fn(dO, dP) receives the iteration's increments as complex128 arrays (object, probe) and
    # must sum them over all shards in place.
    REDUCE = ctypes.CFUNCTYPE(None, ctypes.POINTER(ctypes.c_double), ctypes.c_size_t, ctypes.POINTER(ctypes.c_double),
                              ctypes.c_size_t, ctypes.c_void_p)

    def set_dm_reduce(self, fn):
        def hook(po, no, pp, npr, _user):
            dO = np.ctypeslib.as_array(po, shape=(2 * no,)).view(np.complex128)
            dP = np.ctypeslib.as_array(pp, shape=(2 * npr,)).view(np.complex128)
            fn(dO, dP)
        self._reduce = self.REDUCE(hook)  # keep the callback alive
        lib().orc_set_dm_reduce(self.h, ctypes.cast(self._reduce, ctypes.c_void_p), None)

    def step(self):
        e = ctypes.c_double(0)
        rc = lib().orc_step(self.h, ctypes.byref(e))
        if rc:
            raise RuntimeError(f"oracle step failed ({rc})")
        return e.value

    def state(self):
        o = np.zeros((self.X, self.Y), np.complex128)
        p = np.zeros((self.K, self.N, self.N), np.complex128)
        sc = np.zeros(4, np.float64)
        lib().orc_get(self.h, _p(o), _p(p), _p(sc))
        return o, p, sc

    def psi(self):
        out = np.zeros((self.P, self.N, self.N), np.complex128)
        lib().orc_get_psi(self.h, _p(out))
        return out

    def close(self):
        if self.h:
            lib().orc_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


def dm_baseline_f32(amp, pos, probe, X, Y, iters, nthreads):
    """Multithreaded FP32 DM on the host (the CPU baseline).  Returns (seconds, object)."""
    amp = np.ascontiguousarray(amp, np.float32)
    pos = np.ascontiguousarray(pos, np.float32)
    pr = np.ascontiguousarray(probe.reshape(-1, probe.shape[-1])[: probe.shape[-1]], np.complex64)
    obj = np.zeros((X, Y), np.complex64)
    N = amp.shape[1]
    t = lib().orc_dm_baseline_f32(N, amp.shape[0], X, Y, _p(amp), _p(pos), _p(pr), iters, nthreads, _p(obj))
    return t, obj


def mls_raw_positions(nx, ny, stepx, stepy, dx_s, mirror_x=False, mirror_y=False):
    """Centred Cartesian positions of the ML mesh in pixels, FP32 like src/CartesianScanMesh.cpp:94-177:
    ((i - (nx-1)/2) * step) * float(1/dx_s), row-major over (i, j), x = row, y = column."""
    f = np.float32
    i = np.arange(nx, dtype=f) - f(nx - 1) * f(0.5)
    j = np.arange(ny, dtype=f) - f(ny - 1) * f(0.5)
    if mirror_x:
        i = -i
    if mirror_y:
        j = -j
    inv = f(1.0 / dx_s)
    px = (i * f(stepx)) * inv
    py = (j * f(stepy)) * inv
    out = np.zeros((nx, ny, 2), f)
    out[:, :, 0] = px[:, None]
    out[:, :, 1] = py[None, :]
    return out.reshape(-1, 2)


def mls_geometry(raw_pos, N):
    """ML-mesh geometry from centred pixel positions: (X, Y), window starts (P, 2), object ROI (x0, y0, nx, ny)."""
    raw = np.ascontiguousarray(raw_pos, np.float32)
    P = raw.shape[0]
    xy = np.zeros(2, np.int32)
    starts = np.zeros((P, 2), np.int32)
    roi = np.zeros(4, np.int32)
    lib().orc_mls_geometry(_p(raw), P, N, _p(xy), _p(starts), _p(roi))
    return int(xy[0]), int(xy[1]), starts, roi


def mls_zone_plate_probe(N, lambd, dx_s, beamSize):
    """MLs probe start without a given probe, FP64: the zone-plate guess of Probe::initMLH (src/Probe.cpp:376-420,
    d_initProbeMLH / d_endProbeMLH / d_shiftEnd, src/ProbeKernels.cu:220-360, h_initProbeMLH :592-628):
    fftshift(FFT2(fftshift(kern)) * pf) with kern the apertured zone plate (outer radius D_FZP/2, central stop D_H/2)
    times the Fresnel kernel to z = fl + beamSize, pf the detector-side phase, fl = 2 Rn dRn / lambda."""
    Rn, dRn, D_FZP, D_H = 90e-6, 50e-9, 180e-6, 60e-6
    fl = 2 * Rn * dRn / lambd
    dx_fzp = lambd * fl / (N * dx_s)
    k = 2 * np.pi / lambd
    z = fl + beamSize
    g = -dx_fzp * N / 2 + dx_fzp * N / (N - 1) * np.arange(N)
    s2 = g[None, :] ** 2 + g[:, None] ** 2
    r = np.sqrt(s2)
    kern = ((r <= D_FZP / 2) & (r >= D_H / 2)) * np.exp(1j * (-2 / (lambd * 2 * fl) * np.pi) * s2) \
        * np.exp(1j * (k / (2 * z)) * s2)
    fu = lambd * (fl + beamSize) / dx_fzp
    fs = fu / (N - 1)
    i = np.arange(N)
    lu = np.where(i < N // 2, -fu / 2 + fs * (N // 2) + fs * i, -fu / 2 + fs * (i - N // 2))
    pf = np.exp(1j * k * z) * np.exp(1j * (k / (2 * z)) * (lu[None, :] ** 2 + lu[:, None] ** 2))
    return np.fft.fftshift(np.fft.fft2(np.fft.fftshift(kern)) * pf)


class OracleMls:
    """FP64 MLs (groups, preconditioned LSQ-ML, one probe mode), stepped one iteration at a time.  variable=1 is the
    reference's default path (variable probe and intensity, sub-pixel probe shift, position search from iteration
    PPS); variable=0 the fixed-probe core."""

    def __init__(self, raw_pos, intens, probe, obj=None, seed=0x5EED5EED, delta_p=0.1, variable=0, PPS=20, K=1):
        self.raw = np.ascontiguousarray(raw_pos, np.float32)
        self.I = np.ascontiguousarray(intens, np.float64)
        self.P, self.N = self.I.shape[0], self.I.shape[1]
        self.X, self.Y, self.starts, self.roi = mls_geometry(self.raw, self.N)
        pr = np.ascontiguousarray(np.asarray(probe).reshape(-1, self.N, self.N)[0], np.complex128)  # mode 0
        o = None if obj is None else np.ascontiguousarray(obj, np.complex128)
        self.variable = int(variable)
        self.K = int(K) if self.variable else 1
        self.h = lib().orc_mls_create(_p(self.raw), self.P, self.N, _p(self.I), _p(pr),
                                      _p(o) if o is not None else None, seed, delta_p, self.variable, int(PPS), self.K)

    def step(self):
        e = ctypes.c_double(0)
        lib().orc_mls_step(self.h, ctypes.byref(e))
        return e.value

    def state(self):
        o = np.zeros((self.X, self.Y), np.complex128)
        p = np.zeros((self.K, self.N, self.N), np.complex128)
        sc = np.zeros(1)
        lib().orc_mls_get(self.h, _p(o), _p(p), _p(sc))
        return o, (p[0] if self.K == 1 else p), sc

    def variable_state(self):
        """(E, evo0, evo1, positions) of the variable path."""
        E = np.zeros((self.N, self.N), np.complex128)
        e0 = np.zeros(self.P)
        e1 = np.zeros(self.P)
        pos = np.zeros((self.P, 2), np.float32)
        lib().orc_mls_get_var(self.h, _p(E), _p(e0), _p(e1), _p(pos))
        return E, e0, e1, pos

    def close(self):
        if self.h:
            lib().orc_mls_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


# ---- whole-mode pattern ingest (index work: numpy) ----------------------------------------------------------------
# DiffractionLoader::run (src/DiffractionLoader.cpp:55-131) step by step, in the reference's order.

def read_pattern_file(path, rows, cols):
    """All rows x cols sections of a .bin (raw float32, src/FileManager.cpp:145-183) or .csv file (values
    separated by commas and line breaks, src/FileManager.cpp:185-216) as float32 (n, rows, cols)."""
    ext = os.path.splitext(path)[1].lower()
    if ext == ".bin":
        v = np.fromfile(path, dtype=np.float32)
    elif ext == ".csv":
        with open(path) as f:
            toks = f.read().replace(",", " ").split()
        v = np.array([np.float32(t) for t in toks], np.float32)
    else:
        raise ValueError(f"unsupported pattern file {path}")
    n = v.size // (rows * cols)
    return v[:n * rows * cols].reshape(n, rows, cols)


def symmetrize(raw, S, qx, qy):
    """Crop / zero-pad a rows x cols pattern to S x S around (qx, qy) (src/DiffractionLoader.cpp:81-107); a pattern
    that is already S x S is copied as it is.  Rows / columns the reference would write past the S x S output are
    dropped."""
    rows, cols = raw.shape
    if rows == S and cols == S:
        return raw.astype(np.float32).copy()
    out = np.zeros((S, S), np.float32)
    dx, dy = qx - S // 2, qy - S // 2
    oox, dox = (-dx, 0) if dx < 0 else (0, dx)
    ooy, doy = (-dy, 0) if dy < 0 else (0, dy)
    numX = S if qx + S // 2 < rows else rows - dox
    numY = S if qy + S // 2 < cols else cols - doy
    nX, nY = max(0, min(numX, S - oox)), max(0, min(numY, S - ooy))
    out[oox:oox + nX, ooy:ooy + nY] = raw[dox:dox + nX, doy:doy + nY]
    return out


def rotate90(a, times):
    """h_realRotate90 (src/utilitiesKernels.cu:2031-2049): only times % 4 == 1 moves data, out[S-1-c][r] = in[r][c]."""
    if times % 4 != 1:
        return a.copy()
    S = a.shape[0]
    out = np.empty_like(a)
    r, c = np.meshgrid(np.arange(S), np.arange(S), indexing="ij")
    out[S - 1 - c, r] = a[r, c]
    return out


def fft_shift(a):
    """h_shiftFFT (src/utilitiesKernels.cu:1945-1964): rows then columns shifted circularly by round(S/2)."""
    S = a.shape[0]
    h = int(np.floor(S / 2 + 0.5))
    t = np.empty_like(a)
    t[(np.arange(S) - h) % S, :] = a  # d_shiftX: out[(x - h) mod S][y] = in[x][y]
    out = np.empty_like(a)
    out[:, (np.arange(S) - h) % S] = t  # d_shiftY
    return out


def preprocess_pattern(raw, S, qx, qy, rotate90_times=0, fft_shift_data=0):
    a = symmetrize(raw, S, qx, qy)
    if rotate90_times > 0:
        a = rotate90(a, rotate90_times)
    if fft_shift_data:
        a = fft_shift(a)
    return a


def ingest(fp, P, S, nx, ny, qx, qy, fs=0, dpf=1, rotate90_times=0, fft_shift_data=0):
    """The P patterns of a whole-mode run: pattern i from section i % dpf of the file fp with '#' -> '%' formatted
    with i // dpf + fs (src/Diffractions.cpp:188-209, src/IPhaser.cpp:203-205), then preprocessed."""
    fmt = fp.replace("#", "%", 1)
    out = np.zeros((P, S, S), np.float32)
    cache = {}
    for i in range(P):
        name = fmt % (i // dpf + fs) if "%" in fmt else fmt
        if name not in cache:
            cache = {name: read_pattern_file(name, nx, ny)}
        out[i] = preprocess_pattern(cache[name][i % dpf], S, qx, qy, rotate90_times, fft_shift_data)
    return out


# ---- simulation mode (simulate=1) ---------------------------------------------------------------------------------

def read_pgm(path):
    """8-bit PGM (P5 binary or P2 plain) as a uint8 (rows, cols) array."""
    with open(path, "rb") as f:
        data = f.read()
    toks, pos = [], 0
    while len(toks) < 4:
        while data[pos:pos + 1].isspace():
            pos += 1
        if data[pos:pos + 1] == b"#":
            pos = data.index(b"\n", pos) + 1
            continue
        end = pos
        while not data[end:end + 1].isspace():
            end += 1
        toks.append(data[pos:end].decode())
        pos = end
    magic, w, h = toks[0], int(toks[1]), int(toks[2])
    if magic == "P5":
        return np.frombuffer(data[pos + 1:pos + 1 + w * h], np.uint8).reshape(h, w)
    return np.array(data[pos:].split()[:w * h], dtype=np.uint8).reshape(h, w)


def sim_object(mag_img, phase_img, X, Y):
    """Sample::loadFromFile + h_applyHammingToSample (src/Sample.cpp:109-162, src/SampleKernels.cu:75-90,510-518):
    magnitude (v / max) * 0.9 + 0.1, phase (v / max) * pi/3, times the 2-D Hamming window of period alignUp(w, 32) - 1,
    centred in an X x Y zero object."""
    h, w = mag_img.shape
    mag = (mag_img.astype(np.float64) / mag_img.max()) * np.float64(np.float32(0.9)) + (1.0 - np.float64(np.float32(0.9)))
    ph = (phase_img.astype(np.float64) / phase_img.max()) * 1.0471975512
    aw = (w + 31) // 32 * 32
    ham_c = 0.53836 - 0.46164 * np.cos(np.pi * 2.0 * np.arange(w) / (aw - 1))
    ham_r = 0.53836 - 0.46164 * np.cos(np.pi * 2.0 * np.arange(h) / (aw - 1))
    obj = np.zeros((X, Y), np.complex128)
    ox, oy = X // 2 - h // 2, Y // 2 - w // 2
    obj[ox:ox + h, oy:oy + w] = mag * np.exp(1j * ph) * ham_r[:, None] * ham_c[None, :]
    return obj


def _splitmix64_stream(seed, n):
    out = np.empty(n, np.uint64)
    s = int(seed) & 0xFFFFFFFFFFFFFFFF
    m = 0xFFFFFFFFFFFFFFFF
    for i in range(n):
        s = (s + 0x9E3779B97F4A7C15) & m
        z = s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & m
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & m
        out[i] = z ^ (z >> 31)
    return out


def sim_probe(N, beamSize, dx_s, seed):
    """Probe::simulate (src/Probe.cpp:184-207,332-340; d_initProbeSimulated, src/ProbeKernels.cu:192-205) with the
    random phase field from the seed: SplitMix64 from seed ^ 0xA0761D6478BD642F, u = ((next >> 11) + 0.5) 2^-53,
    circular convolution with a Gaussian of FWHM 10 px centred at (N/2, N/2), divided by its maximum."""
    z = _splitmix64_stream(np.uint64(seed) ^ np.uint64(0xA0761D6478BD642F), N * N)
    u = ((z >> np.uint64(11)).astype(np.float64) + 0.5) * 2.0 ** -53
    u = u.reshape(N, N)
    s = 10.0 / 2.3548
    c = np.arange(N) - N / 2
    g = np.exp(-(c[:, None] ** 2 + c[None, :] ** 2) / s ** 2)
    f = np.real(np.fft.ifft2(np.fft.fft2(u) * np.fft.fft2(g)))
    f = f / f.max()
    window = N / (2 * 2.35)
    factor = float(np.float32(dx_s / beamSize))
    r = np.sqrt(c[:, None] ** 2 + c[None, :] ** 2)
    q = r * factor
    with np.errstate(invalid="ignore", divide="ignore"):
        p = np.where(q != 0, np.sin(np.pi * q) / (np.pi * q), 1.0)
    p = np.abs(p * np.exp(-r * r / window ** 2))
    return p * np.exp(1j * np.pi * f)


def simulate_amplitudes(obj, probe, pos):
    """Diffractions::simulate (src/Diffractions.cpp:80-117): |FFT2(bilinear O at pos * P)| per position."""
    N = probe.shape[0]
    return np.stack([np.abs(fft2(extract_patch(obj, np.float32(q[0]), np.float32(q[1]), N) * probe)) for q in pos])


# ---- result files ---------------------------------------------------------------------------------------------------

def format_complex_csv(a):
    """Cuda2DArray::save in text mode (src/Cuda2DArray.hpp:439-464) with the complex cell of src/Cuda2DArray.cpp:46-52:
    `re`, '+' when im >= 0, `im`, 'j', each number as an ostream prints a float (6 significant digits, %g), cells
    joined by ", ", one line per row."""
    a = np.asarray(a, np.complex64)
    rows = []
    for row in a:
        cells = []
        for v in row:
            re, im = float(np.float32(v.real)), float(np.float32(v.imag))
            cells.append("%g" % re + ("+" if im >= 0 else "") + "%g" % im + "j")
        rows.append(", ".join(cells) + "\n")
    return "".join(rows)


def parse_complex_csv(text):
    """The values of such a file as complex64 (rows, cols)."""
    out = []
    for line in text.splitlines():
        if not line.strip():
            continue
        row = []
        for cell in line.split(","):
            c = cell.strip().rstrip("ji")
            k = max(i for i in range(1, len(c)) if c[i] in "+-" and c[i - 1] not in "eE")
            row.append(complex(np.float32(float(c[:k].rstrip("+"))), np.float32(float(c[k:]))))
        out.append(row)
    return np.array(out, np.complex64)
