"""ctypes binding of the engine's C ABI (include/ptychopy_b200.h) and a small Session wrapper.

This is the same boundary a non-CPython host binds; the CPython module `ptychopy` (the reference-compatible
surface) sits on the same library.  Loading fails loudly when the native library has not been built: there is
no fallback implementation.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libptychopy_b200.so")

PTY_OK = 0
PTY_ERR_INVALID = -1
PTY_ERR_OOM = -2
PTY_ERR_CUDA = -3
PTY_ERR_STATE = -4
PTY_ERR_UNSUPPORTED = -5
PTY_ERR_TIMEOUT = -6
PTY_ERR_IO = -7
PTY_F32 = 0
PTY_F64 = 1

# Entry points declared in include/ptychopy_b200.h (checked by tests/test_abi.py).
EXPORTS = [
    "pty_params_init", "pty_session_create", "pty_session_destroy", "pty_set_patterns", "pty_set_positions",
    "pty_set_object", "pty_set_probe", "pty_init", "pty_step", "pty_run", "pty_get_dims", "pty_get_object",
    "pty_get_probe", "pty_get_positions", "pty_write_results", "pty_set_stream", "pty_kernel_launches",
    "pty_last_error", "pty_fft2_dev", "pty_fft2_dev_noalloc", "pty_batch_run", "pty_simulate",
    "pty_set_shard", "pty_dm_step_local", "pty_dm_increments", "pty_dm_step_finish",
    "pty_nn_conv3x3", "pty_nn_conv3x3_bwd", "pty_nn_relu", "pty_nn_relu_bwd", "pty_nn_pool2", "pty_nn_pool2_bwd",
    "pty_nn_up2", "pty_nn_up2_bwd", "pty_nn_mse", "pty_nn_adam", "pty_warm_input", "pty_warm_stitch",
    "pty_warm_object", "pty_dm_psi_from_object", "pty_tc_weights_size", "pty_tc_pack_weights", "pty_tc_conv3x3",
    "pty_tc_pool2", "pty_tc_up2", "pty_tc_to_bf16", "pty_tc_first_layer", "pty_tc_last_layer", "pty_set_warm_start",
    "pty_selftest_bounded_waits", "pty_fft2_tc", "pty_autotune", "pty_get_mls_state",
    "pty_release_cached_memory", "pty_preprocess_patterns", "pty_get_patterns", "pty_params_from_cmdline",
]


class PtyParams(ctypes.Structure):
    """Mirror of `pty_params` (field order and types must match the header)."""
    _fields_ = [
        ("jobID", ctypes.c_char * 128), ("algorithm", ctypes.c_char * 8), ("fp", ctypes.c_char * 256),
        ("fs", ctypes.c_int), ("hdf5path", ctypes.c_char * 128), ("dpf", ctypes.c_int),
        ("beamSize", ctypes.c_double), ("probeGuess", ctypes.c_char * 256), ("objectGuess", ctypes.c_char * 256),
        ("size", ctypes.c_int), ("qx", ctypes.c_int), ("qy", ctypes.c_int), ("nx", ctypes.c_int),
        ("ny", ctypes.c_int), ("scanDimsx", ctypes.c_int), ("scanDimsy", ctypes.c_int),
        ("spiralScan", ctypes.c_int), ("flipScanAxis", ctypes.c_int), ("mirror1stScanAxis", ctypes.c_int),
        ("mirror2ndScanAxis", ctypes.c_int), ("stepx", ctypes.c_double), ("stepy", ctypes.c_double),
        ("probeModes", ctypes.c_int), ("lambd", ctypes.c_double), ("dx_d", ctypes.c_double),
        ("z", ctypes.c_double), ("iter", ctypes.c_int), ("T", ctypes.c_int), ("jitterRadius", ctypes.c_int),
        ("delta_p", ctypes.c_double), ("threshold", ctypes.c_int), ("rotate90", ctypes.c_int),
        ("sqrtData", ctypes.c_int), ("fftShiftData", ctypes.c_int), ("binaryOutput", ctypes.c_int),
        ("simulate", ctypes.c_int), ("phaseConstraint", ctypes.c_int), ("updateProbe", ctypes.c_int),
        ("updateModes", ctypes.c_int), ("beamstopMask", ctypes.c_int), ("lf", ctypes.c_char * 256),
        ("PPS", ctypes.c_int), ("seed", ctypes.c_uint64), ("calculateRMS", ctypes.c_int),
        ("device", ctypes.c_int), ("wave", ctypes.c_int), ("precision", ctypes.c_int),
        ("mlsCore", ctypes.c_int), ("save", ctypes.c_int), ("outputDir", ctypes.c_char * 256),
        ("driftx", ctypes.c_double), ("drifty", ctypes.c_double), ("bitDepth", ctypes.c_int),
    ]


_lib = None


def lib():
    """The loaded native library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m ptychopy_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        vp, ip, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)
        sig = {
            "pty_params_init": ([ctypes.POINTER(PtyParams)], ctypes.c_int),
            "pty_params_from_cmdline": ([ctypes.c_char_p, ctypes.POINTER(PtyParams)], ctypes.c_int),
            "pty_session_create": ([ctypes.POINTER(PtyParams), ctypes.POINTER(vp)], ctypes.c_int),
            "pty_session_destroy": ([vp], ctypes.c_int),
            "pty_set_patterns": ([vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int], ctypes.c_int),
            "pty_set_positions": ([vp, vp, ctypes.c_int], ctypes.c_int),
            "pty_set_object": ([vp, vp, ctypes.c_int, ctypes.c_int], ctypes.c_int),
            "pty_set_probe": ([vp, vp, ctypes.c_int, ctypes.c_int], ctypes.c_int),
            "pty_init": ([vp], ctypes.c_int),
            "pty_step": ([vp, dp], ctypes.c_int),
            "pty_run": ([vp, ctypes.c_int, vp], ctypes.c_int),
            "pty_get_dims": ([vp, ip, ip, ip, ip, ip, ip], ctypes.c_int),
            "pty_get_object": ([vp, vp, ctypes.c_int, ctypes.c_int], ctypes.c_int),
            "pty_get_probe": ([vp, vp, ctypes.c_int, ctypes.c_int], ctypes.c_int),
            "pty_get_positions": ([vp, vp, ctypes.c_int], ctypes.c_int),
            "pty_get_mls_state": ([vp, vp, vp, vp, ctypes.c_int, ctypes.c_int], ctypes.c_int),
            "pty_release_cached_memory": ([ctypes.c_int], ctypes.c_int),
            "pty_write_results": ([vp, ctypes.c_char_p, ctypes.c_int, ctypes.c_int], ctypes.c_int),
            "pty_set_stream": ([vp, vp], ctypes.c_int),
            "pty_kernel_launches": ([vp], ctypes.c_int64),
            "pty_last_error": ([], ctypes.c_char_p),
            "pty_fft2_dev": ([vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp], ctypes.c_int),
            "pty_fft2_dev_noalloc": ([vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp], ctypes.c_int),
            "pty_preprocess_patterns": ([vp] + [ctypes.c_int] * 8 + [vp, vp], ctypes.c_int),
            "pty_get_patterns": ([vp, vp, ctypes.c_int, ctypes.c_int], ctypes.c_int),
            "pty_batch_run": ([ctypes.POINTER(vp), ctypes.c_int, ctypes.c_int], ctypes.c_int),
            "pty_simulate": ([vp, ctypes.c_int, ctypes.c_int, vp, ctypes.c_int, vp, ctypes.c_int, vp], ctypes.c_int),
            "pty_set_shard": ([vp, ctypes.c_int, ctypes.c_int], ctypes.c_int),
            "pty_dm_step_local": ([vp], ctypes.c_int),
            "pty_dm_increments": ([vp, ctypes.POINTER(vp), ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(vp),
                                   ctypes.POINTER(ctypes.c_size_t)], ctypes.c_int),
            "pty_dm_step_finish": ([vp], ctypes.c_int),
            "pty_dm_psi_from_object": ([vp], ctypes.c_int),
            "pty_set_warm_start": ([vp, vp, ctypes.c_size_t, ctypes.c_int], ctypes.c_int),
            "pty_selftest_bounded_waits": ([vp], ctypes.c_int),
            "pty_fft2_tc": ([vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, vp], ctypes.c_int),
            "pty_autotune": ([vp, ctypes.c_int, ctypes.c_char_p, ctypes.c_int], ctypes.c_int),
            "pty_tc_weights_size": ([ctypes.c_int, ctypes.c_int], ctypes.c_int),
            "pty_tc_pack_weights": ([vp, ctypes.c_int, ctypes.c_int, vp, vp], ctypes.c_int),
            "pty_tc_conv3x3": ([vp, vp, vp, vp] + [ctypes.c_int] * 8 + [ctypes.c_float, vp, vp], ctypes.c_int),
            "pty_tc_pool2": ([vp, vp] + [ctypes.c_int] * 4 + [vp], ctypes.c_int),
            "pty_tc_up2": ([vp, vp] + [ctypes.c_int] * 4 + [vp], ctypes.c_int),
            "pty_tc_to_bf16": ([vp, vp, ctypes.c_size_t, vp], ctypes.c_int),
            "pty_tc_first_layer": ([vp, vp, vp, vp] + [ctypes.c_int] * 4 + [ctypes.c_float, vp], ctypes.c_int),
            "pty_tc_last_layer": ([vp, vp, vp, vp] + [ctypes.c_int] * 5 + [vp], ctypes.c_int),
            "pty_nn_conv3x3": ([vp, vp, vp, vp] + [ctypes.c_int] * 6 + [vp], ctypes.c_int),
            "pty_nn_conv3x3_bwd": ([vp] * 6 + [ctypes.c_int] * 5 + [vp], ctypes.c_int),
            "pty_nn_relu": ([vp, ctypes.c_size_t, vp], ctypes.c_int),
            "pty_nn_relu_bwd": ([vp, vp, ctypes.c_size_t, vp], ctypes.c_int),
            "pty_nn_pool2": ([vp, vp, ctypes.c_size_t, ctypes.c_int, ctypes.c_int, vp], ctypes.c_int),
            "pty_nn_pool2_bwd": ([vp, vp, ctypes.c_size_t, ctypes.c_int, ctypes.c_int, vp], ctypes.c_int),
            "pty_nn_up2": ([vp, vp, ctypes.c_size_t, ctypes.c_int, ctypes.c_int, vp], ctypes.c_int),
            "pty_nn_up2_bwd": ([vp, vp, ctypes.c_size_t, ctypes.c_int, ctypes.c_int, vp], ctypes.c_int),
            "pty_nn_mse": ([vp, vp, vp, ctypes.c_size_t, vp, ctypes.c_size_t, vp, vp], ctypes.c_int),
            "pty_nn_adam": ([vp, vp, vp, vp, ctypes.c_size_t] + [ctypes.c_float] * 4 + [ctypes.c_int, vp],
                            ctypes.c_int),
            "pty_warm_input": ([vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_float, vp], ctypes.c_int),
            "pty_warm_stitch": ([vp, vp, ctypes.c_int, vp, ctypes.c_int, ctypes.c_int] + [ctypes.c_float] * 3 +
                                [vp, ctypes.c_int, ctypes.c_int, vp], ctypes.c_int),
            "pty_warm_object": ([vp, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_float, vp, ctypes.c_int,
                                 vp, ctypes.c_int, vp, vp, vp, vp], ctypes.c_int),
        }
        for name, (args, res) in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


class PtyError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def check(rc):
    if rc != PTY_OK:
        raise PtyError(rc, lib().pty_last_error().decode())


def default_params(**kw):
    p = PtyParams()
    check(lib().pty_params_init(ctypes.byref(p)))
    for k, v in kw.items():
        if not hasattr(p, k):
            raise KeyError(k)
        if isinstance(v, str):
            v = v.encode()
        setattr(p, k, v)
    return p


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data)


class Session:
    """One reconstruction through the C ABI.  Arrays in, arrays out (host numpy)."""

    def __init__(self, **params):
        self.params = default_params(**params)
        h = ctypes.c_void_p()
        check(lib().pty_session_create(ctypes.byref(self.params), ctypes.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            lib().pty_session_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_patterns(self, amp):
        amp = np.ascontiguousarray(amp)
        dt = PTY_F32 if amp.dtype == np.float32 else PTY_F64
        if dt == PTY_F64:
            amp = np.ascontiguousarray(amp, dtype=np.float64)
        check(lib().pty_set_patterns(self.h, _ptr(amp), dt, amp.shape[0], amp.shape[1]))

    def set_patterns_ptr(self, ptr, P, N, dtype=PTY_F32):
        check(lib().pty_set_patterns(self.h, ctypes.c_void_p(ptr), dtype, P, N))

    def set_positions(self, xy_m):
        xy = np.ascontiguousarray(xy_m, dtype=np.float64)
        check(lib().pty_set_positions(self.h, _ptr(xy), xy.shape[0]))

    def set_object(self, obj):
        o = np.ascontiguousarray(obj, dtype=np.complex64)
        check(lib().pty_set_object(self.h, _ptr(o), o.shape[0], o.shape[1]))

    def set_probe(self, probe):
        p = np.ascontiguousarray(probe, dtype=np.complex64)
        if p.ndim == 2:
            p = p[None]
        check(lib().pty_set_probe(self.h, _ptr(p), p.shape[0], p.shape[1]))

    def init(self):
        check(lib().pty_init(self.h))

    def step(self):
        e = ctypes.c_double(0)
        check(lib().pty_step(self.h, ctypes.byref(e)))
        return e.value

    def run(self, iters, errors=False):
        errs = np.zeros(max(iters, 1), np.float64) if errors else None
        check(lib().pty_run(self.h, iters, _ptr(errs) if errors else None))
        return errs[:iters] if errors else None

    def dims(self):
        v = [ctypes.c_int() for _ in range(6)]
        check(lib().pty_get_dims(self.h, *[ctypes.byref(x) for x in v]))
        return dict(zip(["X", "Y", "K", "N", "P", "iters"], [x.value for x in v]))

    def object(self):
        d = self.dims()
        o = np.empty((d["X"], d["Y"]), np.complex64)
        check(lib().pty_get_object(self.h, _ptr(o), d["X"], d["Y"]))
        return o

    def probe(self):
        d = self.dims()
        p = np.empty((d["K"], d["N"], d["N"]), np.complex64)
        check(lib().pty_get_probe(self.h, _ptr(p), d["K"], d["N"]))
        return p

    def patterns(self):
        """The session's diffraction data (P, N, N) float32 as the iterations read them (pty_get_patterns)."""
        d = self.dims()
        out = np.zeros((d["P"], d["N"], d["N"]), np.float32)
        check(lib().pty_get_patterns(self.h, _ptr(out), d["P"], d["N"]))
        return out

    def positions(self):
        d = self.dims()
        q = np.empty((d["P"], 2), np.float32)
        check(lib().pty_get_positions(self.h, _ptr(q), d["P"]))
        return q

    def mls_state(self):
        """MLs default path: (extra probe mode E, evo0, evo1)."""
        d = self.dims()
        E = np.empty((d["N"], d["N"]), np.complex64)
        e0 = np.empty(d["P"])
        e1 = np.empty(d["P"])
        check(lib().pty_get_mls_state(self.h, _ptr(E), _ptr(e0), _ptr(e1), d["N"], d["P"]))
        return E, e0, e1

    def write_results(self, directory, r=0, binary=False):
        check(lib().pty_write_results(self.h, directory.encode(), r, int(binary)))

    def set_stream(self, stream_handle):
        check(lib().pty_set_stream(self.h, ctypes.c_void_p(stream_handle)))

    def launches(self):
        return int(lib().pty_kernel_launches(self.h))

    # ---- DM position shards (multi-GPU) ----
    def set_shard(self, first, total):
        check(lib().pty_set_shard(self.h, first, total))

    def step_local(self):
        check(lib().pty_dm_step_local(self.h))

    def increments(self):
        """(dO pointer, object elements, dP pointer, probe elements): complex64 device buffers."""
        o, p = ctypes.c_void_p(), ctypes.c_void_p()
        no, npr = ctypes.c_size_t(), ctypes.c_size_t()
        check(lib().pty_dm_increments(self.h, ctypes.byref(o), ctypes.byref(no), ctypes.byref(p), ctypes.byref(npr)))
        return o.value, no.value, p.value, npr.value

    def step_finish(self):
        check(lib().pty_dm_step_finish(self.h))

    def set_warm_start(self, params, width=16):
        """Trained warm-start network parameters (warmstart.Net.state()); pty_init builds the start object from
        them (pty_set_warm_start).  None removes them."""
        if params is None:
            check(lib().pty_set_warm_start(self.h, None, 0, 0))
            return
        self._warm = np.ascontiguousarray(params, np.float32)
        check(lib().pty_set_warm_start(self.h, _ptr(self._warm), self._warm.size, int(width)))

    def autotune(self, iters=2):
        """Times the launch variants on temporary sessions and keeps the fastest (pty_autotune, before init);
        returns the summary line."""
        buf = ctypes.create_string_buffer(1024)
        check(lib().pty_autotune(self.h, int(iters), buf, len(buf)))
        return buf.value.decode()

    def psi_from_object(self):
        """DM: exit waves = P * O at every position (pty_dm_psi_from_object), for a given start object."""
        check(lib().pty_dm_psi_from_object(self.h))


def simulate(obj, probe, pos_px):
    """Diffraction amplitudes |FFT2(O_bilinear(pos) * P)| (P, N, N) float32 (pty_simulate)."""
    o = np.ascontiguousarray(obj, np.complex64)
    p = np.ascontiguousarray(probe, np.complex64)
    if p.ndim == 3:
        p = np.ascontiguousarray(p[0])
    q = np.ascontiguousarray(pos_px, np.float32)
    out = np.empty((q.shape[0], p.shape[0], p.shape[0]), np.float32)
    check(lib().pty_simulate(_ptr(o), o.shape[0], o.shape[1], _ptr(p), p.shape[0], _ptr(q), q.shape[0], _ptr(out)))
    return out


def batch_run(sessions, iters):
    """Run `iters` iterations of every session, interleaved on their own streams (pty_batch_run)."""
    arr = (ctypes.c_void_p * len(sessions))(*[s.h.value for s in sessions])
    check(lib().pty_batch_run(arr, len(sessions), iters))


def fft2_dev(data_ptr, work_ptr, batch, N, inverse=False, stream=0):
    """In-place batched 2-D FFT of device memory (complex64), through pty_fft2_dev."""
    check(lib().pty_fft2_dev(ctypes.c_void_p(data_ptr), ctypes.c_void_p(work_ptr), batch, N, int(inverse),
                             ctypes.c_void_p(stream)))
