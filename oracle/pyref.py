"""ctypes binding of oracle/_ref/libptyref.so: the reference's own device functions (compiled unchanged by
oracle/ref_build.py) behind small launch wrappers.  TEST INFRASTRUCTURE ONLY: the GPU stage tests use it to pin
the oracle (oracle/oracle.cpp) to the reference's code; the product never loads it.

All arrays are torch CUDA tensors (complex64 as torch.complex64, reals as float32); layouts follow the reference
(row-major, object rows pitched to alignUp(Y, 32)).
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libptyref.so")

_lib = None


def available():
    return os.path.exists(LIB)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            raise FileNotFoundError(f"{LIB} is missing: build it with oracle/ref_build.py where the reference "
                                    "checkout is present (the built library travels with the tree)")
        L = ctypes.CDLL(LIB)
        vp, i, f = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
        sig = {
            "ref_version": [],
            "ref_dm_calc_psi": [vp, vp, vp, vp, i, i, i, i, i, vp],
            "ref_dm_modulus": [vp, vp, i, i, vp],
            "ref_dm_update": [vp, vp, vp, vp, vp, vp, vp, i, i, i, i, i, vp],
            "ref_extract_patch": [vp, i, i, i, f, f, i, vp],
            "ref_simulate_psi": [vp, i, i, i, vp, f, f, i, vp],
            "ref_adjust_fft": [vp, vp, vp, vp, f, i, i],
            "ref_update_object": [vp, vp, vp, vp, vp, i, i, f, i, i, i, i, i, i],
            "ref_update_probe": [vp, vp, vp, vp, vp, i, i, f, i, i, i, i, i],
            "ref_calculate_er": [vp, vp, i, i, vp],
            "ref_lsq_terms": [vp, vp, vp, vp, f, i, vp, vp, vp, vp, vp],
            "ref_modulus_amplitude": [vp, vp, vp, f, i],
            "ref_cartesian_mesh": [vp, i, i, f, f, f, i, i],
            "ref_mesh": [i, vp, i, i, f, f, f, i, i, f, f],
            "ref_symmetrize": [vp, vp, i, i, i, i, i, i, i, i],
            "ref_rotate90": [vp, vp, i, i],
            "ref_shift_fft": [vp, vp, i],
            "ref_sqrt_patterns": [vp, i, i],
            "ref_preprocess": [vp, i, i, i, f],
        }
        for name, args in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = i
        _lib = L
    return _lib


def ptr(t):
    """Device address of a torch tensor (None for a null pointer)."""
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def call(name, *args):
    rc = getattr(lib(), name)(*args)
    if rc != 0:
        raise RuntimeError(f"{name} returned CUDA error {rc}")


def align32(n):
    return (n + 31) // 32 * 32
