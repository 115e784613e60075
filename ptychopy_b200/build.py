"""Build recipe for the engine's native code (no cmake, no setuptools): nvcc for the sm_100a kernels and the
C ABI (libptychopy_b200.so), g++ for the CPython module `ptychopy` that links against it.  Outputs are written
next to this file so they travel with the source tree; object files go to _build/ (git-ignored).

    python -m ptychopy_b200.build        # incremental
    python -m ptychopy_b200.build -f     # force
"""
import os
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(ROOT, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall"]

CU_SOURCES = ["kernels_common.cu", "kernels_dm.cu", "kernels_epie.cu", "kernels_mls.cu", "session.cu",
              "noalloc.cu", "kernels_nn.cu", "kernels_warm.cu", "kernels_tc.cu",
              "warm_start.cu", "kernels_fft_tc.cu", "autotune.cu", "kernels_mls_var.cu", "kernels_epie_chain.cu",
              "ingest.cu", "sim_mode.cu", "kernels_dm_tc.cu", "cmdline.cpp"]
HEADERS = ["fft_core.cuh", "kernel_util.cuh", "kernels.h", "kernels_epie.h", "kernels_mls.h", "session.h", "umma.cuh", "pdl.cuh", "fftx.cuh"]

LIB = os.path.join(HERE, "libptychopy_b200.so")
EXT = os.path.join(HERE, "ptychopy" + sysconfig.get_config_var("EXT_SUFFIX"))


def _newer(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(force=False, verbose=True):
    """Compile the CUDA kernels + C ABI into libptychopy_b200.so and the CPython module `ptychopy`."""
    os.makedirs(BUILD, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "ptychopy_b200.h")]
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
        if force or _newer(o, [s] + hdrs):
            _run([NVCC] + NVFLAGS + ["-c", s, "-o", o], verbose)
        objs.append(o)
    if force or _newer(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart_static", "-lrt", "-ldl", "-lpthread"],
             verbose)
    import numpy

    pysrc = os.path.join(CSRC, "pymodule.cpp")
    if force or _newer(EXT, [pysrc, LIB, os.path.join(ROOT, "include", "ptychopy_b200.h")]):
        _run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-Wall",
              "-I" + sysconfig.get_paths()["include"], "-I" + numpy.get_include(),
              pysrc, "-o", EXT, "-L" + HERE, "-lptychopy_b200", "-Wl,-rpath,$ORIGIN"], verbose)
    return LIB, EXT


if __name__ == "__main__":
    build(force="-f" in sys.argv)
