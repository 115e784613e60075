"""The C ABI library loads and exports every entry point the header declares (no GPU needed)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    txt = open(os.path.join(ROOT, "include", "ptychopy_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(pty_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    from ptychopy_b200 import abi

    L = ctypes.CDLL(abi.LIB_PATH)
    names = header_functions()
    assert len(names) >= 19
    for n in names:
        assert hasattr(L, n), n
    assert sorted(abi.EXPORTS) == names


def test_params_defaults_are_the_reference_defaults():
    # ptychopy_algorithmnp defaults (src/ptychopy.c:282-323)
    from ptychopy_b200 import abi

    p = abi.default_params()
    assert p.size == 512 and p.scanDimsx == 26 and p.scanDimsy == 26 and p.iter == 100
    assert p.beamSize == 400e-9 and p.stepx == 40e-9 and p.lambd == 2.3843e-10 and p.z == 2.2
    assert p.dx_d == 172e-6 and p.probeModes == 1 and p.phaseConstraint == 1
    assert p.updateProbe == 10 and p.updateModes == 20 and p.PPS == 20 and p.delta_p == 0.1
    assert p.algorithm == b"ePIE"


def test_params_struct_layout_matches_header(tmp_path):
    # compile a probe against the header and compare every field offset with the ctypes mirror
    import subprocess

    from ptychopy_b200 import abi

    fields = [f[0] for f in abi.PtyParams._fields_]
    src = tmp_path / "layout.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "ptychopy_b200.h"\nint main(void){\n'
                   + "".join(f'printf("%zu\\n", offsetof(pty_params, {f}));\n' for f in fields)
                   + 'printf("%zu\\n", sizeof(pty_params));return 0;}\n')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    assert out[:-1] == [getattr(abi.PtyParams, f).offset for f in fields]
    assert out[-1] == ctypes.sizeof(abi.PtyParams)


def test_bad_arguments_are_status_codes_not_crashes():
    from ptychopy_b200 import abi

    L = abi.lib()
    p = abi.default_params(algorithm="nope")
    h = ctypes.c_void_p()
    rc = L.pty_session_create(ctypes.byref(p), ctypes.byref(h))
    assert rc == abi.PTY_ERR_INVALID and not h.value
    assert b"unknown algorithm" in L.pty_last_error()
    p = abi.default_params(size=8)
    assert L.pty_session_create(ctypes.byref(p), ctypes.byref(h)) == abi.PTY_ERR_INVALID
    p = abi.default_params(fp=b"/data/scan#.h5")
    assert L.pty_session_create(ctypes.byref(p), ctypes.byref(h)) == abi.PTY_ERR_UNSUPPORTED
    assert L.pty_step(None, None) == abi.PTY_ERR_STATE
    assert L.pty_params_init(None) == abi.PTY_ERR_INVALID


def test_no_gpu_gives_a_cuda_status():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from ptychopy_b200 import abi

    p = abi.default_params()
    h = ctypes.c_void_p()
    rc = abi.lib().pty_session_create(ctypes.byref(p), ctypes.byref(h))
    assert rc in (abi.PTY_ERR_CUDA, abi.PTY_ERR_INVALID)
