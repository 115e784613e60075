"""The recipe that compiles the reference's own device functions (oracle/ref_build.py): every listed function is
found exactly once in its source file, and the built library exports every launch wrapper the stage tests use.
No GPU needed."""
import ctypes
import os

import pytest

import pyref
import ref_build

REF = ref_build.DEFAULT_REF


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "src")), reason="needs the reference checkout")
def test_every_unit_is_extracted_once():
    for fname, kind, name in ref_build.UNITS:
        with open(os.path.join(REF, "src", fname)) as f:
            line, body = ref_build.extract(f.read(), kind, name)
        assert line > 0 and name in body.split("(")[0] + body.split("{")[0]


def test_extract_picks_the_definition_not_a_declaration():
    src = "__global__ void d_k(int a);\n\ntemplate<bool B>\n__global__ void d_k(int a)\n{\n  if (a) { a++; }\n}\n"
    line, body = ref_build.extract(src, "fn", "d_k")
    assert line == 3 and body.startswith("template<bool B>") and body.endswith("}")


def test_library_exports_the_wrappers():
    if not pyref.available():
        pytest.skip("oracle/_ref/libptyref.so not built here")
    L = ctypes.CDLL(pyref.LIB)
    for name in ["ref_version", "ref_dm_calc_psi", "ref_dm_modulus", "ref_dm_update", "ref_extract_patch",
                 "ref_simulate_psi", "ref_adjust_fft", "ref_update_object", "ref_update_probe", "ref_calculate_er",
                 "ref_lsq_terms", "ref_modulus_amplitude", "ref_cartesian_mesh", "ref_symmetrize", "ref_rotate90",
                 "ref_shift_fft", "ref_sqrt_patterns", "ref_preprocess"]:
        assert hasattr(L, name), name
    assert L.ref_version() == 1
