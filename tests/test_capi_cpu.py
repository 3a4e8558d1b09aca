"""C ABI checks that need no GPU: the library loads, exports every function that
include/owl_ssg.h declares, and refuses to run without a device (no CPU
fallback)."""
import ctypes as C
import os
import re

import pytest

from owl_b200 import _lib as L
from owl_b200.solver import SSGSolver

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    txt = open(os.path.join(ROOT, "include", "owl_ssg.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(owl_\w+)\s*\(", txt)))


def test_header_symbols_exported():
    lib = L.load()
    names = header_functions()
    assert len(names) >= 12
    for n in names:
        assert hasattr(lib, n), n
    assert sorted(L.EXPORTED) == names


def test_queries():
    lib = L.load()
    assert lib.owl_ssg_abi_version() == 10
    assert lib.owl_ssg_nparam(L.OWL_ACOUSTIC_ISO_2D) == 2
    assert lib.owl_ssg_ncomp(L.OWL_ELASTIC_VHTIORT_2D) == 2
    assert lib.owl_ssg_nparam(99) == -1
    d = L.OwlSsgDesc()
    d.medium = L.OWL_ELASTIC_VHTIORT_2D
    for aniso, n in ((L.OWL_ANISO_ISO, 3), (L.OWL_ANISO_THOMSEN, 6), (L.OWL_ANISO_AT, 6), (L.OWL_ANISO_CIJ, 5), (9, -1)):
        d.aniso = aniso
        assert lib.owl_ssg_desc_nparam(C.byref(d)) == n
    d.medium = L.OWL_ACOUSTIC_ISO_3D
    assert lib.owl_ssg_desc_nparam(C.byref(d)) == 2


def test_struct_sizes_match_header():
    # ctypes mirrors the C structs field for field (no padding surprises)
    assert C.sizeof(L.OwlSsgDesc) == 4 * 22
    assert C.sizeof(L.OwlRunOpts) == 4 * 8
    assert C.sizeof(L.OwlReceiver) == 4 * (6 + 54 + 1)


def test_no_device_is_an_error_not_a_fallback():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = L.load()
    assert lib.owl_ssg_device_ok() == 0
    with pytest.raises(L.OwlError) as e:
        SSGSolver(L.OWL_ACOUSTIC_ISO_2D, 32, 32, 10.0, 10.0, 1e-3, 10)
    assert e.value.code == L.OWL_ERR_NO_DEVICE


def test_null_arguments_rejected():
    lib = L.load()
    assert lib.owl_ssg_create(None, None) == L.OWL_ERR_INVALID
    assert b"null" in lib.owl_last_error()
    assert lib.owl_ssg_forward(None, 0, None, None, None, 0, None) == L.OWL_ERR_INVALID
