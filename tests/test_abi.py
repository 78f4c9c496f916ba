"""The C-ABI library loads and exports every entry point include/aimd_b200.h declares (no GPU calls)."""

import ctypes
import os
import re

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "aimd_b200.h")
SCF_HEADER = os.path.join(ROOT, "include", "aimd_scf.h")


def declared_functions(header=HEADER):
    src = open(header).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(aimd_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_the_abi():
    names = declared_functions()
    for must in ["aimd_create", "aimd_destroy", "aimd_set_geometry", "aimd_jk", "aimd_grad2e", "aimd_onee",
                 "aimd_onee_grad", "aimd_schwarz", "aimd_eri_tensor", "aimd_last_error"]:
        assert must in names


def test_library_exports_every_declared_symbol():
    from aimd_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("native library not built in this checkout")
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    assert set(_lib.SIGNATURES) >= set(declared_functions())
    lib.aimd_version.restype = ctypes.c_int
    assert lib.aimd_version() == 1


def test_scf_driver_exports_every_declared_symbol():
    from aimd_b200 import _lib
    if not os.path.exists(_lib.SCF_LIB_PATH):
        pytest.skip("SCF driver not built in this checkout")
    names = declared_functions(SCF_HEADER)
    assert {"aimd_scf_run", "aimd_scf_default_options", "aimd_scf_release", "aimd_scf_last_error"} <= set(names)
    lib = _lib.load_scf()
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(_lib.SCF_SIGNATURES) >= set(names)
    # the defaults of include/aimd_scf.h, through the library (no GPU call)
    import ctypes
    opt = _lib.SCFOptions()
    lib.aimd_scf_default_options(ctypes.byref(opt))
    assert (opt.max_iter, opt.diis_space, opt.conv_energy, opt.conv_commutator) == (100, 8, 1e-10, 1e-7)
