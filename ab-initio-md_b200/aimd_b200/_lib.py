"""
ctypes binding of the C ABI in ``include/aimd_b200.h`` (library
``aimd_b200/_native/libaimd_b200.so``, built by ``aimd_b200/build.py``).

There is no fallback: if the library is missing or no CUDA device is
present, ``load()`` raises, and so does every integral call.
"""

from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_native", "libaimd_b200.so")

AIMD_OK, AIMD_ERR_ARG, AIMD_ERR_CUDA, AIMD_ERR_UNSUPPORTED = 0, 1, 2, 3

_i32p = ctypes.POINTER(ctypes.c_int)
_f64p = ctypes.POINTER(ctypes.c_double)
_i64p = ctypes.POINTER(ctypes.c_int64)
_vp = ctypes.c_void_p
_i = ctypes.c_int
_d = ctypes.c_double

# name -> (restype, argtypes); the exported surface of include/aimd_b200.h
SIGNATURES = {
    "aimd_create": (_i, [ctypes.POINTER(_vp), _i, _i, _i, _i32p, _i32p, _i32p, _i32p, _i32p, _i32p, _i, _f64p, _f64p,
                         _i, _i32p, _i32p, _i32p, _i32p, _i32p, _i, _f64p, _f64p, _f64p]),
    "aimd_destroy": (_i, [_vp]),
    "aimd_set_geometry": (_i, [_vp, _vp, _vp]),
    "aimd_schwarz": (_i, [_vp, _vp, _vp]),
    "aimd_pair_count": (_i, [_vp]),
    "aimd_set_fp32_cutoff": (_i, [_vp, _d]),
    "aimd_set_launch_shape": (_i, [_vp, _i, _i]),
    "aimd_get_launch_shape": (_i, [_vp, ctypes.POINTER(_i), ctypes.POINTER(_i)]),
    "aimd_jk": (_i, [_vp, _i, _vp, _vp, _vp, _d, _vp]),
    "aimd_jk_delta": (_i, [_vp, _i, _vp, _vp, _vp, _d, _d, _vp]),
    "aimd_eri_tensor": (_i, [_vp, _vp, _d, _vp]),
    "aimd_eri_tensor_static": (_i, [_vp, _vp, _d, _vp]),
    "aimd_grad2e": (_i, [_vp, _vp, _i, _vp, _d, _d, _d, _vp, _vp]),
    "aimd_onee": (_i, [_vp, _f64p, _vp, _vp, _vp, _vp, _vp]),
    "aimd_onee_grad": (_i, [_vp, _vp, _vp, _vp, _vp]),
    "aimd_quartet_counts": (_i, [_vp, _i, _i64p]),
    "aimd_pair_data": (_i, [_vp, _i32p, _i32p, _i32p]),
    "aimd_launch_count": (ctypes.c_uint64, [_vp]),
    "aimd_sizes": (_i, [_vp, ctypes.POINTER(_i), ctypes.POINTER(_i)]),
    "aimd_nuclear_repulsion": (_i, [_vp, ctypes.POINTER(_d), _vp]),
    "aimd_last_error": (ctypes.c_char_p, []),
    "aimd_version": (_i, []),
}

_lib = None

# the device SCF driver (include/aimd_scf.h), a second library over the first
SCF_LIB_PATH = os.path.join(_HERE, "_native", "libaimd_scf.so")
AIMD_SCF_CONVERGED, AIMD_SCF_MAX_ITER, AIMD_SCF_NONFINITE = 1, 2, 4


class SCFOptions(ctypes.Structure):
    """aimd_scf_options of include/aimd_scf.h."""
    _fields_ = [("n_alpha", ctypes.c_int), ("n_beta", ctypes.c_int), ("unrestricted", ctypes.c_int),
                ("max_iter", ctypes.c_int), ("diis_space", ctypes.c_int), ("conv_energy", ctypes.c_double),
                ("conv_commutator", ctypes.c_double), ("schwarz_threshold", ctypes.c_double),
                ("lindep_threshold", ctypes.c_double), ("max_coefficient", ctypes.c_double)]


SCF_SIGNATURES = {
    "aimd_scf_default_options": (None, [ctypes.POINTER(SCFOptions)]),
    "aimd_scf_run": (_i, [_vp, ctypes.POINTER(SCFOptions), _vp, _vp, _vp, ctypes.POINTER(_d),
                          ctypes.POINTER(_i), ctypes.POINTER(_i), _vp]),
    "aimd_scf_release": (_i, [_vp]),
    "aimd_scf_last_error": (ctypes.c_char_p, []),
}
_scf = None


def load_scf() -> ctypes.CDLL:
    """The SCF driver library (loaded once, after the integral library); raises if it is not built."""
    global _scf
    if _scf is None:
        load()
        if not os.path.exists(SCF_LIB_PATH):
            raise ImportError(f"SCF driver not built: {SCF_LIB_PATH} (run aimd_b200/build.py)")
        lib = ctypes.CDLL(SCF_LIB_PATH)
        for name, (res, args) in SCF_SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _scf = lib
    return _scf


class NativeError(RuntimeError):
    """A C-ABI call returned a non-zero status."""


def load() -> ctypes.CDLL:
    """The native library (loaded once); raises if it is not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"native library not built: {LIB_PATH} (run aimd_b200/build.py or __graft_entry__.build())")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def check(status: int, what: str) -> None:
    if status != AIMD_OK:
        msg = load().aimd_last_error().decode(errors="replace")
        kind = {AIMD_ERR_ARG: "invalid argument", AIMD_ERR_CUDA: "CUDA error",
                AIMD_ERR_UNSUPPORTED: "unsupported"}.get(status, f"status {status}")
        raise NativeError(f"{what}: {kind}: {msg}")
