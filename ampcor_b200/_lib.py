"""ctypes binding of the C ABI declared in include/ampcor_b200.h.

The shared library ``libampcor_b200.so`` is built in-tree next to this file (see
``ampcor_b200/build.py``).  Loading it needs no GPU; every compute entry point does.
There is no other implementation behind this module: if the library is missing the import of
``load()`` raises, it never falls back to host code.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_float, c_int, c_int32, c_int64, c_uint32, c_uint64, c_void_p

HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY = os.path.join(HERE, "libampcor_b200.so")

# status codes (include/ampcor_b200.h)
OK = 0
E_ARG = 1
E_SHAPE = 2
E_CUDA = 3
E_NOMEM = 4
E_BOUNDS = 5
E_STATE = 6
FLAG_REF_COMPAT = 1
FLAG_PLAIN_FP32 = 2
FLAG_DERAMP = 4

STATUS_NAMES = {
    OK: "AMPCOR_OK",
    E_ARG: "AMPCOR_E_ARG",
    E_SHAPE: "AMPCOR_E_SHAPE",
    E_CUDA: "AMPCOR_E_CUDA",
    E_NOMEM: "AMPCOR_E_NOMEM",
    E_BOUNDS: "AMPCOR_E_BOUNDS",
    E_STATE: "AMPCOR_E_STATE",
}


class Params(ctypes.Structure):
    _fields_ = [
        ("pairs", c_uint64),
        ("ref_lines", c_uint64),
        ("ref_samples", c_uint64),
        ("tgt_lines", c_uint64),
        ("tgt_samples", c_uint64),
        ("refine_factor", c_uint64),
        ("refine_margin", c_uint64),
        ("zoom_factor", c_uint64),
        ("device", c_int32),
        ("flags", c_uint32),
    ]


class PairDiag(ctypes.Structure):
    _fields_ = [
        ("coarse_u", c_int32),
        ("coarse_v", c_int32),
        ("top", c_int32),
        ("left", c_int32),
        ("refined_u", c_int32),
        ("refined_v", c_int32),
        ("fine_p", c_int32),
        ("fine_q", c_int32),
        ("coarse_peak", c_float),
        ("refined_peak", c_float),
        ("zoom_peak", c_float),
        ("reserved", c_float),
    ]


class Job(ctypes.Structure):
    _fields_ = [
        ("ref", c_void_p),
        ("ref_lines", c_int64),
        ("ref_samples", c_int64),
        ("tgt", c_void_p),
        ("tgt_lines", c_int64),
        ("tgt_samples", c_int64),
        ("ulhc", c_void_p),
        ("pairs", c_uint64),
        ("offsets", c_void_p),
        ("diag", c_void_p),
        ("coarse_surfaces", c_void_p),
        ("refined_surfaces", c_void_p),
    ]


# every symbol the header declares, with its signature
SIGNATURES = {
    "ampcor_create": (c_int, [POINTER(Params), POINTER(c_void_p)]),
    "ampcor_destroy": (c_int, [c_void_p]),
    "ampcor_add_reference": (c_int, [c_void_p, c_uint64, c_void_p, c_uint64]),
    "ampcor_add_target": (c_int, [c_void_p, c_uint64, c_void_p, c_uint64]),
    "ampcor_adjust": (c_int, [c_void_p, POINTER(POINTER(c_float))]),
    "ampcor_diagnostics": (c_int, [c_void_p, c_void_p]),
    "ampcor_correlate": (c_int, [c_void_p, POINTER(Job), c_void_p]),
    "ampcor_synchronize": (c_int, [c_void_p, c_void_p]),
    "ampcor_correlate_host": (c_int, [c_void_p, POINTER(Job)]),
    "ampcor_surface_dims": (c_int, [c_void_p, POINTER(c_int32), POINTER(c_int32), POINTER(c_int32)]),
    "ampcor_profile": (c_int, [c_void_p, c_int]),
    "ampcor_stage_times": (c_int, [c_void_p, POINTER(ctypes.c_double), POINTER(ctypes.c_double),
                                   POINTER(ctypes.c_double), POINTER(c_uint64)]),
    "ampcor_kernel_times": (c_int, [c_void_p, POINTER(ctypes.c_double), POINTER(c_uint64)]),
    "ampcor_form": (c_int, [c_void_p]),
    "ampcor_configure": (c_int, [c_void_p, c_int, c_uint64]),
    "ampcor_chunk": (c_int, [c_void_p, POINTER(c_uint64)]),
    "ampcor_inject_timeout": (c_int, [c_void_p, c_int]),
    "ampcor_correlate_noalloc": (c_int, [POINTER(Params), POINTER(Job), c_void_p, ctypes.c_char_p,
                                         ctypes.c_size_t]),
    "ampcor_last_error": (c_char_p, [c_void_p]),
    "ampcor_version": (c_char_p, []),
    "ampcor_copyright": (c_char_p, []),
}

_lib = None


def load(path: str = LIBRARY) -> ctypes.CDLL:
    """Load (once) and return the correlator library with its signatures declared."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(
            f"{path} is missing: build the CUDA library first (python -m ampcor_b200.build)"
        )
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib
