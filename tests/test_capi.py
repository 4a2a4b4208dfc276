"""The C ABI library loads and exports what include/ampcor_b200.h declares (CPU only; no
compute call needs a GPU here)."""
import ctypes
import os
import re

import numpy as np
import pytest

from ampcor_b200 import _lib
from ampcor_b200.worker import Error, Worker

from conftest import cuda_available

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "ampcor_b200.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^(?:int|const char\*)\s+(ampcor_\w+)\s*\(", text, re.M)))


def test_header_declares_the_abi():
    names = declared_functions()
    assert set(names) == set(_lib.SIGNATURES), (names, sorted(_lib.SIGNATURES))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_lib.LIBRARY)
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_version_and_copyright():
    lib = _lib.load()
    assert b"ampcor_b200" in lib.ampcor_version()
    assert lib.ampcor_copyright()


def test_struct_sizes():
    assert ctypes.sizeof(_lib.PairDiag) == 48
    assert ctypes.sizeof(_lib.Params) == 8 * 8 + 8
    assert ctypes.sizeof(_lib.Job) == 12 * 8


def test_rejects_bad_geometry_without_touching_cuda():
    lib = _lib.load()
    h = ctypes.c_void_p()
    p = _lib.Params(pairs=1, ref_lines=32, ref_samples=16, tgt_lines=48, tgt_samples=48,
                    refine_factor=2, refine_margin=4, zoom_factor=4)
    assert lib.ampcor_create(ctypes.byref(p), ctypes.byref(h)) == _lib.E_SHAPE
    assert b"square" in lib.ampcor_last_error(None)
    p = _lib.Params(pairs=1, ref_lines=32, ref_samples=32, tgt_lines=47, tgt_samples=47,
                    refine_factor=2, refine_margin=4, zoom_factor=4)
    assert lib.ampcor_create(ctypes.byref(p), ctypes.byref(h)) == _lib.E_SHAPE
    p = _lib.Params(pairs=1, ref_lines=32, ref_samples=32, tgt_lines=48, tgt_samples=48,
                    refine_factor=2, refine_margin=12, zoom_factor=4)
    assert lib.ampcor_create(ctypes.byref(p), ctypes.byref(h)) == _lib.E_SHAPE  # 32+24 > 48
    assert lib.ampcor_create(None, ctypes.byref(h)) == _lib.E_ARG
    assert lib.ampcor_destroy(None) == _lib.E_ARG


def test_rejects_refinement_not_multiple_of_eight():
    lib = _lib.load()
    h = ctypes.c_void_p()
    p = _lib.Params(pairs=1, ref_lines=30, ref_samples=30, tgt_lines=46, tgt_samples=46,
                    refine_factor=2, refine_margin=4, zoom_factor=4)
    assert lib.ampcor_create(ctypes.byref(p), ctypes.byref(h)) == _lib.E_SHAPE


@pytest.mark.skipif(cuda_available(), reason="checks the no-device failure path")
def test_create_without_a_device_fails_cleanly():
    with pytest.raises(Error) as e:
        Worker(pairs=4, chip=(32, 32), window=(48, 48), refine_factor=2, refine_margin=4,
               zoom_factor=4)
    assert e.value.status == _lib.E_CUDA
