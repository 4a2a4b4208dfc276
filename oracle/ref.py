"""The reference's own CPU correlator, compiled from its sources - TEST INFRASTRUCTURE ONLY.

``oracle/_ref/libampcor_ref.so`` (``make -C oracle``, when the reference source tree is present)
holds lib/libampcor/correlators/Sequential.cc and lib/libampcor/dom/SLC.cc, built unmodified
against the pyre stand-ins of ``oracle/ref_shim``, and the driver ``ref_shim/ref_driver.cc``.
Only the tests (which pin the FP64 oracle to it) and the reference arm of ``bench.py`` (which
times it) load it.

* :func:`sequential` - ``Sequential::adjust`` over a batch of tile pairs cut from two rasters by
  the reference's own ``addReferenceTile`` / ``addTargetTile`` (the rasters are written to raw
  complex64 files, the SLC format of lib/libampcor/dom/SLC.icc:122-126, and memory-mapped);
* :func:`sumarea` - the reference's ``SumArea`` table and box sums (SumArea.icc:66-180).
"""
from __future__ import annotations

import ctypes
import os
import tempfile
from ctypes import c_char_p, c_int, c_long, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libampcor_ref.so")

_lib = None


def available() -> bool:
    return os.path.exists(LIB)


def load():
    global _lib
    if _lib is None:
        if not available():
            raise ImportError(f"{LIB} is missing: build it with `make -C oracle` where the "
                              f"reference source tree is present")
        lib = ctypes.CDLL(LIB)
        lib.ampcor_ref_sequential.restype = c_int
        lib.ampcor_ref_sequential.argtypes = [c_char_p, c_long, c_long, c_char_p, c_long, c_long,
                                              c_void_p, c_long, c_long, c_long, c_void_p, c_int]
        lib.ampcor_ref_sumarea.restype = c_int
        lib.ampcor_ref_sumarea.argtypes = [c_void_p, c_long, c_long, c_void_p, c_void_p, c_long,
                                           c_void_p]
        lib.ampcor_ref_error.restype = c_char_p
        lib.ampcor_ref_error.argtypes = []
        _lib = lib
    return _lib


class Rasters:
    """A raster pair written once to raw complex64 files for the reference's SLC reader."""

    def __init__(self, ref, tgt, directory=None):
        self.ref_shape = tuple(int(s) for s in ref.shape)
        self.tgt_shape = tuple(int(s) for s in tgt.shape)
        self._dir = tempfile.TemporaryDirectory(dir=directory)
        self.ref_path = os.path.join(self._dir.name, "reference.slc")
        self.tgt_path = os.path.join(self._dir.name, "secondary.slc")
        np.ascontiguousarray(ref, np.complex64).tofile(self.ref_path)
        np.ascontiguousarray(tgt, np.complex64).tofile(self.tgt_path)

    def close(self):
        self._dir.cleanup()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def sequential(rasters: Rasters, ulhc, R, W, threads=1):
    """The correlation surfaces ((P, C, C) doubles) of the reference's CPU ``Sequential`` worker
    for the pairs whose chip and window corners are the rows of ``ulhc``."""
    u = np.ascontiguousarray(np.asarray(ulhc).reshape(-1, 4), np.int32)
    C = W - R + 1
    cor = np.zeros((u.shape[0], C, C))
    rc = load().ampcor_ref_sequential(rasters.ref_path.encode(), *rasters.ref_shape,
                                      rasters.tgt_path.encode(), *rasters.tgt_shape,
                                      u.ctypes.data, u.shape[0], R, W, cor.ctypes.data,
                                      int(threads))
    if rc:
        raise RuntimeError(load().ampcor_ref_error().decode())
    return cor


def sumarea(a, boxes=()):
    """The reference's summed-area table of a 2-d array and its sums over ``boxes`` (rows of
    r0, c0, height, width)."""
    a = np.ascontiguousarray(a, np.float64)
    b = np.ascontiguousarray(np.asarray(boxes, np.int64).reshape(-1, 4), dtype=np.int64)
    table = np.empty_like(a)
    sums = np.empty(b.shape[0])
    rc = load().ampcor_ref_sumarea(a.ctypes.data, a.shape[0], a.shape[1], table.ctypes.data,
                                   b.ctypes.data, b.shape[0], sums.ctypes.data)
    if rc:
        raise RuntimeError(load().ampcor_ref_error().decode())
    return table, sums
