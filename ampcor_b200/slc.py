"""SLC rasters on disk: raw row-major complex64, lines x samples, no header.

This mirrors the reference's file-based SLC product (pkg/ampcor/dom/SLC.py, backed by
lib/libampcor/dom/SLC.icc:123-126 and the ext/ampcor/slc.cc:50-93 bindings): the caller gives the
path and the shape, the file is mapped read-only, pixels are read by (line, sample) index or by
flat offset, and ``slice`` refuses regions that leave the raster.  On top of that, ``pinned()``
reads the raster into page-locked host memory, which is what lets
``Worker.correlate`` (``ampcor_correlate_host``) upload it in bands while the correlation of the
pairs already covered runs.
"""
from __future__ import annotations

import os

import numpy as np

PIXEL_DTYPE = np.dtype(np.complex64)


def pixel_size() -> int:
    """Bytes per pixel (slc_pixelSize in the reference extension)."""
    return PIXEL_DTYPE.itemsize


class SLC:
    """A raw complex64 raster file of ``shape = (lines, samples)``."""

    def __init__(self, path, shape):
        lines, samples = (int(s) for s in shape)
        if lines <= 0 or samples <= 0:
            raise ValueError(f"an SLC needs a positive shape, got {shape}")
        self.path = os.fspath(path)
        self.shape = (lines, samples)
        self.raster = None

    def size(self) -> int:
        """Memory footprint of the raster in bytes (SLC.py: size)."""
        lines, samples = self.shape
        return lines * samples * pixel_size()

    def open(self, mode: str = "r") -> "SLC":
        """Map the file (SLC.py: open).  The file must hold at least ``size()`` bytes."""
        if mode not in ("r", "r+"):
            raise ValueError("an SLC opens for reading ('r') or update ('r+')")
        have = os.path.getsize(self.path)
        if have < self.size():
            raise ValueError(f"{self.path}: {have} bytes, a {self.shape[0]} x {self.shape[1]} SLC "
                             f"needs {self.size()}")
        self.raster = np.memmap(self.path, dtype=PIXEL_DTYPE, mode=mode, shape=self.shape)
        return self

    def _mapped(self) -> np.ndarray:
        if self.raster is None:
            self.open()
        return self.raster

    def __getitem__(self, index) -> complex:
        """The pixel at a (line, sample) index or at a flat offset (slc_getitem)."""
        r = self._mapped()
        if isinstance(index, (tuple, list)):
            line, sample = (int(i) for i in index)
            if not (0 <= line < self.shape[0] and 0 <= sample < self.shape[1]):
                raise IndexError(f"pixel {index} outside a {self.shape} raster")
            return complex(r[line, sample])
        offset = int(index)
        if not 0 <= offset < r.size:
            raise IndexError(f"offset {offset} outside a raster of {r.size} pixels")
        return complex(r.reshape(-1)[offset])

    def slice(self, begin, shape):
        """A view of the region at ``begin`` of ``shape``, or None where it leaves the raster
        (SLC.py: slice, with its one-past-the-end convention)."""
        if any(b < 0 for b in begin):
            return None
        if any(b + s > l for b, s, l in zip(begin, shape, self.shape)):
            return None
        (b0, b1), (s0, s1) = begin, shape
        return self._mapped()[b0:b0 + s0, b1:b1 + s1]

    def pinned(self, rows_per_read: int = 1024) -> np.ndarray:
        """The whole raster in page-locked host memory, read ``rows_per_read`` lines at a time.

        Page-locked memory is what lets the host-buffer correlation overlap its upload with the
        correlation; without a CUDA device the buffer is ordinary host memory."""
        lines, samples = self.shape
        out = pinned_empty(self.shape)
        src = self._mapped()
        for y in range(0, lines, max(1, rows_per_read)):
            out[y:y + rows_per_read] = src[y:y + rows_per_read]
        return out

    @staticmethod
    def write(path, raster) -> "SLC":
        """Write a 2-d complex raster as a raw complex64 SLC file and return it, unopened."""
        a = np.ascontiguousarray(raster, dtype=PIXEL_DTYPE)
        if a.ndim != 2:
            raise ValueError("an SLC raster is 2-d (lines x samples)")
        a.tofile(os.fspath(path))
        return SLC(path, a.shape)


def pinned_empty(shape) -> np.ndarray:
    """An uninitialised complex64 host array of ``shape`` in page-locked memory where a CUDA
    device is present (through torch), else in ordinary memory."""
    try:
        import torch

        if torch.cuda.is_available():
            t = torch.empty(tuple(shape), dtype=torch.complex64, pin_memory=True)
            a = t.numpy()
            # keep the tensor (and its page-locked allocation) alive as long as the array
            return _Pinned(a, t)
    except ImportError:  # pragma: no cover
        pass
    return np.empty(tuple(shape), dtype=PIXEL_DTYPE)


class _Pinned(np.ndarray):
    """A numpy view of a page-locked torch buffer that holds on to the buffer."""

    def __new__(cls, view, owner):
        obj = view.view(cls)
        obj._owner = owner
        return obj

    def __array_finalize__(self, obj):
        self._owner = getattr(obj, "_owner", None)
