"""Drop-in for the ``ampcor_cuda`` CPython extension of ampcor (ext/ampcor_cuda/).

Same functions, same argument order and meaning, same return values:

* ``sequential(points, (refLines, refSamples), (tgtLines, tgtSamples), refineMargin,
  refineFactor, zoomFactor)`` -> worker (ext/ampcor_cuda/sequential.cc:40-73; note the Python
  order margin, factor, zoom);
* ``addReference(worker, slc, idx, (bLine, bSample), (eLine, eSample))`` and ``addTarget(...)``
  copy the slice [begin, end) of the raster into the worker (sequential.cc:85-143, :155-213);
* ``adjust(worker)`` -> tuple of ``(dy, dx)`` float pairs in pair order (sequential.cc:225-271);
* ``copyright()``, ``version()`` (ampcor_cuda.cc:25-27) and the exception class ``Error``.

A worker argument that is not a worker raises ``TypeError`` as the capsule checks do
(sequential.cc:108-126).  The raster argument is the SLC: a 2-d complex64 array, or an object
whose ``raster`` attribute is one (pkg/ampcor/dom/SLC.py:79-89 keeps its mapped raster there).
Failures in the library raise ``Error`` instead of aborting the interpreter.  The device is
``AMPCOR_DEVICE`` (default 0) where the reference hard-codes device 4
(pkg/ampcor/correlators/CUDA.py:73).
"""
from __future__ import annotations

import os

import numpy as np

from ..worker import Error, Worker
from ..worker import copyright as _copyright
from ..worker import version as _version

CAPSULE_NAME = "ampcor::cuda::sequential::capsule_t"

__all__ = ["Error", "copyright", "version", "sequential", "addReference", "addTarget", "adjust"]


class SequentialCapsule:
    """Opaque worker handle (the role of the PyCapsule named ``CAPSULE_NAME``)."""

    name = CAPSULE_NAME

    def __init__(self, worker: Worker):
        self.worker = worker


def copyright():
    return _copyright()


def version():
    return _version()


def sequential(points, ref_shape, tgt_shape, refineMargin, refineFactor, zoomFactor):
    """Instantiate a new sequential correlation worker."""
    ref_lines, ref_samples = (int(x) for x in ref_shape)
    tgt_lines, tgt_samples = (int(x) for x in tgt_shape)
    worker = Worker(
        pairs=int(points),
        chip=(ref_lines, ref_samples),
        window=(tgt_lines, tgt_samples),
        refine_factor=int(refineFactor),
        refine_margin=int(refineMargin),
        zoom_factor=int(zoomFactor),
        device=int(os.environ.get("AMPCOR_DEVICE", "0")),
    )
    return SequentialCapsule(worker)


def _worker(capsule) -> Worker:
    if not isinstance(capsule, SequentialCapsule):
        raise TypeError("invalid worker capsule")
    return capsule.worker


def _raster(slc) -> np.ndarray:
    raster = getattr(slc, "raster", slc)
    raster = np.asarray(raster)
    if raster.ndim != 2 or raster.dtype != np.complex64:
        raise TypeError("invalid SLC: expected a 2-d complex64 raster")
    return raster


def _slice(slc, begin, end):
    raster = _raster(slc)
    (bl, bs), (el, es) = ((int(x) for x in begin), (int(x) for x in end))
    return raster[bl:el, bs:es]


def addReference(worker, slc, idx, begin, end):
    """Copy the reference chip [begin, end) of ``slc`` into slot ``idx``."""
    _worker(worker).add_reference(int(idx), _slice(slc, begin, end))
    return None


def addTarget(worker, slc, idx, begin, end):
    """Copy the target search window [begin, end) of ``slc`` into slot ``idx``."""
    _worker(worker).add_target(int(idx), _slice(slc, begin, end))
    return None


def adjust(worker):
    """Perform pixel-level adjustments: returns ((dy, dx), ...) in pair order."""
    offsets = _worker(worker).adjust()
    return tuple((float(dy), float(dx)) for dy, dx in offsets)
