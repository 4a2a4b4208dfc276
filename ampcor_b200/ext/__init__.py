"""Extension modules with the names the ampcor Python package imports.

``ampcor.ext`` resolves ``libampcor_cuda`` to the CPython extension ``ampcor_cuda``
(pkg/ampcor/ext/__init__.py:29-51); :mod:`ampcor_b200.ext.ampcor_cuda` provides the same
module-level functions on top of the C ABI, so the reference's CUDA strategy can bind to it
unchanged (``libampcor_cuda = ampcor_b200.ext.ampcor_cuda``).
"""
from . import ampcor_cuda  # noqa: F401

libampcor_cuda = ampcor_cuda
