"""ampcor_b200: B200-native (sm_100a) batched tile correlator.

The drop-in boundary is the C ABI in ``include/ampcor_b200.h`` (library
``ampcor_b200/libampcor_b200.so``).  On top of it:

* :class:`ampcor_b200.worker.Worker` - the correlator worker (the role of
  ``ampcor::cuda::correlators::Sequential``);
* :mod:`ampcor_b200.ext.ampcor_cuda` - the functions of ampcor's ``ampcor_cuda`` extension;
* :mod:`ampcor_b200.autotune`, :mod:`ampcor_b200.batch`, :mod:`ampcor_b200.serve` - the
  autotuner, uneven raster batches in one CUDA graph and the continuous-batching server;
* :mod:`ampcor_b200.parallel` - row-band sharding of one job over ranks;
* :mod:`ampcor_b200.plan` - tile-pair planning with the reference's grid/plan semantics;
* :mod:`ampcor_b200.synth` - seeded synthetic raster pairs for the benchmark workloads.
"""
from .worker import Error, Worker, copyright, version  # noqa: F401

__all__ = ["Error", "Worker", "copyright", "version"]
