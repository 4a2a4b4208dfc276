"""Python view of the correlator worker (one ``ampcor_handle`` of the C ABI).

``Worker`` mirrors ``ampcor::cuda::correlators::Sequential`` (lib/libampcor_cuda/correlators/
Sequential.h:44-67): it is built from the pair count, the chip and window shapes and the
refinement parameters, takes chips and windows pair by pair (``add_reference``/``add_target``)
and ``adjust()`` returns the offset field.  It also offers ``correlate()``, which cuts the tiles
from whole rasters on the device, for device-resident (``torch`` CUDA tensors) or host (numpy)
buffers.
"""
from __future__ import annotations

import ctypes
from ctypes import byref, c_float, c_int32, c_void_p

import numpy as np

from . import _lib

# correlation forms, indexed by the value ampcor_form returns
FORMS = ("plain", "tensor", "spectral")


class Error(Exception):
    """Raised when the correlator library reports a failure (the extension's ``Error``,
    ext/ampcor_cuda/exceptions.cc:30-40)."""

    def __init__(self, status: int, message: str):
        self.status = status
        super().__init__(f"{_lib.STATUS_NAMES.get(status, status)}: {message}")


def _check(lib, handle, status):
    if status != _lib.OK:
        msg = lib.ampcor_last_error(handle)
        raise Error(status, msg.decode() if msg else "")


class Worker:
    """A correlator bound to one CUDA device."""

    def __init__(self, pairs, chip, window, refine_factor=2, refine_margin=8, zoom_factor=4,
                 device=0, ref_compat=False, plain=False, deramp=False):
        self._lib = _lib.load()
        chip = tuple(int(c) for c in chip)
        window = tuple(int(w) for w in window)
        self.pairs = int(pairs)
        self.chip = chip
        self.window = window
        self.refine_factor = int(refine_factor)
        self.refine_margin = int(refine_margin)
        self.zoom_factor = int(zoom_factor)
        self.device = int(device)
        params = _lib.Params(
            pairs=self.pairs,
            ref_lines=chip[0],
            ref_samples=chip[1],
            tgt_lines=window[0],
            tgt_samples=window[1],
            refine_factor=self.refine_factor,
            refine_margin=self.refine_margin,
            zoom_factor=self.zoom_factor,
            device=self.device,
            flags=(_lib.FLAG_REF_COMPAT if ref_compat else 0) | (_lib.FLAG_PLAIN_FP32 if plain else 0)
            | (_lib.FLAG_DERAMP if deramp else 0),
        )
        handle = c_void_p()
        _check(self._lib, None, self._lib.ampcor_create(byref(params), byref(handle)))
        self._handle = handle
        c, r, z = c_int32(), c_int32(), c_int32()
        self._lib.ampcor_surface_dims(handle, byref(c), byref(r), byref(z))
        self.coarse_dim, self.refined_dim, self.zoomed_dim = c.value, r.value, z.value
        # "spectral": FFT correlation in shared memory; "tensor": bf16x3 split products on the
        # tensor cores; "plain": FP32 FMA direct sums
        self.form = FORMS[self._lib.ampcor_form(handle)]

    # lifetime
    def close(self):
        if getattr(self, "_handle", None):
            self._lib.ampcor_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._handle

    # the pair-by-pair interface of the reference worker
    def _add(self, fn, pid, tile, dim):
        tile = np.asarray(tile)
        if tile.dtype != np.complex64 or tile.ndim != 2:
            raise TypeError("tiles are 2-d complex64 arrays")
        if tile.shape != (dim, dim):
            raise ValueError(f"expected a {dim}x{dim} tile, got {tile.shape}")
        if tile.strides[1] != 8:
            tile = np.ascontiguousarray(tile)
        stride = tile.strides[0] // 8
        _check(self._lib, self._handle,
               fn(self._handle, int(pid), tile.ctypes.data_as(c_void_p), stride))

    def add_reference(self, pid, tile):
        self._add(self._lib.ampcor_add_reference, pid, tile, self.chip[0])

    def add_target(self, pid, tile):
        self._add(self._lib.ampcor_add_target, pid, tile, self.window[0])

    def adjust(self) -> np.ndarray:
        """Correlate every pair; returns a (pairs, 2) float32 array of (dy, dx)."""
        ptr = ctypes.POINTER(c_float)()
        _check(self._lib, self._handle, self._lib.ampcor_adjust(self._handle, byref(ptr)))
        if self.pairs == 0:
            return np.zeros((0, 2), np.float32)
        return np.ctypeslib.as_array(ptr, shape=(self.pairs, 2)).copy()

    def diagnostics(self) -> np.ndarray:
        out = (_lib.PairDiag * max(self.pairs, 1))()
        _check(self._lib, self._handle,
               self._lib.ampcor_diagnostics(self._handle, ctypes.cast(out, c_void_p)))
        return diag_array(out, self.pairs)

    # per-stage device timing
    def profile(self, enable=True):
        _check(self._lib, self._handle, self._lib.ampcor_profile(self._handle, int(bool(enable))))

    def stage_times(self):
        """(coarse_ms, refine_ms, fine_ms, launches) since profiling started or was last read."""
        c, r, f = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        n = ctypes.c_uint64()
        _check(self._lib, self._handle,
               self._lib.ampcor_stage_times(self._handle, byref(c), byref(r), byref(f), byref(n)))
        return c.value, r.value, f.value, n.value

    def configure(self, form=None, chunk=None):
        """Select the form ("spectral", "tensor" or "plain") and the refinement chunk (pairs)."""
        f = -1 if form is None else FORMS.index(form)
        _check(self._lib, self._handle,
               self._lib.ampcor_configure(self._handle, f, int(chunk or 0)))
        self.form = FORMS[self._lib.ampcor_form(self._handle)]

    def inject_timeout(self, batches=1):
        """Failure-detection test hook: the next ``batches`` batches make their tensor-core zoom
        wait on a barrier nothing completes; the bounded wait runs out and the batch raises
        :class:`Error` (AMPCOR_E_CUDA, timed out) at its synchronisation."""
        _check(self._lib, self._handle, self._lib.ampcor_inject_timeout(self._handle, int(batches)))

    @property
    def chunk(self):
        c = ctypes.c_uint64()
        _check(self._lib, self._handle, self._lib.ampcor_chunk(self._handle, byref(c)))
        return c.value

    KERNELS = ("coarse_correlation", "refinement", "fine_correlation", "coarse_statistics",
               "fine_statistics", "zoom")

    def kernel_times(self):
        """{kernel: (ms, launches)} since profiling started or was last read."""
        ms = (ctypes.c_double * 6)()
        n = (ctypes.c_uint64 * 6)()
        _check(self._lib, self._handle, self._lib.ampcor_kernel_times(self._handle, ms, n))
        return {k: (ms[i], n[i]) for i, k in enumerate(self.KERNELS)}

    # whole rasters
    def correlate(self, ref, tgt, ulhc, offsets=None, diag=None, coarse_surfaces=None,
                  refined_surfaces=None, stream=None, synchronize=True):
        """Correlate the pairs whose chip/window corners are the rows of ``ulhc`` (int32,
        pairs x 4: chip line, chip sample, window line, window sample).

        ``ref``/``tgt`` are 2-d complex64 rasters: either all arguments are CUDA tensors
        (device path, enqueued on ``stream``) or all are numpy arrays (host path, copies inside
        the call).  Returns the (pairs, 2) offsets.
        """
        try:
            import torch
        except ImportError:  # pragma: no cover
            torch = None
        if torch is not None and isinstance(ref, torch.Tensor):
            return self._correlate_device(ref, tgt, ulhc, offsets, diag, coarse_surfaces,
                                          refined_surfaces, stream, synchronize)
        return self._correlate_host(ref, tgt, ulhc, diag)

    def _correlate_device(self, ref, tgt, ulhc, offsets, diag, cs, rs, stream, synchronize):
        import torch

        for name, t in (("ref", ref), ("tgt", tgt), ("ulhc", ulhc)):
            if not t.is_cuda or not t.is_contiguous():
                raise ValueError(f"{name} must be a contiguous CUDA tensor")
        if ref.dtype != torch.complex64 or tgt.dtype != torch.complex64:
            raise TypeError("rasters are complex64")
        if ulhc.dtype != torch.int32 or ulhc.ndim != 2 or ulhc.shape[1] != 4:
            raise TypeError("ulhc is an int32 (pairs, 4) tensor")
        pairs = ulhc.shape[0]
        if offsets is None:
            offsets = torch.empty((pairs, 2), dtype=torch.float32, device=ref.device)
        job = _lib.Job(
            ref=ref.data_ptr(), ref_lines=ref.shape[0], ref_samples=ref.shape[1],
            tgt=tgt.data_ptr(), tgt_lines=tgt.shape[0], tgt_samples=tgt.shape[1],
            ulhc=ulhc.data_ptr(), pairs=pairs, offsets=offsets.data_ptr(),
            diag=diag.data_ptr() if diag is not None else None,
            coarse_surfaces=cs.data_ptr() if cs is not None else None,
            refined_surfaces=rs.data_ptr() if rs is not None else None,
        )
        st = c_void_p(torch_stream_handle(stream, ref.device))
        _check(self._lib, self._handle, self._lib.ampcor_correlate(self._handle, byref(job), st))
        if synchronize:
            _check(self._lib, self._handle, self._lib.ampcor_synchronize(self._handle, st))
        return offsets

    def _correlate_host(self, ref, tgt, ulhc, diag):
        ref = np.ascontiguousarray(ref, dtype=np.complex64)
        tgt = np.ascontiguousarray(tgt, dtype=np.complex64)
        ulhc = np.ascontiguousarray(ulhc, dtype=np.int32).reshape(-1, 4)
        pairs = ulhc.shape[0]
        offsets = np.empty((pairs, 2), np.float32)
        dbuf = (_lib.PairDiag * max(pairs, 1))() if diag else None
        job = _lib.Job(
            ref=ref.ctypes.data, ref_lines=ref.shape[0], ref_samples=ref.shape[1],
            tgt=tgt.ctypes.data, tgt_lines=tgt.shape[0], tgt_samples=tgt.shape[1],
            ulhc=ulhc.ctypes.data, pairs=pairs, offsets=offsets.ctypes.data,
            diag=ctypes.cast(dbuf, c_void_p).value if dbuf is not None else None,
        )
        _check(self._lib, self._handle, self._lib.ampcor_correlate_host(self._handle, byref(job)))
        if diag:
            return offsets, diag_array(dbuf, pairs)
        return offsets


def torch_stream_handle(stream, device):
    """The cudaStream_t of a torch stream (the current one when ``stream`` is None), with torch's
    legacy default stream (handle 0) passed as cudaStreamLegacy so the library orders its work
    after torch's."""
    import torch

    if stream is None:
        stream = torch.cuda.current_stream(device)
    h = int(stream.cuda_stream)
    return h if h else 1  # cudaStreamLegacy


DIAG_DTYPE = np.dtype([
    ("coarse_u", np.int32), ("coarse_v", np.int32), ("top", np.int32), ("left", np.int32),
    ("refined_u", np.int32), ("refined_v", np.int32), ("fine_p", np.int32), ("fine_q", np.int32),
    ("coarse_peak", np.float32), ("refined_peak", np.float32), ("zoom_peak", np.float32),
    ("reserved", np.float32),
])


def diag_array(buf, pairs) -> np.ndarray:
    """Structured numpy view (copied) of an array of ampcor_pair_diag."""
    raw = np.ctypeslib.as_array(ctypes.cast(buf, ctypes.POINTER(ctypes.c_uint8)),
                                shape=(max(pairs, 1) * DIAG_DTYPE.itemsize,))
    return raw.view(DIAG_DTYPE)[:pairs].copy()


def version() -> str:
    return _lib.load().ampcor_version().decode()


def copyright() -> str:
    return _lib.load().ampcor_copyright().decode()
