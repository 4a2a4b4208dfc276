"""FP64 CPU oracle of the ampcor batched tile correlator - TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` import
this package, and only to check (or time beside) the CUDA path; the product never calls it.

``oracle.c`` holds the restatements (see its header for the reference file:line of every
step); this module loads ``_build/liboracle.so`` (``make -C oracle``) and exposes:

* :func:`coarse_cpu` - the reference CPU coarse correlator (lib/libampcor/correlators/
  Sequential.cc:17-97), whose integer argmax the GPU must reproduce bit for bit;
* :func:`adjust` - the full FP64 pipeline (coarse NCC, nudge, FFT refinement, refined NCC, zoom,
  offsets) with per-pair diagnostics;
* stage functions for the known-answer tests.

:mod:`oracle.npref` cross-checks the upsampling and zoom against ``numpy.fft``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from ctypes import POINTER, c_double, c_int, c_longlong, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")
REF_COMPAT = 1
DERAMP = 2  # ORACLE_DERAMP: remove each complex tile's linear phase ramp before refining


class Src(ctypes.Structure):
    _fields_ = [
        ("ref_base", c_void_p), ("ref_off", c_void_p), ("ref_stride", c_longlong),
        ("tgt_base", c_void_p), ("tgt_off", c_void_p), ("tgt_stride", c_longlong),
    ]


class Geom(ctypes.Structure):
    _fields_ = [("R", c_int), ("W", c_int), ("f", c_int), ("m", c_int), ("z", c_int),
                ("flags", c_int)]


DIAG_DTYPE = np.dtype([
    ("coarse_u", np.int32), ("coarse_v", np.int32), ("top", np.int32), ("left", np.int32),
    ("fine_p", np.int32), ("fine_q", np.int32), ("refined_u", np.int32), ("refined_v", np.int32),
    ("coarse_peak", np.float64), ("coarse_gap", np.float64), ("refined_peak", np.float64),
    ("zoom_peak", np.float64), ("zoom_gap", np.float64),
])

_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(
                os.path.join(HERE, "oracle.c")):
            build()
        lib = ctypes.CDLL(LIB)
        lib.oracle_coarse_cpu.restype = None
        lib.oracle_coarse_cpu.argtypes = [POINTER(Src), c_longlong, c_int, c_int, c_void_p,
                                          c_void_p, c_void_p, c_int, c_int]
        lib.oracle_adjust.restype = None
        lib.oracle_adjust.argtypes = [POINTER(Src), c_longlong, POINTER(Geom), c_void_p,
                                      c_void_p, c_void_p, c_void_p, c_int]
        lib.oracle_deramp.restype = None
        lib.oracle_deramp.argtypes = [c_void_p, c_int]
        lib.oracle_argmax_first.restype = c_int
        lib.oracle_argmax_first.argtypes = [c_void_p, c_longlong]
        lib.oracle_sat.restype = None
        lib.oracle_sat.argtypes = [c_void_p, c_int, c_int, c_void_p]
        lib.oracle_box.restype = c_double
        lib.oracle_box.argtypes = [c_void_p, c_int, c_int, c_int, c_int, c_int]
        lib.oracle_ncc.restype = c_double
        lib.oracle_ncc.argtypes = [c_void_p, c_int, c_void_p, c_int, c_void_p, c_void_p]
        lib.oracle_nudge.restype = None
        lib.oracle_nudge.argtypes = [c_int, c_int, c_int, c_int, c_int, POINTER(c_int),
                                     POINTER(c_int)]
        lib.oracle_dirichlet.restype = c_double
        lib.oracle_dirichlet.argtypes = [c_int, c_double]
        lib.oracle_interp_matrix.restype = None
        lib.oracle_interp_matrix.argtypes = [c_int, c_int, c_void_p]
        lib.oracle_upsample.restype = None
        lib.oracle_upsample.argtypes = [c_void_p, c_int, c_int, c_void_p, c_void_p, c_void_p]
        lib.oracle_xcorr.restype = None
        lib.oracle_xcorr.argtypes = [c_void_p, c_int, c_void_p, c_int, c_void_p]
        lib.oracle_zoom.restype = None
        lib.oracle_zoom.argtypes = [c_void_p, c_int, c_int, c_void_p, c_int, c_void_p, c_void_p]
        _lib = lib
    return _lib


def _threads(threads):
    return int(threads) if threads else (os.cpu_count() or 1)


class Sources:
    """Tile sources of a batch: rasters + chip/window corners, or a reference-style arena."""

    def __init__(self, ref, tgt, ulhc):
        self.ref = np.ascontiguousarray(ref, np.complex64)
        self.tgt = np.ascontiguousarray(tgt, np.complex64)
        ulhc = np.asarray(ulhc, np.int64).reshape(-1, 4)
        self.ref_off = np.ascontiguousarray(ulhc[:, 0] * self.ref.shape[1] + ulhc[:, 1])
        self.tgt_off = np.ascontiguousarray(ulhc[:, 2] * self.tgt.shape[1] + ulhc[:, 3])
        self.pairs = ulhc.shape[0]
        self.src = Src(self.ref.ctypes.data, self.ref_off.ctypes.data, self.ref.shape[1],
                       self.tgt.ctypes.data, self.tgt_off.ctypes.data, self.tgt.shape[1])


def coarse_cpu(ref, tgt, ulhc, R, W, surfaces=False, threads=None, as_built=False):
    """Reference CPU coarse correlator.  Returns (argmax (P,2) int32, gap (P,), [surfaces]).

    ``as_built=False`` (the default, and the integer-offset gate) centres each placement on its
    window box mean, as the reference intends and its CUDA worker does; ``as_built=True`` repeats
    the arithmetic of the reference's CPU code as written, whose summed-area table is built over
    an empty grid (lib/libampcor/correlators/Sequential.cc:48), so no mean is taken off."""
    s = Sources(ref, tgt, ulhc)
    C = W - R + 1
    arg = np.zeros((s.pairs, 2), np.int32)
    gap = np.zeros(s.pairs, np.float64)
    cor = np.zeros((s.pairs, C, C), np.float64) if surfaces else None
    load().oracle_coarse_cpu(ctypes.byref(s.src), s.pairs, R, W,
                             cor.ctypes.data if surfaces else None, arg.ctypes.data,
                             gap.ctypes.data, _threads(threads), int(bool(as_built)))
    return (arg, gap, cor) if surfaces else (arg, gap)


def adjust(ref, tgt, ulhc, R, W, f, m, z, ref_compat=False, surfaces=False, threads=None,
           deramp=False):
    """Full FP64 pipeline.  Returns (offsets (P,2) float32, diag structured (P,), [coarse and
    refined surfaces]).  ``deramp`` removes each complex tile's linear phase ramp before the
    refinement (oracle_deramp)."""
    s = Sources(ref, tgt, ulhc)
    g = Geom(R, W, f, m, z, (REF_COMPAT if ref_compat else 0) | (DERAMP if deramp else 0))
    C, Cf = W - R + 1, 2 * f * m + 1
    off = np.zeros((s.pairs, 2), np.float32)
    diag = np.zeros(s.pairs, DIAG_DTYPE)
    cs = np.zeros((s.pairs, C, C)) if surfaces else None
    rs = np.zeros((s.pairs, Cf, Cf)) if surfaces else None
    load().oracle_adjust(ctypes.byref(s.src), s.pairs, ctypes.byref(g), off.ctypes.data,
                         diag.ctypes.data, cs.ctypes.data if surfaces else None,
                         rs.ctypes.data if surfaces else None, _threads(threads))
    return (off, diag, cs, rs) if surfaces else (off, diag)


# stage functions ------------------------------------------------------------------------

def deramp(tile):
    """The FP64 deramp of one square complex tile (oracle_deramp), returned as a new array."""
    t = np.ascontiguousarray(tile, np.complex128).copy()
    load().oracle_deramp(t.ctypes.data, t.shape[0])
    return t


def sat(x):
    x = np.ascontiguousarray(x, np.float64)
    out = np.empty_like(x)
    load().oracle_sat(x.ctypes.data, x.shape[0], x.shape[1], out.ctypes.data)
    return out


def box(sat_table, r0, c0, r1, c1):
    t = np.ascontiguousarray(sat_table, np.float64)
    return load().oracle_box(t.ctypes.data, t.shape[1], r0, c0, r1, c1)


def ncc(chip, win):
    chip = np.ascontiguousarray(chip, np.float64)
    win = np.ascontiguousarray(win, np.float64)
    R, W = chip.shape[0], win.shape[0]
    C = W - R + 1
    g = np.empty((C, C))
    scratch = np.empty(W * W + R * R)
    sigma = load().oracle_ncc(chip.ctypes.data, R, win.ctypes.data, W, g.ctypes.data,
                              scratch.ctypes.data)
    return g, sigma


def xcorr(chip, win):
    chip = np.ascontiguousarray(chip, np.float64)
    win = np.ascontiguousarray(win, np.float64)
    R, W = chip.shape[0], win.shape[0]
    out = np.empty((W - R + 1, W - R + 1))
    load().oracle_xcorr(chip.ctypes.data, R, win.ctypes.data, W, out.ctypes.data)
    return out


def argmax_first(a):
    a = np.ascontiguousarray(a, np.float64)
    return int(load().oracle_argmax_first(a.ctypes.data, a.size))


def nudge(u, v, R, W, m):
    t, l = c_int(), c_int()
    load().oracle_nudge(u, v, R, W, m, ctypes.byref(t), ctypes.byref(l))
    return t.value, l.value


def interp_matrix(N, f):
    U = np.empty((f * N, N))
    load().oracle_interp_matrix(N, f, U.ctypes.data)
    return U


def upsample(tile, f):
    tile = np.ascontiguousarray(tile, np.complex128)
    N = tile.shape[0]
    U = interp_matrix(N, f)
    out = np.empty((f * N, f * N), np.complex128)
    tmp = np.empty((N, f * N), np.complex128)
    load().oracle_upsample(tile.ctypes.data, N, f, U.ctypes.data, out.ctypes.data,
                           tmp.ctypes.data)
    return out


def zoom(G, z, use_abs=False):
    G = np.ascontiguousarray(G, np.float64)
    Cf = G.shape[0]
    U = interp_matrix(Cf, z)
    out = np.empty((z * Cf, z * Cf))
    tmp = np.empty((Cf, z * Cf))
    load().oracle_zoom(G.ctypes.data, Cf, z, U.ctypes.data, int(use_abs), out.ctypes.data,
                       tmp.ctypes.data)
    return out
