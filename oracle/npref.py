"""numpy.fft restatement of the refinement and zoom transforms - TEST INFRASTRUCTURE ONLY.

The intended math of the reference's cuFFT stages (lib/libampcor_cuda/correlators/
Sequential.icc:703-873 refine the chip, :915-1087 the target neighbourhood, :1101-1286 zoom the
correlation surface): forward FFT of the N x N tile, spectrum zero-padded to f N x f N with the
negative-frequency quadrants kept at the far corners and, for even N, the Nyquist row/column
split in half between its two images, inverse FFT, scaled so that the original samples are
reproduced (net factor 1/N^2).  ``oracle.c`` computes the same operator as a Dirichlet-kernel
matrix; tests check the two against each other in FP64.
"""
from __future__ import annotations

import numpy as np


def _pad_axis(X, axis, f):
    N = X.shape[axis]
    F = f * N
    shape = list(X.shape)
    shape[axis] = F
    out = np.zeros(shape, dtype=np.complex128)
    X = np.moveaxis(X, axis, 0)
    o = np.moveaxis(out, axis, 0)
    if N % 2:
        h = (N - 1) // 2
        o[: h + 1] = X[: h + 1]
        o[F - h:] = X[N - h:]
    else:
        h = N // 2
        o[:h] = X[:h]
        o[F - h + 1:] = X[h + 1:]
        o[h] = 0.5 * X[h]
        o[F - h] = 0.5 * X[h]
    return np.moveaxis(o, 0, axis)


def upsample_fft(tile, f):
    """Band-limited upsampling of an N x N complex tile to fN x fN (FP64)."""
    tile = np.asarray(tile, np.complex128)
    N = tile.shape[0]
    X = np.fft.fft2(tile)
    X = _pad_axis(_pad_axis(X, 0, f), 1, f)
    return np.fft.ifft2(X) * (f * f)


def zoom_fft(G, z, use_abs=False):
    """Zoom a real Cf x Cf surface by z; real part (or magnitude as the reference's c2r)."""
    out = upsample_fft(np.asarray(G, np.complex128), z)
    return np.abs(out) if use_abs else out.real
